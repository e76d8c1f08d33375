"""The serving throughput that bench.py reports: completions per second between
the first and the last completion, so a loop that keeps up reports about the
offered rate whatever its latency, and a saturated loop reports its capacity.
Checked with a fake server (no GPU): constant latency, and FIFO service at a
fixed capacity."""
import importlib.util
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Info:
    def __init__(self, submit_ms, finish_ms):
        self.submit_ms = submit_ms
        self.finish_ms = finish_ms
        self.latency_ms = finish_ms - submit_ms
        self.state = "done"


class _FakeServer:
    """Finishes request k at max(submit + latency, first submit + latency +
    k / capacity) (FIFO at `capacity` q/s; no cap when capacity is None)."""

    def __init__(self, latency_ms, capacity=None):
        import time
        self._clock = time.perf_counter
        self.latency_ms = latency_ms
        self.capacity = capacity
        self.submits = []

    def submit(self, desc, out=None):
        self.submits.append(self._clock() * 1e3)
        return len(self.submits) - 1

    def drain(self):
        pass

    def wait(self, k):
        sub = self.submits[k]
        fin = sub + self.latency_ms
        if self.capacity is not None:
            fin = max(fin, self.submits[0] + self.latency_ms + k * 1e3 / self.capacity)
        return _Info(sub, fin)


def test_keeping_up_reports_the_offered_rate_despite_long_latency():
    b = _bench()
    srv = _FakeServer(latency_ms=700.0)
    r = b.poisson_run(srv, [None] * 8, rate=400.0, seconds=0.5, seed=3)
    assert r["completed"] == r["requests"] == 200
    # constant latency: the completions repeat the arrivals shifted by 700 ms,
    # so the reported rate is the sampled arrival rate, latency not charged
    arrival_rate = (len(srv.submits) - 1) / ((srv.submits[-1] - srv.submits[0]) / 1e3)
    assert r["throughput_qps"] == pytest.approx(arrival_rate, rel=1e-6)
    assert r["throughput_qps"] == pytest.approx(400.0, rel=0.25)
    assert r["p50_ms"] == pytest.approx(700.0, abs=1.0)


def test_saturated_loop_reports_its_capacity():
    b = _bench()
    r = b.poisson_run(_FakeServer(latency_ms=50.0, capacity=100.0), [None] * 8, rate=400.0,
                      seconds=0.5, seed=4)
    assert r["throughput_qps"] == pytest.approx(100.0, rel=0.05)
    assert not r["sustained"]
