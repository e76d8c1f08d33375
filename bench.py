#!/usr/bin/env python
"""Benchmark of the batched multi-query traversal path.

Workloads (`--workload`, default c2):

  c1  R-MAT scale 16, edge factor 16 (a=.57 b=.19 c=.19), symmetrised,
      deduplicated, no self loops, int32 CSR; 64 BFS sources drawn uniformly
      from non-isolated vertices; one 64-bit query-mask word per vertex.
  c2  R-MAT scale 22, same parameters, uint32 weights uniform in [1,64];
      256 BFS + 256 SSSP sources from the largest component; 4 x 64-bit mask
      words per vertex.  (The default line.)
  c3  2048 x 2048 4-neighbour grid, 10% of the edges deleted, 0.1% random
      shortcuts, symmetrised, f32 weights uniform in [1,100]; 1024 SSSP
      queries (half from the corner region, half uniform) + one WCC pass.
  c5  Chung-Lu power-law graph, 2^25 vertices, exponent 2.1, mean degree 16,
      f32 log-normal(0,1) weights; 4096 queries in four 1024-slot groups
      (two BFS, two SSSP; half of each group's sources from the top 1% of
      hubs, half uniform) + one WCC pass.
  serve  (or --serve) R-MAT 24 serving loop: Poisson arrivals, 60% BFS /
      30% SSSP / 10% k-hop; p50/p99 latency and completed queries/s.

A step is one pass of the workload's batches over device-resident inputs,
with init and output writing included.  Metric: aggregate GTEPS = the sum
over queries of the directed CSR entries of the vertices each query reached
(a WCC pass counts every entry), divided by the time.

  python bench.py [--workload c2] [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) each rank runs its round-robin shard of an N-times
larger query list (cgp_b200.parallel.shard_indices) on its own GPU: queries
are independent, so there is no collective on the data path (weak scaling);
the time is the max over ranks.  `--impl reference` times the reference's own
CPU traversal (cpu_bfs / cpu_sssp compiled from the reference sources into
oracle/_ref) on the host cores, on inputs built by the C generators under
oracle/ (the same arrays), and prints the same config.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L2_BYTES = 126 * 2**20
BFS_INF = 2**31 - 1

# DRAM bytes per level of a level class from ncu captures (dram__bytes_read.sum
# + dram__bytes_write.sum summed over the level's kernels), with where and when
# they were measured.  Reported beside the run's own numbers; never computed
# from files at run time.
NCU_TRAFFIC = {
    ("c2", "sssp_gather"): {
        "bytes_per_level": 5.812e10,
        "source": "profiles/dram_traffic_sssp_gather_rmat22.md (one-pass ncu metrics, full size)",
        "captured": "2026-12-03",
    },
}


WORKLOADS = {
    "c1": {"graph": "rmat", "scale": 16, "edge_factor": 16, "weights": None,
           "groups": [("bfs", 64)], "wcc": False, "sources": "non-isolated"},
    "c2": {"graph": "rmat", "scale": 22, "edge_factor": 16, "weights": ("u32", 1, 64, False),
           "groups": [("bfs", 256), ("sssp", 256)], "wcc": False, "sources": "largest component"},
    "c3": {"graph": "grid", "rows": 2048, "cols": 2048, "delete": 0.1, "shortcut": 0.001,
           "weights": ("f32", 1.0, 100.0, False), "groups": [("sssp", 1024)], "wcc": True,
           "sources": "half corner region, half uniform"},
    "c5": {"graph": "chung_lu", "vertices": 1 << 25, "exponent": 2.1, "mean_degree": 16.0,
           "weights": ("f32", 0.0, 1.0, True),
           "groups": [("bfs", 1024), ("bfs", 1024), ("sssp", 1024), ("sssp", 1024)],
           "wcc": True, "sources": "half top-1% degree hubs, half uniform"},
}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c5", "serve"])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=0, help="timed steps (0: the workload's default)")
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="cgp", choices=["cgp", "reference"])
    p.add_argument("--scale", type=int, default=0, help="override the R-MAT scale")
    p.add_argument("--vertices", type=int, default=0, help="override the Chung-Lu vertex count")
    p.add_argument("--grid-side", type=int, default=0, help="override the grid's rows and columns")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-one-query", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--e2e-layout", default="vertex", choices=["vertex", "query"])
    p.add_argument("--mode", default="hybrid")
    p.add_argument("--pull-edge-ratio", type=float, default=0.20)
    p.add_argument("--pull-frontier-ratio", type=float, default=0.15)
    p.add_argument("--heavy-degree", type=int, default=0)
    p.add_argument("--sssp-pull-edge-ratio", type=float, default=0.5)
    p.add_argument("--sssp-pull-pair-ratio", type=float, default=0.5)
    p.add_argument("--bfs-pull-form", type=int, default=0, choices=[0, 1, 2],
                   help="BFS pull: lane per vertex (0), CTA chunks (1), lane per vertex in "
                        "in-degree order (2)")
    p.add_argument("--levels-per-sync", type=int, default=0)
    p.add_argument("--level-loop", default="", choices=["", "auto", "chunks", "device"],
                   help="level loop form (default: device-looped graph for c3, else chunks)")
    p.add_argument("--no-light-chunks", action="store_true",
                   help="gather light vertices one warp per vertex instead of in CTA chunks")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--no-profile", action="store_true", help="skip the profiled step")
    p.add_argument("--json-out", default="")
    p.add_argument("--serve", action="store_true",
                   help="serving workload: R-MAT 24, Poisson arrivals, p50/p99 latency")
    p.add_argument("--serve-rates", default="500,2000,8000")
    p.add_argument("--serve-seconds", type=float, default=10.0)
    p.add_argument("--serve-slots", type=int, default=256)
    p.add_argument("--serve-out", default="device", choices=["device", "none"],
                   help="serving: write each result to a device buffer (a ring) or discard it")
    p.add_argument("--serve-out-ring", type=int, default=512)
    p.add_argument("--serve-groups", type=int, default=0,
                   help="traversal groups of the serving loop (0 = 1)")
    p.add_argument("--sssp-chunk-direction", type=int, default=0,
                   help="SSSP gather/scatter per 32-slot chunk (1), per group (-1), auto (0)")
    p.add_argument("--serve-admission", default="group", choices=["slots", "chunks", "group"],
                   help="serving admission: any free slot, whole 32-slot chunks, or whole groups")
    p.add_argument("--serve-profile", action="store_true",
                   help="time the serving loop's kernel classes (slower: no CUDA graphs)")
    a = p.parse_args()
    if a.serve:
        a.workload = "serve"
    return a


def default_steps(name):
    return {"c1": 20, "c2": 20, "c3": 3, "c5": 1}.get(name, 1)


# ------------------------------------------------------------------ workload
def workload_spec(args):
    wl = dict(WORKLOADS[args.workload])
    if args.scale and wl["graph"] == "rmat":
        wl["scale"] = args.scale
    if args.vertices and wl["graph"] == "chung_lu":
        wl["vertices"] = args.vertices
    if args.grid_side and wl["graph"] == "grid":
        wl["rows"] = wl["cols"] = args.grid_side
    return wl


def workload_name(args, wl):
    base = {"rmat": f"rmat{wl.get('scale')}_ef{wl.get('edge_factor')}",
            "grid": f"grid{wl.get('rows')}x{wl.get('cols')}",
            "chung_lu": f"chunglu{wl.get('vertices')}_g{wl.get('exponent')}"}[wl["graph"]]
    parts = {}
    for kind, n in wl["groups"]:
        parts[kind] = parts.get(kind, 0) + n
    q = "_".join(f"{k}{n}" for k, n in parts.items())
    return f"{args.workload}_{base}_{q}" + ("_wcc" if wl["wcc"] else "")


def make_graph(gen, wl):
    """Builds the workload graph with `gen` (the library's generators on the
    GPU arm, oracle's C restatement on the reference arm: same arrays)."""
    t = time.perf_counter()
    if wl["graph"] == "rmat":
        g = gen.gen_rmat(wl["scale"], wl["edge_factor"], 0.57, 0.19, 0.19, seed=1)
    elif wl["graph"] == "grid":
        g = gen.gen_grid(wl["rows"], wl["cols"], wl["delete"], wl["shortcut"], seed=1)
    else:
        g = gen.gen_chung_lu(wl["vertices"], wl["exponent"], wl["mean_degree"], seed=1)
    if wl["weights"]:
        kind, p0, p1, logn = wl["weights"]
        g = g.with_weights(kind, p0, p1, seed=2, lognormal=logn)
    return g, time.perf_counter() - t


def component_tables(g, labels):
    """Per-vertex component label -> (size, directed CSR entries)."""
    lab = labels.astype(np.int64)
    deg = g.degrees()
    size = np.bincount(lab, minlength=g.num_vertices)
    edges = np.bincount(lab, weights=deg.astype(np.float64), minlength=g.num_vertices)
    return size, edges


def select_queries(args, wl, g, labels, world):
    """The global query list of every group: [(kind, sources)], identical on
    both arms (the same seeded picks on the same arrays)."""
    V = g.num_vertices
    groups = []
    if args.workload == "c1":
        src = g.pick_sources(64 * world, seed=42)
        groups = [("bfs", src)]
    elif args.workload == "c2":
        size, _ = component_tables(g, labels)
        big = int(np.argmax(size))
        allowed = (labels.astype(np.int64) == big).astype(np.uint8)
        nb, ns = wl["groups"][0][1] * world, wl["groups"][1][1] * world
        src = g.pick_sources(nb + ns, seed=42, allowed=allowed)
        groups = [("bfs", src[:nb]), ("sssp", src[nb:])]
    elif args.workload == "c3":
        rows, cols = wl["rows"], wl["cols"]
        r = np.arange(V) // cols
        c = np.arange(V) % cols
        corner = ((r < max(2, rows // 10)) & (c < max(2, cols // 10))).astype(np.uint8)
        n = 1024 * world
        a = g.pick_sources(n // 2, seed=42, allowed=corner)
        b = g.pick_sources(n - n // 2, seed=43)
        groups = [("sssp", np.concatenate([a, b]))]
    elif args.workload == "c5":
        deg = g.degrees()
        hubs = np.zeros(V, np.uint8)
        hubs[np.argsort(-deg, kind="stable")[: max(1, V // 100)]] = 1
        for i, (kind, n) in enumerate(wl["groups"]):
            m = n * world
            a = g.pick_sources(m // 2, seed=42 + 2 * i, allowed=hubs)
            b = g.pick_sources(m - m // 2, seed=43 + 2 * i)
            groups.append((kind, np.concatenate([a, b])))
    return groups


def shard_groups(groups, rank, world):
    from cgp_b200.parallel import shard_indices
    return [(k, np.asarray(s)[shard_indices(len(s), rank, world)]) for k, s in groups]


def workload_config(args, wl, g, world):
    """The config keys both arms print."""
    cfg = {"workload": workload_name(args, wl), "graph": wl["graph"],
           "V": int(g.num_vertices), "E": int(g.num_edges),
           "weights": (None if not wl["weights"] else
                       f"{wl['weights'][0]} {'lognormal' if wl['weights'][3] else 'uniform'} "
                       f"[{wl['weights'][1]},{wl['weights'][2]}]"),
           "queries_per_gpu": [[k, n] for k, n in wl["groups"]] + ([["wcc", 1]] if wl["wcc"] else []),
           "sources": wl["sources"], "seeds": {"graph": 1, "weights": 2, "sources": 42},
           "parallelism": f"query-sharded x{world}"}
    for k in ("scale", "edge_factor", "rows", "cols", "delete", "shortcut", "vertices", "exponent",
              "mean_degree"):
        if k in wl:
            cfg[k] = wl[k]
    return cfg


def reach_edges(groups, labels, comp_edges):
    """Directed CSR entries reached by each query (a query on a symmetric
    graph reaches exactly its source's component)."""
    lab = labels.astype(np.int64)
    return [comp_edges[lab[np.asarray(s, np.int64)]].astype(np.float64) for _, s in groups]


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        sm, mx, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        busy = [s for s, p in zip(sm, power) if p > 0.5 * max(power)] if power else []
        return {"sm_mhz": statistics.median(busy or sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ----------------------------------------------------------------- roofline
def level_bytes(p, kind, V, W, ob=4, qs=0):
    """Bytes of one level from its device counters, two ways.

    Algorithmic (per unit of work, the per-edge / per-pair counts; L2 hits
    included because every (edge, slot) access is charged):
      BFS push: U(2o+Wb+4) + D(4+2Wb) + 4N + Wb U'
      BFS pull: 2 V Wb + P 2o + S(4+Wb) + 4N
      SSSP scatter: U(2o+Wb+4) + D(4+4+Wb) + 4 sum(popc) + 8 A + Wb U'
      SSSP gather:  2o V + 4 Qs P + S(4+4+Wb) + 4 A + 4 I + Wb U'
    Compulsory (what must cross HBM at least once: every array touched read
    once, every changed entry written once):
      BFS push: U(2o+Wb) + D(4) + N 4 + Wb U' (+ visited words of the
                destinations, D Wb capped at V Wb)
      BFS pull: 3 V Wb + P 2o + S 4 + 4N
      SSSP scatter: U(2o+Wb) + D(4+4) + 4 sum(popc) + min(A, V Qs) 4 + 4 I + Wb U'
      SSSP gather:  o V + S(4+4) + 4 Qs P + 4 I + Wb (P + U')
    (U, U' = frontier sizes, D = their out-degree sum, N = newly reached pairs,
    P, S = vertices and in-edges a pull level scanned, A = (edge, slot) pairs,
    I = improved entries, Qs = SSSP slots, Wb = mask bytes per vertex.)"""
    Wb = 8 * W
    U, D, N, Un = p.frontier_size, p.frontier_edges, p.new_pairs, p.next_size
    if kind == "bfs":
        if p.mode == "push":
            alg = U * (2 * ob + Wb + 4) + D * (4 + 2 * Wb) + 4 * N + Wb * Un
            comp = U * (2 * ob + Wb) + 4 * D + min(D, V) * Wb + 4 * N + Wb * Un
            return "bfs_push", alg, comp
        alg = 2 * V * Wb + p.pull_vertices * 2 * ob + p.pull_edges * (4 + Wb) + 4 * N
        comp = 3 * V * Wb + p.pull_vertices * 2 * ob + p.pull_edges * 4 + 4 * N
        return "bfs_pull", alg, comp
    if p.sssp_mode == "push":
        alg = (U * (2 * ob + Wb + 4) + D * (4 + 4 + Wb) + 4 * p.sssp_active + 8 * p.sssp_pairs
               + Wb * Un)
        comp = (U * (2 * ob + Wb) + D * 8 + 4 * p.sssp_active + 4 * min(p.sssp_pairs, V * qs)
                + 4 * p.improved + Wb * Un)
        return "sssp_scatter", alg, comp
    P, S = p.sssp_pull_vertices, p.sssp_pull_edges
    alg = 2 * ob * V + 4 * qs * P + S * (4 + 4 + Wb) + 4 * p.sssp_pairs + 4 * p.improved + Wb * Un
    comp = ob * V + S * 8 + 4 * qs * P + 4 * p.improved + Wb * (P + Un)
    return "sssp_gather", alg, comp


# kernels that do the work of each level class
CLASS_KERNELS = {
    "bfs_push": "k_bfs_push, k_bfs_push_heavy",
    "bfs_pull": "k_bfs_pull, k_bfs_pull_heavy(_commit)",
    "sssp_scatter": "k_sssp_push, k_sssp_dense, k_sssp_push_heavy",
    "sssp_gather": "k_sssp_pull_chunked, k_sssp_pull_heavy_vec",
}


def level_classes(profiles, kind, V, W, ob=4, qs=0):
    """Per level class: levels, kernel ms (CUDA events on the launching
    stream, every kernel of the level), algorithmic and compulsory bytes."""
    out = {}
    for p in profiles:
        name, alg, comp = level_bytes(p, kind, V, W, ob=ob, qs=qs)
        c = out.setdefault(name, {"ms": 0.0, "launches": 0, "bytes": 0, "compulsory": 0})
        c["ms"] += p.kernel_ms
        c["launches"] += 1
        c["bytes"] += alg
        c["compulsory"] += comp
    return out


def merge_classes(a, b):
    for k, v in b.items():
        c = a.setdefault(k, {"ms": 0.0, "launches": 0, "bytes": 0, "compulsory": 0})
        for f in c:
            c[f] += v[f]
    return a


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def roofline_line(args, kclass):
    peak, peak_src = measured_peaks()
    if not kclass:
        return None
    dom = max(kclass, key=lambda k: kclass[k]["ms"])
    k = kclass[dom]
    n = max(1, k["launches"])
    sec = k["ms"] / 1e3
    achieved = k["compulsory"] / sec / 1e9
    alg = k["bytes"] / sec / 1e9
    tr = NCU_TRAFFIC.get((args.workload, dom))
    line = {"bound": "hbm", "kernel": f"{dom} levels ({CLASS_KERNELS[dom]})",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
            else "fallback 6650 GB/s",
            "bytes": "compulsory: each array the level touches read once, each changed entry "
                     "written once",
            "per": "level", "compulsory_bytes_per_launch": k["compulsory"] / n,
            "ms_per_launch": k["ms"] / n,
            "traffic": tr["bytes_per_level"] if tr else None,
            "traffic_source": (f"{tr['source']}, captured {tr['captured']}" if tr else None),
            "dram_frac": (tr["bytes_per_level"] / (k["ms"] / n / 1e3) / 1e9 / peak if tr else None),
            "l2_inclusive": {"achieved": alg, "frac": alg / peak,
                             "bytes_per_launch": k["bytes"] / n,
                             "note": "every (edge, slot) access charged, L2 hits included"},
            "classes": {c: {"ms": v["ms"], "launches": v["launches"],
                            "GBps_algorithmic": v["bytes"] / max(v["ms"], 1e-9) / 1e6,
                            "GBps_compulsory": v["compulsory"] / max(v["ms"], 1e-9) / 1e6,
                            "frac_algorithmic": v["bytes"] / max(v["ms"], 1e-9) / 1e6 / peak}
                        for c, v in kclass.items()}}
    return line


# -------------------------------------------------------------- CPU sides
def cpu_sample_sizes(args, groups, threads):
    """A bounded sample of each group's queries for the CPU reference: about
    10-30 s of host work, BFS and SSSP in the workload's own ratio."""
    per = {"c1": 64, "c2": max(1, threads // 2), "c3": max(1, threads), "c5": max(1, threads // 4)}
    n = per.get(args.workload, 1)
    kinds = [k for k, _ in groups]
    out = []
    for k, s in groups:
        share = n if args.workload == "c1" else max(1, n // max(1, kinds.count(k)))
        out.append(min(len(s), share))
    return out


def cpu_reference_sample(g, groups, sizes, threads):
    """The reference's cpu_bfs / cpu_sssp (oracle/_ref) when compiled here,
    else the C restatement, over `threads` host threads.  Returns (seconds,
    edges, kind, outputs per group)."""
    import oracle
    gf = type(g)(g.row_offsets, g.col_indices,
                 None if g.weights is None else g.weights.astype(np.float32))
    deg = g.degrees()
    t = time.perf_counter()
    outs = []
    kind = "reference" if oracle.has_ref() else "port"
    for (k, s), n in zip(groups, sizes):
        src = np.asarray(s[:n], np.int32)
        if kind == "reference":
            outs.append(oracle.ref_batch("bfs" if k == "bfs" else "sssp", gf, src, threads=threads))
        else:
            outs.append(oracle.batch(k, g, src, threads=threads)[0])
    dt = time.perf_counter() - t
    edges = 0
    for o in outs:
        if o.dtype == np.float32:
            reached = np.isfinite(o)
        elif o.dtype == np.uint32:
            reached = o != np.uint32(0xFFFFFFFF)
        else:
            reached = o != BFS_INF
        edges += int((reached * deg[None, :]).sum()) if reached.size else 0
    return dt, edges, kind, outs


def as_u32_words(cpu_out, weight_kind):
    """The reference's float distances as the 4-byte words the library writes
    (uint32 distances for integer weights, f32 bits for float weights)."""
    if cpu_out.dtype != np.float32:
        return cpu_out.view(np.uint32)
    if weight_kind == "f32":
        return cpu_out.view(np.uint32)
    u = np.full(cpu_out.shape, 2**32 - 1, np.uint32)
    fin = np.isfinite(cpu_out)
    u[fin] = cpu_out[fin].astype(np.uint32)
    return u


def run_reference_arm(args):
    """The reference's CPU traversal on the same workload, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    import oracle
    wl = workload_spec(args)
    if args.workload == "serve":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no serving loop to time on the host cores"}))
        return 0
    steps = args.steps or default_steps(args.workload)
    g, _ = make_graph(oracle, wl)
    labels = oracle.wcc_components(g)
    groups = shard_groups(select_queries(args, wl, g, labels, world), 0, world)
    threads = os.cpu_count() or 1
    sizes = cpu_sample_sizes(args, groups, threads)
    for _ in range(args.warmup):
        cpu_reference_sample(g, groups, [min(2, n) for n in sizes], threads)
    times, edges, kind = [], 0, "port"
    for _ in range(steps):
        dt, e, kind, _ = cpu_reference_sample(g, groups, sizes, threads)
        times.append(dt)
        edges = e
    t = sum(times)
    value = steps * edges / t / 1e9
    sample = (" + ".join(f"{n} {k.upper()}" for (k, _), n in zip(groups, sizes))
              + f" queries of the workload per step, reference cpu_bfs/cpu_sssp, one query "
                f"per host thread")
    line = {
        "impl": "reference", "metric": "aggregate GTEPS", "value": value, "unit": "GTEPS",
        "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1000 * t / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": wl["weights"][0] if wl["weights"] else "i32",
        "data": "synthetic", "config": workload_config(args, wl, g, world),
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ serving
def serve_mix(g, n, seed, allowed=None):
    """60% BFS, 30% SSSP, 10% k-hop BFS (k uniform in 2..6), sources uniform
    over non-isolated vertices (seeded)."""
    import cgp_b200 as cgp
    rng = np.random.default_rng(seed)
    src = g.pick_sources(n, seed=seed, allowed=allowed)
    u = rng.random(n)
    ks = rng.integers(2, 7, n)
    out = []
    for i in range(n):
        kind = "bfs" if u[i] < 0.6 else ("sssp" if u[i] < 0.9 else "khop")
        out.append(cgp.QueryDescriptor(int(src[i]), kind, int(ks[i]) if kind == "khop" else 0))
    return out


def poisson_run(server, descs, rate, seconds, seed, outs=None):
    """Submits requests at Poisson arrival times for `seconds`, waits for all,
    returns latency percentiles and throughput.  Throughput is the completion
    rate between the first and the last completion: it equals the offered rate
    while latency stays stationary and falls to the service capacity when the
    queue grows (the first request's latency, the pipeline fill, is not
    charged to the window).  The p50 latencies of the first and the last third
    of the arrivals show whether the queue grows.  With `outs`, request i's
    result is written to device buffer outs[i % len(outs)] (a ring)."""
    rng = np.random.default_rng(seed)
    n = max(1, int(rate * seconds))
    gaps = rng.exponential(1.0 / rate, n)
    t_arr = np.cumsum(gaps)
    tickets = []
    t0 = time.perf_counter()
    for i in range(n):
        target = t0 + t_arr[i]
        while True:
            now = time.perf_counter()
            if now >= target:
                break
            if target - now > 0.002:
                time.sleep(target - now - 0.001)
        tickets.append(server.submit(descs[i % len(descs)],
                                     outs[i % len(outs)] if outs else None))
    server.drain()
    infos = [server.wait(t) for t in tickets]
    lat = np.array([i.latency_ms for i in infos])
    third = max(1, n // 3)
    done = [i for i in infos if i.state == "done"]
    fin = sorted(i.finish_ms for i in done)
    span = max(fin[-1] - fin[0], 1e-3) / 1e3
    tput = (len(done) - 1) / span if len(done) > 1 else 0.0
    return {"rate_qps": rate, "requests": n, "completed": len(done),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "throughput_qps": tput,
            "p50_first_third_ms": float(np.percentile(lat[:third], 50)),
            "p50_last_third_ms": float(np.percentile(lat[-third:], 50)),
            "sustained": bool(tput >= 0.9 * rate)}


def run_serve(args):
    import cgp_b200 as cgp
    scale = args.scale or 24
    t = time.perf_counter()
    g = cgp.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=1)
    g = g.with_weights("u32", 1, 255, seed=2)
    gen_s = time.perf_counter() - t
    graph = cgp.CsrGraph(g, offsets64=True, symmetric=True)
    descs = serve_mix(g, 4096, seed=42)
    rows = []
    with cgp.Server(graph, slots=args.serve_slots,
                    options=cgp.RunOptions(traversal_mode=args.mode,
                                           pull_edge_ratio=args.pull_edge_ratio,
                                           heavy_degree=args.heavy_degree,
                                           sssp_pull_edge_ratio=args.sssp_pull_edge_ratio,
                                           sssp_pull_pair_ratio=args.sssp_pull_pair_ratio,
                                           sssp_chunk_direction=args.sssp_chunk_direction,
                                           serve_admission=args.serve_admission,
                                           serve_groups=args.serve_groups,
                                           profile_kernels=args.serve_profile)) as srv:
        outs = None
        if args.serve_out == "device":
            import torch
            outs = [torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
                    for _ in range(args.serve_out_ring)]
        poisson_run(srv, descs[:64], 200, 0.3, seed=7, outs=outs)  # warm-up
        for i, rate in enumerate(float(r) for r in args.serve_rates.split(",")):
            s0 = srv.stats()
            row = poisson_run(srv, descs, rate, args.serve_seconds, seed=100 + i, outs=outs)
            s1 = srv.stats()
            row["levels"] = s1["levels"] - s0["levels"]
            row["level_ms"] = (s1["busy_ms"] - s0["busy_ms"]) / max(1, row["levels"])
            row["retire_ms"] = s1["retire_ms"] - s0["retire_ms"]
            row["retire_passes"] = s1["retire_passes"] - s0["retire_passes"]
            row["admit_ms"] = s1["admit_ms"] - s0["admit_ms"]
            sc = s1["sssp_chunk_levels"] - s0["sssp_chunk_levels"]
            row["gathering_chunk_frac"] = ((s1["gather_chunk_levels"] - s0["gather_chunk_levels"])
                                           / sc if sc else None)
            if args.serve_profile:
                row["kernel_ms"] = {k: s1["kernel_ms"].get(k, 0) - s0["kernel_ms"].get(k, 0)
                                    for k in s1["kernel_ms"]}
            rows.append(row)
        st = srv.stats()
    line = {"metric": "serve p50/p99 latency", "unit": "ms", "workload":
            f"rmat{scale}_serving_mix60_30_10", "V": g.num_vertices, "E": g.num_edges,
            "offsets": "int64", "slots": st["slots"], "state_bytes": st["state_bytes"],
            "sssp_direction": {1: "per 32-slot chunk", -1: "per group"}.get(
                args.sssp_chunk_direction, "auto (per 32-slot chunk)"),
            "sssp_pull_edge_ratio": args.sssp_pull_edge_ratio,
            "admission": {"slots": "any free slot", "chunks": "whole 32-slot cohorts",
                          "group": "group cohorts"}[args.serve_admission],
            "groups": args.serve_groups or 1,
            "results": ({"device": f"written to a ring of {args.serve_out_ring} device buffers",
                         "none": "discarded"})[args.serve_out],
            "seconds_per_rate": args.serve_seconds, "rates": rows, "graph_gen_s": gen_s}
    print(json.dumps(line), flush=True)
    if args.json_out:
        Path(args.json_out).write_text(json.dumps(line) + "\n")
    return 0


# ------------------------------------------------------------------ GPU arm
def unreached_word(kind, wk):
    if kind in ("bfs", "khop"):
        return BFS_INF
    return 0x7f800000 if wk == "f32" else -1


def reached_counts(out, kind, wk, chunk=1 << 20):
    """Per-column count of reached vertices of a device output [V][Q]
    (chunked over vertices to bound temporary memory)."""
    import torch
    miss = unreached_word(kind, wk)
    cnt = torch.zeros(out.shape[1], dtype=torch.int64, device=out.device)
    for v0 in range(0, out.shape[0], chunk):
        cnt += (out[v0:v0 + chunk] != miss).sum(0)
    return cnt.cpu().numpy()


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "serve":
        return run_serve(args)
    import torch
    import torch.distributed as dist
    import cgp_b200 as cgp

    wl = workload_spec(args)
    steps = args.steps or default_steps(args.workload)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and world > 1:
        print(f"warning: WORLD_SIZE={world} but --gpus={args.gpus}", file=sys.stderr)
    torch.cuda.set_device(local)
    cgp.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def allreduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return t.item()

    MAX = dist.ReduceOp.MAX if world > 1 else None
    SUM = dist.ReduceOp.SUM if world > 1 else None

    g, gen_s = make_graph(cgp, wl)
    wk = wl["weights"][0] if wl["weights"] else None
    graph = cgp.CsrGraph(g, symmetric=True)
    V = g.num_vertices
    labels = cgp.run("wcc", graph, [0]).values[:, 0]
    comp_size, comp_edges = component_tables(g, labels)
    groups = shard_groups(select_queries(args, wl, g, labels, world), rank, world)
    descs = [[cgp.QueryDescriptor(int(s), k) for s in src] for k, src in groups]
    edges_q = reach_edges(groups, labels, comp_edges)
    expect_reach = [comp_size[labels.astype(np.int64)[np.asarray(s, np.int64)]] for _, s in groups]
    edges_step = float(sum(e.sum() for e in edges_q)) + (g.num_edges if wl["wcc"] else 0)
    nq_step = sum(len(d) for d in descs) + (1 if wl["wcc"] else 0)

    stream = torch.cuda.current_stream(dev)
    tuning = dict(traversal_mode=args.mode, pull_edge_ratio=args.pull_edge_ratio,
                  pull_frontier_ratio=args.pull_frontier_ratio, heavy_degree=args.heavy_degree,
                  sssp_pull_edge_ratio=args.sssp_pull_edge_ratio,
                  sssp_pull_pair_ratio=args.sssp_pull_pair_ratio,
                  bfs_pull_form=args.bfs_pull_form,
                  light_chunks=not args.no_light_chunks, levels_per_sync=args.levels_per_sync,
                  level_loop=args.level_loop or ("device" if args.workload == "c3" else "chunks"))
    base = cgp.RunOptions(stream=stream.cuda_stream, **tuning)
    if args.workload == "c5":
        # 1024-slot groups; depths written at discovery into the output, which
        # doubles as the working values (the bit-plane form would need another
        # 34 GB beside the 137 GB output)
        base = dataclasses.replace(base, mask_words=16, depth_mode="direct")
    if args.workload == "c3":
        base = dataclasses.replace(base, mask_words=16)

    # outputs: one device buffer per group, except that c5's four 1024-slot
    # groups share one (137 GB each): every group's values are written, the
    # next group's run overwrites them
    outs = []
    for k, src in groups:
        if args.workload == "c5" and outs:
            outs.append(outs[0])
        else:
            outs.append(torch.empty((V, len(src)), dtype=torch.int32, device=dev))
    out_w = torch.empty((V, 1), dtype=torch.int32, device=dev) if wl["wcc"] else None
    wcc_d = [cgp.QueryDescriptor(0, "wcc")]

    # autotuner (untimed): mask width, heavy threshold, pull thresholds per batch
    opts = []
    tune_s = time.perf_counter()
    tuned = {}
    for (k, src), d in zip(groups, descs):
        o = base
        if not args.no_autotune and args.workload in ("c1", "c2"):
            key = (k, len(d))
            if key not in tuned:
                tuned[key] = cgp.autotune(graph, d, base, reps=2)
            o = tuned[key]
        opts.append(o)
    tune_s = time.perf_counter() - tune_s

    def step():
        res = []
        for d, o, out in zip(descs, opts, outs):
            res.append(cgp.run_batch(graph, d, o, out=out))
        if wl["wcc"]:
            res.append(cgp.run_batch(graph, wcc_d, base, out=out_w))
        return res

    # warm-up; the first pass checks every column's reach against its component
    for w in range(max(3, args.warmup)):
        if w == 0:
            for gi, (d, o, (k, src)) in enumerate(zip(descs, opts, groups)):
                out = outs[gi]
                cgp.run_batch(graph, d, o, out=out)
                got = reached_counts(out, k, wk)
                assert np.array_equal(got, expect_reach[gi]), (args.workload, k, gi)
            if wl["wcc"]:
                cgp.run_batch(graph, wcc_d, base, out=out_w)
                assert np.array_equal(out_w[:, 0].cpu().numpy().view(np.uint32), labels)
        else:
            step()

    launches = 0
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    per_group_ms = [0.0] * (len(groups) + (1 if wl["wcc"] else 0))
    last = None
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            last = step()
            for i, r in enumerate(last):
                launches += r.kernel_launches
                per_group_ms[i] += r.gpu_time_ms
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_max = allreduce(ms, MAX)
    total_edges = allreduce(edges_step * steps, SUM)
    value = total_edges / (ms_max / 1e3) / 1e9
    qps = allreduce(nq_step * steps, SUM) / (ms_max / 1e3)

    group_lines = []
    for i, r in enumerate(last):
        kind = groups[i][0] if i < len(groups) else "wcc"
        e = float(edges_q[i].sum()) if i < len(groups) else float(g.num_edges)
        gm = per_group_ms[i] / steps
        group_lines.append({"kind": kind, "queries": len(descs[i]) if i < len(groups) else 1,
                            "ms": gm, "gteps": e / max(gm / 1e3, 1e-12) / 1e9,
                            "iterations": r.iterations, "push_levels": r.push_levels,
                            "pull_levels": r.pull_levels, "mask_words": r.mask_words,
                            "ms_per_level": gm / max(1, r.iterations)})

    # ---- profiled step: per-kernel-class CUDA-event times + level counters
    kclass, level_trace = {}, {}
    if not args.no_profile and args.workload in ("c1", "c2", "c3"):
        for i, (d, o, (k, src)) in enumerate(zip(descs, opts, groups)):
            p = cgp.run_batch(graph, d, dataclasses.replace(o, profile_kernels=True,
                                                            profile_iterations=True),
                              out=outs[i])
            qs = len(d) if k == "sssp" else 0
            merge_classes(kclass, level_classes(p.iteration_profiles, k, V, p.mask_words, qs=qs))
            if k == "bfs":
                level_trace[f"{k}{i}"] = [[q.mode, q.frontier_size, q.frontier_edges, q.new_pairs,
                                           q.pull_edges, round(q.kernel_ms, 3)]
                                          for q in p.iteration_profiles]
            else:
                level_trace[f"{k}{i}"] = [[q.sssp_mode, q.frontier_size, q.frontier_edges,
                                           q.sssp_active, q.sssp_pairs, q.improved,
                                           q.sssp_pull_edges, round(q.kernel_ms, 3)]
                                          for q in p.iteration_profiles]
            level_trace[f"kernel_ms_{k}{i}"] = p.kernel_profile
        level_trace["columns"] = {
            "bfs": ["mode", "frontier", "frontier_edges", "new_pairs", "pull_edges", "ms"],
            "sssp": ["mode", "frontier", "frontier_edges", "active_bits", "pairs", "improved",
                     "pull_edges", "ms"]}
    roofline = roofline_line(args, kclass)

    # ---- one-query form: the same kernels with Q = 1, back to back (sampled)
    one_query = None
    if not args.no_one_query and rank == 0:
        o1 = torch.empty((V, 1), dtype=torch.int32, device=dev)
        t_one = 0.0
        sample_txt = []
        per_kind_opts = {}
        for gi, (d, (k, src)) in enumerate(zip(descs, groups)):
            n1 = {"c1": 64, "c2": 16 if k == "bfs" else 8, "c3": 4, "c5": 2}[args.workload]
            n1 = min(n1, len(d))
            if k not in per_kind_opts:
                o = dataclasses.replace(base, mask_words=0, depth_mode="auto")
                per_kind_opts[k] = (o if args.no_autotune or args.workload not in ("c1", "c2")
                                    else cgp.autotune(graph, d[:1], o, reps=2))
            o = per_kind_opts[k]
            cgp.run_batch(graph, d[:1], o, out=o1)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for q in d[:n1]:
                cgp.run_batch(graph, [q], o, out=o1)
            e1.record(stream)
            torch.cuda.synchronize()
            per_q = e0.elapsed_time(e1) / n1
            t_one += per_q * len(d)
            sample_txt.append(f"{n1} of {len(d)} {k.upper()}")
        if wl["wcc"]:
            t_one += per_group_ms[-1] / steps
        edges_rank = float(sum(e.sum() for e in edges_q)) + (g.num_edges if wl["wcc"] else 0)
        one_query = {"gteps": edges_rank / (t_one / 1e3) / 1e9,
                     "ms_per_step": t_one,
                     "sample": "single-query runs (" + ", ".join(sample_txt) +
                               "), scaled to the batch"}

    # ---- e2e: the public API with host buffers (pinned), copies inside
    e2e = None
    e2e_skip = None
    host_bytes = 4 * V * nq_step
    if args.workload == "c5":
        e2e_skip = (f"the step's results ({host_bytes / 1e9:.0f} GB) exceed the host's memory; "
                    f"each group's device output is overwritten by the next")
    elif args.e2e_steps > 0:
        qmaj = args.e2e_layout == "query"
        all_d = [q for d in descs for q in d] + (wcc_d if wl["wcc"] else [])
        nq = len(all_d)
        try:
            host = torch.empty((nq, V) if qmaj else (V, nq), dtype=torch.int32, pin_memory=True)
        except RuntimeError as ex:
            host = None
            e2e_skip = f"pinned host buffer of {host_bytes / 1e9:.1f} GB failed: {ex}"
        if host is not None:
            # one call for every group: the last group's options, with the BFS
            # group's pull thresholds when there is one
            eopts = dataclasses.replace(opts[-1], stream=0)
            for (k, _), o in zip(groups, opts):
                if k == "bfs":
                    eopts = dataclasses.replace(eopts, pull_edge_ratio=o.pull_edge_ratio,
                                                pull_frontier_ratio=o.pull_frontier_ratio)
                    break
            batch = cgp.HybridQueryBatch(all_d)

            def e2e_step():
                return cgp.run_heterogeneous(graph, batch, options=eopts, out=host,
                                             layout="query" if qmaj else "vertex")
            r_e2e = e2e_step()
            barrier()
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                e2e_step()
            t_e2e = time.perf_counter() - t0
            t_e2e = allreduce(t_e2e, MAX)
            e_edges = allreduce(edges_step * args.e2e_steps, SUM)
            # spot check: the host copy equals the device-resident results
            hv = host.numpy()
            col = (lambda j: hv[j]) if qmaj else (lambda j: hv[:, j])
            same = True
            j0 = 0
            for gi, (k, src) in enumerate(groups):
                dev_out = outs[gi]
                if args.workload != "c5":
                    for j in (0, len(src) - 1):
                        same &= bool(np.array_equal(col(j0 + j), dev_out[:, j].cpu().numpy()))
                j0 += len(src)
            e2e = {"value": e_edges / t_e2e / 1e9, "unit": "GTEPS",
                   "h2d_bytes_per_step": 16 * nq, "d2h_bytes_per_step": 4 * V * nq,
                   "steps": args.e2e_steps, "ms_per_step": 1e3 * t_e2e / args.e2e_steps,
                   "groups": r_e2e.groups, "matches_device": same,
                   "output": f"one pinned host buffer, {'query' if qmaj else 'vertex'}-major "
                             f"4-byte values [{'Q][V' if qmaj else 'V][Q'}]"}
            del host

    # ---- serving on the default workload's graph: continuous batching
    serving = None
    if rank == 0 and args.workload == "c2" and args.serve_seconds > 0:
        mix = serve_mix(g, 2048, seed=43,
                        allowed=(labels == labels[groups[0][1][0]]).astype(np.uint8))
        with cgp.Server(graph, slots=args.serve_slots,
                        options=cgp.RunOptions(traversal_mode=args.mode)) as srv:
            poisson_run(srv, mix[:64], 200, 0.3, seed=7)
            serving = poisson_run(srv, mix, 2000.0, args.serve_seconds, seed=8)
            serving["slots"] = srv.stats()["slots"]
            serving["mix"] = "60% BFS / 30% SSSP / 10% k-hop (k in 2..6)"

    # ---- CPU baseline (rank 0, N = 1): the reference CPU traversal, bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sizes = cpu_sample_sizes(args, groups, threads)
        dt, edges, kind, couts = cpu_reference_sample(g, groups, sizes, threads)
        match = True
        for gi, ((k, src), n, co) in enumerate(zip(groups, sizes, couts)):
            out = outs[gi]
            if args.workload == "c5":  # groups share one output: re-run this one
                cgp.run_batch(graph, descs[gi], opts[gi], out=out)
            got = out[:, :n].cpu().numpy().T.copy()
            ref = co.view(np.uint32) if k == "bfs" else as_u32_words(co, wk)
            match &= bool(np.array_equal(got.view(np.uint32), ref))
        cpu = {"value": edges / dt / 1e9, "unit": "GTEPS", "cores": threads, "kind": kind,
               "sample": (" + ".join(f"{n} {k.upper()}" for (k, _), n in zip(groups, sizes)) +
                          f" queries of the workload, one query per host thread ({dt:.1f} s)"),
               "matches_gpu": match}

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": "aggregate GTEPS", "value": value, "unit": "GTEPS", "n_gpus": world,
            "steps": steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms_max / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": wk or "i32", "data": "synthetic",
            "config": workload_config(args, wl, g, world),
            "engine": {"traversal_mode": args.mode, "level_loop": base.level_loop,
                       "options": [{"kind": k, "mask_words": o.mask_words,
                                    "heavy_degree": o.heavy_degree,
                                    "pull_edge_ratio": o.pull_edge_ratio,
                                    "sssp_pull_edge_ratio": o.sssp_pull_edge_ratio,
                                    "sssp_pull_pair_ratio": o.sssp_pull_pair_ratio,
                                    "dense_unroll": o.dense_unroll, "depth_mode": o.depth_mode}
                                   for (k, _), o in zip(groups, opts)],
                       "autotuned": not args.no_autotune and args.workload in ("c1", "c2"),
                       "tuning_s": tune_s,
                       "l2": (f"inputs larger than L2: CSR "
                              f"{4 * (V + 1 + 2 * g.num_edges) / 2**20:.0f} MiB + outputs "
                              f"{4 * V * nq_step / 2**30:.1f} GiB per step, re-initialised "
                              f"every step (no flush)")},
            "queries_per_s": qps,
            "groups": group_lines,
            "one_query": one_query,
            "batched_vs_one_query": (value / world / one_query["gteps"]) if one_query else None,
            "clocks": clocks, "e2e": e2e, "e2e_unavailable": e2e_skip,
            "gpu_launches": launches, "roofline": roofline,
            "serving": serving, "level_trace": level_trace or None,
            "cpu_baseline": cpu, "graph_gen_s": gen_s,
        }
        s = json.dumps(line)
        print(s, flush=True)
        if args.json_out:
            Path(args.json_out).write_text(s + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
