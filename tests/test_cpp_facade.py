"""The C++ host API (include/cgp_b200.hpp) compiles against the C ABI, and
its known-answer validator passes on the device."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "validate_facade.cpp"
BIN = ROOT / "_build" / "validate_facade"


def _compile():
    BIN.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", str(SRC),
           f"-L{ROOT / 'cgp_b200'}", "-lcgp_b200", f"-Wl,-rpath,{ROOT / 'cgp_b200'}",
           "-o", str(BIN)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return BIN


def test_facade_compiles_and_links():
    assert _compile().exists()


@pytest.mark.gpu
def test_facade_validator_passes():
    b = _compile()
    r = subprocess.run([str(b)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASS" in r.stdout
