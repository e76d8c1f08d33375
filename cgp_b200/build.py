"""Builds the in-tree native library ``cgp_b200/libcgp_b200.so``.

CUDA sources are compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); host C++ sources with g++ and OpenMP.  The
objects go to ``_build/`` at the repository root and the shared library is
written next to this file, so it travels with the working tree.
"""
from __future__ import annotations

import concurrent.futures
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libcgp_b200.so"
STAMP = PKG / "libcgp_b200.so.sha256"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp",
            "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-fopenmp", f"-I{INCLUDE}", f"-I{CSRC}",
             f"-I{CUDA_HOME / 'include'}"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(obj, [src, *_headers()]):
        return obj
    if src.suffix == ".cu":
        cmd = [NVCC, *CU_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def _digest() -> str:
    h = hashlib.sha256()
    for f in [*_sources(), *_headers()]:
        h.update(f.name.encode())
        h.update(f.read_bytes())
    h.update(" ".join(CU_FLAGS + CXX_FLAGS).encode())
    return h.hexdigest()


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compiles every source that changed and links the shared library.
    A library whose recorded source digest matches is left as it is."""
    digest = _digest()
    if LIB.exists() and STAMP.exists() and STAMP.read_text().strip() == digest:
        return LIB
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lgomp",
               "-Xlinker", "-z,defs", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"linking failed:\n{r.stdout}\n{r.stderr}")
        shutil.move(str(tmp), str(LIB))
    STAMP.write_text(digest + "\n")
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Builds the CPU checker libraries under oracle/ (test infrastructure)."""
    cmd = ["make", "-s", "-C", str(ROOT / "oracle")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose:
        print(r.stdout, r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
