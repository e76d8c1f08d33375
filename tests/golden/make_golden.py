"""Generates tests/golden/golden.json from the reference.

Run where the reference tree is available: $CGP_REFERENCE, else a
directory named `reference` beside the repository:

    python tests/golden/make_golden.py

It records
  * the reference's Matrix Market fixtures (puercgp/examples/matrices/*.mm),
    the CSR the reference loader builds from them, and the reference's own
    cpu_bfs / cpu_sssp results for the validators' default sources "0,1,2,3"
    (validate_bfs.cu:62, validate_sssp.cu:62), computed by oracle/_ref;
  * the known-answer toy tests of the reference examples, with the expected
    vectors as the reference test files state them (file:line in "source");
  * reference cpu_bfs / cpu_sssp / cpu_wcc outputs on two small seeded graphs
    (R-MAT scale 8 and a 12x12 grid) generated by this library, so the CPU
    restatement is pinned on more than toy inputs.
The JSON is committed; the tests read only the JSON.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
import cgp_b200 as cgp  # noqa: E402

REF = Path(os.environ.get("CGP_REFERENCE", str(ROOT.parent / "reference")))
INF_I = 2**31 - 1


def csr_json(row, col, w=None):
    d = {"row_offsets": [int(x) for x in row], "col_indices": [int(x) for x in col]}
    if w is not None:
        d["weights"] = [float(x) for x in w]
    return d


def main():
    if not oracle.has_ref():
        raise SystemExit("oracle/_ref/libcgpref.so missing: run `make -C oracle` with the reference present")
    out = {"generator": "tests/golden/make_golden.py", "inf_int32": INF_I, "cases": []}

    # --- reference Matrix Market fixtures through the reference loader + oracle
    for name, kind in (("unweighted", "bfs"), ("weighted", "sssp")):
        p = REF / "puercgp/examples/matrices" / f"{name}.mm"
        row, col, w = oracle.ref_load_matrix_market(str(p))
        g = cgp.HostCsr(row, col, w)
        sources = [0, 1, 2, 3]
        if kind == "bfs":
            expect = [oracle.ref_bfs(g, s).tolist() for s in sources]
        else:
            expect = [[float(x) for x in oracle.ref_sssp(g, s)] for s in sources]
        out["cases"].append({
            "name": f"{name}_mm", "kind": kind,
            "source": f"puercgp/examples/matrices/{name}.mm via load_matrix_market "
                      f"(mtx_loader.hxx:99-187) and cpu_{kind} (mtx_loader.hxx)",
            "mtx": p.read_text(), "graph": csr_json(row, col, w),
            "sources": sources, "expect": expect})

    toy_row, toy_col = [0, 2, 3, 3, 3], [1, 2, 3]
    out["cases"] += [
        {"name": "hybrid_toy", "kind": "mixed",
         "source": "puercgp/examples/validate_hybrid.cu:41-106",
         "graph": csr_json(toy_row, toy_col, [2.0, 5.0, 1.0]), "directed": True,
         "queries": [["bfs", 0], ["sssp", 0], ["wcc", 0]],
         "expect": [[0, 1, 1, 2], [0.0, 2.0, 5.0, 3.0], [0, 0, 0, 0]]},
        {"name": "replenish_toy", "kind": "mixed",
         "source": "puercgp/examples/validate_replenish.cu:33-112",
         "graph": csr_json(toy_row, toy_col, [2.0, 5.0, 3.0]), "directed": True,
         "queries": [["bfs", 0], ["sssp", 0], ["bfs", 1], ["sssp", 1]],
         "expect": [[0, 1, 1, 2], [0.0, 2.0, 5.0, 5.0], [INF_I, 0, INF_I, 1],
                    ["inf", 0.0, "inf", 3.0]]},
        {"name": "wcc_toy", "kind": "mixed",
         "source": "puercgp/examples/validate_wcc.cu:33-72",
         "graph": csr_json(toy_row, toy_col), "directed": True,
         "queries": [["wcc", 0]], "expect": [[0, 0, 0, 0]]},
        {"name": "push_one_level", "kind": "one_level",
         "source": "puercgp/examples/smoke_hybrid_push.cu:45-173",
         "graph": csr_json(toy_row, toy_col, [2.0, 5.0, 1.0]), "directed": True,
         "queries": [["bfs", 0], ["sssp", 0]],
         "expect": [[0, 1, 1, INF_I], [0.0, 2.0, 5.0, "inf"]],
         "expect_next_frontier": {"vertices": [1, 2], "mask": 3}, "expect_active_union": 3},
        {"name": "hybrid_init", "kind": "init",
         "source": "puercgp/examples/smoke_hybrid_init.cu:41-135",
         "graph": csr_json([0, 1, 2, 3, 3], [1, 2, 3]), "directed": True,
         "queries": [["bfs", 0], ["sssp", 1]],
         "expect_frontier": {"0": 1, "1": 2},
         "expect": [[0, INF_I, INF_I, INF_I], ["inf", 0.0, "inf", "inf"]]},
        {"name": "convergence_levels", "kind": "levels",
         "source": "puercgp/examples/smoke_replenish.cu:49-116 (BFS/SSSP slots)",
         "graph": csr_json(toy_row, toy_col, [2.0, 5.0, 1.0]), "directed": True,
         "queries": [["bfs", 0], ["sssp", 0]],
         "expect_iterations": 3, "expect_masks": [3, 3, 0]},
    ]

    # --- reference outputs on seeded graphs from this library's generators
    rm = cgp.gen_rmat(8, 8, seed=7).with_weights("f32", 1.0, 10.0, seed=3)
    grid = cgp.gen_grid(12, 12, 0.1, 0.02, seed=5).with_weights("f32", 1.0, 100.0, seed=6)
    for name, g in (("rmat8", rm), ("grid12", grid)):
        V = g.num_vertices
        deg = g.degrees()
        srcs = [int(v) for v in np.flatnonzero(deg > 0)[:: max(1, V // 6)][:6]]
        out["cases"].append({
            "name": f"{name}_ref", "kind": "ref_outputs",
            "source": "reference cpu_bfs / cpu_sssp / cpu_wcc (mtx_loader.hxx:269-356) run here",
            "graph": csr_json(g.row_offsets, g.col_indices, g.weights), "sources": srcs,
            "bfs": [oracle.ref_bfs(g, s).tolist() for s in srcs],
            "sssp": [[float(x) for x in oracle.ref_sssp(g, s)] for s in srcs],
            "wcc": [float(x) for x in oracle.ref_wcc(g)]})

    dst = Path(__file__).with_name("golden.json")
    dst.write_text(json.dumps(out, indent=1, allow_nan=True))
    print(f"wrote {dst} ({dst.stat().st_size} bytes, {len(out['cases'])} cases)")


if __name__ == "__main__":
    main()
