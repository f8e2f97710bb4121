"""Regenerates tests/golden/golden.npz from the REFERENCE ITSELF.

Run in a checkout where the reference tree is present and oracle/_ref/ref_harness_omp has been
built (`make -C oracle`).  Every graph below is passed to the compiled reference
(oracle/ref_harness.cpp over the unmodified ParButterfly headers) and its dense results are
stored.  tests/test_oracle_golden.py pins the C restatement (oracle/pb_oracle.c) to these
vectors; the GPU tests compare against the restatement.

Modes recorded: the reference paths that give correct results.  Ranked HASH/HIST per-vertex
credits use the wrong filter (butterfly_count.h:364-367), SERIAL+SIDE+VERT writes unstrided
results (:1371-1372), TOTAL has no branch for the A* types (butterfly_count_total.h:970-974),
and wing peeling is only correct with PBATCHS/PBATCHWA.
  counts : BATCHS with every rank type, per VERT / EDGE / TOTAL
  tip    : PBATCHS peeling of ADEG/BATCHS per-vertex counts
  wing   : PBATCHS peeling of ADEG/BATCHS per-edge counts
  extra  : SERIAL (ranked), BATCHWA, SORT counts for cross-checks
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from parbutterfly_b200.graph import BipartiteGraph  # noqa: E402

RANKS = ["SIDE", "COCORE", "ACOCORE", "DEG", "ADEG"]


def kab(a, b):
    v = np.repeat(np.arange(a), b)
    u = np.tile(np.arange(b), a)
    return BipartiteGraph.from_edges(a, b, v, u)


def star(k):
    return BipartiteGraph.from_edges(1, k, np.zeros(k, dtype=np.int64), np.arange(k))


def disjoint(g1, g2):
    v1, u1 = g1.edge_list()
    v2, u2 = g2.edge_list()
    return BipartiteGraph.from_edges(g1.nv + g2.nv, g1.nu + g2.nu, np.concatenate([v1, v2 + g1.nv]),
                                     np.concatenate([u1, u2 + g1.nu]))


def graphs():
    gs = {
        "k34": kab(3, 4),
        "k55": kab(5, 5),
        "star12": star(12),
        "single_edge": BipartiteGraph.from_edges(2, 3, [1], [2]),
        "isolated": BipartiteGraph.from_edges(40, 30, [0, 0, 5, 5, 7, 39], [0, 29, 0, 29, 29, 0]),
        "kab_union": disjoint(kab(4, 6), kab(3, 3)),
        "uniform_50x40": BipartiteGraph.uniform(50, 40, 300, 11),
        "uniform_300x200": BipartiteGraph.uniform(300, 200, 3000, 12),
        "zipf_200x300": BipartiteGraph.zipf(200, 300, 2500, 1.5, 13),
        "rmat_512x256": BipartiteGraph.rmat(9, 8, 6000, 0.55, 0.15, 0.15, 0.15, 14),
        "dense_60x50": BipartiteGraph.uniform(60, 50, 1800, 15),
        "skew_u": BipartiteGraph.powerlaw_u(300, 600, 6000, 2.0, 300, 16),
    }
    return gs


def main():
    assert oracle.have_reference(), "build oracle/_ref first (make -C oracle)"
    out = {}
    for name, g in graphs().items():
        out[f"{name}/offsetsV"] = g.offsetsV
        out[f"{name}/edgesV"] = g.edgesV
        out[f"{name}/offsetsU"] = g.offsetsU
        out[f"{name}/edgesU"] = g.edgesU
        out[f"{name}/dims"] = np.array([g.nv, g.nu, g.m], dtype=np.int64)
        for per in ["VERT", "EDGE", "TOTAL"]:
            for rank in RANKS:
                r = oracle.run_reference(g, per, "BATCHS", rank, threads=2)
                out[f"{name}/{per}/BATCHS/{rank}"] = r["count"]
                out[f"{name}/use_v"] = np.array([int(r["use_v"]), r["w_side"]], dtype=np.int64)
            for ct, rank in [("SERIAL", "ADEG"), ("BATCHWA", "DEG"), ("SORT", "ACOCORE")]:
                r = oracle.run_reference(g, per, ct, rank, threads=2)
                out[f"{name}/{per}/{ct}/{rank}"] = r["count"]
        r = oracle.run_reference(g, "VERT", "BATCHS", "ADEG", "BATCHS", threads=2)
        out[f"{name}/tip"] = r["peel"]
        r = oracle.run_reference(g, "EDGE", "BATCHS", "ADEG", "BATCHS", threads=2)
        out[f"{name}/wing"] = r["peel"]
        print(name, g.nv, g.nu, g.m, "total", int(out[f"{name}/TOTAL/BATCHS/ADEG"][0]))
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz"), **out)


if __name__ == "__main__":
    main()
