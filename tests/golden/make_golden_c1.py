"""Regenerates tests/golden/golden_c1.npz from the REFERENCE ITSELF: the small plain-method
workload (uniform 4096 x 4096, m = 131072 distinct edges, seed 1), counted with
-countType BATCHS -rankType ADEG -per VERT and -per TOTAL, no peeling.

Run in a checkout where the reference tree is present and oracle/_ref/ref_harness_omp has been
built (`make -C oracle`).  Stored: the graph's CSR digest, the reference's (use_v, W_side),
per-vertex counts in full and the total of both runs.

    python tests/golden/make_golden_c1.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from parbutterfly_b200.graph import workload  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_c1.npz")


def graph_digest(g) -> str:
    h = hashlib.sha256()
    h.update(np.array([g.nv, g.nu, g.m], dtype="<i8").tobytes())
    for a in (g.offsetsV, g.edgesV, g.offsetsU, g.edgesU):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


def main():
    g = workload("c1")
    vert = oracle.run_reference(g, "VERT", "BATCHS", "ADEG", "NONE", threads=4)
    total = oracle.run_reference(g, "TOTAL", "BATCHS", "ADEG", "NONE", threads=4)
    np.savez_compressed(
        OUT,
        graph_sha=np.array(graph_digest(g)),
        use_v_wside=np.array([int(vert["use_v"]), vert["w_side"]], dtype=np.int64),
        vert_count=vert["count"].astype(np.int64),
        vert_total=np.array(vert["total"], dtype=np.int64),
        total=np.array(total["total"], dtype=np.int64),
        provenance=np.array("oracle/_ref/ref_harness_omp (the reference's headers, BATCHS, ADEG)"),
    )
    print(f"wrote {OUT}: use_v={vert['use_v']} w_side={vert['w_side']} total={total['total']}")


if __name__ == "__main__":
    main()
