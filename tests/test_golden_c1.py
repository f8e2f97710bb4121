"""The small plain-method workload (uniform 4096 x 4096, m = 131072, seed 1; -countType BATCHS
-rankType ADEG -per VERT and -per TOTAL) pinned to the reference's own results
(tests/golden/golden_c1.npz, written by tests/golden/make_golden_c1.py from the compiled
reference).  CPU: the generator reproduces the reference's input, and the C restatement
matches.  GPU: the CUDA path matches, through every count type."""
import hashlib
import os

import numpy as np
import pytest

import oracle
from parbutterfly_b200.graph import workload

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_c1.npz")


@pytest.fixture(scope="module")
def c1():
    return workload("c1"), np.load(FIXTURE)


def _digest(g):
    h = hashlib.sha256()
    h.update(np.array([g.nv, g.nu, g.m], dtype="<i8").tobytes())
    for a in (g.offsetsV, g.edgesV, g.offsetsU, g.edgesU):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


def test_generator_reproduces_the_reference_input(c1):
    g, z = c1
    assert _digest(g) == str(z["graph_sha"])


def test_oracle_matches_reference(c1):
    g, z = c1
    use_v, w, _, _ = oracle.cmp_wedge_counts(g)
    assert [int(use_v), w] == [int(x) for x in z["use_v_wside"]]
    np.testing.assert_array_equal(oracle.count(g, "VERT", "ADEG")[0], z["vert_count"])
    assert oracle.count(g, "TOTAL", "ADEG")[0] == int(z["total"]) == int(z["vert_total"])


@pytest.mark.gpu
def test_gpu_matches_reference(ctx, c1):
    from parbutterfly_b200 import butterflies as pb
    g, z = c1
    dg = ctx.upload(g)
    try:
        use_v, w = pb.cmp_wedge_counts(dg)
        assert [int(use_v), w] == [int(x) for x in z["use_v_wside"]]
        for ct in ["BATCHS", "SERIAL", "BATCHWA", "HASH", "SORT", "HIST"]:
            np.testing.assert_array_equal(pb.count(dg, ct, "ADEG"), z["vert_count"], err_msg=ct)
            assert pb.count_total(dg, ct, "ADEG") == int(z["total"]), ct
    finally:
        dg.close()
