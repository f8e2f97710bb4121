"""The two-phase peel schedule (a coarse pass cutting the items into partitions by ranges of their
final numbers, then every partition's exact rounds as an independent instance of one launch)
gives the same tip and wing numbers as one instance running every round over the whole GPU,
and as the reference: its golden vectors, the 2^18-edge R-MAT with the benchmark's flags and
the 2^20-edge / 1e7-edge tip fixtures.  The exact rounds summed over the partitions equal the
rounds of the one-instance peel."""
import hashlib
import os

import numpy as np
import pytest

import oracle
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu

GOLDEN_LARGE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_large.npz")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i8").tobytes()).hexdigest()


@pytest.mark.parametrize("parts", [1, 7, 300, 5000])
def test_two_phase_golden_tip_and_wing(ctx, golden, parts):
    for name, (g, rec) in golden.items():
        dg = ctx.upload(g)
        c = pb.count(dg, "BATCHS", "ADEG")
        e = pb.count_e(dg, "BATCHS", "ADEG")
        t1 = pb.peel(dg, c)
        r1 = ctx.stats()["peel_rounds"]
        w1 = pb.peel_e(dg, e)
        rw1 = ctx.stats()["peel_rounds"]
        t2 = pb.peel(dg, c, peel_parts=parts)
        r2 = ctx.stats()["peel_rounds"]
        w2 = pb.peel_e(dg, e, peel_parts=parts)
        st = ctx.stats()
        dg.close()
        np.testing.assert_array_equal(t2, rec["tip"], err_msg=name)
        np.testing.assert_array_equal(w2, rec["wing"], err_msg=name)
        np.testing.assert_array_equal(t1, t2, err_msg=name)
        np.testing.assert_array_equal(w1, w2, err_msg=name)
        assert (r1, rw1) == (r2, st["peel_rounds"]), name
        assert st["peel_parts"] >= 1


@pytest.mark.parametrize("parts", [64, 600])
def test_two_phase_benchmark_flags_sample(ctx, parts):
    with np.load(GOLDEN_LARGE) as z:
        cnt = z["rmat18/count"].astype(np.int64)
        wing_ref = z["rmat18/peel"].astype(np.int64)
    g = BipartiteGraph.rmat(14, 12, 1 << 18, 0.55, 0.15, 0.15, 0.15, 2)
    dg = ctx.upload(g)
    try:
        e = pb.count_e(dg, "HASH", "ACOCORE")
        np.testing.assert_array_equal(e, cnt)
        w = pb.peel_e(dg, e, peel_parts=parts)
        np.testing.assert_array_equal(w, wing_ref)
        assert ctx.stats()["peel_rounds"] == oracle.peel_edge_fast(g, cnt)[1]
    finally:
        dg.close()


@pytest.mark.parametrize("name", ["rmat16", "plaw10m"])
def test_two_phase_tip_fixtures(ctx, name):
    with np.load(GOLDEN_LARGE) as z:
        sha = str(z[f"{name}/peel_sha"])
    g = (BipartiteGraph.rmat(16, 14, 1 << 20, 0.55, 0.15, 0.15, 0.15, 2) if name == "rmat16" else
         BipartiteGraph.powerlaw_u(100_000, 1_000_000, 10_000_000, 2.0, 100_000, 3))
    dg = ctx.upload(g)
    try:
        c = pb.count(dg, "BATCHS", "ADEG")
        tip = pb.peel(dg, c, peel_parts=600)
        assert _sha(tip) == sha
    finally:
        dg.close()


def test_two_phase_random_graphs_vs_oracle(ctx):
    for seed in range(4):
        g = BipartiteGraph.rmat(11, 10, 20000, 0.55, 0.15, 0.15, 0.15, 900 + seed)
        dg = ctx.upload(g)
        e = pb.count_e(dg, "HASH", "ADEG")
        c = pb.count(dg, "BATCHS", "ADEG")
        w = pb.peel_e(dg, e, peel_parts=100 + 50 * seed)
        t = pb.peel(dg, c, peel_parts=100 + 50 * seed)
        dg.close()
        np.testing.assert_array_equal(w, oracle.peel_edge_fast(g, e)[0])
        np.testing.assert_array_equal(t, oracle.peel_vert(g, c)[0])


@pytest.mark.parametrize("parts", [16, 500])
def test_two_phase_batch_of_graphs(ctx, parts):
    graphs = [BipartiteGraph.batch_member(k) for k in range(24)]
    dgs = [ctx.upload(g) for g in graphs]
    try:
        counts = pb.count_batch(dgs, "BATCHS", "ADEG")
        plain = pb.peel_batch(dgs, counts)
        two = pb.peel_batch(dgs, counts, peel_parts=parts)
        assert ctx.stats()["peel_parts"] >= 1
        for g, c, a, b in zip(graphs, counts, plain, two):
            np.testing.assert_array_equal(a, b)
            np.testing.assert_array_equal(b, oracle.peel_vert(g, c)[0])
    finally:
        for dg in dgs:
            dg.close()
