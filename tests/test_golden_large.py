"""Parity at the benchmark's sizes against vectors produced by the reference itself
(tests/golden/make_golden_large.py ran the compiled reference on these graphs).

  rmat18  : the benchmark workload's generator and flags (-rankType ACOCORE -per EDGE
            -countType HASH, wing peel) at 2^18 edges: per-edge counts and wing numbers, in full.
  rmat16  : R-MAT at 2^20 edges, ADEG per-vertex counts and tip numbers (SHA-256 digests).
  plaw10m : the skewed power-law-degree workload at 1e7 edges: per-vertex counts (largest above
            2^32) and tip numbers (digests).
  c2count : the full benchmark graph (2^24 edges): per-edge counts (digest) and the total.
  c3tip   : the skewed power-law-degree workload at full size (1e8 edges): per-vertex counts and
            tip numbers (digests) from the oracle (64-bit buckets; the counts exceed 2^32, where
            the reference's 32-bit buckets are not exact), pinned to the reference on plaw10m.
  c2wing  : the full benchmark graph's wing numbers (digest), from the oracle's bucket-queue
            wing peel (oracle/pb_oracle_fast.c, pinned to the reference on every smaller fixture)
            run on per-edge counts equal to the reference's; the reference's own wing peel of
            this graph does not finish within hours.

The CPU tests check that the generators still produce the graphs the reference saw; the GPU
tests compare the CUDA path with the reference's results bit for bit.
"""
import hashlib
import os

import numpy as np
import pytest

from parbutterfly_b200.graph import BipartiteGraph

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_large.npz")
MODEL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "parbutterfly_b200", "models",
                     "sched_b200.bin")

GRAPHS = {
    "rmat18": lambda: BipartiteGraph.rmat(14, 12, 1 << 18, 0.55, 0.15, 0.15, 0.15, 2),
    "rmat16": lambda: BipartiteGraph.rmat(16, 14, 1 << 20, 0.55, 0.15, 0.15, 0.15, 2),
    "plaw10m": lambda: BipartiteGraph.powerlaw_u(100_000, 1_000_000, 10_000_000, 2.0, 100_000, 3),
    "c2count": lambda: BipartiteGraph.rmat(20, 18, 1 << 24, 0.55, 0.15, 0.15, 0.15, 2),
}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i8").tobytes()).hexdigest()


def graph_digest(g) -> str:
    h = hashlib.sha256()
    h.update(np.array([g.nv, g.nu, g.m], dtype="<i8").tobytes())
    for a in (g.offsetsV, g.edgesV, g.offsetsU, g.edgesU):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def large():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def _rec(large, name):
    return {k[len(name) + 1:]: v for k, v in large.items() if k.startswith(name + "/")}


@pytest.mark.parametrize("name", ["rmat18", "rmat16", "plaw10m"])
def test_generators_reproduce_reference_inputs(large, name):
    g = GRAPHS[name]()
    assert graph_digest(g) == str(_rec(large, name)["graph_sha"])


def test_full_vectors_match_their_digests(large):
    r = _rec(large, "rmat18")
    assert digest(r["count"].astype(np.int64)) == str(r["count_sha"])
    assert digest(r["peel"].astype(np.int64)) == str(r["peel_sha"])
    assert int(r["count"].astype(np.int64).sum()) // 4 == int(r["use_v_wside_total"][2])


def _check(res, r, key, name):
    idx = r["sample_idx"]
    np.testing.assert_array_equal(res[idx], r[f"{key}_sample"], err_msg=f"{name}: sampled {key} entries differ")
    assert digest(res) == str(r[f"{key}_sha"]), f"{name}: {key} digest differs from the reference's"


@pytest.mark.gpu
def test_rmat18_benchmark_flags_count_and_wing(ctx, large):
    from parbutterfly_b200 import butterflies as pb
    r = _rec(large, "rmat18")
    g = GRAPHS["rmat18"]()
    dg = ctx.upload(g)
    try:
        use_v, w = pb.cmp_wedge_counts(dg)
        assert [int(use_v), w] == [int(x) for x in r["use_v_wside_total"][:2]]
        e = pb.count_e(dg, "HASH", "ACOCORE")
        np.testing.assert_array_equal(e, r["count"].astype(np.int64))
        wing = pb.peel_e(dg, e)
        np.testing.assert_array_equal(wing, r["peel"].astype(np.int64))
        # Learned scheduling (the shipped cost models) changes how the work runs, never the result.
        model = pb.SchedModel(ctx)
        model.load(MODEL)
        model.attach()
        try:
            e2 = pb.count_e(dg, "HASH", "ACOCORE", sched="learned")
            np.testing.assert_array_equal(e2, e)
            wing2 = pb.peel_e(dg, e, sched="learned")
            np.testing.assert_array_equal(wing2, wing)
        finally:
            pb.detach_sched_model(ctx)
            model.close()
    finally:
        dg.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["rmat16", "plaw10m"])
def test_tip_numbers_match_reference(ctx, large, name):
    from parbutterfly_b200 import butterflies as pb
    r = _rec(large, name)
    g = GRAPHS[name]()
    dg = ctx.upload(g)
    try:
        c = pb.count(dg, "BATCHS", "ADEG")
        _check(c, r, "count", name)
        assert int(c.sum()) // 2 == int(r["use_v_wside_total"][2])
        tip = pb.peel(dg, c)
        _check(tip, r, "peel", name)
    finally:
        dg.close()


@pytest.mark.gpu
def test_power_law_workload_tip_numbers(ctx, large):
    from parbutterfly_b200 import butterflies as pb
    r = _rec(large, "c3tip")
    g = BipartiteGraph.powerlaw_u(100_000, 1_000_000, 100_000_000, 2.0, 100_000, 3)
    assert graph_digest(g) == str(r["graph_sha"])
    dg = ctx.upload(g)
    del g
    try:
        c = pb.count(dg, "BATCHS", "ADEG")
        _check(c, r, "count", "c3tip")
        total, rounds, w_rank = (int(x) for x in r["total_rounds_wrank"])
        assert int(c.sum()) // 2 == total
        tip = pb.peel(dg, c, peel_parts=1200)  # the two-phase schedule; same numbers as one round at a time
        assert ctx.stats()["peel_rounds"] == rounds
        _check(tip, r, "peel", "c3tip")
    finally:
        dg.close()


def test_benchmark_wing_record_is_consistent(large):
    r = _rec(large, "c2wing")
    assert str(r["graph_sha"]) == str(_rec(large, "c2count")["graph_sha"])
    rounds, wmax = (int(x) for x in r["rounds_max"])
    assert rounds == 131618 and int(r["peel_sample"].max()) <= wmax


@pytest.mark.gpu
def test_benchmark_graph_wing_numbers(ctx, large):
    from parbutterfly_b200 import butterflies as pb
    r = _rec(large, "c2wing")
    g = GRAPHS["c2count"]()
    dg = ctx.upload(g)
    try:
        e = pb.count_e(dg, "HASH", "ACOCORE")
        wing = pb.peel_e(dg, e)
        assert ctx.stats()["peel_rounds"] == int(r["rounds_max"][0])
        _check(wing, r, "peel", "c2wing")
    finally:
        dg.close()


@pytest.mark.gpu
def test_benchmark_graph_edge_counts_match_reference(ctx, large):
    from parbutterfly_b200 import butterflies as pb
    r = _rec(large, "c2count")
    g = GRAPHS["c2count"]()
    assert graph_digest(g) == str(r["graph_sha"])
    dg = ctx.upload(g)
    try:
        e = pb.count_e(dg, "HASH", "ACOCORE")
        _check(e, r, "count", "c2count")
        assert int(e.sum()) // 4 == int(r["use_v_wside_total"][2]) == 23_556_852_288
        assert pb.count_total(dg, "BATCHS", "ADEG") == 23_556_852_288
    finally:
        dg.close()
