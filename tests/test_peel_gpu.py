"""Parity of the CUDA tip / wing peeling with the golden vectors (the reference's PBATCHS
peeling) and with the oracle; integer results, bit-exact."""
import numpy as np
import pytest

import oracle
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu

PEEL_TYPES = ["SORT", "HASH", "HIST", "BATCHS", "BATCHWA"]


def test_golden_tip_and_wing(ctx, golden):
    for name, (g, rec) in golden.items():
        dg = ctx.upload(g)
        c = pb.count(dg, "BATCHS", "ADEG")
        np.testing.assert_array_equal(pb.peel(dg, c), rec["tip"], err_msg=name)
        e = pb.count_e(dg, "BATCHS", "ADEG")
        np.testing.assert_array_equal(pb.peel_e(dg, e), rec["wing"], err_msg=name)
        dg.close()


@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("kind", ["uniform", "zipf", "rmat", "powerlaw"])
def test_tip_random_vs_oracle(ctx, kind, seed):
    if kind == "uniform":
        g = BipartiteGraph.uniform(2000, 1500, 20000, 500 + seed)
    elif kind == "zipf":
        g = BipartiteGraph.zipf(1500, 2500, 20000, 1.4, 600 + seed)
    elif kind == "rmat":
        g = BipartiteGraph.rmat(11, 11, 30000, 0.55, 0.15, 0.15, 0.15, 700 + seed)
    else:
        g = BipartiteGraph.powerlaw_u(1000, 4000, 40000, 2.0, 1000, 800 + seed)
    dg = ctx.upload(g)
    for uv in (False, True):
        c, _ = oracle.count(g, "VERT", "ADEG", use_v=uv)
        tip, rounds = oracle.peel_vert(g, c, use_v=uv)
        got = pb.peel(dg, c, PEEL_TYPES[seed % 5], use_v=uv)
        np.testing.assert_array_equal(got, tip)
        assert ctx.stats()["peel_rounds"] == rounds


@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("kind", ["uniform", "zipf", "rmat"])
def test_wing_random_vs_oracle(ctx, kind, seed):
    if kind == "uniform":
        g = BipartiteGraph.uniform(600, 500, 6000, 900 + seed)
    elif kind == "zipf":
        g = BipartiteGraph.zipf(500, 700, 6000, 1.3, 1000 + seed)
    else:
        g = BipartiteGraph.rmat(10, 9, 8000, 0.55, 0.15, 0.15, 0.15, 1100 + seed)
    dg = ctx.upload(g)
    for uv in (False, True):
        e, _ = oracle.count(g, "EDGE", "ADEG", use_v=uv)
        wing, rounds = oracle.peel_edge(g, e, use_v=uv)
        got = pb.peel_e(dg, e, PEEL_TYPES[seed % 5], use_v=uv)
        np.testing.assert_array_equal(got, wing)
        assert ctx.stats()["peel_rounds"] == rounds


def test_wing_hub_edges_use_cta_path(ctx):
    """Hubs whose neighbour lists exceed a warp table (and a CTA table) go through the
    CTA-level aggregator and the global-memory markers."""
    nv, nu = 20000, 60
    rng = np.random.default_rng(5)
    v = np.concatenate([np.zeros(18000, dtype=np.int64), rng.integers(0, nv, 4000)])
    u = np.concatenate([rng.integers(0, nu, 18000), rng.integers(0, nu, 4000)])
    v = np.concatenate([v, np.arange(9000)])
    u = np.concatenate([u, np.full(9000, 7)])
    g = BipartiteGraph.from_edges(nv, nu, v, u)
    dg = ctx.upload(g)
    for uv in (False, True):
        e, _ = oracle.count(g, "EDGE", "DEG", use_v=uv)
        np.testing.assert_array_equal(pb.count_e(dg, "HASH", "DEG", use_v=uv), e)
        np.testing.assert_array_equal(pb.peel_e(dg, e, use_v=uv), oracle.peel_edge(g, e, use_v=uv)[0])
        c, _ = oracle.count(g, "VERT", "DEG", use_v=uv)
        np.testing.assert_array_equal(pb.peel(dg, c, use_v=uv), oracle.peel_vert(g, c, use_v=uv)[0])


@pytest.mark.parametrize("a,b", [(3, 4), (8, 5)])
def test_complete_bipartite_peel(ctx, a, b):
    g = BipartiteGraph.from_edges(a, b, np.repeat(np.arange(a), b), np.tile(np.arange(b), a))
    dg = ctx.upload(g)
    c = pb.count(dg)
    np.testing.assert_array_equal(pb.peel(dg, c), c)
    e = pb.count_e(dg)
    np.testing.assert_array_equal(pb.peel_e(dg, e), e)


def test_peel_inputs_on_device(ctx):
    import torch
    g = BipartiteGraph.zipf(900, 700, 7000, 1.3, 21)
    dg = ctx.upload(g)
    use_v, _ = pb.cmp_wedge_counts(dg)
    e = pb.count_e(dg, "HASH", "ACOCORE")
    e_dev = torch.from_numpy(e).cuda()
    out = torch.zeros_like(e_dev)
    pb.peel_e(dg, e_dev, out=out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.peel_edge(g, e)[0])


@pytest.mark.parametrize("small,huge,chunk", [("0", "1000000000000", "8192"), ("0", "1000000000000", "1"),
                                              ("0", "64", "8192"), ("8192", "200", "16")])
def test_peel_levels_warp_cta_grid(ctx, monkeypatch, small, huge, chunk):
    """Forces frontier items through the CTA-level (small=0), chunked (chunk=1: every item split
    into as many work units as it has first-level entries) and grid-level (low huge) paths."""
    monkeypatch.setenv("PB_PEEL_SMALL_WORK", small)
    monkeypatch.setenv("PB_PEEL_HUGE_WORK", huge)
    monkeypatch.setenv("PB_PEEL_CHUNK_WORK", chunk)
    for g in [BipartiteGraph.zipf(500, 700, 6000, 1.3, 1201), BipartiteGraph.rmat(10, 9, 8000, 0.55, 0.15, 0.15, 0.15, 1202)]:
        dg = ctx.upload(g)
        for uv in (False, True):
            e, _ = oracle.count(g, "EDGE", "ADEG", use_v=uv)
            np.testing.assert_array_equal(pb.peel_e(dg, e, use_v=uv), oracle.peel_edge(g, e, use_v=uv)[0])
            c, _ = oracle.count(g, "VERT", "ADEG", use_v=uv)
            np.testing.assert_array_equal(pb.peel(dg, c, use_v=uv), oracle.peel_vert(g, c, use_v=uv)[0])


def test_barrier_timeout_reports_status_and_context_survives(ctx, monkeypatch):
    """A grid-barrier wait that cannot complete (a phantom arrival, set by a test hook) runs out
    after the configured bound; the call returns PB_ETIMEOUT and the context keeps working."""
    import time
    from parbutterfly_b200._ffi import PBError, PB_ETIMEOUT
    g = BipartiteGraph.zipf(300, 400, 3000, 1.3, 1301)
    dg = ctx.upload(g)
    e = pb.count_e(dg)
    monkeypatch.setenv("PB_PEEL_BARRIER_TIMEOUT_MS", "500")
    monkeypatch.setenv("PB_PEEL_TEST_STUCK_BARRIER", "1")
    t0 = time.time()
    with pytest.raises(PBError) as ex:
        pb.peel_e(dg, e)
    assert ex.value.status == PB_ETIMEOUT
    assert time.time() - t0 < 30
    monkeypatch.delenv("PB_PEEL_TEST_STUCK_BARRIER")
    monkeypatch.delenv("PB_PEEL_BARRIER_TIMEOUT_MS")
    np.testing.assert_array_equal(pb.peel_e(dg, e), oracle.peel_edge(g, e)[0])
    np.testing.assert_array_equal(pb.count_e(dg), e)
