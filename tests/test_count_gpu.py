"""Parity of the CUDA counting path with the golden vectors and the oracle, through the C ABI.
Integer results: bit-exact."""
import numpy as np
import pytest

import oracle
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu

RANKS = ["SIDE", "COCORE", "ACOCORE", "DEG", "ADEG"]
COUNT_TYPES = ["SORT", "ASORT", "HASH", "AHASH", "HIST", "AHIST", "BATCHS", "BATCHWA", "SERIAL"]


def test_golden_all_ranks_and_pers(ctx, golden):
    for name, (g, rec) in golden.items():
        dg = ctx.upload(g)
        use_v, w = pb.cmp_wedge_counts(dg)
        assert [int(use_v), w] == list(rec["use_v"]), name
        for rank in RANKS:
            np.testing.assert_array_equal(pb.count(dg, "BATCHS", rank), rec[f"VERT/BATCHS/{rank}"], err_msg=f"{name} {rank}")
            np.testing.assert_array_equal(pb.count_e(dg, "BATCHS", rank), rec[f"EDGE/BATCHS/{rank}"], err_msg=f"{name} {rank}")
            assert pb.count_total(dg, "BATCHS", rank) == int(rec[f"TOTAL/BATCHS/{rank}"][0]), name
        dg.close()


def test_golden_every_count_type(ctx, golden):
    for name, (g, rec) in golden.items():
        dg = ctx.upload(g)
        for ct in COUNT_TYPES:
            np.testing.assert_array_equal(pb.count(dg, ct, "ADEG"), rec["VERT/BATCHS/ADEG"], err_msg=f"{name} {ct}")
            np.testing.assert_array_equal(pb.count_e(dg, ct, "ACOCORE"), rec["EDGE/BATCHS/ACOCORE"], err_msg=f"{name} {ct}")
            assert pb.count_total(dg, ct, "DEG") == int(rec["TOTAL/BATCHS/DEG"][0]), f"{name} {ct}"
        dg.close()


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("kind", ["uniform", "zipf", "rmat", "powerlaw"])
def test_random_graphs_vs_oracle(ctx, kind, seed):
    if kind == "uniform":
        g = BipartiteGraph.uniform(3000, 2000, 40000, 100 + seed)
    elif kind == "zipf":
        g = BipartiteGraph.zipf(2000, 3000, 40000, 1.3, 200 + seed)
    elif kind == "rmat":
        g = BipartiteGraph.rmat(12, 11, 60000, 0.55, 0.15, 0.15, 0.15, 300 + seed)
    else:
        g = BipartiteGraph.powerlaw_u(2000, 8000, 80000, 2.0, 2000, 400 + seed)
    dg = ctx.upload(g)
    rank = RANKS[seed % len(RANKS)]
    ov, wr = oracle.count(g, "VERT", rank)
    oe, _ = oracle.count(g, "EDGE", rank)
    ot, _ = oracle.count(g, "TOTAL", rank)
    np.testing.assert_array_equal(pb.count(dg, "HASH", rank), ov)
    assert ctx.stats()["w_rank"] == wr  # same order, same ranked wedge count
    np.testing.assert_array_equal(pb.count_e(dg, "BATCHS", rank), oe)
    assert pb.count_total(dg, "SORT", rank) == ot
    # both count sides
    for uv in (False, True):
        np.testing.assert_array_equal(pb.count(dg, "BATCHS", rank, use_v=uv), oracle.count(g, "VERT", rank, use_v=uv)[0])


def test_config1_full_size(ctx):
    """The 4096 x 4096, m = 131072 uniform workload, -per VERT and -per TOTAL (BATCHS, ADEG)."""
    g = BipartiteGraph.uniform(4096, 4096, 131072, 1)
    dg = ctx.upload(g)
    ov, wr = oracle.count(g, "VERT", "ADEG")
    np.testing.assert_array_equal(pb.count(dg, "BATCHS", "ADEG"), ov)
    assert ctx.stats()["w_rank"] == wr
    assert pb.count_total(dg, "BATCHS", "ADEG") == oracle.count(g, "TOTAL", "ADEG")[0] == ov.sum() // 2


def test_large_rmat_invariants(ctx):
    """At the 2^20 x 2^18, m = 2^24 R-MAT size the oracle is too slow; check the identities that
    hold at any size: sum(vertex counts)/2 = sum(edge counts)/4 = total, for every rank type,
    and per-edge counts identical across aggregation strategies."""
    g = BipartiteGraph.rmat(20, 18, 1 << 24, 0.55, 0.15, 0.15, 0.15, 2)
    dg = ctx.upload(g)
    totals = set()
    e_ref = None
    for rank, ct in [("ACOCORE", "HASH"), ("ADEG", "BATCHS"), ("DEG", "SORT"), ("SIDE", "HASH")]:
        t = pb.count_total(dg, ct, rank)
        v = pb.count(dg, ct, rank)
        e = pb.count_e(dg, ct, rank)
        assert v.sum() % 2 == 0 and e.sum() % 4 == 0
        totals.update({t, int(v.sum()) // 2, int(e.sum()) // 4})
        if e_ref is None:
            e_ref = e
        else:
            np.testing.assert_array_equal(e, e_ref)
    assert len(totals) == 1


def test_edge_cases(ctx):
    # isolated vertices, single edge, a star (no wedges on one side), K_{a,b}
    cases = [
        BipartiteGraph.from_edges(5, 4, [1], [2]),
        BipartiteGraph.from_edges(1, 9, np.zeros(9, dtype=np.int64), np.arange(9)),
        BipartiteGraph.from_edges(4, 6, np.repeat(np.arange(4), 6), np.tile(np.arange(6), 4)),
        BipartiteGraph.from_edges(50, 60, [0, 0, 49, 49], [0, 59, 0, 59]),
    ]
    for g in cases:
        dg = ctx.upload(g)
        for rank in RANKS:
            np.testing.assert_array_equal(pb.count(dg, "HASH", rank), oracle.count(g, "VERT", rank)[0])
            np.testing.assert_array_equal(pb.count_e(dg, "HASH", rank), oracle.count(g, "EDGE", rank)[0])
            assert pb.count_total(dg, "HASH", rank) == oracle.count(g, "TOTAL", rank)[0]


def test_empty_graph(ctx):
    g = BipartiteGraph.from_edges(3, 2, [], [])
    dg = ctx.upload(g)
    assert pb.count_total(dg) == 0
    assert (pb.count(dg) == 0).all()


def test_device_pointer_outputs(ctx):
    import torch
    g = BipartiteGraph.zipf(800, 600, 9000, 1.4, 9)
    dg = ctx.upload(g)
    use_v, _ = pb.cmp_wedge_counts(dg)
    out = torch.zeros(g.nu if use_v else g.nv, dtype=torch.int64, device="cuda")
    pb.count(dg, "HASH", "ADEG", out=out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.count(g, "VERT", "ADEG")[0])


def test_graph_from_device_and_validation(ctx):
    import torch
    g = BipartiteGraph.uniform(200, 300, 2500, 4)
    arrs = [torch.from_numpy(a.astype(np.int32)).cuda() for a in (g.offsetsV, g.edgesV, g.offsetsU, g.edgesU)]
    dg = pb.DeviceGraph(ctx, device_arrays=(g.nv, g.nu, *arrs))
    np.testing.assert_array_equal(pb.count(dg, "HASH", "DEG"), oracle.count(g, "VERT", "DEG")[0])
    bad = arrs[1].clone()
    bad[0], bad[1] = arrs[1][1], arrs[1][0]
    from parbutterfly_b200._ffi import PBError
    with pytest.raises(PBError):
        pb.DeviceGraph(ctx, device_arrays=(g.nv, g.nu, arrs[0], bad, arrs[2], arrs[3]))


def test_eti_matches_oracle(ctx, golden):
    for name, (g, rec) in golden.items():
        dg = ctx.upload(g)
        for uv in (False, True):
            np.testing.assert_array_equal(pb.edge_to_idxs(dg, uv), oracle.edge_to_idxs(g, uv), err_msg=name)
            np.testing.assert_array_equal(pb.idxs_to_edge(dg, uv), oracle.edge_to_idxs(g, not uv), err_msg=name)


@pytest.mark.parametrize("smem,small_w,acc64", [("16384", "0", "0"), ("20000", "64", "1"), ("196608", "512", "1")])
def test_cta_modes_vs_oracle(ctx, monkeypatch, smem, small_w, acc64):
    """Small CTA tables push endpoints into the hash, hybrid and global-scratch modes; acc64
    forces 64-bit per-edge accumulation (otherwise 32-bit when the degrees allow)."""
    monkeypatch.setenv("PB_COUNT_SMEM", smem)
    monkeypatch.setenv("PB_COUNT_SMALL_W", small_w)
    monkeypatch.setenv("PB_EDGE_ACC64", acc64)
    for g in [BipartiteGraph.rmat(14, 12, 150000, 0.55, 0.15, 0.15, 0.15, 41),
              BipartiteGraph.powerlaw_u(3000, 20000, 200000, 2.0, 3000, 42)]:
        dg = ctx.upload(g)
        for rank in ["ADEG", "SIDE", "ACOCORE"]:
            np.testing.assert_array_equal(pb.count(dg, "HASH", rank), oracle.count(g, "VERT", rank)[0])
            np.testing.assert_array_equal(pb.count_e(dg, "HASH", rank), oracle.count(g, "EDGE", rank)[0])
            assert pb.count_total(dg, "HASH", rank) == oracle.count(g, "TOTAL", rank)[0]
        dg.close()


@pytest.mark.parametrize("ct", ["SORT", "ASORT", "HIST", "AHIST"])
@pytest.mark.parametrize("max_wedges", [2577500000, 5000])
def test_materialized_aggregators_vs_oracle(ctx, ct, max_wedges):
    """SORT (radix sort + runs) and HIST (semisort histogram) over wedge batches of at most
    max_wedges wedges (-m); small -m forces many batches."""
    for g in [BipartiteGraph.rmat(12, 11, 40000, 0.55, 0.15, 0.15, 0.15, 51),
              BipartiteGraph.zipf(1500, 2500, 30000, 1.4, 52)]:
        dg = ctx.upload(g)
        for rank in ["ADEG", "SIDE", "COCORE"]:
            np.testing.assert_array_equal(pb.count(dg, ct, rank, max_wedges=max_wedges), oracle.count(g, "VERT", rank)[0])
            np.testing.assert_array_equal(pb.count_e(dg, ct, rank, max_wedges=max_wedges), oracle.count(g, "EDGE", rank)[0])
            assert pb.count_total(dg, ct, rank, max_wedges=max_wedges) == oracle.count(g, "TOTAL", rank)[0]
        dg.close()


def test_hist_heavy_keys_overflow_path(ctx):
    """A complete bipartite block makes a few (endpoint, u2) keys carry huge multiplicities and
    fills semisort buckets with repeated keys; results must match the oracle."""
    a, b = 40, 300
    v = np.repeat(np.arange(a), b)
    u = np.tile(np.arange(b), a)
    extra_v = np.random.default_rng(3).integers(0, 400, 3000)
    extra_u = np.random.default_rng(4).integers(0, 2000, 3000)
    g = BipartiteGraph.from_edges(400, 2000, np.concatenate([v, extra_v]), np.concatenate([u, extra_u]))
    dg = ctx.upload(g)
    for ct in ["HIST", "SORT"]:
        np.testing.assert_array_equal(pb.count(dg, ct, "ADEG"), oracle.count(g, "VERT", "ADEG")[0])
        np.testing.assert_array_equal(pb.count_e(dg, ct, "DEG"), oracle.count(g, "EDGE", "DEG")[0])
