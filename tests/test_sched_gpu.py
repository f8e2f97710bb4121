"""Learned scheduler: the tensor-core GEMM against a torch fp32 reference, MLP training, trace
logging, and learned / exploring choices giving results identical to the plain path and the
oracle."""
import numpy as np
import pytest

import oracle
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu


@pytest.fixture
def small_items(monkeypatch):
    """Every endpoint with wedges goes to the block aggregator, whose table is shrunk so small
    graphs reach all four aggregation modes."""
    monkeypatch.setenv("PB_COUNT_SMALL_W", "0")
    monkeypatch.setenv("PB_COUNT_SMEM", "16384")
    monkeypatch.setenv("PB_SCHED_MIN_WEDGES", "0")  # the learned choice scores every item here


def _rmat(seed, lv=11, lu=10, m=20000):
    return BipartiteGraph.rmat(lv, lu, m, 0.55, 0.15, 0.15, 0.15, seed)


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (128, 16, 16), (130, 64, 64), (300, 100, 200), (1000, 128, 70),
                                   (257, 8, 33), (64, 120, 1)])
def test_tc_gemm_matches_fp32(ctx, M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 131 + N * 7 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    D = pb.tc_gemm_bf16(ctx, A, B)
    ref = A.float() @ B.float().T
    # BF16 products are exact in FP32; only the accumulation order differs.
    torch.testing.assert_close(D, ref, rtol=1e-4, atol=1e-3)


def test_tc_gemm_transposed_operands(ctx):
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    At = torch.randn(96, 200, device="cuda", generator=g).to(torch.bfloat16)  # K x M storage
    Bt = torch.randn(96, 48, device="cuda", generator=g).to(torch.bfloat16)   # K x N storage
    A, B = At.T, Bt.T  # M x K and N x K views with element strides (1, M) and (1, N)
    D = pb.tc_gemm_bf16(ctx, A, B)
    torch.testing.assert_close(D, A.float() @ B.float().T, rtol=1e-4, atol=1e-3)


def test_mlp_learns_held_out_function(ctx):
    rng = np.random.default_rng(0)
    X = rng.normal(size=(8192, 16)).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] ** 2 - 0.7 * X[:, 2] * X[:, 3] + 0.3 * X[:, 4]).astype(np.float32)
    m = pb.SchedModel(ctx, seed=3)
    mse = m.train(m.COUNT, X[:6144], y[:6144], epochs=80, batch=512, lr=3e-3)
    pred = m.predict(m.COUNT, X[6144:])
    assert mse < 0.2
    assert np.corrcoef(pred, y[6144:])[0, 1] > 0.85


def test_model_save_load_roundtrip(ctx, tmp_path):
    rng = np.random.default_rng(1)
    X = rng.normal(size=(1024, 16)).astype(np.float32)
    y = X[:, 0] * 2 + 1
    m = pb.SchedModel(ctx, seed=4)
    m.train(m.PEEL, X, y, epochs=5, batch=256)
    p = str(tmp_path / "sched.bin")
    m.save(p)
    m2 = pb.SchedModel(ctx, seed=99)
    m2.load(p)
    np.testing.assert_array_equal(m.predict(m.PEEL, X[:50]), m2.predict(m2.PEEL, X[:50]))


def test_explore_modes_exact_and_traced(ctx, small_items):
    g = _rmat(7)
    dg = ctx.upload(g)
    use_v = oracle.cmp_wedge_counts(g)[0]
    ov, _ = oracle.count(g, "VERT", "ADEG", use_v=use_v)
    oe, _ = oracle.count(g, "EDGE", "ADEG", use_v=use_v)
    pb.trace_clear(ctx)
    pb.trace_set(ctx, "explore", seed=11)
    try:
        for seed_round in range(2):
            np.testing.assert_array_equal(pb.count(dg, "HASH", "ADEG"), ov)
            np.testing.assert_array_equal(pb.count_e(dg, "BATCHS", "ADEG"), oe)
            assert pb.count_total(dg, "HASH", "ADEG") == int(ov.sum()) // 2
    finally:
        pb.trace_set(ctx, "off")
    X, y = pb.trace_rows(ctx, pb.SchedModel.COUNT)
    assert X.shape[0] > 100 and X.shape[0] == y.shape[0]
    modes = X[:, 12:].argmax(1)
    assert np.all(X[:, 12:].sum(1) == 1)
    assert len(set(modes.tolist())) >= 3  # the exploration covers the modes
    assert np.all(np.isfinite(y)) and y.min() > 0


def _collect_count_traces(ctx, seeds):
    pb.trace_clear(ctx)
    pb.trace_set(ctx, "explore", seed=21)
    try:
        for s in seeds:
            dg = ctx.upload(_rmat(s))
            pb.count(dg, "HASH", "ADEG")
            pb.count_e(dg, "HASH", "ADEG")
    finally:
        pb.trace_set(ctx, "off")
    return pb.trace_rows(ctx, pb.SchedModel.COUNT)


def test_learned_count_exact_and_reported(ctx, small_items):
    X, y = _collect_count_traces(ctx, [31, 32, 33])
    m = pb.SchedModel(ctx, seed=5)
    m.train(m.COUNT, X, y, epochs=40, batch=512)
    m.attach()
    try:
        g = _rmat(40)
        dg = ctx.upload(g)
        for per_fn in (pb.count, pb.count_e):
            plain = per_fn(dg, "HASH", "ADEG")
            learned = per_fn(dg, "HASH", "ADEG", sched="learned")
            np.testing.assert_array_equal(learned, plain)
            st = ctx.stats()
            assert st["sched_used"] == 1 and st["sched_items"] > 0
            assert st["sched_pred"] > 0 and st["sched_meas"] > 0 and st["sched_mae_log2"] >= 0
        assert pb.count_total(dg, "BATCHS", "ADEG", sched="learned") == pb.count_total(dg, "BATCHS", "ADEG")
    finally:
        pb.detach_sched_model(ctx)


def test_learned_without_model_runs_plain(ctx):
    dg = ctx.upload(_rmat(41, 9, 9, 3000))
    np.testing.assert_array_equal(pb.count(dg, "HASH", "ADEG", sched="learned"), pb.count(dg, "HASH", "ADEG"))
    assert ctx.stats()["sched_used"] == 0


def test_peel_explore_every_setting_exact_and_learned(ctx):
    graphs = [_rmat(50 + k, 10, 9, 6000 + 1500 * k) for k in range(3)]
    graphs.append(BipartiteGraph.zipf(600, 400, 9000, 1.3, 57))
    pb.trace_clear(ctx)
    pb.trace_set(ctx, "explore", seed=77)
    choices = set()
    try:
        for g in graphs:
            dg = ctx.upload(g)
            use_v = oracle.cmp_wedge_counts(g)[0]
            c = pb.count(dg, "BATCHS", "ADEG")
            ce = pb.count_e(dg, "BATCHS", "ADEG")
            tip_ref = oracle.peel_vert(g, c, use_v=use_v)[0]
            wing_ref = oracle.peel_edge(g, ce, use_v=use_v)[0]
            for _ in range(4):
                np.testing.assert_array_equal(pb.peel(dg, c), tip_ref)
                choices.add(ctx.stats()["sched_choice"])
                np.testing.assert_array_equal(pb.peel_e(dg, ce), wing_ref)
                choices.add(ctx.stats()["sched_choice"])
    finally:
        pb.trace_set(ctx, "off")
    assert len(choices) > 4
    X, y = pb.trace_rows(ctx, pb.SchedModel.PEEL)
    assert X.shape[0] == 8 * len(graphs)
    m = pb.SchedModel(ctx, seed=6)
    m.train(m.PEEL, X, y, epochs=60, batch=16)
    m.attach()
    try:
        g = graphs[1]
        dg = ctx.upload(g)
        c = pb.count(dg, "BATCHS", "ADEG")
        ce = pb.count_e(dg, "BATCHS", "ADEG")
        np.testing.assert_array_equal(pb.peel(dg, c, sched="learned"), pb.peel(dg, c))
        np.testing.assert_array_equal(pb.peel_e(dg, ce, sched="learned"), pb.peel_e(dg, ce))
        pb.peel_e(dg, ce, sched="learned")
        st = ctx.stats()
        assert st["sched_used"] == 1 and 0 <= st["sched_choice"] < 3 and st["sched_pred"] > 0
        pb.peel(dg, c, sched="learned")
        assert 0 <= ctx.stats()["sched_choice"] < 48
    finally:
        pb.detach_sched_model(ctx)
        m.close()


def test_autotune_picks_a_geometry_once_and_keeps_results(ctx):
    g = _rmat(61, 12, 11, 60000)
    dg = ctx.upload(g)
    plain = pb.count(dg, "HASH", "ADEG")
    first = pb.count(dg, "HASH", "ADEG", autotune=True)
    st1 = ctx.stats()
    again = pb.count(dg, "HASH", "ADEG", autotune=True)
    st2 = ctx.stats()
    np.testing.assert_array_equal(first, plain)
    np.testing.assert_array_equal(again, plain)
    assert st1["autotuned"] == 1 and st2["autotuned"] == 0
    geom = (st2["count_smem_bytes"], st2["count_blocks_per_sm"], st2["count_small_w"])
    assert geom == (st1["count_smem_bytes"], st1["count_blocks_per_sm"], st1["count_small_w"])
    assert geom[0] in (32 << 10, 48 << 10, 96 << 10, 200 << 10) and geom[2] in (256, 512)
    e = pb.count_e(dg, "HASH", "ADEG", autotune=True)
    np.testing.assert_array_equal(e, pb.count_e(dg, "HASH", "ADEG"))
    assert pb.count_total(dg, "BATCHS", "ADEG", autotune=True) == int(plain.sum()) // 2
