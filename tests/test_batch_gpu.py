"""Many graphs in one pass (pb_count_vert_batch / pb_peel_vert_batch): every graph's counts and
tip numbers equal its own single-graph results (oracle / separate calls), bit-exact."""
import numpy as np
import pytest

import oracle
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu


def _mixed_graphs():
    gs = []
    for k in range(12):
        if k % 3 == 0:
            gs.append(BipartiteGraph.uniform(100 + 37 * k, 80 + 11 * k, 600 + 50 * k, 900 + k))
        elif k % 3 == 1:
            gs.append(BipartiteGraph.zipf(300 + 5 * k, 120 + 40 * k, 2000 + 90 * k, 1.4, 950 + k))
        else:
            gs.append(BipartiteGraph.rmat(8, 9, 3000 + 100 * k, 0.55, 0.15, 0.15, 0.15, 980 + k))
    gs.append(BipartiteGraph.from_edges(5, 7, np.repeat(np.arange(5), 7), np.tile(np.arange(7), 5)))
    gs.append(BipartiteGraph.from_edges(3, 2, [], []))
    return gs


def test_batch_matches_oracle_per_graph(ctx):
    gs = _mixed_graphs()
    dgs = [ctx.upload(g) for g in gs]
    counts = pb.count_batch(dgs, "BATCHS", "ADEG")
    tips = pb.peel_batch(dgs, counts)
    sides = set()
    for g, c, t in zip(gs, counts, tips):
        use_v = oracle.cmp_wedge_counts(g)[0]
        sides.add(use_v)
        oc, _ = oracle.count(g, "VERT", "ADEG", use_v=use_v)
        np.testing.assert_array_equal(c, oc)
        np.testing.assert_array_equal(t, oracle.peel_vert(g, oc, use_v=use_v)[0])
    assert sides == {True, False}  # both count-side orientations are in the batch


def test_batch_members_match_single_calls(ctx):
    gs = [BipartiteGraph.batch_member(k) for k in range(0, 256, 32)]
    dgs = [ctx.upload(g) for g in gs]
    counts = pb.count_batch(dgs, "HASH", "ADEG")
    tips = pb.peel_batch(dgs, counts)
    for dg, c, t in zip(dgs, counts, tips):
        single = pb.count(dg, "HASH", "ADEG")
        np.testing.assert_array_equal(c, single)
        np.testing.assert_array_equal(t, pb.peel(dg, single))


def test_batch_graph_replays_match_oracle(ctx):
    """The planned CUDA graph (ranking + counting + one persistent peel launch for the whole
    batch) gives every graph's oracle counts and tip numbers on every replay."""
    gs = _mixed_graphs()
    dgs = [ctx.upload(g) for g in gs]
    bg = pb.BatchGraph(dgs, "BATCHS", "ADEG")
    for rep in range(3):
        counts, tips = bg.run()
        for g, c, t in zip(gs, counts, tips):
            use_v = oracle.cmp_wedge_counts(g)[0]
            oc, _ = oracle.count(g, "VERT", "ADEG", use_v=use_v)
            np.testing.assert_array_equal(c, oc)
            np.testing.assert_array_equal(t, oracle.peel_vert(g, oc, use_v=use_v)[0])
    assert ctx.stats()["ms_count"] > 0
    bg.close()


def test_batch_graph_autotuned_cocore_hash(ctx):
    """ACOCORE ranking (a data-dependent number of bucket rounds, recorded and captured) with
    the HASH aggregator and autotuned geometry; equals the single-graph calls."""
    gs = [BipartiteGraph.batch_member(k) for k in range(3, 256, 23)]
    dgs = [ctx.upload(g) for g in gs]
    bg = pb.BatchGraph(dgs, "HASH", "ACOCORE", autotune=True)
    counts, tips = bg.run()
    counts2, tips2 = bg.run()
    for dg, c, t, c2, t2 in zip(dgs, counts, tips, counts2, tips2):
        single = pb.count(dg, "HASH", "ACOCORE")
        np.testing.assert_array_equal(c, single)
        np.testing.assert_array_equal(t, pb.peel(dg, single))
        np.testing.assert_array_equal(c2, c)
        np.testing.assert_array_equal(t2, t)
    bg.close()


def test_batch_graph_rejects_materialising_aggregators(ctx):
    dgs = [ctx.upload(BipartiteGraph.uniform(50, 40, 300, 5))]
    with pytest.raises(pb._ffi.PBError) as ei:
        pb.BatchGraph(dgs, "SORT", "ADEG")
    assert ei.value.status == pb._ffi.PB_EUNSUPPORTED


def test_batch_more_graphs_than_ctas_share_them(ctx):
    """More graphs than resident CTAs: light graphs run one after another on shared CTAs, the
    heavy one on a CTA range of its own; every graph keeps its own peel rounds."""
    gs = [BipartiteGraph.uniform(20 + k % 17, 15 + k % 11, 60 + k % 40, 5000 + k) for k in range(400)]
    gs.append(BipartiteGraph.rmat(12, 11, 40000, 0.55, 0.15, 0.15, 0.15, 5400))
    dgs = [ctx.upload(g) for g in gs]
    counts = pb.count_batch(dgs, "BATCHS", "ADEG")
    tips = pb.peel_batch(dgs, counts)
    for g, c, t in zip(gs, counts, tips):
        use_v = oracle.cmp_wedge_counts(g)[0]
        oc, _ = oracle.count(g, "VERT", "ADEG", use_v=use_v)
        np.testing.assert_array_equal(c, oc)
        np.testing.assert_array_equal(t, oracle.peel_vert(g, oc, use_v=use_v)[0])
