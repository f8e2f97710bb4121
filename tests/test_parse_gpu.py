"""readBipartite on the device (pb_graph_parse_text / pb_graph_read_text): graphs parsed by the
GPU kernels count exactly like the host-parsed ones and the oracle, from host bytes, device
bytes and files; every error readBipartite aborts on comes back as a status."""
import numpy as np
import pytest

import oracle
from parbutterfly_b200 import _ffi
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu


def _text(g, tmp_path, name="g.hyper"):
    p = str(tmp_path / name)
    g.write_text(p)
    return p, open(p, "rb").read()


@pytest.mark.parametrize("make", [
    lambda: BipartiteGraph.rmat(10, 9, 7000, 0.55, 0.15, 0.15, 0.15, 71),
    lambda: BipartiteGraph.zipf(700, 900, 5000, 1.3, 72),
    lambda: BipartiteGraph.uniform(300, 200, 4000, 73),
    lambda: BipartiteGraph.from_edges(4, 3, [0, 0, 1, 3], [0, 2, 1, 2]),
])
def test_device_parse_counts_like_host_parse(ctx, tmp_path, make):
    import torch
    g = make()
    path, data = _text(g, tmp_path)
    ref_e, _ = oracle.count(g, "EDGE", "ADEG")
    for dg in (pb.read_text_device(ctx, path), pb.graph_from_text(ctx, data),
               pb.graph_from_text(ctx, torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()).cuda())):
        assert (dg.nv, dg.nu, dg.m) == (g.nv, g.nu, g.m)
        np.testing.assert_array_equal(pb.count_e(dg, "HASH", "ADEG"), ref_e)
        np.testing.assert_array_equal(pb.count(dg, "BATCHS", "ADEG"), oracle.count(g, "VERT", "ADEG")[0])


def test_device_parse_tolerates_whitespace_layout(ctx):
    # one number per line (the writer's layout) and everything on one line parse the same
    text = b"AdjacencyHypergraph\n2\n3\n2\n3\n0 2\n0 1 1\n0\t1\r\n0 0 1  \n"
    dg = pb.graph_from_text(ctx, text)
    assert (dg.nv, dg.nu, dg.m) == (2, 2, 3)
    g = BipartiteGraph.from_edges(2, 2, [0, 0, 1], [0, 1, 1])
    np.testing.assert_array_equal(pb.count_e(dg, "HASH", "ADEG"), oracle.count(g, "EDGE", "ADEG")[0])


@pytest.mark.parametrize("text,status", [
    (b"AdjacencyGraph\n2\n3\n2\n3\n0 2\n0 1 1\n0 1\n0 1 0\n", _ffi.PB_EIO),     # wrong header word
    (b"AdjacencyHypergraph\n2\n3\n2\n3\n0 2\n0 1 1\n0 1\n0 1\n", _ffi.PB_EIO),  # token count
    (b"AdjacencyHypergraph\n2\n3\n2\n2\n0 2\n0 1 1\n0 1\n0 1\n", _ffi.PB_EIO),  # mv != mu
    (b"AdjacencyHypergraph\n2\n3\n2\n3\n0 2\n0 1 5\n0 1\n0 1 0\n", _ffi.PB_EINVAL),  # id out of range
    (b"AdjacencyHypergraph\n2\n3\n2\n3\n0 2\n0 1 x\n0 1\n0 1 0\n", _ffi.PB_EIO),  # not a number
    (b"AdjacencyHypergraph\n2\n3\n2\n3\n0 2\n1 0 1\n0 1\n0 1 0\n", _ffi.PB_EINVAL),  # unsorted list
    (b"AdjacencyHypergraph\n", _ffi.PB_EIO),                                     # no sizes
])
def test_device_parse_errors_are_statuses(ctx, text, status):
    with pytest.raises(_ffi.PBError) as ei:
        pb.graph_from_text(ctx, text)
    assert ei.value.status == status
    # the context stays usable
    dg = pb.graph_from_text(ctx, b"AdjacencyHypergraph 1 1 1 1 0 0 0 0")
    assert pb.count_total(dg) == 0
