"""Host-side checks that need no GPU: the C ABI library loads and exports every declared
symbol, generators are deterministic and valid, file IO round-trips, validation rejects bad
CSRs, and a context on a GPU-less host fails with a status instead of crashing."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from parbutterfly_b200 import _ffi
from parbutterfly_b200.graph import BipartiteGraph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "parbutterfly_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(pb_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    decl = declared_symbols()
    assert decl == sorted(_ffi.EXPORTS)
    L = _ffi.lib()
    missing = [s for s in decl if not hasattr(L, s)]
    assert missing == []
    assert L.pb_abi_version() == 2


def test_opts_defaults_match_reference_cli():
    o = _ffi.Opts()
    _ffi.lib().pb_opts_default(C.byref(o))
    # BipartiteButterflies.C: countType SERIAL (:92), rankType ADEG (:118), -m (:172), -a (:173)
    assert o.count_type == 8 and o.rank_type == 4 and o.per_type == 0
    assert o.max_wedges == 2577500000 and o.max_array_size == 23090996160
    assert o.use_v == -1 and o.sched == 0


@pytest.mark.parametrize("maker", [
    lambda s: BipartiteGraph.uniform(300, 200, 4000, s),
    lambda s: BipartiteGraph.rmat(10, 9, 20000, 0.55, 0.15, 0.15, 0.15, s),
    lambda s: BipartiteGraph.zipf(500, 400, 8000, 1.5, s),
    lambda s: BipartiteGraph.powerlaw_u(400, 2000, 30000, 2.0, 400, s),
])
def test_generators_deterministic_and_valid(maker):
    a, b, c = maker(7), maker(7), maker(8)
    for x, y in [(a.offsetsV, b.offsetsV), (a.edgesV, b.edgesV), (a.offsetsU, b.offsetsU), (a.edgesU, b.edgesU)]:
        np.testing.assert_array_equal(x, y)
    assert not np.array_equal(a.edgesV, c.edgesV)
    a.validate()
    v, u = a.edge_list()
    assert np.unique(v * a.nu + u).size == a.m


def test_generator_sizes():
    g = BipartiteGraph.uniform(4096, 4096, 131072, 1)
    assert (g.nv, g.nu, g.m) == (4096, 4096, 131072)
    g = BipartiteGraph.powerlaw_u(1000, 5000, 60000, 2.0, 1000, 3)
    assert g.m == 60000
    for k in (0, 1, 100, 255):
        b = BipartiteGraph.batch_member(k)
        assert 64 <= b.nv <= 65536 and 64 <= b.nu <= 65536 and b.m >= 4 * min(b.nu, b.nv) // 2
        b.validate()


def test_text_roundtrip(tmp_path):
    g = BipartiteGraph.zipf(120, 90, 700, 1.2, 5)
    p = str(tmp_path / "g.hyper")
    g.write_text(p)
    assert open(p).readline().strip() == "AdjacencyHypergraph"
    h = BipartiteGraph.read_text(p)
    for x, y in [(g.offsetsV, h.offsetsV), (g.edgesV, h.edgesV), (g.offsetsU, h.offsetsU), (g.edgesU, h.edgesU)]:
        np.testing.assert_array_equal(x, y)


def test_text_reader_rejects_bad_files(tmp_path):
    bad_header = tmp_path / "a"
    bad_header.write_text("AdjacencyGraph\n1\n0\n1\n0\n0\n0\n")
    with pytest.raises(_ffi.PBError):
        BipartiteGraph.read_text(str(bad_header))
    mv_ne_mu = tmp_path / "b"
    mv_ne_mu.write_text("AdjacencyHypergraph\n1\n1\n1\n2\n0\n0\n0\n0\n0\n")
    with pytest.raises(_ffi.PBError):
        BipartiteGraph.read_text(str(mv_ne_mu))
    out_of_range = tmp_path / "c"
    out_of_range.write_text("AdjacencyHypergraph\n1\n1\n1\n1\n0\n5\n0\n0\n")
    with pytest.raises(_ffi.PBError):
        BipartiteGraph.read_text(str(out_of_range))
    truncated = tmp_path / "d"
    truncated.write_text("AdjacencyHypergraph\n2\n2\n2\n2\n0\n1\n")
    with pytest.raises(_ffi.PBError):
        BipartiteGraph.read_text(str(truncated))
    with pytest.raises(_ffi.PBError):
        BipartiteGraph.read_text(str(tmp_path / "missing"))


def test_validation_rejects_unsorted_and_mismatched():
    g = BipartiteGraph.uniform(30, 20, 100, 3)
    g.validate()
    bad = BipartiteGraph(g.nv, g.nu, g.offsetsV.copy(), g.edgesV.copy(), g.offsetsU.copy(), g.edgesU.copy())
    i = int(np.argmax(np.diff(g.offsetsV) >= 2))
    b = int(bad.offsetsV[i])
    bad.edgesV[b], bad.edgesV[b + 1] = bad.edgesV[b + 1], bad.edgesV[b]
    with pytest.raises(_ffi.PBError) as e:
        bad.validate()
    assert e.value.status == _ffi.PB_EINVAL
    bad2 = BipartiteGraph(g.nv, g.nu, g.offsetsV.copy(), g.edgesV.copy(), g.offsetsU.copy(), g.edgesU.copy())
    bad2.edgesU[0] = (bad2.edgesU[0] + 1) % g.nv
    with pytest.raises(_ffi.PBError):
        bad2.validate()


def test_context_without_gpu_reports_status():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    h = C.c_void_p()
    st = _ffi.lib().pb_ctx_create(0, None, C.byref(h))
    assert st == _ffi.PB_ECUDA and not h.value


def test_binary_format_roundtrip(tmp_path):
    g = BipartiteGraph.rmat(9, 8, 3000, 0.55, 0.15, 0.15, 0.15, 31)
    base = str(tmp_path / "g")
    g.write_binary(base)
    cfg = open(base + ".config").read().split()
    assert [int(x) for x in cfg] == [g.nv, g.m, g.nu, g.m]
    assert os.path.getsize(base + ".vidx") == 4 * g.nv  # offsets without the final m
    h = BipartiteGraph.read_binary(base)
    for name in ("offsetsV", "edgesV", "offsetsU", "edgesU"):
        np.testing.assert_array_equal(getattr(h, name), getattr(g, name))
    with pytest.raises(_ffi.PBError):
        BipartiteGraph.read_binary(str(tmp_path / "missing"))
