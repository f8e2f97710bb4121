"""The pbb command line against the reference's own BipartiteButterflies driver (built from the
reference sources by oracle/Makefile as oracle/_ref/BipartiteButterflies): same input file
(AdjacencyHypergraph text written by the library), same flags and aliases
(BipartiteButterflies.C:79-194), same result lines ("number of butterflies: N" / "number of
edge butterflies: N", :222-268) and the same stage names in the timer lines.

CPU: the reference driver's lines equal the oracle's totals for every flag set (this pins the
file writer and the flag table).  GPU: pbb prints the reference driver's lines."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from parbutterfly_b200.graph import BipartiteGraph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "BipartiteButterflies")
PBB = os.path.join(ROOT, "parbutterfly_b200", "cli", "pbb")

# (flags, per) — long names, numeric aliases, peeling on and off.
FLAG_SETS = [
    (["-countType", "BATCHS", "-rankType", "ADEG", "-per", "VERT"], "VERT"),
    (["-countType", "SERIAL", "-rankType", "ACOCORE", "-per", "EDGE", "-nopeel"], "EDGE"),
    (["-t", "5", "-w", "2", "-e", "1", "-tp", "3"], "EDGE"),
    (["-t", "8", "-w", "3", "-e", "0", "-tp", "4"], "VERT"),
    (["-per", "TOTAL", "-countType", "HASH"], "TOTAL"),
    (["-e", "0", "-total", "-t", "1"], "TOTAL"),
    (["-countType", "SORT", "-rankType", "DEG", "-per", "VERT", "-peelType", "BATCHS"], "VERT"),
]

needs_ref = pytest.mark.skipif(not os.path.exists(REF_CLI), reason="reference driver not built (reference tree absent)")


def _lines(out):
    return [ln for ln in out.splitlines() if ln.startswith("number of")]


def _stages(out):
    return [ln.split(" : ")[0] for ln in out.splitlines() if re.match(r"^(Par|Serial|WedgePar|SortCE|Sort|HashCE|Hash|"
                                                                      r"HistCE|Hist)( Peel)? : ", ln)]


def _run(exe, flags, path, env=None):
    e = dict(os.environ, OMP_NUM_THREADS="2", **(env or {}))
    r = subprocess.run([exe, *flags, "-r", "0", path], capture_output=True, text=True, env=e, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    return r.stdout


@pytest.fixture(scope="module")
def hyper(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    g = BipartiteGraph.rmat(10, 9, 6000, 0.55, 0.15, 0.15, 0.15, 31)
    p = str(d / "g.hyper")
    g.write_text(p)
    return g, p


@needs_ref
@pytest.mark.parametrize("flags,per", FLAG_SETS)
def test_reference_driver_matches_oracle(hyper, flags, per):
    g, path = hyper
    lines = _lines(_run(REF_CLI, flags, path))
    total = oracle.count(g, "TOTAL", "ADEG")[0]
    word = "edge butterflies" if per == "EDGE" else "butterflies"
    assert lines == [f"number of {word}: {total}"]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("flags,per", FLAG_SETS)
def test_pbb_prints_the_reference_lines(hyper, flags, per):
    _, path = hyper
    ref = _run(REF_CLI, flags, path)
    ours = _run(PBB, flags, path)
    assert _lines(ours) == _lines(ref)
    assert _stages(ours) == _stages(ref)


# Sparsification (BipartiteButterflies.C:175-193, 213-214, 333-340): long and numeric flags.
SPARSE_SETS = [
    (["-sparseType", "EDGE", "-d", "2"], "EDGE", 2),
    (["-sparseType", "COLOR", "-d", "3"], "COLOR", 3),
    (["-s", "2", "-d", "5"], "EDGE", 5),
    (["-s", "1", "-d", "25", "-per", "VERT"], "COLOR", 25),
]


@needs_ref
@pytest.mark.parametrize("flags,kind,denom", SPARSE_SETS)
def test_reference_driver_sparse_matches_host_sparsifier(hyper, flags, kind, denom):
    """The reference driver's estimate equals the host sparsifier's graph counted by the oracle
    and scaled as the reference scales it: pins pb_sparsify_bipartite and pb_sparse_estimate."""
    g, path = hyper
    lines = _lines(_run(REF_CLI, flags, path))
    h = g.sparsify(kind, denom)
    est = BipartiteGraph.sparse_estimate(oracle.count(h, "TOTAL", "ADEG")[0], kind, denom)
    assert lines == [f"number of butterflies: {est}"]


def test_sparsify_keeps_a_valid_graph():
    g = BipartiteGraph.zipf(300, 200, 4000, 1.3, 33)
    for kind in ("EDGE", "COLOR"):
        h = g.sparsify(kind, 4)
        assert 0 < h.m < g.m
        assert h.offsetsV[-1] == h.m and h.offsetsU[-1] == h.m
        assert (np.diff(h.offsetsV) > 0).all() and (np.diff(h.offsetsU) > 0).all()  # no vertex without edges
        assert h.sparsify(kind, 1).m == h.m  # one colour keeps everything


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("flags,kind,denom", SPARSE_SETS)
def test_pbb_sparse_prints_the_reference_lines(hyper, flags, kind, denom):
    _, path = hyper
    assert _lines(_run(PBB, flags, path)) == _lines(_run(REF_CLI, flags, path))
