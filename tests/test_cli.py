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
