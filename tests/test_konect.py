"""KONECT edge lists (pb_read_konect) against the reference's own converter
(utils/KONECTtoHyperAdj.C, built by oracle/Makefile as oracle/_ref/KONECTtoHyperAdj): the same
AdjacencyHypergraph file from the same edge list — comment lines, weight and time columns,
repeated pairs, sparse and unsorted ids."""
import os
import subprocess

import numpy as np
import pytest

from parbutterfly_b200.graph import BipartiteGraph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_KONECT = os.path.join(ROOT, "oracle", "_ref", "KONECTtoHyperAdj")


def _write_konect(path, seed, cols):
    rng = np.random.default_rng(seed)
    m = 3000
    v = rng.integers(1, 5000, size=m) * 3
    u = rng.integers(1, 800, size=m) * 7
    v = np.concatenate([v, v[:200]])  # repeated pairs
    u = np.concatenate([u, u[:200]])
    with open(path, "w") as f:
        f.write("% bip unweighted\n% 3200 5000 800\n")
        for a, b in zip(v, u):
            extra = " ".join(str(int(x)) for x in rng.integers(1, 9, size=cols - 2))
            f.write(f"{a} {b}{(' ' + extra) if extra else ''}\n")


def test_konect_small_known_answer(tmp_path):
    p = tmp_path / "k.txt"
    p.write_text("% c\n3 10 1\n3 12 1\n7 10 1\n3 10 1\n20 12 1\n7 30 1\n20 30 1\n1 10 2\n")
    g = BipartiteGraph.read_konect(str(p))
    # V ids {1,3,7,20} -> 0..3, U ids {10,12,30} -> 0..2; (3,10) appears twice.
    want = BipartiteGraph.from_edges(4, 3, [1, 1, 2, 3, 2, 3, 0], [0, 1, 0, 1, 2, 2, 0])
    for name in ("offsetsV", "edgesV", "offsetsU", "edgesU"):
        np.testing.assert_array_equal(getattr(g, name), getattr(want, name), err_msg=name)


@pytest.mark.skipif(not os.path.exists(REF_KONECT), reason="reference converter not built (reference tree absent)")
@pytest.mark.parametrize("cols", [2, 4])
def test_konect_matches_reference_converter(tmp_path, cols):
    src = str(tmp_path / "edges.txt")
    _write_konect(src, 11 + cols, cols)
    ref_out = str(tmp_path / "ref.hyper")
    r = subprocess.run([REF_KONECT, src, ref_out], capture_output=True, text=True, timeout=120,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr
    ours = str(tmp_path / "ours.hyper")
    BipartiteGraph.read_konect(src).write_text(ours)
    assert open(ours).read().split() == open(ref_out).read().split()
