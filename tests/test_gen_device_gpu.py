"""The device R-MAT generator (pb_gen_rmat_device) produces exactly the graph of the host
generator (pb_gen_rmat) for the same arguments: same draw stream, same first-m-distinct rule,
both CSR sides sorted.  Cases include skewed parameters where most draws repeat a pair (the
generator then grows its draw count), rectangular grids both ways and the benchmark's R-MAT
parameters."""
import numpy as np
import pytest

from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu

CASES = [
    (10, 8, 20000, 0.55, 0.15, 0.15, 0.15, 2),
    (8, 6, 8000, 0.57, 0.19, 0.19, 0.05, 5),      # m close to the 16384 pairs: many repeats
    (6, 11, 30000, 0.45, 0.25, 0.15, 0.15, 9),    # U side longer than V side
    (14, 12, 1 << 18, 0.55, 0.15, 0.15, 0.15, 2),  # the benchmark's 2^18-edge sample
    (5, 5, 0, 0.25, 0.25, 0.25, 0.25, 1),
]


@pytest.mark.parametrize("args", CASES)
def test_device_rmat_equals_host_rmat(ctx, args):
    host = BipartiteGraph.rmat(*args)
    dg = pb.gen_rmat_device(ctx, *args)
    try:
        dev = dg.download()
    finally:
        dg.close()
    assert (dev.nv, dev.nu, dev.m) == (host.nv, host.nu, host.m)
    for name in ("offsetsV", "edgesV", "offsetsU", "edgesU"):
        np.testing.assert_array_equal(getattr(dev, name)[:len(getattr(host, name))], getattr(host, name), err_msg=name)
