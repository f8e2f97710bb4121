"""pb_count_total_noalloc: the total-count entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc where they need a count (code inside another
framework's memory pool, paths that must not synchronise the device, callers near the memory
limit).  Its output is checked, exactly (integer counts), against the existing pb_count_total
entry point, against the CPU oracle's total and, for the fixtures produced by the reference
itself, against the reference's own total, on two calls in a row: the static scratch array
keeps the previous call's contents, so the second call also checks that the entry point clears
what must start at zero.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from parbutterfly_b200 import _ffi
from parbutterfly_b200 import butterflies as pb
from parbutterfly_b200.graph import BipartiteGraph

pytestmark = pytest.mark.gpu


def _device_csr(g):
    import torch
    arrs = [torch.from_numpy(a.astype(np.int32)).cuda() for a in (g.offsetsV, g.edgesV, g.offsetsU, g.edgesU)]
    s = _ffi.CSR(g.nv, g.nu, g.m, arrs[0].data_ptr(), arrs[1].data_ptr(), arrs[2].data_ptr(), arrs[3].data_ptr())
    return s, arrs


def _noalloc_total(s):
    import torch
    out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    msg = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = _ffi.lib().pb_count_total_noalloc(C.byref(s), C.c_void_p(stream), C.c_void_p(out.data_ptr()), msg, 256)
    assert st == _ffi.PB_OK, msg.value.decode()
    torch.cuda.synchronize()
    return int(out.item())


@pytest.mark.parametrize("make", [
    lambda: BipartiteGraph.uniform(3000, 2000, 40000, 71),
    lambda: BipartiteGraph.zipf(2000, 3000, 40000, 1.3, 72),
    lambda: BipartiteGraph.rmat(12, 11, 60000, 0.55, 0.15, 0.15, 0.15, 73),
    lambda: BipartiteGraph.from_edges(4, 6, np.repeat(np.arange(4), 6), np.tile(np.arange(6), 4)),
])
def test_noalloc_total_matches_count_total_twice(make):
    g = make()
    with pb.Context(0) as ctx:
        dg = ctx.upload(g)
        expect = pb.count_total(dg, "BATCHS", "ADEG")
        dg.close()
    assert expect == oracle.count(g, "TOTAL", "ADEG")[0]
    s, keep = _device_csr(g)
    first = _noalloc_total(s)
    second = _noalloc_total(s)
    assert first == expect
    assert second == expect


def test_noalloc_total_matches_reference_golden(golden):
    # Totals the reference itself printed for the fixture graphs (BATCHS, ADEG).
    for name, (g, rec) in golden.items():
        expect = int(rec["TOTAL/BATCHS/ADEG"][0])
        s, keep = _device_csr(g)
        for _ in range(2):
            assert _noalloc_total(s) == expect, name


def test_noalloc_rejects_oversized_side():
    import torch
    n = (1 << 22)
    offs = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    one = torch.zeros(2, dtype=torch.int32, device="cuda")
    s = _ffi.CSR(n, 1, 0, offs.data_ptr(), one.data_ptr(), one.data_ptr(), one.data_ptr())
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    msg = C.create_string_buffer(256)
    st = _ffi.lib().pb_count_total_noalloc(C.byref(s), None, C.c_void_p(out.data_ptr()), msg, 256)
    assert st == _ffi.PB_ETOOBIG
    assert b"limit" in msg.value
