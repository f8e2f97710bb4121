"""Host-side mirror of ParButterfly's entry points over the C ABI.

Names and argument meanings follow the C++ functions that BipartiteButterflies' Compute()
calls (apps/hyper/BipartiteButterflies.C:75-277):

  cmp_wedge_counts(G)                -> cmpWedgeCounts   (butterfly_utils.h:1080-1086)
  edge_to_idxs(G, use_v)             -> edgeToIdxs       (butterfly_utils.h:2034-2062)
  idxs_to_edge(G, use_v)             -> idxsToEdge       (butterfly_utils.h:2065-2067)
  count(G, count_type, rank_type)    -> Count            (butterfly_count.h:1634-1731)
  count_e(G, count_type, rank_type)  -> CountE           (butterfly_ecount.h:1766-1899)
  count_total(G, ...)                -> CountTotal       (butterfly_count_total.h:1014-1102)
  peel(G, counts, peel_type)         -> Peel             (butterfly_peel.h:896-934)
  peel_e(G, ecounts, peel_type)      -> PeelE            (butterfly_epeel.h:519-569)

Results are dense int64 numpy arrays (the reference strides its arrays by 8 longs).  Unlike
the reference, errors raise PBError instead of exiting, and PeelE leaves the graph intact.
Inputs may be numpy (host) or torch CUDA tensors (device); outputs follow `out=` when given.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _ffi
from .graph import BipartiteGraph

COUNT_TYPES = {"SORT": 0, "ASORT": 1, "HASH": 2, "AHASH": 3, "HIST": 4, "AHIST": 5, "BATCHS": 6, "BATCHWA": 7,
               "SERIAL": 8}
RANK_TYPES = {"SIDE": 0, "COCORE": 1, "ACOCORE": 2, "DEG": 3, "ADEG": 4}
PEEL_TYPES = {"SORT": 0, "HASH": 1, "HIST": 2, "BATCHS": 3, "BATCHWA": 4}
PER_TYPES = {"VERT": 0, "EDGE": 1, "TOTAL": 2}


def _enum(table, v, what):
    if isinstance(v, str):
        if v not in table:
            raise ValueError(f"unknown {what} {v!r}; expected one of {sorted(table)}")
        return table[v]
    return int(v)


def make_opts(count_type="SERIAL", rank_type="ADEG", peel_type="BATCHS", per="VERT", use_v: Optional[bool] = None,
              max_wedges=2577500000, max_array_size=23090996160, sched="plain", autotune=False,
              peel_parts=0) -> _ffi.Opts:
    """pb_opts.  peel_parts: batching of the peel's exact rounds (0: the scheduler's choice when
    sched="learned", else one round at a time; n > 0: the two-phase schedule with about n
    partitions; -1: one round at a time even when learned).  Results never depend on it."""
    o = _ffi.Opts()
    _ffi.lib().pb_opts_default(C.byref(o))
    o.count_type = _enum(COUNT_TYPES, count_type, "count type")
    o.rank_type = _enum(RANK_TYPES, rank_type, "rank type")
    o.peel_type = _enum(PEEL_TYPES, peel_type, "peel type")
    o.per_type = _enum(PER_TYPES, per, "per type")
    o.max_wedges = int(max_wedges)
    o.max_array_size = int(max_array_size)
    o.sched = 1 if str(sched).lower() == "learned" else 0
    o.autotune = 1 if autotune else 0
    o.use_v = -1 if use_v is None else int(bool(use_v))
    o.peel_parts = int(peel_parts)
    return o


class Context:
    """A pb_ctx: one CUDA device and stream.  Use one per host thread."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self._lib = _ffi.lib()
        self._h = C.c_void_p()
        _ffi.check(self._lib.pb_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(self._h)),
                   what="pb_ctx_create")
        self.device = device

    def close(self):
        if self._h:
            self._lib.pb_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def check(self, st, what=""):
        _ffi.check(st, self._h, what)

    def stats(self) -> dict:
        s = _ffi.Stats()
        self.check(self._lib.pb_get_stats(self._h, C.byref(s)), "pb_get_stats")
        return {name: getattr(s, name) for name, _ in _ffi.Stats._fields_}

    def kernel_launches(self) -> int:
        return int(self._lib.pb_kernel_launches(self._h))

    def upload(self, g: BipartiteGraph) -> "DeviceGraph":
        return DeviceGraph(self, g)


class DeviceGraph:
    """A pb_graph: the two-sided CSR resident in device memory."""

    def __init__(self, ctx: Context, g: Optional[BipartiteGraph] = None, *, device_arrays=None):
        self.ctx = ctx
        self._h = C.c_void_p()
        lib = ctx._lib
        if g is not None:
            s = g.csr_struct()
            ctx.check(lib.pb_graph_upload(ctx.handle, C.byref(s), C.byref(self._h)), "pb_graph_upload")
            self.nv, self.nu, self.m = g.nv, g.nu, g.m
        else:
            nv, nu, offV, edgV, offU, edgU = device_arrays
            m = int(edgV.numel())
            s = _ffi.CSR(nv, nu, m, offV.data_ptr(), edgV.data_ptr(), offU.data_ptr(), edgU.data_ptr())
            ctx.check(lib.pb_graph_from_device(ctx.handle, C.byref(s), C.byref(self._h)), "pb_graph_from_device")
            self.nv, self.nu, self.m = nv, nu, m

    @classmethod
    def _adopt(cls, ctx: Context, handle) -> "DeviceGraph":
        dg = cls.__new__(cls)
        dg.ctx, dg._h = ctx, handle
        nv, nu, m = C.c_int64(), C.c_int64(), C.c_int64()
        ctx.check(ctx._lib.pb_graph_dims(handle, C.byref(nv), C.byref(nu), C.byref(m)), "pb_graph_dims")
        dg.nv, dg.nu, dg.m = nv.value, nu.value, m.value
        return dg

    def close(self):
        if self._h:
            self.ctx._lib.pb_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def download(self) -> BipartiteGraph:
        """The graph copied back to host memory."""
        s = _ffi.CSR()
        self.ctx.check(self.ctx._lib.pb_graph_download(self._h, C.byref(s)), "pb_graph_download")
        return BipartiteGraph._from_owned(s)


def graph_from_text(ctx: Context, data) -> DeviceGraph:
    """readBipartite on the device: `data` is the AdjacencyHypergraph text as bytes (host) or a
    torch uint8 CUDA tensor; tokenised, parsed and validated by GPU kernels."""
    h = C.c_void_p()
    if isinstance(data, (bytes, bytearray)):
        buf = C.create_string_buffer(bytes(data), len(data))
        ctx.check(ctx._lib.pb_graph_parse_text(ctx.handle, buf, len(data), C.byref(h)), "pb_graph_parse_text")
    else:
        import torch
        torch.cuda.synchronize()
        ctx.check(ctx._lib.pb_graph_parse_text(ctx.handle, data.data_ptr(), data.numel(), C.byref(h)),
                  "pb_graph_parse_text")
    return DeviceGraph._adopt(ctx, h)


def gen_rmat_device(ctx: Context, log_nv: int, log_nu: int, m: int, a: float, b: float, c: float, d: float,
                    seed: int) -> DeviceGraph:
    """The graph of BipartiteGraph.rmat (same arguments) generated on the device."""
    h = C.c_void_p()
    ctx.check(ctx._lib.pb_gen_rmat_device(ctx.handle, log_nv, log_nu, m, a, b, c, d, seed, C.byref(h)),
              "pb_gen_rmat_device")
    return DeviceGraph._adopt(ctx, h)


def read_text_device(ctx: Context, path: str) -> DeviceGraph:
    """An AdjacencyHypergraph file read into pinned memory and parsed on the device."""
    h = C.c_void_p()
    ctx.check(ctx._lib.pb_graph_read_text(ctx.handle, path.encode(), C.byref(h)), "pb_graph_read_text")
    return DeviceGraph._adopt(ctx, h)


def _ptr(a):
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _out(n, out):
    if out is not None:
        return out
    return np.zeros(max(n, 1), dtype=np.int64)


def cmp_wedge_counts(dg: DeviceGraph):
    uv, w = C.c_int32(), C.c_int64()
    dg.ctx.check(dg.ctx._lib.pb_cmp_wedge_counts(dg.ctx.handle, dg.handle, C.byref(uv), C.byref(w)),
                 "pb_cmp_wedge_counts")
    return bool(uv.value), int(w.value)


def edge_to_idxs(dg: DeviceGraph, use_v: bool):
    """edgeToIdxs (butterfly_utils.h:2034-2062): for every edge in the use_v orientation, its
    position in the other orientation's lists."""
    eti = np.zeros(max(dg.m, 1), dtype=np.uint32)
    dg.ctx.check(dg.ctx._lib.pb_edge_to_idxs(dg.ctx.handle, dg.handle, int(use_v), eti.ctypes.data),
                 "pb_edge_to_idxs")
    return eti[:dg.m]


def idxs_to_edge(dg: DeviceGraph, use_v: bool):
    """idxsToEdge (butterfly_utils.h:2065-2067): edgeToIdxs of the other orientation."""
    return edge_to_idxs(dg, not use_v)


def count(dg: DeviceGraph, count_type="SERIAL", rank_type="ADEG", use_v=None, out=None, **kw):
    """Per-vertex butterfly counts of the count side (original vertex ids)."""
    if use_v is None:
        use_v = cmp_wedge_counts(dg)[0]
    n = dg.nu if use_v else dg.nv
    res = _out(n, out)
    o = make_opts(count_type, rank_type, per="VERT", use_v=use_v, **kw)
    dg.ctx.check(dg.ctx._lib.pb_count_vert(dg.ctx.handle, dg.handle, C.byref(o), _ptr(res)), "pb_count_vert")
    return res[:n] if out is None else res


def count_e(dg: DeviceGraph, count_type="SERIAL", rank_type="ADEG", use_v=None, out=None, **kw):
    """Per-edge butterfly counts, indexed like the reference's CountE result."""
    if use_v is None:
        use_v = cmp_wedge_counts(dg)[0]
    res = _out(dg.m, out)
    o = make_opts(count_type, rank_type, per="EDGE", use_v=use_v, **kw)
    dg.ctx.check(dg.ctx._lib.pb_count_edge(dg.ctx.handle, dg.handle, C.byref(o), _ptr(res)), "pb_count_edge")
    return res[:dg.m] if out is None else res


def count_total(dg: DeviceGraph, count_type="SERIAL", rank_type="ADEG", use_v=None, **kw) -> int:
    res = np.zeros(1, dtype=np.int64)
    o = make_opts(count_type, rank_type, per="TOTAL", use_v=use_v, **kw)
    dg.ctx.check(dg.ctx._lib.pb_count_total(dg.ctx.handle, dg.handle, C.byref(o), res.ctypes.data), "pb_count_total")
    return int(res[0])


def peel(dg: DeviceGraph, counts, peel_type="BATCHS", use_v=None, out=None, **kw):
    """Tip numbers from per-vertex counts."""
    if use_v is None:
        use_v = cmp_wedge_counts(dg)[0]
    n = dg.nu if use_v else dg.nv
    c = counts if not isinstance(counts, np.ndarray) else np.ascontiguousarray(counts, dtype=np.int64)
    res = _out(n, out)
    o = make_opts(peel_type=peel_type, per="VERT", use_v=use_v, **kw)
    dg.ctx.check(dg.ctx._lib.pb_peel_vert(dg.ctx.handle, dg.handle, C.byref(o), _ptr(c), _ptr(res)), "pb_peel_vert")
    return res[:n] if out is None else res


def peel_e(dg: DeviceGraph, ecounts, peel_type="BATCHS", use_v=None, out=None, **kw):
    """Wing numbers from per-edge counts."""
    if use_v is None:
        use_v = cmp_wedge_counts(dg)[0]
    c = ecounts if not isinstance(ecounts, np.ndarray) else np.ascontiguousarray(ecounts, dtype=np.int64)
    res = _out(dg.m, out)
    o = make_opts(peel_type=peel_type, per="EDGE", use_v=use_v, **kw)
    dg.ctx.check(dg.ctx._lib.pb_peel_edge(dg.ctx.handle, dg.handle, C.byref(o), _ptr(c), _ptr(res)), "pb_peel_edge")
    return res[:dg.m] if out is None else res


def count_batch(dgs, count_type="BATCHS", rank_type="ADEG", **kw):
    """Per-vertex counts of several graphs in one pass (each with its own count side)."""
    k = len(dgs)
    sides = [(dg.nu if cmp_wedge_counts(dg)[0] else dg.nv) for dg in dgs]
    outs = [np.zeros(max(n, 1), dtype=np.int64) for n in sides]
    ctx = dgs[0].ctx
    hs = (C.c_void_p * k)(*[dg.handle for dg in dgs])
    ps = (C.c_void_p * k)(*[o.ctypes.data for o in outs])
    o = make_opts(count_type, rank_type, per="VERT", **kw)
    ctx.check(ctx._lib.pb_count_vert_batch(ctx.handle, hs, k, C.byref(o), ps), "pb_count_vert_batch")
    return [out[:n] for out, n in zip(outs, sides)]


def peel_batch(dgs, counts, peel_type="BATCHS", **kw):
    """Tip numbers of several graphs in one persistent launch."""
    k = len(dgs)
    cs = [np.ascontiguousarray(c, dtype=np.int64) for c in counts]
    tips = [np.zeros(max(c.size, 1), dtype=np.int64) for c in cs]
    ctx = dgs[0].ctx
    hs = (C.c_void_p * k)(*[dg.handle for dg in dgs])
    pc = (C.c_void_p * k)(*[c.ctypes.data if c.size else None for c in cs])
    pt = (C.c_void_p * k)(*[t.ctypes.data for t in tips])
    o = make_opts(peel_type=peel_type, per="VERT", **kw)
    ctx.check(ctx._lib.pb_peel_vert_batch(ctx.handle, hs, k, C.byref(o), pc, pt), "pb_peel_vert_batch")
    return [t[:c.size] for t, c in zip(tips, cs)]


class BatchGraph:
    """k graphs planned as one CUDA graph (pb_batch): every run() replays ranking, per-vertex
    counting and tip peeling of the whole batch and returns (counts, tips) per graph."""

    def __init__(self, dgs, count_type="BATCHS", rank_type="ADEG", **kw):
        self.ctx = dgs[0].ctx
        self.sides = [(dg.nu if cmp_wedge_counts(dg)[0] else dg.nv) for dg in dgs]
        self._h = C.c_void_p()
        k = len(dgs)
        hs = (C.c_void_p * k)(*[dg.handle for dg in dgs])
        o = make_opts(count_type, rank_type, per="VERT", **kw)
        self.ctx.check(self.ctx._lib.pb_batch_create(self.ctx.handle, hs, k, C.byref(o), C.byref(self._h)),
                       "pb_batch_create")
        self.counts = [np.zeros(max(n, 1), dtype=np.int64) for n in self.sides]
        self.tips = [np.zeros(max(n, 1), dtype=np.int64) for n in self.sides]

    def run(self, copy_out=True):
        k = len(self.sides)
        pc = (C.c_void_p * k)(*[c.ctypes.data for c in self.counts]) if copy_out else None
        pt = (C.c_void_p * k)(*[t.ctypes.data for t in self.tips]) if copy_out else None
        self.ctx.check(self.ctx._lib.pb_batch_run(self.ctx.handle, self._h, pc, pt), "pb_batch_run")
        return [c[:n] for c, n in zip(self.counts, self.sides)], [t[:n] for t, n in zip(self.tips, self.sides)]

    def close(self):
        if self._h:
            self.ctx._lib.pb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SchedModel:
    """The learned scheduler's cost models (a pb_sched_model): one for the per-item aggregation
    modes of counting, one for the work-unit setting of peeling."""

    COUNT, PEEL = _ffi.SCHED_COUNT, _ffi.SCHED_PEEL

    def __init__(self, ctx: Context, seed: int = 1):
        self.ctx = ctx
        self._h = C.c_void_p()
        ctx.check(ctx._lib.pb_sched_model_create(ctx.handle, seed, C.byref(self._h)), "pb_sched_model_create")

    def close(self):
        if self._h:
            self.ctx._lib.pb_sched_model_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def train(self, target: int, X, y, epochs=60, batch=1024, lr=3e-3) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, _ffi.SCHED_FEATURES)
        y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1)
        assert X.shape[0] == y.shape[0]
        mse = C.c_float()
        self.ctx.check(self.ctx._lib.pb_sched_train(self.ctx.handle, self._h, target, X.ctypes.data, y.ctypes.data,
                                                    X.shape[0], epochs, batch, lr, C.byref(mse)), "pb_sched_train")
        return float(mse.value)

    def predict(self, target: int, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, _ffi.SCHED_FEATURES)
        y = np.zeros(X.shape[0], dtype=np.float32)
        self.ctx.check(self.ctx._lib.pb_sched_predict(self.ctx.handle, self._h, target, X.ctypes.data, X.shape[0],
                                                      y.ctypes.data), "pb_sched_predict")
        return y

    def save(self, path: str):
        self.ctx.check(self.ctx._lib.pb_sched_save(self.ctx.handle, self._h, path.encode()), "pb_sched_save")

    def load(self, path: str):
        self.ctx.check(self.ctx._lib.pb_sched_load(self.ctx.handle, self._h, path.encode()), "pb_sched_load")

    def attach(self):
        """LEARNED calls on the model's context use this model from now on."""
        self.ctx.check(self.ctx._lib.pb_ctx_set_sched_model(self.ctx.handle, self._h), "pb_ctx_set_sched_model")


def detach_sched_model(ctx: Context):
    ctx.check(ctx._lib.pb_ctx_set_sched_model(ctx.handle, None), "pb_ctx_set_sched_model")


def trace_set(ctx: Context, mode: str = "plain", seed: int = 0):
    """Trace logging of scheduler rows on ctx: mode "off", "plain" or "explore"."""
    m = {"off": _ffi.TRACE_OFF, "plain": _ffi.TRACE_PLAIN, "explore": _ffi.TRACE_EXPLORE}[mode]
    ctx.check(ctx._lib.pb_trace_set(ctx.handle, m, seed), "pb_trace_set")


def trace_rows(ctx: Context, target: int):
    """The rows logged for target (SchedModel.COUNT or .PEEL): X [n, 16] and y [n] (log2 time)."""
    n = C.c_int64()
    ctx.check(ctx._lib.pb_trace_rows(ctx.handle, target, None, None, 0, C.byref(n)), "pb_trace_rows")
    X = np.zeros((n.value, _ffi.SCHED_FEATURES), dtype=np.float32)
    y = np.zeros(n.value, dtype=np.float32)
    if n.value:
        ctx.check(ctx._lib.pb_trace_rows(ctx.handle, target, X.ctypes.data, y.ctypes.data, n.value, C.byref(n)),
                  "pb_trace_rows")
    return X, y


def trace_clear(ctx: Context):
    ctx.check(ctx._lib.pb_trace_clear(ctx.handle), "pb_trace_clear")


def tc_gemm_bf16(ctx: Context, A, B):
    """D = A @ B.T on the tensor cores for torch bf16 CUDA tensors A [M, K] and B [N, K]
    (any strides); returns an fp32 [M, N] tensor."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    D = torch.empty((M, N), dtype=torch.float32, device=A.device)
    torch.cuda.synchronize()  # the context's stream is not ordered after torch's
    ctx.check(ctx._lib.pb_tc_gemm_bf16(ctx.handle, M, N, K, A.data_ptr(), A.stride(0), A.stride(1), B.data_ptr(),
                                       B.stride(0), B.stride(1), D.data_ptr(), N), "pb_tc_gemm_bf16")
    return D
