"""ctypes binding of libpbgpu.so (the C ABI declared in include/parbutterfly_b200.h).

The library is built in-tree (parbutterfly_b200/_lib/libpbgpu.so).  There is no fallback:
if the library is missing, every call raises ``PBLibraryMissing``.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpbgpu.so")

PB_OK, PB_EINVAL, PB_ENOMEM, PB_ETOOBIG, PB_ETIMEOUT, PB_ECUDA, PB_EUNSUPPORTED, PB_EIO = range(8)
STATUS_NAMES = {
    PB_OK: "PB_OK", PB_EINVAL: "PB_EINVAL", PB_ENOMEM: "PB_ENOMEM", PB_ETOOBIG: "PB_ETOOBIG",
    PB_ETIMEOUT: "PB_ETIMEOUT", PB_ECUDA: "PB_ECUDA", PB_EUNSUPPORTED: "PB_EUNSUPPORTED", PB_EIO: "PB_EIO",
}

# Exported symbols, exactly those declared in include/parbutterfly_b200.h.
EXPORTS = [
    "pb_abi_version", "pb_opts_default", "pb_ctx_create", "pb_ctx_destroy", "pb_last_error",
    "pb_get_stats", "pb_kernel_launches", "pb_graph_upload", "pb_graph_from_device", "pb_graph_destroy",
    "pb_graph_dims", "pb_cmp_wedge_counts", "pb_edge_to_idxs", "pb_count_vert", "pb_count_edge",
    "pb_count_total", "pb_peel_vert", "pb_peel_edge", "pb_csr_free", "pb_read_adjacency_hypergraph",
    "pb_write_adjacency_hypergraph", "pb_csr_validate", "pb_gen_uniform", "pb_gen_rmat",
    "pb_gen_powerlaw_u", "pb_gen_zipf", "pb_gen_batch_member", "pb_count_total_noalloc",
    "pb_count_vert_batch", "pb_peel_vert_batch", "pb_sched_model_create", "pb_sched_model_destroy",
    "pb_sched_train", "pb_sched_predict", "pb_sched_save", "pb_sched_load", "pb_ctx_set_sched_model",
    "pb_trace_set", "pb_trace_rows", "pb_trace_clear", "pb_tc_gemm_bf16", "pb_batch_create", "pb_batch_run",
    "pb_batch_destroy", "pb_graph_parse_text", "pb_graph_read_text", "pb_read_binary_hypergraph",
    "pb_write_binary_hypergraph", "pb_gen_rmat_device", "pb_graph_download", "pb_read_konect",
    "pb_sparsify_bipartite", "pb_sparse_estimate",
]

SCHED_FEATURES = 16
SCHED_WING_CANDIDATES = 3
SCHED_TIP_CANDIDATES = 48
SCHED_COUNT, SCHED_PEEL = 0, 1
TRACE_OFF, TRACE_PLAIN, TRACE_EXPLORE = 0, 1, 2
SPARSE = {"NONE": 0, "COLOR": 1, "EDGE": 2}  # SparseType, butterfly_utils.h:28


class PBLibraryMissing(RuntimeError):
    pass


class PBError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


class Opts(C.Structure):
    _fields_ = [
        ("count_type", C.c_int32), ("rank_type", C.c_int32), ("peel_type", C.c_int32),
        ("per_type", C.c_int32), ("max_wedges", C.c_int64), ("max_array_size", C.c_int64),
        ("sched", C.c_int32), ("autotune", C.c_int32), ("use_v", C.c_int32), ("peel_parts", C.c_int32),
    ]


class CSR(C.Structure):
    _fields_ = [
        ("nv", C.c_int64), ("nu", C.c_int64), ("m", C.c_int64),
        ("offsetsV", C.c_void_p), ("edgesV", C.c_void_p),
        ("offsetsU", C.c_void_p), ("edgesU", C.c_void_p),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("w_side", C.c_int64), ("w_rank", C.c_int64), ("use_v", C.c_int32), ("n_big", C.c_int32),
        ("ms_rank", C.c_double), ("ms_relabel", C.c_double), ("ms_scan", C.c_double),
        ("ms_count", C.c_double), ("ms_convert", C.c_double), ("ms_peel", C.c_double),
        ("peel_rounds", C.c_int64), ("peel_work", C.c_int64), ("ms_agg_kernel", C.c_double),
        ("sched_used", C.c_int32), ("sched_choice", C.c_int32), ("sched_items", C.c_int64),
        ("ms_sched", C.c_double), ("sched_pred", C.c_double), ("sched_meas", C.c_double),
        ("sched_mae_log2", C.c_double), ("count_smem_bytes", C.c_int32), ("count_blocks_per_sm", C.c_int32),
        ("count_small_w", C.c_int32), ("autotuned", C.c_int32),
        ("peel_parts", C.c_int64), ("peel_coarse_rounds", C.c_int64), ("peel_fine_rounds_max", C.c_int64),
    ]


_lib = None


def lib():
    """Loads libpbgpu.so once; raises PBLibraryMissing when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PBLibraryMissing(
            f"{LIB_PATH} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C parbutterfly_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    P, I32, I64, U64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_double
    S = C.c_int  # pb_status
    sig = {
        "pb_abi_version": (C.c_int, []),
        "pb_opts_default": (None, [C.POINTER(Opts)]),
        "pb_ctx_create": (S, [C.c_int, P, C.POINTER(P)]),
        "pb_ctx_destroy": (S, [P]),
        "pb_last_error": (C.c_char_p, [P]),
        "pb_get_stats": (S, [P, C.POINTER(Stats)]),
        "pb_kernel_launches": (I64, [P]),
        "pb_graph_upload": (S, [P, C.POINTER(CSR), C.POINTER(P)]),
        "pb_graph_from_device": (S, [P, C.POINTER(CSR), C.POINTER(P)]),
        "pb_graph_destroy": (S, [P]),
        "pb_graph_dims": (S, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
        "pb_cmp_wedge_counts": (S, [P, P, C.POINTER(I32), C.POINTER(I64)]),
        "pb_edge_to_idxs": (S, [P, P, I32, P]),
        "pb_count_vert": (S, [P, P, C.POINTER(Opts), P]),
        "pb_count_edge": (S, [P, P, C.POINTER(Opts), P]),
        "pb_count_total": (S, [P, P, C.POINTER(Opts), P]),
        "pb_peel_vert": (S, [P, P, C.POINTER(Opts), P, P]),
        "pb_peel_edge": (S, [P, P, C.POINTER(Opts), P, P]),
        "pb_csr_free": (None, [C.POINTER(CSR)]),
        "pb_read_adjacency_hypergraph": (S, [C.c_char_p, C.POINTER(CSR)]),
        "pb_write_adjacency_hypergraph": (S, [C.c_char_p, C.POINTER(CSR)]),
        "pb_csr_validate": (S, [C.POINTER(CSR), C.c_char_p, C.c_size_t]),
        "pb_gen_uniform": (S, [I64, I64, I64, U64, C.POINTER(CSR)]),
        "pb_gen_rmat": (S, [I32, I32, I64, D, D, D, D, U64, C.POINTER(CSR)]),
        "pb_gen_powerlaw_u": (S, [I64, I64, I64, D, I64, U64, C.POINTER(CSR)]),
        "pb_gen_zipf": (S, [I64, I64, I64, D, U64, C.POINTER(CSR)]),
        "pb_gen_batch_member": (S, [I32, C.POINTER(CSR)]),
        "pb_gen_rmat_device": (S, [P, I32, I32, I64, D, D, D, D, U64, C.POINTER(P)]),
        "pb_graph_download": (S, [P, C.POINTER(CSR)]),
        "pb_read_konect": (S, [C.c_char_p, C.POINTER(CSR)]),
        "pb_sparsify_bipartite": (S, [C.POINTER(CSR), I32, I64, I64, C.POINTER(CSR)]),
        "pb_sparse_estimate": (I64, [I64, I32, I64]),
        "pb_count_total_noalloc": (S, [C.POINTER(CSR), P, P, C.c_char_p, C.c_size_t]),
        "pb_count_vert_batch": (S, [P, C.POINTER(P), I32, C.POINTER(Opts), C.POINTER(P)]),
        "pb_peel_vert_batch": (S, [P, C.POINTER(P), I32, C.POINTER(Opts), C.POINTER(P), C.POINTER(P)]),
        "pb_sched_model_create": (S, [P, U64, C.POINTER(P)]),
        "pb_sched_model_destroy": (S, [P]),
        "pb_sched_train": (S, [P, P, I32, P, P, I64, I32, I32, C.c_float, C.POINTER(C.c_float)]),
        "pb_sched_predict": (S, [P, P, I32, P, I64, P]),
        "pb_sched_save": (S, [P, P, C.c_char_p]),
        "pb_sched_load": (S, [P, P, C.c_char_p]),
        "pb_ctx_set_sched_model": (S, [P, P]),
        "pb_trace_set": (S, [P, I32, U64]),
        "pb_trace_rows": (S, [P, I32, P, P, I64, C.POINTER(I64)]),
        "pb_trace_clear": (S, [P]),
        "pb_tc_gemm_bf16": (S, [P, I64, I32, I64, P, I64, I64, P, I64, I64, P, I64]),
        "pb_batch_create": (S, [P, C.POINTER(P), I32, C.POINTER(Opts), C.POINTER(P)]),
        "pb_batch_run": (S, [P, P, C.POINTER(P), C.POINTER(P)]),
        "pb_batch_destroy": (S, [P]),
        "pb_graph_parse_text": (S, [P, P, C.c_size_t, C.POINTER(P)]),
        "pb_graph_read_text": (S, [P, C.c_char_p, C.POINTER(P)]),
        "pb_read_binary_hypergraph": (S, [C.c_char_p, C.POINTER(CSR)]),
        "pb_write_binary_hypergraph": (S, [C.c_char_p, C.POINTER(CSR)]),
    }
    for name, (res, args) in sig.items():
        try:
            f = getattr(L, name)
        except AttributeError:
            continue  # reported by missing_exports(); calling it raises AttributeError
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def missing_exports() -> list:
    """Symbols declared in include/parbutterfly_b200.h that the built library lacks."""
    L = lib()
    return [name for name in EXPORTS if not hasattr(L, name)]


def check(status: int, ctx=None, what: str = "") -> None:
    if status != PB_OK:
        msg = what
        if ctx:
            m = lib().pb_last_error(ctx)
            if m:
                msg = f"{what}: {m.decode()}" if what else m.decode()
        raise PBError(status, msg)
