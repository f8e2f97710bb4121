"""CPU checkers for the CUDA path (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm import this
package.  It wraps:
  * oracle/_build/libpboracle.so — the C restatement in pb_oracle.c (functions cite the
    reference file:line they follow), and
  * oracle/_ref/ref_harness_{omp,ser} — the reference itself, compiled from its own sources by
    oracle/Makefile (only where the reference tree is present at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libpboracle.so")
HARNESS_OMP = os.path.join(HERE, "_ref", "ref_harness_omp")
HARNESS_SER = os.path.join(HERE, "_ref", "ref_harness_ser")
HARNESS_FWD = os.path.join(HERE, "_ref", "ref_harness_fwd")  # built without INVERSE

RANK = {"SIDE": 0, "COCORE": 1, "ACOCORE": 2, "DEG": 3, "ADEG": 4}
PER = {"VERT": 0, "EDGE": 1, "TOTAL": 2}


class _G(C.Structure):
    _fields_ = [("nv", C.c_int64), ("nu", C.c_int64), ("m", C.c_int64), ("offV", C.c_void_p),
                ("edgV", C.c_void_p), ("offU", C.c_void_p), ("edgU", C.c_void_p)]


_lib = None


def build() -> None:
    """Builds the C restatement and, when the reference tree is present, the reference harness."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        L = C.CDLL(ORACLE_LIB)
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        L.pbo_cmp_wedge_counts.restype = I64
        L.pbo_cmp_wedge_counts.argtypes = [C.POINTER(_G), C.POINTER(I32), C.POINTER(I64), C.POINTER(I64)]
        L.pbo_vertex_order.restype = None
        L.pbo_vertex_order.argtypes = [C.POINTER(_G), I32, I32, P, P]
        L.pbo_edge_to_idxs.restype = None
        L.pbo_edge_to_idxs.argtypes = [C.POINTER(_G), I32, P]
        L.pbo_count.restype = I64
        L.pbo_count.argtypes = [C.POINTER(_G), I32, I32, I32, P]
        L.pbo_peel_vert.restype = I64
        L.pbo_peel_vert.argtypes = [C.POINTER(_G), I32, P, P]
        L.pbo_peel_edge.restype = I64
        L.pbo_peel_edge.argtypes = [C.POINTER(_G), I32, P, P]
        L.pbo_peel_edge_fast.restype = I64
        L.pbo_peel_edge_fast.argtypes = [C.POINTER(_G), I32, P, P]
        L.pbo_ranked_wedges.restype = I64
        L.pbo_ranked_wedges.argtypes = [C.POINTER(_G), I32, I32]
        _lib = L
    return _lib


def _gs(g):
    return _G(g.nv, g.nu, g.m, g.offsetsV.ctypes.data, g.edgesV.ctypes.data, g.offsetsU.ctypes.data,
              g.edgesU.ctypes.data)


def cmp_wedge_counts(g):
    """(use_v, num_wedges, W_V, W_U) as cmpWedgeCounts (butterfly_utils.h:1080-1086)."""
    uv, wv, wu = C.c_int32(), C.c_int64(), C.c_int64()
    w = lib().pbo_cmp_wedge_counts(C.byref(_gs(g)), C.byref(uv), C.byref(wv), C.byref(wu))
    return bool(uv.value), int(w), int(wv.value), int(wu.value)


def count(g, per="VERT", rank="ADEG", use_v=None):
    """Returns (result, W_rank).  VERT: int64[nCount]; EDGE: int64[m]; TOTAL: int."""
    if use_v is None:
        use_v = cmp_wedge_counts(g)[0]
    if per == "VERT":
        out = np.zeros((g.nu if use_v else g.nv) or 1, dtype=np.int64)
    elif per == "EDGE":
        out = np.zeros(max(g.m, 1), dtype=np.int64)
    else:
        out = np.zeros(1, dtype=np.int64)
    w = lib().pbo_count(C.byref(_gs(g)), RANK[rank], PER[per], int(use_v), out.ctypes.data)
    if per == "VERT":
        out = out[:(g.nu if use_v else g.nv)]
    elif per == "EDGE":
        out = out[:g.m]
    else:
        return int(out[0]), int(w)
    return out, int(w)


def ranked_wedges(g, rank="ADEG", use_v=None):
    if use_v is None:
        use_v = cmp_wedge_counts(g)[0]
    return int(lib().pbo_ranked_wedges(C.byref(_gs(g)), RANK[rank], int(use_v)))


def vertex_order(g, rank="ADEG", use_v=None):
    if use_v is None:
        use_v = cmp_wedge_counts(g)[0]
    order = np.zeros(max(g.n, 1), dtype=np.uint32)
    rk = np.zeros(max(g.n, 1), dtype=np.uint32)
    lib().pbo_vertex_order(C.byref(_gs(g)), RANK[rank], int(use_v), order.ctypes.data, rk.ctypes.data)
    return order[:g.n], rk[:g.n]


def edge_to_idxs(g, use_v):
    eti = np.zeros(max(g.m, 1), dtype=np.uint32)
    lib().pbo_edge_to_idxs(C.byref(_gs(g)), int(use_v), eti.ctypes.data)
    return eti[:g.m]


def peel_vert(g, counts, use_v=None):
    """Tip numbers (64-bit buckets).  Returns (tip, rounds)."""
    if use_v is None:
        use_v = cmp_wedge_counts(g)[0]
    c = np.ascontiguousarray(counts, dtype=np.int64)
    d = np.zeros(max(c.size, 1), dtype=np.int64)
    r = lib().pbo_peel_vert(C.byref(_gs(g)), int(use_v), c.ctypes.data, d.ctypes.data)
    return d[:c.size], int(r)


def peel_edge(g, ecounts, use_v=None):
    """Wing numbers.  Returns (wing, rounds)."""
    if use_v is None:
        use_v = cmp_wedge_counts(g)[0]
    c = np.ascontiguousarray(ecounts, dtype=np.int64)
    d = np.zeros(max(c.size, 1), dtype=np.int64)
    r = lib().pbo_peel_edge(C.byref(_gs(g)), int(use_v), c.ctypes.data, d.ctypes.data)
    return d[:c.size], int(r)


def peel_edge_fast(g, ecounts, use_v=None):
    """Wing numbers by the bucket-queue, multi-threaded restatement (pb_oracle_fast.c): same
    results as peel_edge, fast enough for the 2^24-edge benchmark graph.  Returns (wing, rounds)."""
    if use_v is None:
        use_v = cmp_wedge_counts(g)[0]
    c = np.ascontiguousarray(ecounts, dtype=np.int64)
    d = np.zeros(max(c.size, 1), dtype=np.int64)
    r = lib().pbo_peel_edge_fast(C.byref(_gs(g)), int(use_v), c.ctypes.data, d.ctypes.data)
    return d[:c.size], int(r)


# ---- the reference itself ------------------------------------------------------------------
def have_reference(serial: bool = False) -> bool:
    return os.path.exists(HARNESS_SER if serial else HARNESS_OMP)


def run_reference(g, per="VERT", count_type="BATCHS", rank="ADEG", peel="NONE", rounds=1, threads=None,
                  serial=False, timeout=None, forward=False):
    """Runs the compiled reference on g.  Returns dict(use_v, w_side, total, count, peel, count_s, peel_s).
    forward: the build without INVERSE (the reference's other wedge direction)."""
    exe = HARNESS_FWD if forward else (HARNESS_SER if serial else HARNESS_OMP)
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as td:
        gp = os.path.join(td, "g.bin")
        g.save_bin(gp)
        outp = os.path.join(td, "out")
        r = subprocess.run([exe, gp, per, count_type, rank, peel, outp, str(rounds)], capture_output=True,
                           text=True, env=env, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]} {r.stdout[-2000:]}")
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("use_v=")][-1]
        kv = dict(tok.split("=") for tok in line.split())
        res = {"use_v": bool(int(kv["use_v"])), "w_side": int(kv["w_side"]), "total": int(kv["total"]),
               "count_s": float(kv["count_s"]), "peel_s": float(kv["peel_s"]), "stdout": r.stdout}
        res["count"] = np.fromfile(outp + ".count", dtype=np.int64)
        res["peel"] = np.fromfile(outp + ".peel", dtype=np.int64) if peel != "NONE" else None
        return res
