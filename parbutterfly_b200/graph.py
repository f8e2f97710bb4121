"""Host-side bipartite graph in the reference's two-sided CSR layout (bipartiteCSR,
apps/hyper/butterfly_utils.h:184-197): offsetsV[nv+1], edgesV[m], offsetsU[nu+1], edgesU[m],
uint32 offsets and ids, every adjacency list sorted ascending.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _ffi


@dataclass
class BipartiteGraph:
    nv: int
    nu: int
    offsetsV: np.ndarray
    edgesV: np.ndarray
    offsetsU: np.ndarray
    edgesU: np.ndarray

    @property
    def m(self) -> int:
        return int(self.edgesV.shape[0])

    @property
    def n(self) -> int:
        return self.nv + self.nu

    def csr_struct(self) -> _ffi.CSR:
        """ctypes view (the arrays must stay alive while the struct is used)."""
        for a in (self.offsetsV, self.edgesV, self.offsetsU, self.edgesU):
            assert a.dtype == np.uint32 and a.flags.c_contiguous
        return _ffi.CSR(self.nv, self.nu, self.m, self.offsetsV.ctypes.data, self.edgesV.ctypes.data,
                        self.offsetsU.ctypes.data, self.edgesU.ctypes.data)

    def validate(self) -> None:
        s = self.csr_struct()
        buf = C.create_string_buffer(512)
        st = _ffi.lib().pb_csr_validate(C.byref(s), buf, 512)
        if st != _ffi.PB_OK:
            raise _ffi.PBError(st, buf.value.decode())

    def degrees(self):
        return np.diff(self.offsetsV.astype(np.int64)), np.diff(self.offsetsU.astype(np.int64))

    @property
    def nbytes(self) -> int:
        return sum(a.nbytes for a in (self.offsetsV, self.edgesV, self.offsetsU, self.edgesU))

    # ---- construction -------------------------------------------------------------------
    @staticmethod
    def from_edges(nv: int, nu: int, v, u) -> "BipartiteGraph":
        """Builds both sorted sides from an edge list (duplicates removed)."""
        v = np.asarray(v, dtype=np.int64)
        u = np.asarray(u, dtype=np.int64)
        if v.size:
            if v.min() < 0 or v.max() >= nv or u.min() < 0 or u.max() >= nu:
                raise ValueError("edge endpoint out of range")
        keys = np.unique(v * nu + u)
        v = keys // nu
        u = keys % nu
        offV = np.zeros(nv + 1, dtype=np.uint32)
        np.cumsum(np.bincount(v, minlength=nv), out=offV[1:])
        edgV = u.astype(np.uint32)
        order = np.lexsort((v, u))
        offU = np.zeros(nu + 1, dtype=np.uint32)
        np.cumsum(np.bincount(u, minlength=nu), out=offU[1:])
        edgU = v[order].astype(np.uint32)
        return BipartiteGraph(nv, nu, offV, edgV, offU, edgU)

    def edge_list(self):
        """(v, u) arrays in edgesV order."""
        dv, _ = self.degrees()
        v = np.repeat(np.arange(self.nv, dtype=np.int64), dv)
        return v, self.edgesV.astype(np.int64)

    @staticmethod
    def _from_owned(s: _ffi.CSR) -> "BipartiteGraph":
        nv, nu, m = int(s.nv), int(s.nu), int(s.m)

        def take(ptr, n):
            if n == 0:
                return np.zeros(0, dtype=np.uint32)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint32)), shape=(n,)).copy()

        g = BipartiteGraph(nv, nu, take(s.offsetsV, nv + 1), take(s.edgesV, m), take(s.offsetsU, nu + 1),
                           take(s.edgesU, m))
        _ffi.lib().pb_csr_free(C.byref(s))
        return g

    # ---- generators (seeded, C++ side) ------------------------------------------------------
    @staticmethod
    def uniform(nv: int, nu: int, m: int, seed: int) -> "BipartiteGraph":
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_gen_uniform(nv, nu, m, seed, C.byref(s)), what="pb_gen_uniform")
        return BipartiteGraph._from_owned(s)

    @staticmethod
    def rmat(log_nv: int, log_nu: int, m: int, a: float, b: float, c: float, d: float, seed: int):
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_gen_rmat(log_nv, log_nu, m, a, b, c, d, seed, C.byref(s)), what="pb_gen_rmat")
        return BipartiteGraph._from_owned(s)

    @staticmethod
    def powerlaw_u(nv: int, nu: int, m: int, alpha: float, dmax: int, seed: int):
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_gen_powerlaw_u(nv, nu, m, alpha, dmax, seed, C.byref(s)), what="pb_gen_powerlaw_u")
        return BipartiteGraph._from_owned(s)

    @staticmethod
    def zipf(nv: int, nu: int, m: int, s_exp: float, seed: int):
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_gen_zipf(nv, nu, m, s_exp, seed, C.byref(s)), what="pb_gen_zipf")
        return BipartiteGraph._from_owned(s)

    @staticmethod
    def batch_member(g: int):
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_gen_batch_member(g, C.byref(s)), what="pb_gen_batch_member")
        return BipartiteGraph._from_owned(s)

    # ---- files -------------------------------------------------------------------------------
    def save_bin(self, path: str) -> None:
        """Binary layout read by oracle/ref_harness.cpp: b"PBBGRAPH", int64 nv, nu, m, then the
        four uint32 arrays."""
        with open(path, "wb") as f:
            f.write(b"PBBGRAPH")
            f.write(np.array([self.nv, self.nu, self.m], dtype=np.int64).tobytes())
            for a in (self.offsetsV, self.edgesV, self.offsetsU, self.edgesU):
                f.write(np.ascontiguousarray(a, dtype=np.uint32).tobytes())

    @staticmethod
    def load_bin(path: str) -> "BipartiteGraph":
        with open(path, "rb") as f:
            if f.read(8) != b"PBBGRAPH":
                raise ValueError("not a PBBGRAPH file")
            nv, nu, m = (int(x) for x in np.frombuffer(f.read(24), dtype=np.int64))
            arr = np.frombuffer(f.read(), dtype=np.uint32)
        o = 0
        offV = arr[o:o + nv + 1].copy(); o += nv + 1
        edgV = arr[o:o + m].copy(); o += m
        offU = arr[o:o + nu + 1].copy(); o += nu + 1
        edgU = arr[o:o + m].copy()
        return BipartiteGraph(nv, nu, offV, edgV, offU, edgU)

    def write_text(self, path: str) -> None:
        s = self.csr_struct()
        _ffi.check(_ffi.lib().pb_write_adjacency_hypergraph(os.fsencode(path), C.byref(s)), what=path)

    @staticmethod
    def read_text(path: str) -> "BipartiteGraph":
        """readBipartite (butterfly_utils.h:1008-1058)."""
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_read_adjacency_hypergraph(os.fsencode(path), C.byref(s)), what=path)
        return BipartiteGraph._from_owned(s)

    @staticmethod
    def read_konect(path: str) -> "BipartiteGraph":
        """A KONECT edge list (utils/KONECTtoHyperAdj.C semantics)."""
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_read_konect(os.fsencode(path), C.byref(s)), what=path)
        return BipartiteGraph._from_owned(s)

    def sparsify(self, sparse_type: str, denom: int = 25, seed: int = 0) -> "BipartiteGraph":
        """Sparsified copy for approximate total counts: "EDGE" (eSparseBipartite) or "COLOR"
        (clrSparseBipartite), denom = -d, seed 0 as in the reference's driver
        (butterfly_utils.h:744-996).  Scale the copy's total count with sparse_estimate."""
        s = self.csr_struct()
        o = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_sparsify_bipartite(C.byref(s), _ffi.SPARSE[sparse_type], int(denom), int(seed),
                                                     C.byref(o)), what="pb_sparsify_bipartite")
        return BipartiteGraph._from_owned(o)

    @staticmethod
    def sparse_estimate(sparse_count: int, sparse_type: str, denom: int = 25) -> int:
        """The reference's estimate from a sparsified graph's total (BipartiteButterflies.C:213-214)."""
        return int(_ffi.lib().pb_sparse_estimate(int(sparse_count), _ffi.SPARSE[sparse_type], int(denom)))

    def write_binary(self, base: str) -> None:
        """hyperAdjToBinary's layout: base.config, .vidx, .vadj, .hidx, .hadj."""
        s = self.csr_struct()
        _ffi.check(_ffi.lib().pb_write_binary_hypergraph(os.fsencode(base), C.byref(s)), what=base)

    @staticmethod
    def read_binary(base: str) -> "BipartiteGraph":
        s = _ffi.CSR()
        _ffi.check(_ffi.lib().pb_read_binary_hypergraph(os.fsencode(base), C.byref(s)), what=base)
        return BipartiteGraph._from_owned(s)


# ---- the benchmark workloads -----------------------------------------------------------------
def workload(name: str) -> BipartiteGraph:
    """Seeded synthetic stand-ins for the benchmark configurations (no public dataset is named).

    c1 : uniform 4096 x 4096, m = 131072, seed 1
    c2 : bipartite R-MAT 2^20 (V) x 2^18 (U), (a,b,c,d) = (.55,.15,.15,.15), m = 2^24, seed 2
    c3 : |U| = 1e6 power-law degrees (alpha 2.0, max degree capped at |V| = 1e5), m = 1e8, seed 3
    c5 : bipartite R-MAT 2^26 x 2^24, (.57,.19,.19,.05), m = 1e9, seed 5
    """
    if name == "c1":
        return BipartiteGraph.uniform(4096, 4096, 131072, 1)
    if name == "c2":
        return BipartiteGraph.rmat(20, 18, 1 << 24, 0.55, 0.15, 0.15, 0.15, 2)
    if name == "c3":
        return BipartiteGraph.powerlaw_u(100_000, 1_000_000, 100_000_000, 2.0, 100_000, 3)
    if name == "c5":
        return BipartiteGraph.rmat(26, 24, 1_000_000_000, 0.57, 0.19, 0.19, 0.05, 5)
    raise ValueError(name)
