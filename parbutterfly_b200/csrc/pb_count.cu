// Wedge aggregation and butterfly accumulation on the ranked CSR.
//
// Semantics (CountWorkEfficientParallel, butterfly_count.h:1218-1320; the per-edge and total
// variants butterfly_ecount.h:1334-1429 and butterfly_count_total.h:662-749): for every
// endpoint i, the wedges are (i, v, u2) with v in N(i), u2 in N(v), u2 < min(i, v); w(u2) is
// the number of wedges of i that end in u2.  Then
//   VERT : tagged endpoints i and u2 gain C(w,2); tagged centres v gain w-1 per wedge;
//   EDGE : edges (i,v) and (v,u2) gain w-1 per wedge;
//   TOTAL: the sum of C(w,2).
// Endpoint and centre are on opposite sides, so for one endpoint either the centre credits or
// the endpoint credits matter, never both.
//
// Aggregators (the multiplicity table w):
//   warp  : endpoints with W_i <= small_w; one warp, an open-addressing table in shared memory
//           (keys u2, values w), linear probing, insert by atomicCAS / atomicAdd.
//   block : larger endpoints, one CTA per endpoint taken from a global work counter; the table
//           is a dense shared-memory window over [0, i) (BATCHS-style dense counters), a
//           shared-memory hash table, or a per-CTA dense array in global scratch memory when
//           neither fits.
// The wedge list of an endpoint is flattened: each chunk of neighbours gets an inclusive scan
// of its prefix lengths, and lane/thread t locates its neighbour by a branchless binary search
// over that scan, so consecutive threads read consecutive entries of N(v) (coalesced).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "pb_engine.cuh"
#include "pb_mlp.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kWarpTable = 1024;  // slots per warp (keys + values = 8 KiB)
constexpr int kWarpsPerBlockSmall = 8;

enum Per { VERT = 0, EDGE = 1, TOTAL = 2 };

struct Params {
  const uint32_t* __restrict__ off;
  const uint32_t* __restrict__ adj;
  const uint32_t* __restrict__ pref;
  const uint32_t* __restrict__ eout;
  const int64_t* __restrict__ wsum;
  int64_t n;
  int per;
  int64_t* out;
  int64_t out_len;  // entries of out
  int64_t m2;       // slots of the ranked CSR
  uint32_t* err;    // record of the first bounds violation {code, index lo, index hi, aux}
  uint32_t* out32;  // per-edge counts accumulated in 32 bits when every count fits (else null)
  unsigned long long* mstats;  // per mode (dense, hash, hybrid, global): endpoints, wedges
  // Scheduler hooks of the block aggregator (all null on the plain path):
  const uint8_t* modes;        // modes[q]: aggregation mode of item q chosen by the scheduler
  uint8_t* mode_out;           // mode_out[q]: mode item q ran with
  unsigned long long* cycles;  // cycles[q]: SM cycles item q took (clock64, thread 0)
};

// Records the first bounds violation (checked mode only).
__device__ __noinline__ void record_violation(uint32_t* err, uint32_t code, uint64_t idx, uint32_t aux) {
  if (atomicCAS(&err[0], 0u, code) == 0u) {
    err[1] = (uint32_t)idx;
    err[2] = (uint32_t)(idx >> 32);
    err[3] = aux;
  }
}

// out[idx] += v.  Indices derived from memory are bounds-checked; a violation is recorded
// (and reported as an error by the host) instead of being accessed.
__device__ __forceinline__ void credit(const Params& P, uint64_t idx, int64_t v, uint32_t code) {
  if (idx >= (uint64_t)P.out_len) { record_violation(P.err, code, idx, 0); return; }
  if (P.out32) atomicAdd(&P.out32[idx], (uint32_t)v);  // L2-resident 32-bit accumulation
  else atomic_add_i64(&P.out[idx], v);
}

__device__ __forceinline__ bool slot_ok(const Params& P, uint64_t slot, uint32_t code) {
  if (slot >= (uint64_t)P.m2) { record_violation(P.err, code, slot, 0); return false; }
  return true;
}

// Fibonacci hashing: the high bits of key * 2^32/phi, folded into the table size.
__device__ __forceinline__ uint32_t hash_slot(uint32_t key, uint32_t mask) {
  return __umulhi(key * 0x9E3779B1u, mask + 1u) & mask;
}

// Insert-or-increment.  Tables are sized to at least twice the wedge count, so a probe
// sequence never exceeds the table size; the bound turns a broken invariant into a recorded
// error instead of an endless loop.
__device__ __forceinline__ bool table_insert(uint32_t* keys, uint32_t* vals, uint32_t mask, uint32_t key) {
  uint32_t h = hash_slot(key, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    uint32_t k = keys[h];
    if (k == key) { atomicAdd(&vals[h], 1u); return true; }
    if (k == kEmpty) {
      uint32_t prev = atomicCAS(&keys[h], kEmpty, key);
      if (prev == kEmpty || prev == key) { atomicAdd(&vals[h], 1u); return true; }
    }
    h = (h + 1) & mask;
  }
  return false;
}

__device__ __forceinline__ uint32_t table_find(const uint32_t* keys, const uint32_t* vals, uint32_t mask,
                                               uint32_t key) {
  uint32_t h = hash_slot(key, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    uint32_t k = keys[h];
    if (k == key) return vals[h];
    if (k == kEmpty) return 0;  // unreachable for keys that were inserted
    h = (h + 1) & mask;
  }
  return 0;
}

__device__ __forceinline__ uint32_t next_pow2(uint32_t x) { return x <= 1 ? 1u : 1u << (32 - __clz(x - 1)); }

// Iterates every wedge of endpoint i (slots [b, e) of the ranked CSR) with one warp.
// f(j, vt, slot2, u2t): j = slot of (i, v), vt = tagged v, slot2 = slot of (v, u2), u2t = tagged u2.
template <class F>
__device__ __forceinline__ void warp_wedges(uint32_t b, uint32_t e, const Params& P, F&& f) {
  const unsigned lane = lane_id();
  for (uint32_t j0 = b; j0 < e; j0 += 32) {
    const uint32_t j = j0 + lane;
    uint32_t L = 0, vt = 0, vs = 0;
    if (j < e) {
      L = P.pref[j];
      vt = P.adj[j];
      if ((vt >> 1) < P.n) vs = P.off[vt >> 1];
      else { record_violation(P.err, 28, vt, j); L = 0; }
    }
    const uint32_t incl = warp_inclusive_scan(L);
    const uint32_t excl = incl - L;
    const uint32_t T = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t t0 = 0; t0 < T; t0 += 32) {
      const uint32_t t = t0 + lane;
      uint32_t lo = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        uint32_t x = __shfl_sync(0xffffffffu, incl, lo + step - 1);
        if (x <= t) lo += step;
      }
      const uint32_t ex = __shfl_sync(0xffffffffu, excl, lo);
      const uint32_t vsj = __shfl_sync(0xffffffffu, vs, lo);
      const uint32_t vtj = __shfl_sync(0xffffffffu, vt, lo);
      if (t < T) {
        const uint32_t slot2 = vsj + (t - ex);
        if (slot_ok(P, slot2, 20)) f(j0 + lo, vtj, slot2, P.adj[slot2]);
      }
    }
  }
}

// Per-thread accumulator of per-(i,v) credits, flushed when the neighbour slot changes.
struct SlotAcc {
  uint32_t j = kEmpty;
  int64_t acc = 0;
  __device__ __forceinline__ void flush(const Params& P) {
    if (j != kEmpty && acc) {
      if (!slot_ok(P, j, 10)) return;
      if (P.per == VERT) credit(P, P.adj[j] >> 1, acc, 11);
      else credit(P, P.eout[j], acc, 12);
    }
    acc = 0;
  }
  __device__ __forceinline__ void add(const Params& P, uint32_t jj, int64_t x) {
    if (jj != j) { flush(P); j = jj; }
    acc += x;
  }
};

// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) count_warp_kernel(Params P, int small_w) {
  extern __shared__ uint32_t smem_w[];
  const unsigned lane = lane_id();
  const int wib = threadIdx.x >> 5;
  uint32_t* keys = smem_w + wib * (2 * kWarpTable);
  uint32_t* vals = keys + kWarpTable;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int64_t total = 0;
  for (int64_t i = warp; i < P.n; i += nwarps) {
    const int64_t W = P.wsum[i + 1] - P.wsum[i];
    if (W <= 0 || W > small_w) {
      if (W < 0 && lane == 0) record_violation(P.err, 34, (uint64_t)i, 0);
      continue;
    }
    const uint32_t b = P.off[i], e = P.off[i + 1];
    const bool tag_i = !(P.adj[b] & 1u);
    const bool need_center = P.per == EDGE || (P.per == VERT && !tag_i);
    const uint32_t tsize = max(64u, next_pow2(2u * (uint32_t)W));
    const uint32_t mask = tsize - 1;
    for (uint32_t s = lane; s < tsize; s += 32) { keys[s] = kEmpty; vals[s] = 0; }
    __syncwarp();
    warp_wedges(b, e, P, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
      if (!table_insert(keys, vals, mask, u2t >> 1)) record_violation(P.err, 25, u2t >> 1, (uint32_t)i);
    });
    __syncwarp();
    if (need_center) {
      SlotAcc acc;
      warp_wedges(b, e, P, [&](uint32_t jj, uint32_t, uint32_t slot2, uint32_t u2t) {
        const uint32_t w = table_find(keys, vals, mask, u2t >> 1);
        if (w > 1) {
          if (P.per == EDGE) credit(P, P.eout[slot2], (int64_t)(w - 1), 13);
          acc.add(P, jj, (int64_t)(w - 1));
        }
      });
      acc.flush(P);
    } else {
      int64_t mine = 0;
      for (uint32_t s = lane; s < tsize; s += 32) {
        const uint32_t k = keys[s];
        if (k == kEmpty) continue;
        const int64_t w = vals[s];
        if (w < 2) continue;
        const int64_t bf = w * (w - 1) / 2;
        mine += bf;
        if (P.per == VERT) credit(P, k, bf, 14);
      }
      if (P.per == VERT) {
        mine = warp_sum(mine);
        if (lane == 0 && mine) credit(P, i, mine, 15);
      } else {
        total += mine;
      }
    }
    __syncwarp();
  }
  if (P.per == TOTAL) {
    total = warp_sum(total);
    if (lane == 0 && total) atomic_add_i64(P.out, total);
  }
}

// ---------------------------------------------------------------------------------------------
constexpr int kBlock = 512;

struct BlockShared {
  uint32_t incl[kBlock];
  uint32_t vs[kBlock];
  uint32_t vt[kBlock];
  uint32_t len[kBlock];
  uint32_t scan[32];
  int64_t red[32];
  uint32_t item;
  uint32_t cursor;
};

__device__ __forceinline__ uint32_t block_inclusive_scan_u32(uint32_t x, uint32_t* smem, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t incl = warp_inclusive_scan(x);
  if (lane == 31) smem[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t v = lane < nwarps ? smem[lane] : 0u;
    v = warp_inclusive_scan(v);
    smem[lane] = v;
  }
  __syncthreads();
  incl += warp > 0 ? smem[warp - 1] : 0u;
  total = smem[nwarps - 1];
  return incl;
}

__device__ __forceinline__ int64_t block_sum_i64(int64_t x, int64_t* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  x = warp_sum(x);
  __syncthreads();
  if (lane == 0) smem[warp] = x;
  __syncthreads();
  int64_t t = 0;
  if (warp == 0) {
    t = lane < nwarps ? smem[lane] : 0;
    t = warp_sum(t);
  }
  return t;  // valid in thread 0
}

// Iterates every wedge of endpoint i with the whole CTA.  Per chunk of kBlock neighbours, each
// neighbour's prefix N(v)[0, L) is cut into pieces of at most kPiece wedges; warps claim pieces
// from a shared-memory counter, locate a piece's neighbour once (binary search over the
// chunk's inclusive piece counts) and walk it with 32 lanes, so consecutive lanes read
// consecutive entries of N(v) and no per-wedge search is needed.
constexpr uint32_t kPiece = 256;

template <class F>
__device__ __forceinline__ void block_wedges(uint32_t b, uint32_t e, const Params& P, BlockShared& S, F&& f) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  for (uint32_t j0 = b; j0 < e; j0 += kBlock) {
    const uint32_t j = j0 + tid;
    uint32_t L = 0, vt = 0, vs = 0;
    if (j < e) {
      L = P.pref[j];
      vt = P.adj[j];
      if ((vt >> 1) < P.n) vs = P.off[vt >> 1];
      else { record_violation(P.err, 29, vt, j); L = 0; }
    }
    uint32_t T;
    const uint32_t incl = block_inclusive_scan_u32((L + kPiece - 1) / kPiece, S.scan, T);
    S.incl[tid] = incl;
    S.vs[tid] = vs;
    S.vt[tid] = vt;
    S.len[tid] = L;
    if (tid == 0) S.cursor = 0;
    __syncthreads();
    while (true) {
      uint32_t p = 0;
      if (lane == 0) p = atomicAdd(&S.cursor, 1u);
      p = __shfl_sync(0xffffffffu, p, 0);
      if (p >= T) break;
      uint32_t lo = 0;
#pragma unroll
      for (uint32_t step = kBlock / 2; step > 0; step >>= 1)
        if (S.incl[lo + step - 1] <= p) lo += step;
      const uint32_t first_piece = lo ? S.incl[lo - 1] : 0u;
      const uint32_t k0 = (p - first_piece) * kPiece;
      const uint32_t kend = min(k0 + kPiece, S.len[lo]);
      const uint32_t vsj = S.vs[lo], vtj = S.vt[lo];
      // Vectorised walk: lane t takes the aligned group of four entries at g + 4t (one 16-byte
      // load; the adjacency array is 16-byte aligned and padded to whole groups), and uses the
      // entries inside the piece [vsj + k0, vsj + kend).
      const uint32_t pbeg = vsj + k0, pend = vsj + kend;
      for (uint32_t g = (pbeg & ~3u) + 4u * lane; g < pend; g += 128u) {
        if (!slot_ok(P, g, 21)) break;
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(P.adj + g));
        const uint32_t x[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (uint32_t r = 0; r < 4; ++r) {
          const uint32_t slot2 = g + r;
          if (slot2 >= pbeg && slot2 < pend && slot_ok(P, slot2, 21)) f(j0 + lo, vtj, slot2, x[r]);
        }
      }
    }
    __syncthreads();
  }
}

enum Mode : uint32_t { MODE_DENSE = 0, MODE_HASH = 1, MODE_GLOBAL = 2, MODE_HYBRID = 3 };
// A scheduler mode entry that leaves the item to the plain rule (items too light for the
// choice to matter are not scored by the learned scheduler).
constexpr uint8_t kPlainRule = 0xFF;
// Items with fewer wedges are left to the plain rule when the learned scheduler runs.
constexpr int64_t kSchedMinWedges = 2048;

__global__ void __launch_bounds__(kBlock) count_block_kernel(Params P, const uint32_t* __restrict__ items,
                                                             const uint32_t* __restrict__ n_items_dev,
                                                             uint32_t* cursor, uint32_t* gscratch,
                                                             uint32_t cap_dense, uint32_t cap_hash,
                                                             uint32_t hy_dense, uint32_t hy_hash) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BlockShared& S = *reinterpret_cast<BlockShared*>(smem_raw);
  uint32_t* table = reinterpret_cast<uint32_t*>(smem_raw + ((sizeof(BlockShared) + 15) & ~size_t(15)));
  uint32_t* gcnt = gscratch ? gscratch + (size_t)blockIdx.x * (size_t)P.n : nullptr;
  const uint32_t n_items = *n_items_dev;
  int64_t total = 0;
  while (true) {
    if (threadIdx.x == 0) S.item = atomicAdd(cursor, 1u);
    __syncthreads();
    const uint32_t q = S.item;
    __syncthreads();
    if (q >= n_items) break;
    const long long t_item = clock64();
    const uint32_t i = items[q];
    const int64_t W = P.wsum[i + 1] - P.wsum[i];
    const uint32_t b = P.off[i], e = P.off[i + 1];
    const bool tag_i = !(P.adj[b] & 1u);
    const bool need_center = P.per == EDGE || (P.per == VERT && !tag_i);
    Mode mode;
    if (P.modes && P.modes[q] != kPlainRule) mode = (Mode)(P.modes[q] & 3u);
    else if (i <= cap_dense && (uint64_t)i <= 4ull * (uint64_t)W) mode = MODE_DENSE;
    else if ((uint64_t)2 * W <= cap_hash) mode = MODE_HASH;
    else if (i <= cap_dense) mode = MODE_DENSE;
    else {
      // Hybrid: dense counters for u2 < hy_dense (the low ranks, where R-MAT-like graphs put
      // most wedge ends) plus a hash table for the rest, when the rest is small enough.  The
      // number of wedges ending at or above hy_dense is exact: per neighbour, the prefix length
      // minus the entries below hy_dense (one binary search each).
      unsigned long long lo_w = 0;
      for (uint32_t j = b + threadIdx.x; j < e; j += kBlock) {
        const uint32_t v = P.adj[j] >> 1;
        if (v >= P.n) continue;
        const uint32_t vb = P.off[v];
        const uint32_t below = lower_bound_u32(P.adj, vb, P.off[v + 1], hy_dense << 1) - vb;
        lo_w += min(below, P.pref[j]);
      }
      const int64_t lo_total = block_sum_i64((int64_t)lo_w, S.red);
      if (threadIdx.x == 0) S.item = (uint32_t)(W - lo_total > 0x7fffffff ? 0x7fffffff : W - lo_total);
      __syncthreads();
      const uint32_t hi_w = S.item;
      __syncthreads();
      mode = (2ull * hi_w <= hy_hash) ? MODE_HYBRID : MODE_GLOBAL;
    }
    if (threadIdx.x == 0 && P.mstats) {
      atomicAdd(&P.mstats[mode], 1ull);
      atomicAdd(&P.mstats[4 + mode], (unsigned long long)W);
    }
    uint32_t tsize = 0, mask = 0;
    uint32_t* keys = table;
    uint32_t* vals = table + cap_hash;
    if (mode == MODE_HYBRID) {
      keys = table + hy_dense;
      vals = keys + hy_hash;
      tsize = hy_hash;
      mask = tsize - 1;
    }
    if (mode == MODE_DENSE) {
      for (uint32_t s = threadIdx.x; s < i; s += kBlock) table[s] = 0;
    } else if (mode == MODE_HASH) {
      tsize = max(64u, next_pow2(2u * (uint32_t)W));
      mask = tsize - 1;
      for (uint32_t s = threadIdx.x; s < tsize; s += kBlock) { keys[s] = kEmpty; vals[s] = 0; }
    } else if (mode == MODE_HYBRID) {
      for (uint32_t s = threadIdx.x; s < hy_dense; s += kBlock) table[s] = 0;
      for (uint32_t s = threadIdx.x; s < tsize; s += kBlock) { keys[s] = kEmpty; vals[s] = 0; }
    }
    __syncthreads();
    // Phase 1: multiplicities.
    if (mode == MODE_DENSE) {
      block_wedges(b, e, P, S, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
        if ((u2t >> 1) >= i) { record_violation(P.err, 22, u2t >> 1, i); return; }
        atomicAdd(&table[u2t >> 1], 1u);
      });
    } else if (mode == MODE_HASH) {
      block_wedges(b, e, P, S, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
        if (!table_insert(keys, vals, mask, u2t >> 1)) record_violation(P.err, 26, u2t >> 1, i);
      });
    } else if (mode == MODE_HYBRID) {
      block_wedges(b, e, P, S, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
        const uint32_t u2 = u2t >> 1;
        if (u2 < hy_dense) atomicAdd(&table[u2], 1u);
        else if (!table_insert(keys, vals, mask, u2)) record_violation(P.err, 35, u2, i);
      });
    } else {
      block_wedges(b, e, P, S, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
        if ((u2t >> 1) >= P.n) { record_violation(P.err, 23, u2t >> 1, i); return; }
        atomicAdd(&gcnt[u2t >> 1], 1u);
      });
    }
    __syncthreads();
    if (need_center) {
      // Phase 2: centre / edge credits.
      SlotAcc acc;
      block_wedges(b, e, P, S, [&](uint32_t jj, uint32_t, uint32_t slot2, uint32_t u2t) {
        const uint32_t u2 = u2t >> 1;
        uint32_t w;
        if (u2 >= (mode == MODE_DENSE ? i : (uint32_t)P.n)) { record_violation(P.err, 24, u2, i); return; }
        if (mode == MODE_DENSE) w = table[u2];
        else if (mode == MODE_HASH) w = table_find(keys, vals, mask, u2);
        else if (mode == MODE_HYBRID) w = u2 < hy_dense ? table[u2] : table_find(keys, vals, mask, u2);
        else w = gcnt[u2];
        if (w > 1) {
          if (P.per == EDGE) credit(P, P.eout[slot2], (int64_t)(w - 1), 13);
          acc.add(P, jj, (int64_t)(w - 1));
        }
      });
      acc.flush(P);
      __syncthreads();
      if (mode == MODE_GLOBAL) {  // restore the zero invariant of the scratch array
        block_wedges(b, e, P, S, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
          if ((u2t >> 1) < P.n) gcnt[u2t >> 1] = 0;
        });
        __syncthreads();
      }
    } else {
      // Phase 3: endpoint credits, once per distinct u2.
      int64_t mine = 0;
      if (mode == MODE_DENSE) {
        for (uint32_t s = threadIdx.x; s < i; s += kBlock) {
          const int64_t w = table[s];
          if (w >= 2) {
            const int64_t bf = w * (w - 1) / 2;
            mine += bf;
            if (P.per == VERT) credit(P, s, bf, 16);
          }
        }
      } else if (mode == MODE_HASH || mode == MODE_HYBRID) {
        if (mode == MODE_HYBRID) {
          for (uint32_t s = threadIdx.x; s < hy_dense; s += kBlock) {
            const int64_t w = table[s];
            if (w >= 2) {
              const int64_t bf = w * (w - 1) / 2;
              mine += bf;
              if (P.per == VERT) credit(P, s, bf, 36);
            }
          }
        }
        for (uint32_t s = threadIdx.x; s < tsize; s += kBlock) {
          const uint32_t k = keys[s];
          if (k == kEmpty) continue;
          const int64_t w = vals[s];
          if (w >= 2) {
            const int64_t bf = w * (w - 1) / 2;
            mine += bf;
            if (P.per == VERT) credit(P, k, bf, 17);
          }
        }
      } else {
        block_wedges(b, e, P, S, [&](uint32_t, uint32_t, uint32_t, uint32_t u2t) {
          if ((u2t >> 1) >= P.n) { record_violation(P.err, 27, u2t >> 1, i); return; }
          const int64_t w = atomicExch(&gcnt[u2t >> 1], 0u);
          if (w >= 2) {
            const int64_t bf = w * (w - 1) / 2;
            mine += bf;
            if (P.per == VERT) credit(P, u2t >> 1, bf, 18);
          }
        });
      }
      if (P.per == VERT) {
        const int64_t s = block_sum_i64(mine, S.red);
        if (threadIdx.x == 0 && s) credit(P, i, s, 19);
      } else {
        total += mine;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (P.mode_out) P.mode_out[q] = (uint8_t)mode;
      if (P.cycles) P.cycles[q] = (unsigned long long)(clock64() - t_item);
    }
  }
  if (P.per == TOTAL) {
    const int64_t s = block_sum_i64(total, S.red);
    if (threadIdx.x == 0 && s) atomic_add_i64(P.out, s);
  }
}

__global__ void widen_u32_kernel(const uint32_t* __restrict__ in, int64_t n, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)in[i];
}

__global__ void classify_endpoints_kernel(const int64_t* __restrict__ wsum, int64_t n, int small_w, uint32_t cap_dense,
                                          uint32_t cap_hash, uint32_t* items, uint32_t* counts /* [0]=big [1]=global */) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t W = wsum[i + 1] - wsum[i];
    if (W <= small_w) continue;
    items[atomicAdd(&counts[0], 1u)] = (uint32_t)i;
    const bool dense_ok = (uint64_t)i <= cap_dense;
    const bool hash_ok = (uint64_t)2 * W <= cap_hash;
    if (!dense_ok && !hash_ok) atomicAdd(&counts[1], 1u);
  }
}

// ---- scheduler support ---------------------------------------------------------------------
constexpr int kItemFeatures = 12;  // features per item; 4 one-hot mode slots follow

// One warp per block-aggregator item: cost-model features and the valid modes (bit m set when
// mode m can hold the item's multiplicity table; the global mode always can).
__global__ void item_features_kernel(Params P, const uint32_t* __restrict__ items, uint32_t n_items,
                                     uint32_t cap_dense, uint32_t cap_hash, uint32_t hy_dense, uint32_t hy_hash,
                                     float* F, uint8_t* valid) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t q = warp; q < n_items; q += nwarps) {
    const uint32_t i = items[q];
    const int64_t W = P.wsum[i + 1] - P.wsum[i];
    const uint32_t b = P.off[i], e = P.off[i + 1];
    unsigned long long lo_w = 0, sumdeg = 0;
    for (uint32_t j = b + lane; j < e; j += 32) {
      const uint32_t v = P.adj[j] >> 1;
      if (v >= P.n) continue;
      const uint32_t vb = P.off[v], ve = P.off[v + 1];
      sumdeg += ve - vb;
      const uint32_t below = lower_bound_u32(P.adj, vb, ve, hy_dense << 1) - vb;
      lo_w += min(below, P.pref[j]);
    }
    lo_w = warp_sum(lo_w);
    sumdeg = warp_sum(sumdeg);
    if (lane == 0) {
      const int64_t hi = W - (int64_t)lo_w;
      const uint64_t hi_c = hi > 0x7fffffff ? 0x7fffffffull : (uint64_t)(hi > 0 ? hi : 0);
      const bool tag_i = !(P.adj[b] & 1u);
      const bool need_center = P.per == EDGE || (P.per == VERT && !tag_i);
      const uint32_t deg = e - b;
      float* f = F + q * kMlpIn;
      f[0] = log2f(1.f + (float)W);
      f[1] = log2f(1.f + (float)i);
      f[2] = log2f(1.f + (float)deg);
      f[3] = log2f(1.f + (float)hi_c);
      f[4] = log2f(1.f + (float)lo_w);
      f[5] = log2f(1.f + (float)sumdeg);
      f[6] = need_center ? 1.f : 0.f;
      f[7] = P.per == EDGE ? 1.f : 0.f;
      f[8] = log2f(1.f + (float)P.n);
      f[9] = f[1] - f[0];
      f[10] = P.out32 ? 1.f : 0.f;
      f[11] = log2f(1.f + (float)W / (float)(deg ? deg : 1u));
      for (int k = kItemFeatures; k < kMlpIn; ++k) f[k] = 0.f;
      const bool dense_ok = i <= cap_dense, hash_ok = (uint64_t)2 * W <= cap_hash, hybrid_ok = 2ull * hi_c <= hy_hash;
      // The plain rule's choice (count_block_kernel) rides in the top bits.
      const uint32_t rule = (dense_ok && (uint64_t)i <= 4ull * (uint64_t)W) ? MODE_DENSE
                            : hash_ok                                     ? MODE_HASH
                            : dense_ok                                    ? MODE_DENSE
                            : hybrid_ok                                   ? MODE_HYBRID
                                                                          : MODE_GLOBAL;
      valid[q] = (uint8_t)((dense_ok ? 1u : 0u) | (hash_ok ? 2u : 0u) | 4u | (hybrid_ok ? 8u : 0u) | (rule << 4));
    }
  }
}

// Candidate modes of the learned choice: the shared-memory modes (the global-scratch mode is
// the fallback of items no shared-memory mode can hold; it is never cheaper).
__constant__ int kCandMode[3] = {MODE_DENSE, MODE_HASH, MODE_HYBRID};

// Cost-model rows: item q with candidate c is row 3q + c (features, then the one-hot mode).
__global__ void sched_candidates_kernel(const float* __restrict__ F, uint32_t n_items, float* X) {
  const int64_t total = (int64_t)n_items * 3 * kMlpIn;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / kMlpIn;
    const int f = (int)(e - r * kMlpIn);
    const int64_t q = r / 3;
    const int m = kCandMode[r - 3 * q];
    X[e] = f < kItemFeatures ? F[q * kMlpIn + f] : (f - kItemFeatures == m ? 1.f : 0.f);
  }
}

// The valid shared-memory mode with the least predicted log2 cycles; the plain rule's mode is
// kept unless another one is predicted at least kSchedMargin (log2 units, 10%) cheaper.  Items
// no shared-memory mode can hold take the global mode.
constexpr float kSchedMargin = 0.1375f;
__global__ void sched_choose_kernel(const float* __restrict__ y, const uint8_t* __restrict__ valid, uint32_t n_items,
                                    uint8_t* modes, float* pred, uint32_t* n_global) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n_items; q += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t vq = valid[q], rule = vq >> 4;
    int best = MODE_GLOBAL;
    float by = 1e30f, ry = 1e30f;
    for (int c = 0; c < 3; ++c) {
      const int m = kCandMode[c];
      if (!(vq & (1u << m))) continue;
      const float v = y[q * 3 + c];
      if (v < by) { by = v; best = m; }
      if ((uint32_t)m == rule) ry = v;
    }
    if (rule != MODE_GLOBAL && ry - by < kSchedMargin) {
      best = (int)rule;
      by = ry;
    }
    modes[q] = (uint8_t)best;
    pred[q] = best == MODE_GLOBAL ? -1.f : by;  // no prediction for the fallback
    if (best == MODE_GLOBAL) atomicAdd(n_global, 1u);
  }
}

// sub[k]: the positions q of block-aggregator items with at least min_w wedges.
__global__ void heavy_items_kernel(const uint32_t* __restrict__ items, uint32_t n_items,
                                   const int64_t* __restrict__ wsum, int64_t min_w, uint32_t* sub, uint32_t* n_sub) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n_items; q += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t i = items[q];
    if (wsum[i + 1] - wsum[i] >= min_w) sub[atomicAdd(n_sub, 1u)] = (uint32_t)q;
  }
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, uint32_t n,
                                  uint32_t* dst) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = src[idx[k]];
}

// Scatters the scored items' modes, predictions and features back to their positions.
__global__ void scatter_scored_kernel(const uint32_t* __restrict__ sub, uint32_t n, const uint8_t* __restrict__ msub,
                                      const float* __restrict__ psub, const float* __restrict__ fsub, uint8_t* modes,
                                      float* pred, float* F) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t q = sub[k];
    modes[q] = msub[k];
    pred[q] = psub[k];
    for (int f = 0; f < kMlpIn; ++f) F[(size_t)q * kMlpIn + f] = fsub[(size_t)k * kMlpIn + f];
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// A seeded random valid mode per item (exploration for trace collection).
__global__ void sched_explore_kernel(const uint8_t* __restrict__ valid, uint32_t n_items, uint64_t seed,
                                     uint8_t* modes, uint32_t* n_global) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n_items; q += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t vm = valid[q] & 15u;
    const uint32_t c = __popc(vm);
    uint32_t k = (uint32_t)(mix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(q + 1)) % c);
    int m = 0;
    for (; m < 4; ++m)
      if (vm & (1u << m)) {
        if (k == 0) break;
        --k;
      }
    modes[q] = (uint8_t)m;
    if (m == MODE_GLOBAL) atomicAdd(n_global, 1u);
  }
}

}  // namespace

CountResult count_ranked(const Ranked& R, int per, int64_t* out, const CountConfig& cfg, cudaStream_t s) {
  CountResult res;
  const int64_t n = R.n;
  const int64_t out_len = per == VERT ? n : (per == EDGE ? R.m2 / 2 : 1);
  if (out_len > 0) PB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t) * out_len, s));
  if (n == 0 || R.w_rank == 0) return res;
  Params P{R.off.get(), R.adj.get(), R.pref.get(), per == EDGE ? R.eout.get() : nullptr, R.wsum.get(), n, per, out,
           out_len, R.m2, nullptr, nullptr, nullptr};
  DevBuf<uint32_t> err_local;
  if (cfg.err) {
    P.err = cfg.err;
  } else {
    err_local.alloc(4, s);
    PB_CUDA_TRY(cudaMemsetAsync(err_local.get(), 0, 4 * sizeof(uint32_t), s));
    P.err = err_local.get();
  }
  DevBuf<unsigned long long> mstats(8, s);
  PB_CUDA_TRY(cudaMemsetAsync(mstats.get(), 0, 8 * sizeof(unsigned long long), s));
  P.mstats = mstats.get();
  // Per-edge counts fit 32 bits when (max degree - 1)^2 < 2^32: accumulate them in a 4-byte
  // array (67 MB for 2^24 edges, L2-resident) and widen once at the end.
  DevBuf<uint32_t> out32;
  const uint64_t md = R.max_deg > 0 ? R.max_deg - 1 : 0;
  const char* acc64 = getenv("PB_EDGE_ACC64");  // test hook: force 64-bit per-edge accumulation
  const bool force64 = acc64 && *acc64 == '1';
  if (per == EDGE && out_len > 0 && md * md < (1ull << 32) && !force64) {
    out32.alloc(out_len, s);
    PB_CUDA_TRY(cudaMemsetAsync(out32.get(), 0, out32.bytes(), s));
    P.out32 = out32.get();
  }
  const int sms = sm_count();
  int small_w = std::min(cfg.small_w, kWarpTable / 2);
  int smem_bytes = cfg.smem_bytes;
  // Test hooks: shrink the CTA table / the warp threshold so small graphs reach every CTA mode.
  if (const char* ev = getenv("PB_COUNT_SMEM")) smem_bytes = std::max(16384, std::min(atoi(ev), cfg.smem_bytes));
  if (const char* ev = getenv("PB_COUNT_SMALL_W")) small_w = std::max(0, std::min(atoi(ev), small_w));
  int blocks_per_sm = cfg.blocks_per_sm;
  if (const char* ev = getenv("PB_COUNT_BPS")) blocks_per_sm = std::max(1, std::min(atoi(ev), 4));

  // Block aggregator geometry.
  const size_t shared_fixed = (sizeof(BlockShared) + 15) & ~size_t(15);
  const size_t table_bytes = (size_t)smem_bytes > shared_fixed ? (size_t)smem_bytes - shared_fixed : 0;
  const uint32_t cap_dense = (uint32_t)(table_bytes / 4);
  uint32_t cap_hash = 1;
  while ((size_t)cap_hash * 2 * 8 <= table_bytes) cap_hash <<= 1;  // slots; keys + values
  if (cap_hash < 64) cap_hash = 64;

  // Hybrid mode: half the table area as dense counters, the other half as a hash table.
  const uint32_t hy_dense = (uint32_t)(table_bytes / 2 / 4);
  uint32_t hy_hash = 1;
  while ((size_t)hy_hash * 2 * 8 <= table_bytes / 2) hy_hash <<= 1;
  DevBuf<uint32_t> items(n, s), counts(3, s);
  PB_CUDA_TRY(cudaMemsetAsync(counts.get(), 0, 3 * sizeof(uint32_t), s));
  PB_LAUNCH(classify_endpoints_kernel, std::max(1, std::min(ceil_div(n, 256), sms * 8)), 256, 0, s, R.wsum.get(), n,
            small_w, cap_dense, cap_hash, items.get(), counts.get());
  uint32_t hc[2];
  readback(hc, counts.get(), sizeof(hc), s);
  res.n_big = (int)hc[0];

  // Under graph capture nothing is timed or read back here (the recording run checked).
  const bool cap = capturing();
  cudaEvent_t e0, e1;
  PB_CUDA_TRY(cudaEventCreate(&e0));
  PB_CUDA_TRY(cudaEventCreate(&e1));
  if (!cap) PB_CUDA_TRY(cudaEventRecord(e0, s));
  {
    const int smem = kWarpsPerBlockSmall * 2 * kWarpTable * (int)sizeof(uint32_t);
    static bool attr_set = false;
    if (!attr_set) {
      PB_CUDA_TRY(cudaFuncSetAttribute(count_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      attr_set = true;
    }
    PB_LAUNCH(count_warp_kernel, sms * 3, kWarpsPerBlockSmall * 32, smem, s, P, small_w);
  }
  // Scheduler: per-item modes (learned or exploring) and the record of what each item ran
  // with and how long it took.
  SchedHooks* sh = cfg.sched;
  const bool sched_on = sh && hc[0] > 0 && (sh->model || sh->explore || sh->trace_X);
  DevBuf<float> sF, sPred;
  DevBuf<uint8_t> sValid, sModes, sUsed;
  DevBuf<uint32_t> sNG;
  DevBuf<unsigned long long> sCyc;
  bool need_global = hc[1] > 0;
  if (sched_on) {
    const uint32_t ni = hc[0];
    cudaEvent_t a0, a1;
    PB_CUDA_TRY(cudaEventCreate(&a0));
    PB_CUDA_TRY(cudaEventCreate(&a1));
    PB_CUDA_TRY(cudaEventRecord(a0, s));
    sF.alloc((size_t)ni * kMlpIn, s);
    sValid.alloc(ni, s);
    sUsed.alloc(ni, s);
    sCyc.alloc(ni, s);
    sNG.alloc(1, s);
    PB_CUDA_TRY(cudaMemsetAsync(sNG.get(), 0, sizeof(uint32_t), s));
    const int g1 = std::max(1, std::min(ceil_div(ni, 256), sms * 8));
    // Learned choices score only the items heavy enough for the mode to matter (the rest keep
    // the plain rule, so the scheduler's own cost stays small); tracing covers every item.
    if (sh->model && !sh->trace_X) {
      DevBuf<uint32_t> sub(ni, s), nsub(1, s);
      PB_CUDA_TRY(cudaMemsetAsync(nsub.get(), 0, sizeof(uint32_t), s));
      int64_t min_w = kSchedMinWedges;
      if (const char* ev = getenv("PB_SCHED_MIN_WEDGES")) min_w = atoll(ev);  // test hook: score light items too
      PB_LAUNCH(heavy_items_kernel, g1, 256, 0, s, items.get(), ni, R.wsum.get(), min_w, sub.get(), nsub.get());
      uint32_t nh = 0;
      readback(&nh, nsub.get(), sizeof(nh), s);
      sModes.alloc(ni, s);
      sPred.alloc(ni, s);
      PB_CUDA_TRY(cudaMemsetAsync(sModes.get(), kPlainRule, ni, s));
      PB_CUDA_TRY(cudaMemsetAsync(sPred.get(), 0xFF, sizeof(float) * ni, s));  // NaN: no prediction
      PB_CUDA_TRY(cudaMemsetAsync(sF.get(), 0, sF.bytes(), s));
      if (nh > 0) {
        DevBuf<uint32_t> hitems(nh, s);
        DevBuf<float> hF((size_t)nh * kMlpIn, s), hPr(nh, s);
        DevBuf<uint8_t> hValid(nh, s), hModes(nh, s);
        const int gh = std::max(1, std::min(ceil_div(nh, 256), sms * 8));
        PB_LAUNCH(gather_u32_kernel, gh, 256, 0, s, items.get(), sub.get(), nh, hitems.get());
        PB_LAUNCH(item_features_kernel, std::max(1, std::min(ceil_div((int64_t)nh * 32, 256), sms * 8)), 256, 0, s, P,
                  hitems.get(), nh, cap_dense, cap_hash, hy_dense, hy_hash, hF.get(), hValid.get());
        DevBuf<float> X((size_t)nh * 3 * kMlpIn, s), y((size_t)nh * 3, s);
        PB_LAUNCH(sched_candidates_kernel, std::max(1, std::min(ceil_div((int64_t)nh * 3 * kMlpIn, 256), sms * 8)), 256,
                  0, s, hF.get(), nh, X.get());
        sh->model->predict_dev(X.get(), (int64_t)nh * 3, y.get(), s);
        PB_LAUNCH(sched_choose_kernel, gh, 256, 0, s, y.get(), hValid.get(), nh, hModes.get(), hPr.get(), sNG.get());
        PB_LAUNCH(scatter_scored_kernel, gh, 256, 0, s, sub.get(), nh, hModes.get(), hPr.get(), hF.get(), sModes.get(),
                  sPred.get(), sF.get());
      }
    } else {
      PB_LAUNCH(item_features_kernel, std::max(1, std::min(ceil_div((int64_t)ni * 32, 256), sms * 8)), 256, 0, s, P,
                items.get(), ni, cap_dense, cap_hash, hy_dense, hy_hash, sF.get(), sValid.get());
    }
    if (sh->model && sh->trace_X) {
      DevBuf<float> X((size_t)ni * 3 * kMlpIn, s), y((size_t)ni * 3, s);
      PB_LAUNCH(sched_candidates_kernel, std::max(1, std::min(ceil_div((int64_t)ni * 3 * kMlpIn, 256), sms * 8)), 256,
                0, s, sF.get(), ni, X.get());
      sh->model->predict_dev(X.get(), (int64_t)ni * 3, y.get(), s);
      sModes.alloc(ni, s);
      sPred.alloc(ni, s);
      PB_LAUNCH(sched_choose_kernel, g1, 256, 0, s, y.get(), sValid.get(), ni, sModes.get(), sPred.get(), sNG.get());
    } else if (sh->explore) {
      sModes.alloc(ni, s);
      PB_LAUNCH(sched_explore_kernel, g1, 256, 0, s, sValid.get(), ni, sh->seed, sModes.get(), sNG.get());
    }
    P.modes = sModes.get();  // null when only the plain choices are traced
    P.mode_out = sUsed.get();
    P.cycles = sCyc.get();
    uint32_t ng = 0;
    PB_CUDA_TRY(cudaMemcpyAsync(&ng, sNG.get(), sizeof(ng), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaEventRecord(a1, s));
    PB_CUDA_TRY(cudaEventSynchronize(a1));
    if (P.modes) need_global = ng > 0 || hc[1] > 0;  // unscored items follow the plain rule
    float ms = 0;
    PB_CUDA_TRY(cudaEventElapsedTime(&ms, a0, a1));
    sh->ms = ms;
    cudaEventDestroy(a0);
    cudaEventDestroy(a1);
  }
  DevBuf<uint32_t> gscratch;
  if (hc[0] > 0) {
    int grid = (int)std::min<int64_t>(hc[0], (int64_t)sms * blocks_per_sm);
    if (need_global) {
      // One dense counter array of n entries per CTA: at very large n (the 1e9-edge R-MAT) the
      // CTA count is capped so the arrays stay within half of the free device memory (64 GB at
      // most).
      size_t free_b = 0, total_b = 0;
      PB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
      const size_t budget = std::min<size_t>(free_b / 2, size_t(64) << 30);
      const size_t per_cta = (size_t)n * sizeof(uint32_t);
      grid = (int)std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)(budget / per_cta)));
      gscratch.alloc((size_t)grid * (size_t)n, s);
      PB_CUDA_TRY(cudaMemsetAsync(gscratch.get(), 0, gscratch.bytes(), s));
    }
    PB_CUDA_TRY(cudaFuncSetAttribute(count_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
    PB_LAUNCH(count_block_kernel, grid, kBlock, smem_bytes, s, P, items.get(), counts.get(), counts.get() + 2,
              gscratch.get(), cap_dense, cap_hash, hy_dense, hy_hash);
  }
  if (P.out32)
    PB_LAUNCH(widen_u32_kernel, std::max(1, std::min(ceil_div(out_len, 256), sms * 8)), 256, 0, s, P.out32, out_len, out);
  if (cap) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return res;
  }
  PB_CUDA_TRY(cudaEventRecord(e1, s));
  PB_CUDA_TRY(cudaEventSynchronize(e1));
  {
    unsigned long long h[8];
    PB_CUDA_TRY(cudaMemcpy(h, P.mstats, sizeof(h), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 4; ++k) { res.mode_items[k] = h[k]; res.mode_wedges[k] = h[4 + k]; }
  }
  {
    uint32_t h[4];
    PB_CUDA_TRY(cudaMemcpy(h, P.err, sizeof(h), cudaMemcpyDeviceToHost));
    PB_REQUIRE(h[0] == 0, PB_ECUDA,
               "aggregation: bounds violation code " + std::to_string(h[0]) + " index " +
                   std::to_string(((uint64_t)h[2] << 32) | h[1]) + " aux " + std::to_string(h[3]));
  }
  if (sched_on) {
    const uint32_t ni = hc[0];
    std::vector<float> hF((size_t)ni * kMlpIn), hPred;
    std::vector<uint8_t> hUsed(ni);
    std::vector<unsigned long long> hCyc(ni);
    PB_CUDA_TRY(cudaMemcpy(hF.data(), sF.get(), sF.bytes(), cudaMemcpyDeviceToHost));
    PB_CUDA_TRY(cudaMemcpy(hUsed.data(), sUsed.get(), sUsed.bytes(), cudaMemcpyDeviceToHost));
    PB_CUDA_TRY(cudaMemcpy(hCyc.data(), sCyc.get(), sCyc.bytes(), cudaMemcpyDeviceToHost));
    if (sh->model) {
      hPred.resize(ni);
      PB_CUDA_TRY(cudaMemcpy(hPred.data(), sPred.get(), sPred.bytes(), cudaMemcpyDeviceToHost));
    }
    double pc = 0, mc = 0, mae = 0;
    int64_t npred = 0;
    for (uint32_t q = 0; q < ni; ++q) {
      const double cyc = (double)std::max<unsigned long long>(hCyc[q], 1ull);
      const double lc = std::log2(cyc);
      if (sh->trace_X) {
        for (int f = 0; f < kMlpIn; ++f)
          sh->trace_X->push_back(f < kItemFeatures ? hF[(size_t)q * kMlpIn + f]
                                                   : (f - kItemFeatures == (int)hUsed[q] ? 1.f : 0.f));
        sh->trace_y->push_back((float)lc);
      }
      if (sh->model && hPred[q] >= 0.f) {  // items the model predicted (not the fallback)
        mc += cyc;
        pc += std::exp2((double)hPred[q]);
        mae += std::fabs((double)hPred[q] - lc);
        ++npred;
      }
    }
    sh->items = ni;
    sh->meas_cycles = mc;
    sh->pred_cycles = pc;
    sh->mae_log2 = npred ? mae / npred : 0.0;
  }
  float ms = 0;
  PB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  res.agg_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return res;
}

}  // namespace pb
