// Ranking stage: degrees, count-side choice, vertex orders (SIDE/DEG/ADEG/COCORE/ACOCORE),
// the ranked CSR with tag bits, and the per-endpoint wedge scan.
#include <algorithm>
#include <cstdlib>

#include "pb_engine.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

// Neighbour list of combined id x (V ids first, then nv + U id).  `shift` converts a list
// entry to a combined id.
struct Lists {
  const uint32_t* offV;
  const uint32_t* edgV;
  const uint32_t* offU;
  const uint32_t* edgU;
  int64_t nv;
  __device__ __forceinline__ void get(int64_t x, uint32_t& b, uint32_t& e, const uint32_t*& a, int64_t& shift) const {
    if (x < nv) { b = offV[x]; e = offV[x + 1]; a = edgV; shift = nv; }
    else { b = offU[x - nv]; e = offU[x - nv + 1]; a = edgU; shift = 0; }
  }
};

__global__ void degrees_kernel(Lists L, int64_t n, uint32_t* deg) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    uint32_t b, e; const uint32_t* a; int64_t sh;
    L.get(x, b, e, a, sh);
    deg[x] = e - b;
  }
}

// wedgeF (butterfly_utils.h:1061-1070): (v_deg * (v_deg - 1)) / 2 in 32-bit unsigned
// arithmetic, summed per side in 64 bits (cmpWedgeCounts, :1080-1086).
__global__ void side_wedges_kernel(const uint32_t* __restrict__ off, int64_t n, unsigned long long* acc) {
  unsigned long long s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t d = off[i + 1] - off[i];
    s += (unsigned long long)((uint32_t)(d * (d - 1u)) / 2u);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(acc, s);
}

// Sort key (ascending = earlier rank) for the degree-based orders.
__global__ void order_keys_kernel(const uint32_t* __restrict__ deg, int64_t n, int64_t nv, int rank_type, int use_v,
                                  uint32_t kmax, uint32_t* keys, uint32_t* ids) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    uint32_t k;
    if (rank_type == PB_SIDE) {
      bool on_count = use_v ? (x >= nv) : (x < nv);
      k = on_count ? 0u : 1u;
    } else if (rank_type == PB_DEG) {
      k = kmax - deg[x];
    } else {  // PB_ADEG
      k = kmax - log_key(deg[x]);
    }
    keys[x] = k;
    ids[x] = (uint32_t)x;
  }
}

__global__ void cocore_init_kernel(const uint32_t* __restrict__ deg, int64_t n, int approx, uint32_t* key,
                                   uint32_t* dact, uint8_t* done) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    dact[x] = deg[x];
    key[x] = approx ? log_key(deg[x]) : deg[x];
    done[x] = 0;
  }
}

__global__ void cocore_max_kernel(const uint32_t* __restrict__ key, const uint8_t* __restrict__ done, int64_t n,
                                  uint32_t* out /* [0]=max key+1 of undone (0: none) */) {
  uint32_t m = 0;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x)
    if (!done[x]) m = max(m, key[x] + 1u);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// One bucket round of getCoCoreRanks / getApproxCoCoreRanks (butterfly_utils.h:448-559):
// every undone vertex with key k is finished; each neighbour with key < k (undone, outside
// the bucket) loses one degree per finished neighbour and its key becomes f(new degree)
// (min with k is implied, since f(new) <= key < k).  Keys only decrease, so atomicMin of
// f over all decrements leaves f(final degree).
__global__ void cocore_round_kernel(Lists L, int64_t n, int approx, const uint32_t* __restrict__ kbuf, uint32_t* key,
                                    uint32_t* dact, uint8_t* done) {
  const uint32_t k = kbuf[0] - 1u;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t x = warp; x < n; x += nwarps) {
    if (done[x] || key[x] != k) continue;
    uint32_t b, e; const uint32_t* a; int64_t sh;
    L.get(x, b, e, a, sh);
    for (uint32_t j = b + lane; j < e; j += 32) {
      int64_t y = (int64_t)a[j] + sh;
      if (key[y] < k) {
        uint32_t old = atomicSub(&dact[y], 1u);
        uint32_t nd = old - 1u;
        atomicMin(&key[y], approx ? log_key(nd) : nd);
      }
    }
    __syncwarp();
    if (lane == 0) done[x] = 1;
  }
}

__global__ void cocore_keys_kernel(const uint32_t* __restrict__ key, int64_t n, uint32_t kmax, uint32_t* skeys,
                                   uint32_t* ids) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
    skeys[x] = kmax - key[x];
    ids[x] = (uint32_t)x;
  }
}

__global__ void invert_order_kernel(const uint32_t* __restrict__ order, int64_t n, uint32_t* rank) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    rank[order[r]] = (uint32_t)r;
}

__global__ void ranked_degrees_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ deg, int64_t n,
                                      uint32_t* rdeg) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    rdeg[r] = deg[order[r]];
}

// Fills row r of the ranked CSR with (rank(y) << 1 | on_count_side(y)) for every neighbour y
// of order[r] (rankGraph, butterfly_utils.h:579-623).  With eout, also the output edge index
// of each slot (CountERank's conversion, butterfly_ecount.h:1728-1738): slots whose neighbour
// is on the count side index the center side's lists directly; the others hold the index of
// the same edge in the neighbour's (center side) list, found by binary search (edgeToIdxs,
// butterfly_utils.h:2034-2062).
__global__ void ranked_fill_kernel(Lists L, const uint32_t* __restrict__ order, const uint32_t* __restrict__ rank,
                                   const uint32_t* __restrict__ roff, int64_t n, int use_v, uint32_t* adj,
                                   uint32_t* eout) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t r = warp; r < n; r += nwarps) {
    const int64_t x = order[r];
    uint32_t b, e; const uint32_t* a; int64_t sh;
    L.get(x, b, e, a, sh);
    const uint32_t dst = roff[r];
    const uint32_t x_local = (uint32_t)(x < L.nv ? x : x - L.nv);
    for (uint32_t j = b + lane; j < e; j += 32) {
      const uint32_t yl = a[j];
      const int64_t y = (int64_t)yl + sh;
      const bool y_v = y < L.nv;
      const uint32_t tag = use_v ? (y_v ? 0u : 1u) : (y_v ? 1u : 0u);
      adj[dst + (j - b)] = (rank[y] << 1) | tag;
      if (eout) {
        uint32_t o;
        if (tag) {
          o = j;
        } else {
          const uint32_t* yo = y_v ? L.offV : L.offU;
          const uint32_t* ya = y_v ? L.edgV : L.edgU;
          o = lower_bound_u32(ya, yo[yl], yo[yl + 1], x_local);
        }
        eout[dst + (j - b)] = o;
      }
    }
  }
}

// below[v] = #{u2 in N(v) : u2 < v} in the ranked CSR.
__global__ void below_self_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj, int64_t n,
                                  uint32_t* below) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    uint32_t b = off[v];
    below[v] = lower_bound_u32(adj, b, off[v + 1], (uint32_t)v << 1) - b;
  }
}

// countWedgesScan on the ranked graph (butterfly_utils.h:1192-1239, INVERSE direction): for
// slot (i, v) the wedges are the u2 in N(v) with u2 < min(i, v).  Lists are ascending, so that
// prefix length is a binary search for i in N(v) (when i < v) or the per-vertex below[v].
__global__ void wedge_scan_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj,
                                  const uint32_t* __restrict__ below, int64_t n, uint32_t* pref, int64_t* wcount) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < n; i += nwarps) {
    const uint32_t b = off[i], e = off[i + 1];
    int64_t sum = 0;
    for (uint32_t j = b + lane; j < e; j += 32) {
      const uint32_t v = adj[j] >> 1;
      uint32_t L;
      if ((uint32_t)i < v) {
        const uint32_t vb = off[v];
        L = lower_bound_u32(adj, vb, off[v + 1], (uint32_t)i << 1) - vb;
      } else {
        L = below[v];
      }
      pref[j] = L;
      sum += L;
    }
    sum = warp_sum(sum);
    if (lane == 0) wcount[i] = sum;
  }
}

// eti for the orientation of use_v (edgeToIdxs, butterfly_utils.h:2034-2062).
__global__ void eti_kernel(const uint32_t* __restrict__ offC, const uint32_t* __restrict__ edgC,
                           const uint32_t* __restrict__ offK, const uint32_t* __restrict__ edgK, int64_t nk,
                           uint32_t* eti) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < nk; i += nwarps) {
    for (uint32_t e = offK[i] + lane; e < offK[i + 1]; e += 32) {
      uint32_t v = edgK[e];
      eti[e] = lower_bound_u32(edgC, offC[v], offC[v + 1], (uint32_t)i);
    }
  }
}

// Checked mode: rows strictly ascending, values < 2n, output edge indices < m and each
// output edge index used by exactly two slots (one per direction).
__global__ void validate_ranked_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj,
                                       const uint32_t* __restrict__ eout, int64_t n, int64_t m, uint32_t* uses,
                                       uint32_t* err) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = off[r], e = off[r + 1];
    if (e < b || (int64_t)e > 2 * m) { if (atomicCAS(&err[0], 0u, 30u) == 0u) { err[1] = (uint32_t)r; err[3] = e; } continue; }
    for (uint32_t k = b; k < e; ++k) {
      const uint32_t t = adj[k];
      if ((int64_t)t >= 2 * n || (k > b && t <= adj[k - 1])) {
        if (atomicCAS(&err[0], 0u, 31u) == 0u) { err[1] = k; err[3] = t; }
        break;
      }
      if (eout) {
        const uint32_t o = eout[k];
        if ((int64_t)o >= m) {
          if (atomicCAS(&err[0], 0u, 32u) == 0u) { err[1] = k; err[3] = o; }
          break;
        }
        atomicAdd(&uses[o], 1u);
      }
    }
  }
}

__global__ void validate_uses_kernel(const uint32_t* __restrict__ uses, int64_t m, uint32_t* err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    if (uses[i] != 2u && atomicCAS(&err[0], 0u, 33u) == 0u) { err[1] = (uint32_t)i; err[3] = uses[i]; }
}

int bits_for(uint64_t x) {
  int b = 0;
  while (b < 64 && (x >> b) != 0) ++b;
  return b;
}

Lists lists_of(const pb_graph& g) {
  return Lists{g.offV.get(), g.edgV.get(), g.offU.get(), g.edgU.get(), g.nv};
}

int grid_for(int64_t n, int per_block = 256) { return std::max(1, std::min(ceil_div(n, per_block), sm_count() * 16)); }

}  // namespace

void degrees_combined(const pb_graph& g, uint32_t* deg, cudaStream_t s) {
  const int64_t n = g.nv + g.nu;
  if (n == 0) return;
  PB_LAUNCH(degrees_kernel, grid_for(n), 256, 0, s, lists_of(g), n, deg);
}

void cmp_wedge_counts(const pb_graph& g, int* use_v, int64_t* w_min, int64_t* wv, int64_t* wu, cudaStream_t s) {
  DevBuf<unsigned long long> acc(2, s);
  PB_CUDA_TRY(cudaMemsetAsync(acc.get(), 0, 2 * sizeof(unsigned long long), s));
  if (g.nv) PB_LAUNCH(side_wedges_kernel, grid_for(g.nv), 256, 0, s, g.offV.get(), g.nv, acc.get());
  if (g.nu) PB_LAUNCH(side_wedges_kernel, grid_for(g.nu), 256, 0, s, g.offU.get(), g.nu, acc.get() + 1);
  unsigned long long h[2];
  readback(h, acc.get(), sizeof(h), s);
  *wv = (int64_t)h[0];
  *wu = (int64_t)h[1];
  *use_v = *wv <= *wu;
  *w_min = *wv <= *wu ? *wv : *wu;
}

void vertex_order(const pb_graph& g, int rank_type, int use_v, Ranked& R, cudaStream_t s) {
  const int64_t n = g.nv + g.nu;
  R.n = n;
  R.use_v = use_v;
  R.order.alloc(n, s);
  R.rank.alloc(n, s);
  if (n == 0) return;
  DevBuf<uint32_t> deg(n, s), keys(n, s), keys2(n, s), ids2(n, s);
  degrees_combined(g, deg.get(), s);
  uint32_t kmax = 0;
  int nbits = 0;
  uint32_t* ids = R.order.get();
  if (rank_type == PB_COCORE || rank_type == PB_ACOCORE) {
    const int approx = rank_type == PB_ACOCORE;
    DevBuf<uint32_t> key(n, s), dact(n, s), kbuf(1, s);
    DevBuf<uint8_t> done(n, s);
    PB_LAUNCH(cocore_init_kernel, grid_for(n), 256, 0, s, deg.get(), n, approx, key.get(), dact.get(), done.get());
    while (true) {
      PB_CUDA_TRY(cudaMemsetAsync(kbuf.get(), 0, sizeof(uint32_t), s));
      PB_LAUNCH(cocore_max_kernel, grid_for(n), 256, 0, s, key.get(), done.get(), n, kbuf.get());
      uint32_t k1 = 0;
      readback(&k1, kbuf.get(), sizeof(uint32_t), s);
      if (k1 == 0) break;
      kmax = std::max(kmax, k1 - 1);
      PB_LAUNCH(cocore_round_kernel, grid_for(n * 32), 256, 0, s, lists_of(g), n, approx, kbuf.get(), key.get(),
                dact.get(), done.get());
    }
    PB_LAUNCH(cocore_keys_kernel, grid_for(n), 256, 0, s, key.get(), n, kmax, keys.get(), ids);
    nbits = bits_for(kmax);
  } else {
    if (rank_type == PB_DEG) kmax = g.max_deg;
    else if (rank_type == PB_ADEG) kmax = g.max_deg ? 32u - (uint32_t)__builtin_clz(g.max_deg) : 0u;
    else kmax = 1;
    PB_LAUNCH(order_keys_kernel, grid_for(n), 256, 0, s, deg.get(), n, g.nv, rank_type, use_v, kmax, keys.get(), ids);
    nbits = bits_for(kmax);
  }
  // Stable sort by key: ties keep combined-id order.
  bool alt = radix_sort_pairs_u32(keys.get(), ids, keys2.get(), ids2.get(), n, 0, nbits, s);
  if (alt) PB_CUDA_TRY(cudaMemcpyAsync(ids, ids2.get(), sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
  PB_LAUNCH(invert_order_kernel, grid_for(n), 256, 0, s, R.order.get(), n, R.rank.get());
}

void build_ranked_csr(const pb_graph& g, Ranked& R, bool with_eout, cudaStream_t s) {
  const int64_t n = R.n;
  R.m2 = 2 * g.m;
  R.off.alloc(n + 1, s);
  // Padded to whole 16-byte groups: the aggregators walk rows with 16-byte loads of aligned
  // groups of four entries (entries outside the row are masked, never used).
  R.adj.alloc((size_t)((R.m2 + 3) & ~int64_t(3)) + 4, s);
  if (with_eout) R.eout.alloc(R.m2 > 0 ? R.m2 : 1, s);
  R.max_deg = g.max_deg;
  if (n == 0) {
    PB_CUDA_TRY(cudaMemsetAsync(R.off.get(), 0, sizeof(uint32_t), s));
    return;
  }
  {
    DevBuf<uint32_t> deg(n, s), rdeg(n, s);
    degrees_combined(g, deg.get(), s);
    PB_LAUNCH(ranked_degrees_kernel, grid_for(n), 256, 0, s, R.order.get(), deg.get(), n, rdeg.get());
    exclusive_scan_u32(rdeg.get(), R.off.get(), n, s);
  }
  if (R.m2 == 0) return;
  PB_LAUNCH(ranked_fill_kernel, grid_for(n * 32), 256, 0, s, lists_of(g), R.order.get(), R.rank.get(), R.off.get(), n,
            R.use_v, R.adj.get(), with_eout ? R.eout.get() : nullptr);
  segmented_sort_rows(R.off.get(), n, R.adj.get(), with_eout ? R.eout.get() : nullptr, bits_for((uint64_t)(2 * n)),
                      g.max_deg, s);
}

void wedge_scan(Ranked& R, cudaStream_t s) {
  const int64_t n = R.n;
  R.wsum.alloc(n + 1, s);
  R.pref.alloc(R.m2 > 0 ? R.m2 : 1, s);
  if (n == 0) {
    PB_CUDA_TRY(cudaMemsetAsync(R.wsum.get(), 0, sizeof(int64_t), s));
    R.w_rank = 0;
    return;
  }
  DevBuf<uint32_t> below(n, s);
  DevBuf<int64_t> wc(n, s);
  PB_LAUNCH(below_self_kernel, grid_for(n), 256, 0, s, R.off.get(), R.adj.get(), n, below.get());
  PB_LAUNCH(wedge_scan_kernel, grid_for(n * 32), 256, 0, s, R.off.get(), R.adj.get(), below.get(), n, R.pref.get(),
            wc.get());
  exclusive_scan_i64(wc.get(), R.wsum.get(), n, s);
  readback(&R.w_rank, R.wsum.get() + n, sizeof(int64_t), s);
}

bool check_mode() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("PB_CHECK");
    on = (e && *e && *e != '0') ? 1 : 0;
  }
  return on == 1;
}

void validate_ranked(const Ranked& R, int64_t m, uint32_t* err, cudaStream_t s) {
  if (R.n == 0) return;
  DevBuf<uint32_t> uses;
  if (R.eout.get()) {
    uses.alloc(m > 0 ? m : 1, s);
    PB_CUDA_TRY(cudaMemsetAsync(uses.get(), 0, uses.bytes(), s));
  }
  PB_LAUNCH(validate_ranked_kernel, grid_for(R.n), 256, 0, s, R.off.get(), R.adj.get(), R.eout.get(), R.n, m,
            uses.get(), err);
  if (R.eout.get() && m > 0) PB_LAUNCH(validate_uses_kernel, grid_for(m), 256, 0, s, uses.get(), m, err);
}

void edge_to_idxs(const pb_graph& g, int use_v, uint32_t* eti, cudaStream_t s) {
  const int64_t nk = use_v ? g.nu : g.nv;
  if (nk == 0 || g.m == 0) return;
  const uint32_t* offC = use_v ? g.offV.get() : g.offU.get();
  const uint32_t* edgC = use_v ? g.edgV.get() : g.edgU.get();
  const uint32_t* offK = use_v ? g.offU.get() : g.offV.get();
  const uint32_t* edgK = use_v ? g.edgU.get() : g.edgV.get();
  PB_LAUNCH(eti_kernel, grid_for(nk * 32), 256, 0, s, offC, edgC, offK, edgK, nk, eti);
}

}  // namespace pb
