// Seeded bipartite R-MAT generation on the device, for graphs whose host generation would not
// fit host memory (the 1e9-edge R-MAT workload).  It produces exactly the graph of the host
// generator pb_gen_rmat (pb_gen.cpp): the same SplitMix64 stream (call i returns the mix of
// seed + i * 0x9E3779B97F4A7C15, so it is counter-addressable), the same 32-bit fixed-point
// quadrant thresholds, the same two levels per 64-bit draw, and the same "first m distinct pairs
// in draw order" rule; both CSR sides come out sorted.
//
// Steps: draw D >= m pairs (key = v * nu + u, value = draw index); stable radix sort by key; a
// draw is the first occurrence of its pair when its key differs from its predecessor's; the
// first occurrences are ranked in draw order (scatter into a per-draw flag array, exclusive
// scan); the pairs whose first occurrence ranks below m are kept, already sorted by (v, u),
// which is the V side; the U side is a second sort by (u, v).  D grows by 1/4 until the draws
// hold m distinct pairs.
#include <algorithm>
#include <cmath>

#include "pb_engine.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t i) {
  uint64_t z = seed + i * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct RmatParams {
  uint64_t seed;
  int log_nv, log_nu, levels, calls;  // calls = next() calls per pair
  uint32_t ta, tab, tabc, t_row1, t_col1;
};

// keys[k] = v * nu + u of draw k0 + k, vals[k] = its draw index.
__global__ void rmat_draw_kernel(RmatParams R, uint64_t k0, int64_t n, uint64_t* keys, uint32_t* vals) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = k0 + (uint64_t)t;
    uint64_t call = k * (uint64_t)R.calls;  // next() calls before this draw
    uint64_t row = 0, col = 0, bits = 0;
    int have = 0;
    for (int lvl = 0; lvl < R.levels; ++lvl) {
      if (have == 0) {
        bits = splitmix_at(R.seed, ++call);
        have = 2;
      }
      const uint32_t x = (uint32_t)bits;
      bits >>= 32;
      --have;
      const bool row_live = lvl < R.log_nv, col_live = lvl < R.log_nu;
      uint32_t rb, cb;
      if (row_live && col_live) {
        rb = x >= R.tab;
        cb = (x >= R.ta && x < R.tab) || x >= R.tabc;
      } else if (row_live) {
        rb = x < R.t_row1;
        cb = 0;
      } else {
        rb = 0;
        cb = x < R.t_col1;
      }
      if (row_live) row = (row << 1) | rb;
      if (col_live) col = (col << 1) | cb;
    }
    keys[t] = (row << R.log_nu) | col;
    vals[t] = (uint32_t)k;
  }
}

// first[idx[j]] = 1 when sorted position j starts a new key.
__global__ void first_occurrence_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ idx,
                                        int64_t n, uint32_t* first) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    first[idx[j]] = (j == 0 || keys[j] != keys[j - 1]) ? 1u : 0u;
}

// keep[j] = 1 when sorted position j is the first occurrence of its pair and that occurrence
// ranks below m among first occurrences in draw order (rank = exclusive scan of first[]).
__global__ void keep_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ idx,
                            const uint32_t* __restrict__ rank, int64_t n, uint64_t m, uint8_t* keep) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    keep[j] = ((j == 0 || keys[j] != keys[j - 1]) && rank[idx[j]] < m) ? 1 : 0;
}

__global__ void gather_keys_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ pos, int64_t n,
                                   uint64_t* out) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = keys[pos[j]];
}

// One CSR side from keys sorted by (row << col_bits | col): per-row counts and the columns.
__global__ void side_from_keys_kernel(const uint64_t* __restrict__ keys, int64_t n, int col_bits, uint32_t* cnt,
                                      uint32_t* cols) {
  const uint64_t mask = (1ull << col_bits) - 1ull;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[j];
    atomicAdd(&cnt[k >> col_bits], 1u);
    cols[j] = (uint32_t)(k & mask);
  }
}

// (row << col_bits | col) -> (col << row_bits | row)
__global__ void transpose_keys_kernel(const uint64_t* __restrict__ keys, int64_t n, int col_bits, int row_bits,
                                      uint64_t* out) {
  const uint64_t mask = (1ull << col_bits) - 1ull;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[j];
    out[j] = ((k & mask) << row_bits) | (k >> col_bits);
  }
}

int grid_of(int64_t n) { return std::max(1, std::min(ceil_div(n, 256), sm_count() * 16)); }

uint32_t threshold(double p) {
  if (p <= 0) return 0;
  if (p >= 1) return 0xFFFFFFFFu;
  return (uint32_t)std::llround(p * 4294967296.0);
}

}  // namespace

void gen_rmat_device(int log_nv, int log_nu, int64_t m, double a, double b, double c, double d, uint64_t seed,
                     ParsedCSR& out, cudaStream_t s) {
  PB_REQUIRE(log_nv >= 0 && log_nu >= 0 && log_nv + log_nu <= 62 && log_nv <= 31 && log_nu <= 31, PB_EINVAL,
             "R-MAT sides out of range");
  const int64_t nv = int64_t(1) << log_nv, nu = int64_t(1) << log_nu;
  PB_REQUIRE(m >= 0 && (double)m <= (double)nv * (double)nu, PB_EINVAL, "more edges than pairs");
  PB_REQUIRE(2 * m <= (int64_t)UINT32_MAX && nv + nu < (int64_t(1) << 31), PB_ETOOBIG,
             "graph too large for 32-bit ids and offsets");
  const double tot = a + b + c + d;
  PB_REQUIRE(tot > 0, PB_EINVAL, "R-MAT probabilities sum to zero");
  a /= tot; b /= tot; c /= tot; d /= tot;
  RmatParams R;
  R.seed = seed;
  R.log_nv = log_nv;
  R.log_nu = log_nu;
  R.levels = std::max(log_nv, log_nu);
  R.calls = (R.levels + 1) / 2;
  R.ta = threshold(a);
  R.tab = threshold(a + b);
  R.tabc = threshold(a + b + c);
  R.t_row1 = threshold(c + d);
  R.t_col1 = threshold(b + d);
  const int key_bits = std::max(1, log_nv + log_nu);
  out.nv = nv;
  out.nu = nu;
  out.m = m;
  out.offV.alloc(nv + 1, s);
  out.offU.alloc(nu + 1, s);
  out.edgV.alloc(m > 0 ? m : 1, s);
  out.edgU.alloc(m > 0 ? m : 1, s);
  PB_CUDA_TRY(cudaMemsetAsync(out.offV.get(), 0, out.offV.bytes(), s));
  PB_CUDA_TRY(cudaMemsetAsync(out.offU.get(), 0, out.offU.bytes(), s));
  if (m == 0) return;
  // Draws: start at 1.25 m (R-MAT skew repeats pairs), grow by 1/4 until m distinct pairs exist.
  int64_t D = m + m / 4 + 1024;
  DevBuf<uint64_t> sorted_keys;
  for (int attempt = 0;; ++attempt) {
    PB_REQUIRE(attempt < 40 && D < (int64_t)UINT32_MAX - 1, PB_EINVAL,
               "R-MAT parameters too skewed to reach m distinct pairs");
    DevBuf<uint64_t> k1(D, s), k2(D, s);
    DevBuf<uint32_t> v1(D, s), v2(D, s);
    PB_LAUNCH(rmat_draw_kernel, grid_of(D), 256, 0, s, R, (uint64_t)0, D, k1.get(), v1.get());
    const bool alt = radix_sort_pairs_u64(k1.get(), v1.get(), k2.get(), v2.get(), D, 0, key_bits, s);
    uint64_t* keys = alt ? k2.get() : k1.get();
    uint32_t* idx = alt ? v2.get() : v1.get();
    DevBuf<uint32_t> rank(D + 1, s);
    PB_LAUNCH(first_occurrence_kernel, grid_of(D), 256, 0, s, keys, idx, D, rank.get());
    exclusive_scan_u32(rank.get(), rank.get(), D, s);
    uint32_t distinct = 0;
    readback(&distinct, rank.get() + D, sizeof(distinct), s);
    if ((int64_t)distinct < m) {
      D += D / 4;
      continue;
    }
    DevBuf<uint8_t> keep(D, s);
    PB_LAUNCH(keep_kernel, grid_of(D), 256, 0, s, keys, idx, rank.get(), D, (uint64_t)m, keep.get());
    // The kept positions are the first m entries of a compaction in sorted order.
    DevBuf<uint32_t> pos(D, s), npos(1, s);
    compact_flags(keep.get(), D, pos.get(), npos.get(), s);
    uint32_t kept = 0;
    readback(&kept, npos.get(), sizeof(kept), s);
    PB_REQUIRE((int64_t)kept == m, PB_ECUDA, "device R-MAT: kept pair count mismatch");
    // compact_flags may emit positions out of order; sort them to keep the key order.
    DevBuf<uint32_t> pos2(m, s);
    const bool palt = radix_sort_pairs_u32(pos.get(), nullptr, pos2.get(), nullptr, m, 0, 32, s);
    sorted_keys.alloc(m, s);
    PB_LAUNCH(gather_keys_kernel, grid_of(m), 256, 0, s, keys, palt ? pos2.get() : pos.get(), m, sorted_keys.get());
    break;
  }
  // V side: keys are (v << log_nu | u), sorted.
  DevBuf<uint32_t> cnt(std::max(nv, nu) + 1, s);
  PB_CUDA_TRY(cudaMemsetAsync(cnt.get(), 0, sizeof(uint32_t) * (nv + 1), s));
  PB_LAUNCH(side_from_keys_kernel, grid_of(m), 256, 0, s, sorted_keys.get(), m, log_nu, cnt.get(), out.edgV.get());
  exclusive_scan_u32(cnt.get(), out.offV.get(), nv, s);
  // U side: keys (u << log_nv | v), sorted.
  DevBuf<uint64_t> tk(m, s), tk2(m, s);
  PB_LAUNCH(transpose_keys_kernel, grid_of(m), 256, 0, s, sorted_keys.get(), m, log_nu, log_nv, tk.get());
  sorted_keys.release();
  const bool talt = radix_sort_pairs_u64(tk.get(), nullptr, tk2.get(), nullptr, m, 0, key_bits, s);
  PB_CUDA_TRY(cudaMemsetAsync(cnt.get(), 0, sizeof(uint32_t) * (nu + 1), s));
  PB_LAUNCH(side_from_keys_kernel, grid_of(m), 256, 0, s, talt ? tk2.get() : tk.get(), m, log_nv, cnt.get(),
            out.edgU.get());
  exclusive_scan_u32(cnt.get(), out.offU.get(), nu, s);
}

}  // namespace pb
