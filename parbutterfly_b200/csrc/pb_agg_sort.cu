// SORT and HIST wedge aggregation (count types SORT/ASORT and HIST/AHIST).
//
// Reference: CountSort / CountSortCE (butterfly_count.h:43-313) materialise the wedges of a batch
// of endpoints, sort them by endpoint pair and read multiplicities off the runs; CountHist /
// CountHistCE (:572-893) reduce the wedge keys with a semisort histogram
// (pbbsa::sparse_histogram, lib/histogram.h:252-345).  Batches hold at most max_wedges wedges
// (the -m option, getNextWedgeIdx, butterfly_utils.h:1700-1714).
//
// Device version.  A batch of endpoints [i0, i1) is flattened: wedge t of the batch lives at
// position t, with key ((i - i0) << 32) | u2, the slot j of (i, v) and the slot of (v, u2) in
// side arrays.  Warps materialise chunks of consecutive wedges (one binary search over the
// per-slot wedge prefix per chunk, then a forward walk).
//   SORT: stable LSD radix sort of (key, position) pairs; run boundaries give w.
//   HIST: one radix pass on the top bits of a key hash groups each key's wedges into one
//         bucket; one CTA per bucket builds the bucket's histogram in a shared-memory table,
//         with __match_any_sync combining equal keys of a warp into one atomic; a bucket whose
//         distinct keys overflow the table is redone against a global-memory table.
// Credits then follow the ranked semantics: C(w,2) per distinct pair to tagged endpoints (and to
// the total), w-1 per wedge to tagged centres (VERT) or to both wedge edges (EDGE).
#include <algorithm>

#include "pb_engine.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

enum Per { VERT = 0, EDGE = 1, TOTAL = 2 };
constexpr uint32_t kChunk = 1024;  // wedges per materialising warp

__global__ void widen_pref_kernel(const uint32_t* __restrict__ pref, int64_t m2, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = pref[i];
}

// First index s in [lo, hi) with a[s + 1] > t, i.e. the segment of a (exclusive prefix) holding t.
__device__ __forceinline__ int64_t seg_of(const int64_t* __restrict__ a, int64_t lo, int64_t hi, int64_t t) {
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Materialises wedges [t_begin, t_end) (global flattened indices) at positions t - t_begin.
__global__ void materialize_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ adj,
                                   const uint32_t* __restrict__ pref, const int64_t* __restrict__ spre, int64_t n,
                                   int64_t m2, int64_t t_begin, int64_t t_end, uint32_t i0, uint64_t* keys,
                                   uint32_t* vals, uint32_t* jarr, uint32_t* s2arr) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t c0 = t_begin + warp * (int64_t)kChunk; c0 < t_end; c0 += nwarps * (int64_t)kChunk) {
    const int64_t c1 = min(c0 + (int64_t)kChunk, t_end);
    int64_t s = 0, row = 0;
    if (lane == 0) {
      s = seg_of(spre, 0, m2, c0);  // slot holding wedge c0 (slots of zero length are skipped)
      int64_t lo = 0, hi = n;       // row of slot s: last r with off[r] <= s
      while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)off[mid] <= s) lo = mid;
        else hi = mid;
      }
      row = lo;
    }
    s = __shfl_sync(0xffffffffu, s, 0);
    row = __shfl_sync(0xffffffffu, row, 0);
    int64_t t = c0;
    while (t < c1 && s < m2) {
      while ((int64_t)off[row + 1] <= s) ++row;
      const uint32_t L = pref[s];
      const int64_t base = spre[s];
      if (base + L > t) {  // slots are visited in order; zero-length ones are passed over
        const uint32_t vt = adj[s];
        const uint32_t vs = off[vt >> 1];
        const int64_t kb = t - base, ke = min((int64_t)L, c1 - base);
        for (int64_t k = kb + lane; k < ke; k += 32) {
          const uint32_t slot2 = vs + (uint32_t)k;
          const uint32_t u2 = adj[slot2] >> 1;
          const int64_t pos = base + k - t_begin;
          keys[pos] = ((uint64_t)((uint32_t)row - i0) << 32) | u2;
          vals[pos] = (uint32_t)pos;
          jarr[pos] = (uint32_t)s;
          s2arr[pos] = slot2;
        }
        t = base + ke;
      }
      ++s;
    }
  }
}

struct Credit {
  const uint32_t* off;
  const uint32_t* adj;
  const uint32_t* eout;
  int per;
  uint32_t i0;
  int64_t* out;
  uint32_t* out32;
  unsigned long long* total;
  __device__ __forceinline__ void add(uint64_t idx, int64_t v) const {
    if (out32) atomicAdd(&out32[idx], (uint32_t)v);
    else atomic_add_i64(&out[idx], v);
  }
  // One wedge of multiplicity w: centre / edge credits.
  __device__ __forceinline__ void wedge(uint32_t i, uint32_t j, uint32_t slot2, int64_t w) const {
    if (w < 2) return;
    if (per == EDGE) {
      add(eout[j], w - 1);
      add(eout[slot2], w - 1);
    } else if (per == VERT) {
      const uint32_t vt = adj[j];
      if (vt & 1u) add(vt >> 1, w - 1);
    }
  }
  // One distinct (i, u2) of multiplicity w: endpoint credits.  i is on the count side when
  // its neighbours are not (tag bit of any entry of its row).
  __device__ __forceinline__ void pair(uint32_t i, uint32_t u2, int64_t w) const {
    if (w < 2) return;
    const int64_t b = w * (w - 1) / 2;
    if (per == TOTAL) atomicAdd(total, (unsigned long long)b);
    else if (per == VERT && !(adj[off[i]] & 1u)) {
      add(i, b);
      add(u2, b);
    }
  }
};

// SORT: sorted keys -> run heads.
__global__ void run_heads_kernel(const uint64_t* __restrict__ keys, int64_t n, uint32_t* head) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    head[p] = (p == 0 || keys[p] != keys[p - 1]) ? 1u : 0u;
}

__global__ void run_starts_kernel(const uint32_t* __restrict__ head, const uint32_t* __restrict__ rid, int64_t n,
                                  uint32_t* start) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    if (head[p]) start[rid[p]] = (uint32_t)p;
}

__global__ void sort_credit_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                   const uint32_t* __restrict__ jarr, const uint32_t* __restrict__ s2arr,
                                   const uint32_t* __restrict__ head, const uint32_t* __restrict__ rid,
                                   const uint32_t* __restrict__ start, int64_t n, Credit C) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t r = rid[p] - (head[p] ? 0u : 1u);  // rid = heads strictly before p
    const int64_t w = (int64_t)start[r + 1] - start[r];
    const uint64_t key = keys[p];
    const uint32_t i = C.i0 + (uint32_t)(key >> 32), u2 = (uint32_t)key;
    const uint32_t pos = vals[p];
    const uint32_t j = jarr[pos];
    C.wedge(i, j, s2arr[pos], w);
    if (head[p]) C.pair(i, u2, w);
  }
}

// HIST: bucket of a key (top bits of a 64-bit mix), the radix digit of the semisort pass.
__device__ __forceinline__ uint32_t key_bucket(uint64_t k, int bits) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  return (uint32_t)(k >> (64 - bits));
}

__global__ void bucket_keys_kernel(const uint64_t* __restrict__ keys, int64_t n, int bits, uint32_t* bkey) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    bkey[p] = key_bucket(keys[p], bits);
}

__global__ void bucket_bounds_kernel(const uint32_t* __restrict__ bkey_sorted, int64_t n, uint32_t nb, uint32_t* bstart) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = bkey_sorted[p];
    const uint32_t prev = p ? bkey_sorted[p - 1] : 0xFFFFFFFFu;
    if (b != prev)
      for (uint32_t q = (prev == 0xFFFFFFFFu ? 0u : prev + 1u); q <= b; ++q) bstart[q] = (uint32_t)p;
    if (p == n - 1)
      for (uint32_t q = b + 1; q <= nb; ++q) bstart[q] = (uint32_t)n;
  }
}

constexpr int kHistThreads = 256;
constexpr uint32_t kHistSlots = 2048;  // 64-bit keys + 32-bit counts: 24 KiB
constexpr unsigned long long kNoKey = ~0ull;

__device__ __forceinline__ uint32_t hslot64(uint64_t k, uint32_t mask) {
  return (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> 40) & mask;
}

// Insert-or-add with a bounded probe; false when the table is full.
__device__ __forceinline__ bool h64_add(unsigned long long* keys, uint32_t* cnt, uint32_t mask, uint64_t k, uint32_t c) {
  uint32_t h = hslot64(k, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    unsigned long long cur = keys[h];
    if (cur == k) { atomicAdd(&cnt[h], c); return true; }
    if (cur == kNoKey) {
      unsigned long long prev = atomicCAS(&keys[h], kNoKey, (unsigned long long)k);
      if (prev == kNoKey || prev == k) { atomicAdd(&cnt[h], c); return true; }
    }
    h = (h + 1) & mask;
  }
  return false;
}

__device__ __forceinline__ uint32_t h64_get(const unsigned long long* keys, const uint32_t* cnt, uint32_t mask, uint64_t k) {
  uint32_t h = hslot64(k, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    const unsigned long long cur = keys[h];
    if (cur == k) return cnt[h];
    if (cur == kNoKey) return 0;
    h = (h + 1) & mask;
  }
  return 0;
}

// One CTA per bucket.  Equal keys of a warp are combined with __match_any_sync before the
// shared-memory insert.  Overflowing buckets are flagged and redone by hist_global_kernel.
__global__ void __launch_bounds__(kHistThreads) hist_bucket_kernel(const uint64_t* __restrict__ keys,
                                                                   const uint32_t* __restrict__ vals,
                                                                   const uint32_t* __restrict__ jarr,
                                                                   const uint32_t* __restrict__ s2arr,
                                                                   const uint32_t* __restrict__ bstart, uint32_t nb,
                                                                   Credit C, uint32_t* overflow) {
  __shared__ unsigned long long tk[kHistSlots];
  __shared__ uint32_t tc[kHistSlots];
  __shared__ int failed;
  const unsigned lane = threadIdx.x & 31u;
  for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const uint32_t p0 = bstart[b], p1 = bstart[b + 1];
    if (p0 == p1) continue;
    for (uint32_t s = threadIdx.x; s < kHistSlots; s += kHistThreads) { tk[s] = kNoKey; tc[s] = 0; }
    if (threadIdx.x == 0) failed = 0;
    __syncthreads();
    for (uint32_t q0 = p0; q0 < p1; q0 += kHistThreads) {
      const uint32_t q = q0 + threadIdx.x;
      const bool valid = q < p1;
      const uint64_t k = valid ? keys[q] : kNoKey;
      const unsigned peers = __match_any_sync(0xffffffffu, k);
      if (valid && lane == (unsigned)(__ffs(peers) - 1))
        if (!h64_add(tk, tc, kHistSlots - 1, k, (uint32_t)__popc(peers))) failed = 1;
    }
    __syncthreads();
    if (failed) {
      if (threadIdx.x == 0) overflow[atomicAdd(&overflow[0], 1u) + 1] = b;
      __syncthreads();
      continue;
    }
    for (uint32_t q = p0 + threadIdx.x; q < p1; q += kHistThreads) {
      const uint64_t k = keys[q];
      const int64_t w = h64_get(tk, tc, kHistSlots - 1, k);
      const uint32_t pos = vals[q];
      C.wedge(C.i0 + (uint32_t)(k >> 32), jarr[pos], s2arr[pos], w);
    }
    for (uint32_t s = threadIdx.x; s < kHistSlots; s += kHistThreads) {
      const unsigned long long k = tk[s];
      if (k == kNoKey) continue;
      C.pair(C.i0 + (uint32_t)(k >> 32), (uint32_t)k, tc[s]);
    }
    __syncthreads();
  }
}

// Redo of overflowing buckets against a global open-addressing table (one bucket per CTA,
// regions of the table carved by bucket start).
__global__ void hist_global_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                   const uint32_t* __restrict__ jarr, const uint32_t* __restrict__ s2arr,
                                   const uint32_t* __restrict__ bstart, const uint32_t* __restrict__ overflow,
                                   unsigned long long* gk, uint32_t* gc, Credit C) {
  const uint32_t nover = overflow[0];
  for (uint32_t o = blockIdx.x; o < nover; o += gridDim.x) {
    const uint32_t b = overflow[o + 1];
    const uint32_t p0 = bstart[b], p1 = bstart[b + 1];
    // Region of 4 x bucket length; the table is the largest power of two inside it (load <= 1/2).
    unsigned long long* tk = gk + 4ull * p0;
    uint32_t* tc = gc + 4ull * p0;
    const uint32_t cap = 4 * (p1 - p0);
    uint32_t mask = 1;
    while (mask * 2 <= cap) mask *= 2;
    mask -= 1;
    for (uint32_t s = threadIdx.x; s <= mask; s += blockDim.x) { tk[s] = kNoKey; tc[s] = 0; }
    __syncthreads();
    for (uint32_t q = p0 + threadIdx.x; q < p1; q += blockDim.x) h64_add(tk, tc, mask, keys[q], 1u);
    __syncthreads();
    for (uint32_t q = p0 + threadIdx.x; q < p1; q += blockDim.x) {
      const uint64_t k = keys[q];
      const uint32_t pos = vals[q];
      C.wedge(C.i0 + (uint32_t)(k >> 32), jarr[pos], s2arr[pos], h64_get(tk, tc, mask, k));
    }
    for (uint32_t s = threadIdx.x; s <= mask; s += blockDim.x)
      if (tk[s] != kNoKey) C.pair(C.i0 + (uint32_t)(tk[s] >> 32), (uint32_t)tk[s], tc[s]);
    __syncthreads();
  }
}

__global__ void gather_keys_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ perm, int64_t n,
                                   uint64_t* out) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    out[q] = keys[perm[q]];
}

__global__ void widen_kernel(const uint32_t* __restrict__ in, int64_t n, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)in[i];
}

int grid_for(int64_t n) { return std::max(1, std::min(ceil_div(n, 256), sm_count() * 16)); }

int bits_for(uint64_t x) {
  int b = 0;
  while (b < 64 && (x >> b) != 0) ++b;
  return b;
}

}  // namespace

CountResult count_ranked_materialized(const Ranked& R, int per, int64_t* out, bool hist, int64_t max_wedges,
                                      cudaStream_t s) {
  CountResult res;
  const int64_t n = R.n, m2 = R.m2;
  const int64_t out_len = per == VERT ? n : (per == EDGE ? m2 / 2 : 1);
  if (out_len > 0) PB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t) * out_len, s));
  if (n == 0 || R.w_rank == 0) return res;
  cudaEvent_t e0, e1;
  PB_CUDA_TRY(cudaEventCreate(&e0));
  PB_CUDA_TRY(cudaEventCreate(&e1));
  PB_CUDA_TRY(cudaEventRecord(e0, s));
  // Per-slot exclusive wedge prefix (the flattened wedge index of each slot's first wedge).
  DevBuf<int64_t> spre(m2 + 1, s);
  PB_LAUNCH(widen_pref_kernel, grid_for(m2), 256, 0, s, R.pref.get(), m2, spre.get());
  exclusive_scan_i64(spre.get(), spre.get(), m2, s);
  // Endpoint wedge prefix on the host, to cut batches at endpoint boundaries.
  std::vector<int64_t> wsum(n + 1);
  PB_CUDA_TRY(cudaMemcpyAsync(wsum.data(), R.wsum.get(), sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  // Batch budget: -m, capped so that one batch's arrays stay within a few GiB.
  const int64_t cap = std::min<int64_t>(max_wedges > 0 ? max_wedges : (int64_t)1 << 27, (int64_t)1 << 27);
  const uint64_t md = R.max_deg > 0 ? R.max_deg - 1 : 0;
  DevBuf<uint32_t> out32;
  if (per == EDGE && md * md < (1ull << 32)) {
    out32.alloc(out_len, s);
    PB_CUDA_TRY(cudaMemsetAsync(out32.get(), 0, out32.bytes(), s));
  }
  DevBuf<unsigned long long> total(1, s);
  PB_CUDA_TRY(cudaMemsetAsync(total.get(), 0, sizeof(unsigned long long), s));
  int64_t i0 = 0;
  while (i0 < n) {
    // Largest i1 with wsum[i1] - wsum[i0] <= cap (at least one endpoint).
    int64_t i1 = std::upper_bound(wsum.begin() + i0 + 1, wsum.end(), wsum[i0] + cap) - wsum.begin() - 1;
    if (i1 <= i0) i1 = i0 + 1;
    const int64_t tb = wsum[i0], te = wsum[i1], cnt = te - tb;
    PB_REQUIRE(cnt < (int64_t)UINT32_MAX, PB_ETOOBIG, "a single endpoint's wedges exceed 2^32");
    if (cnt > 0) {
      DevBuf<uint64_t> keys(cnt, s), keys2(cnt, s);
      DevBuf<uint32_t> vals(cnt, s), vals2(cnt, s), jarr(cnt, s), s2arr(cnt, s);
      PB_LAUNCH(materialize_kernel, std::max(1, std::min(ceil_div(cnt, (int64_t)kChunk * 8), sm_count() * 32)), 256, 0,
                s, R.off.get(), R.adj.get(), R.pref.get(), spre.get(), n, m2, tb, te, (uint32_t)i0, keys.get(),
                vals.get(), jarr.get(), s2arr.get());
      Credit C{R.off.get(), R.adj.get(), R.eout.get(), per, (uint32_t)i0, out, out32.get(), total.get()};
      const int key_bits = 32 + bits_for((uint64_t)(i1 - i0));
      if (!hist) {
        const bool alt = radix_sort_pairs_u64(keys.get(), vals.get(), keys2.get(), vals2.get(), cnt, 0, key_bits, s);
        uint64_t* k = alt ? keys2.get() : keys.get();
        uint32_t* v = alt ? vals2.get() : vals.get();
        DevBuf<uint32_t> head(cnt, s), rid(cnt + 1, s), start(cnt + 1, s);
        PB_LAUNCH(run_heads_kernel, grid_for(cnt), 256, 0, s, k, cnt, head.get());
        exclusive_scan_u32(head.get(), rid.get(), cnt, s);
        PB_LAUNCH(run_starts_kernel, grid_for(cnt), 256, 0, s, head.get(), rid.get(), cnt, start.get());
        uint32_t nruns = 0;
        PB_CUDA_TRY(cudaMemcpyAsync(&nruns, rid.get() + cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        PB_CUDA_TRY(cudaStreamSynchronize(s));
        const uint32_t cnt32 = (uint32_t)cnt;
        PB_CUDA_TRY(cudaMemcpyAsync(start.get() + nruns, &cnt32, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        PB_LAUNCH(sort_credit_kernel, grid_for(cnt), 256, 0, s, k, v, jarr.get(), s2arr.get(), head.get(),
                  rid.get(), start.get(), cnt, C);
        PB_CUDA_TRY(cudaStreamSynchronize(s));
      } else {
        // Semisort: bucket keys by hash (about 1024 wedges per bucket), one stable radix pass.
        int bits = bits_for((uint64_t)std::max<int64_t>(1, cnt / 1024));
        bits = std::max(1, std::min(bits, 24));
        const uint32_t nb = 1u << bits;
        DevBuf<uint32_t> bkey(cnt, s), bkey2(cnt, s), perm(cnt, s), perm2(cnt, s);
        PB_LAUNCH(bucket_keys_kernel, grid_for(cnt), 256, 0, s, keys.get(), cnt, bits, bkey.get());
        // sort (bucket, original position) pairs; positions double as the permutation
        PB_CUDA_TRY(cudaMemcpyAsync(perm.get(), vals.get(), sizeof(uint32_t) * cnt, cudaMemcpyDeviceToDevice, s));
        const bool alt = radix_sort_pairs_u32(bkey.get(), perm.get(), bkey2.get(), perm2.get(), cnt, 0, bits, s);
        uint32_t* bs = alt ? bkey2.get() : bkey.get();
        uint32_t* pm = alt ? perm2.get() : perm.get();
        DevBuf<uint32_t> bstart(nb + 1, s);
        PB_LAUNCH(bucket_bounds_kernel, grid_for(cnt), 256, 0, s, bs, cnt, nb, bstart.get());
        // gather keys into bucket order
        DevBuf<uint32_t> overflow(nb + 1, s);
        PB_CUDA_TRY(cudaMemsetAsync(overflow.get(), 0, sizeof(uint32_t), s));
        PB_LAUNCH(gather_keys_kernel, grid_for(cnt), 256, 0, s, keys.get(), pm, cnt, keys2.get());
        PB_LAUNCH(hist_bucket_kernel, std::min<int>(nb, sm_count() * 8), kHistThreads, 0, s, keys2.get(), pm,
                  jarr.get(), s2arr.get(), bstart.get(), nb, C, overflow.get());
        uint32_t nover = 0;
        PB_CUDA_TRY(cudaMemcpyAsync(&nover, overflow.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        PB_CUDA_TRY(cudaStreamSynchronize(s));
        if (nover) {
          DevBuf<unsigned long long> gk(4 * cnt + 64, s);
          DevBuf<uint32_t> gc(4 * cnt + 64, s);
          PB_LAUNCH(hist_global_kernel, std::min<int>(nover, sm_count() * 4), 512, 0, s, keys2.get(), pm, jarr.get(),
                    s2arr.get(), bstart.get(), overflow.get(), gk.get(), gc.get(), C);
        }
        PB_CUDA_TRY(cudaStreamSynchronize(s));
      }
    }
    i0 = i1;
  }
  if (per == TOTAL)
    PB_CUDA_TRY(cudaMemcpyAsync(out, total.get(), sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
  if (out32.get()) PB_LAUNCH(widen_kernel, grid_for(out_len), 256, 0, s, out32.get(), out_len, out);
  PB_CUDA_TRY(cudaEventRecord(e1, s));
  PB_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0;
  PB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  res.agg_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return res;
}

}  // namespace pb
