// Device primitives: scan, stable LSD radix sort, segmented row sort, compaction.
#include "pb_prims.cuh"

namespace pb {

namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

template <class T>
__device__ T block_exclusive_scan(T x, T* smem /*[32]*/, T& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  T incl = warp_inclusive_scan(x);
  if (lane == 31) smem[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T v = lane < nwarps ? smem[lane] : T(0);
    v = warp_inclusive_scan(v);
    smem[lane] = v;
  }
  __syncthreads();
  T warp_prefix = warp > 0 ? smem[warp - 1] : T(0);
  total = smem[nwarps - 1];
  __syncthreads();
  return warp_prefix + incl - x;
}

template <class T>
__global__ void scan_reduce_kernel(const T* __restrict__ in, int64_t n, T* __restrict__ partials) {
  __shared__ T smem[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = base + (int64_t)k * kScanBlock + threadIdx.x;
    if (idx < n) sum += in[idx];
  }
  T total;
  block_exclusive_scan(sum, smem, total);
  if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

template <class T>
__global__ void scan_tile_kernel(const T* in, T* out, int64_t n, const T* __restrict__ tile_offsets) {
  __shared__ T smem[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = base + k;
    v[k] = idx < n ? in[idx] : T(0);
    sum += v[k];
  }
  T total;
  T prefix = block_exclusive_scan(sum, smem, total) + tile_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = base + k;
    if (idx < n) out[idx] = prefix;
    prefix += v[k];
  }
}

template <class T>
__global__ void scan_small_kernel(const T* in, T* out, int64_t n) {
  // one block, n <= kScanTile; writes out[n] = total
  __shared__ T smem[32];
  const int64_t base = (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = base + k;
    v[k] = idx < n ? in[idx] : T(0);
    sum += v[k];
  }
  T total;
  T prefix = block_exclusive_scan(sum, smem, total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t idx = base + k;
    if (idx < n) out[idx] = prefix;
    prefix += v[k];
  }
  if (threadIdx.x == 0) out[n] = total;
}

template <class T>
void exclusive_scan_impl(const T* in, T* out, int64_t n, cudaStream_t s) {
  if (n <= kScanTile) {
    PB_LAUNCH(scan_small_kernel<T>, 1, kScanBlock, 0, s, in, out, n);
    return;
  }
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  DevBuf<T> partials(tiles + 1, s);
  PB_LAUNCH(scan_reduce_kernel<T>, (unsigned)tiles, kScanBlock, 0, s, in, n, partials.get());
  exclusive_scan_impl<T>(partials.get(), partials.get(), tiles, s);
  PB_LAUNCH(scan_tile_kernel<T>, (unsigned)tiles, kScanBlock, 0, s, in, out, n, partials.get());
  PB_CUDA_TRY(cudaMemcpyAsync(out + n, partials.get() + tiles, sizeof(T), cudaMemcpyDeviceToDevice, s));
}

// ---------------------------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits.  A tile is 256 threads x 16 items; warp w of a tile owns
// items [w*512, (w+1)*512) in 16 rounds of 32, so (warp, round, lane) order is input order.
// Per-item ranks inside a warp come from __match_any_sync on the digit (warp multisplit).
constexpr int kRadixThreads = 256;
constexpr int kRadixRounds = 16;
constexpr int kRadixWarps = kRadixThreads / 32;
constexpr int kRadixTile = kRadixThreads * kRadixRounds;

template <class K>
__global__ void radix_upsweep_kernel(const K* __restrict__ keys, int64_t n, int shift, int64_t tiles,
                                     uint32_t* __restrict__ counts) {
  __shared__ uint32_t hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int k = 0; k < kRadixRounds; ++k) {
    int64_t idx = base + (int64_t)k * kRadixThreads + threadIdx.x;
    if (idx < n) atomicAdd(&hist[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = hist[threadIdx.x];
}

template <class K>
__global__ void radix_downsweep_kernel(const K* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t n,
                                       int shift, int64_t tiles, const uint32_t* __restrict__ offsets,
                                       K* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
  __shared__ uint32_t wcnt[kRadixWarps][256];
  __shared__ uint32_t toff[256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kRadixWarps * 256; d += kRadixThreads) (&wcnt[0][0])[d] = 0;
  toff[threadIdx.x] = offsets[(int64_t)threadIdx.x * tiles + blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRadixTile + (int64_t)warp * (32 * kRadixRounds);
  K kreg[kRadixRounds];
  uint32_t vreg[kRadixRounds];
  uint32_t rank[kRadixRounds];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kRadixRounds; ++r) {
    int64_t idx = base + r * 32 + lane;
    bool valid = idx < n;
    K key = valid ? keys[idx] : K(0);
    kreg[r] = key;
    vreg[r] = (valid && vals) ? vals[idx] : 0u;
    uint32_t d = valid ? ((uint32_t)(key >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    uint32_t pre = valid ? wcnt[warp][d] : 0u;
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = pre + __popc(peers);
    __syncwarp();
    rank[r] = pre + __popc(peers & lt);
  }
  __syncthreads();
  {  // exclusive prefix over warps, per digit
    uint32_t run = 0;
    for (int w = 0; w < kRadixWarps; ++w) {
      uint32_t c = wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRadixRounds; ++r) {
    int64_t idx = base + r * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)(kreg[r] >> shift) & 255u;
      uint32_t pos = toff[d] + wcnt[warp][d] + rank[r];
      keys_out[pos] = kreg[r];
      if (vals) vals_out[pos] = vreg[r];
    }
  }
}

template <class K>
bool radix_sort_impl(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int64_t n, int begin_bit,
                     int end_bit, cudaStream_t s) {
  if (n <= 1 || end_bit <= begin_bit) return false;
  PB_REQUIRE(n < (int64_t)UINT32_MAX, PB_ETOOBIG, "radix sort supports < 2^32 items");
  const int64_t tiles = (n + kRadixTile - 1) / kRadixTile;
  DevBuf<uint32_t> counts(256 * tiles + 1, s);
  bool alt = false;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    K* kin = alt ? keys_alt : keys;
    K* kout = alt ? keys : keys_alt;
    uint32_t* vin = vals ? (alt ? vals_alt : vals) : nullptr;
    uint32_t* vout = vals ? (alt ? vals : vals_alt) : nullptr;
    PB_LAUNCH(radix_upsweep_kernel<K>, (unsigned)tiles, kRadixThreads, 0, s, kin, n, shift, tiles, counts.get());
    exclusive_scan_u32(counts.get(), counts.get(), 256 * tiles, s);
    PB_LAUNCH(radix_downsweep_kernel<K>, (unsigned)tiles, kRadixThreads, 0, s, kin, vin, n, shift, tiles,
              counts.get(), kout, vout);
    alt = !alt;
  }
  return alt;
}

// ---------------------------------------------------------------------------------------------
// Segmented row sort.  Rows hold distinct keys; payload packed as (key << 32 | val).
__global__ void rowsort_warp_kernel(const uint32_t* __restrict__ off, int64_t nrows, uint32_t* keys,
                                    uint32_t* vals) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t r = warp; r < nrows; r += nwarps) {
    const uint32_t b = off[r], e = off[r + 1], len = e - b;
    if (len <= 1 || len > 32) continue;
    uint64_t x = ~0ull;
    if (lane < len) x = ((uint64_t)keys[b + lane] << 32) | (vals ? vals[b + lane] : 0u);
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        uint64_t y = __shfl_xor_sync(0xffffffffu, x, j);
        bool up = (lane & k) == 0;
        bool lower = (lane & j) == 0;
        x = (lower == up) ? (x < y ? x : y) : (x > y ? x : y);
      }
    }
    if (lane < len) {
      keys[b + lane] = (uint32_t)(x >> 32);
      if (vals) vals[b + lane] = (uint32_t)x;
    }
  }
}

constexpr int kRowBlockMax = 4096;  // rows in (32, 4096] sort in shared memory

__global__ void rowsort_block_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ rows,
                                     const uint32_t* __restrict__ nrows_dev, uint32_t* keys, uint32_t* vals) {
  __shared__ uint64_t s[kRowBlockMax];
  const uint32_t nr = *nrows_dev;
  for (uint32_t q = blockIdx.x; q < nr; q += gridDim.x) {
    const uint32_t r = rows[q];
    const uint32_t b = off[r], len = off[r + 1] - b;
    uint32_t N = 64;
    while (N < len) N <<= 1;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
      s[i] = i < len ? (((uint64_t)keys[b + i] << 32) | (vals ? vals[b + i] : 0u)) : ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= N; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
          uint32_t ixj = i ^ j;
          if (ixj > i) {
            uint64_t a = s[i], c = s[ixj];
            bool up = (i & k) == 0;
            if ((a > c) == up) { s[i] = c; s[ixj] = a; }
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
      keys[b + i] = (uint32_t)(s[i] >> 32);
      if (vals) vals[b + i] = (uint32_t)s[i];
    }
    __syncthreads();
  }
}

__global__ void classify_rows_kernel(const uint32_t* __restrict__ off, int64_t nrows, uint32_t* mid_rows,
                                     uint32_t* mid_count, uint32_t* big_rows, uint32_t* big_count) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += (int64_t)gridDim.x * blockDim.x) {
    uint32_t len = off[r + 1] - off[r];
    if (len > 32 && len <= (uint32_t)kRowBlockMax) mid_rows[atomicAdd(mid_count, 1u)] = (uint32_t)r;
    else if (len > (uint32_t)kRowBlockMax) big_rows[atomicAdd(big_count, 1u)] = (uint32_t)r;
  }
}

__global__ void big_row_sizes_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ big_rows,
                                     uint32_t nbig, uint32_t* sizes) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nbig; q += gridDim.x * blockDim.x) {
    uint32_t r = big_rows[q];
    sizes[q] = off[r + 1] - off[r];
  }
}

__global__ void big_row_gather_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ big_rows,
                                      uint32_t nbig, const uint32_t* __restrict__ tstart, const uint32_t* keys,
                                      const uint32_t* vals, int key_bits, uint64_t* tkeys, uint32_t* tvals) {
  for (uint32_t q = blockIdx.x; q < nbig; q += gridDim.x) {
    const uint32_t r = big_rows[q], b = off[r], len = off[r + 1] - b, t0 = tstart[q];
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
      tkeys[t0 + i] = ((uint64_t)q << key_bits) | keys[b + i];
      if (vals) tvals[t0 + i] = vals[b + i];
    }
  }
}

__global__ void big_row_scatter_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ big_rows,
                                       uint32_t nbig, const uint32_t* __restrict__ tstart, const uint64_t* tkeys,
                                       const uint32_t* tvals, int key_bits, uint32_t* keys, uint32_t* vals) {
  const uint64_t mask = key_bits >= 64 ? ~0ull : ((1ull << key_bits) - 1ull);
  for (uint32_t q = blockIdx.x; q < nbig; q += gridDim.x) {
    const uint32_t r = big_rows[q], b = off[r], len = off[r + 1] - b, t0 = tstart[q];
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
      keys[b + i] = (uint32_t)(tkeys[t0 + i] & mask);
      if (vals) vals[b + i] = tvals[t0 + i];
    }
  }
}

__global__ void reduce_max_u32_kernel(const uint32_t* __restrict__ in, int64_t n, uint32_t* out) {
  uint32_t m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, in[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void compact_flags_kernel(const uint8_t* __restrict__ flags, int64_t n, uint32_t* ids,
                                     uint32_t* count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (flags[i]) ids[atomicAdd(count, 1u)] = (uint32_t)i;
}

int bits_for(uint64_t x) {  // bits needed to represent values < x+1
  int b = 0;
  while (b < 64 && (x >> b) != 0) ++b;
  return b;
}

}  // namespace

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
  exclusive_scan_impl<int64_t>(in, out, n, s);
}
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, cudaStream_t s) {
  exclusive_scan_impl<uint32_t>(in, out, n, s);
}

bool radix_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n,
                          int begin_bit, int end_bit, cudaStream_t s) {
  return radix_sort_impl<uint64_t>(keys, vals, keys_alt, vals_alt, n, begin_bit, end_bit, s);
}
bool radix_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, int64_t n,
                          int begin_bit, int end_bit, cudaStream_t s) {
  return radix_sort_impl<uint32_t>(keys, vals, keys_alt, vals_alt, n, begin_bit, end_bit, s);
}

void segmented_sort_rows(const uint32_t* off, int64_t nrows, uint32_t* keys, uint32_t* vals, int key_bits,
                         uint32_t max_row, cudaStream_t s) {
  if (nrows <= 0 || max_row <= 1) return;
  const int sms = sm_count();
  PB_LAUNCH(rowsort_warp_kernel, sms * 8, 256, 0, s, off, nrows, keys, vals);
  if (max_row <= 32) return;
  DevBuf<uint32_t> lists(2 * nrows + 2, s);
  DevBuf<uint32_t> cnt(2, s);
  PB_CUDA_TRY(cudaMemsetAsync(cnt.get(), 0, 2 * sizeof(uint32_t), s));
  uint32_t* mid_rows = lists.get();
  uint32_t* big_rows = lists.get() + nrows + 1;
  PB_LAUNCH(classify_rows_kernel, sms * 4, 256, 0, s, off, nrows, mid_rows, cnt.get(), big_rows, cnt.get() + 1);
  PB_LAUNCH(rowsort_block_kernel, sms * 4, 512, 0, s, off, mid_rows, cnt.get(), keys, vals);
  if (max_row <= (uint32_t)kRowBlockMax) return;
  uint32_t nbig = 0;
  readback(&nbig, cnt.get() + 1, sizeof(uint32_t), s);
  if (nbig == 0) return;
  DevBuf<uint32_t> tstart(nbig + 1, s);
  PB_LAUNCH(big_row_sizes_kernel, ceil_div(nbig, 256), 256, 0, s, off, big_rows, nbig, tstart.get());
  exclusive_scan_u32(tstart.get(), tstart.get(), nbig, s);
  uint32_t tot = 0;
  readback(&tot, tstart.get() + nbig, sizeof(uint32_t), s);
  DevBuf<uint64_t> tk(tot, s), tk2(tot, s);
  DevBuf<uint32_t> tv, tv2;
  if (vals) { tv.alloc(tot, s); tv2.alloc(tot, s); }
  PB_LAUNCH(big_row_gather_kernel, std::min<uint32_t>(nbig, sms * 4), 256, 0, s, off, big_rows, nbig, tstart.get(),
            keys, vals, key_bits, tk.get(), tv.get());
  const int total_bits = key_bits + bits_for(nbig - 1);
  bool alt = radix_sort_pairs_u64(tk.get(), tv.get(), tk2.get(), tv2.get(), tot, 0, total_bits, s);
  PB_LAUNCH(big_row_scatter_kernel, std::min<uint32_t>(nbig, sms * 4), 256, 0, s, off, big_rows, nbig,
            tstart.get(), alt ? tk2.get() : tk.get(), alt ? tv2.get() : tv.get(), key_bits, keys, vals);
}

void reduce_max_u32(const uint32_t* in, int64_t n, uint32_t* out_dev, cudaStream_t s) {
  PB_CUDA_TRY(cudaMemsetAsync(out_dev, 0, sizeof(uint32_t), s));
  if (n <= 0) return;
  PB_LAUNCH(reduce_max_u32_kernel, std::min(ceil_div(n, 256), sm_count() * 8), 256, 0, s, in, n, out_dev);
}

void compact_flags(const uint8_t* flags, int64_t n, uint32_t* ids_out, uint32_t* count_dev, cudaStream_t s) {
  PB_CUDA_TRY(cudaMemsetAsync(count_dev, 0, sizeof(uint32_t), s));
  if (n <= 0) return;
  PB_LAUNCH(compact_flags_kernel, std::min(ceil_div(n, 256), sm_count() * 8), 256, 0, s, flags, n, ids_out,
            count_dev);
}

}  // namespace pb
