// pb_count_total_noalloc: total butterfly count without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a count: code that
// runs inside another framework's memory budget (a caching allocator that owns the device
// memory), code on a path that must not synchronise the device (cudaMalloc/cudaFree can), or
// callers running close to the memory limit.  This entry point takes the graph and the output
// in device memory supplied by the caller, and keeps every byte of scratch it needs in one
// file-scope device array of fixed size, reserved on every GPU that loads the library until
// the process exits.
//
// Algorithm: the per-endpoint dense-counter aggregation of the side order (endpoints on the
// count side chosen as cmpWedgeCounts does, wedges (i, v, u2) with u2 < i; the wedge set of
// CountOrigCompactParallelTotal in the reference), one warp per endpoint, each warp owning a
// dense counter window of nCount entries inside the static scratch.
#include <cstring>
#include <mutex>
#include <string>

#include "pb_common.cuh"

namespace pb {
namespace {

// Scratch layout, in 32-bit words: [0, 64) header (W_V and W_U as 64-bit sums, the endpoint
// cursor), then the per-warp dense counter windows.
constexpr size_t kNoAllocWords = size_t(1) << 22;  // 16 MiB
constexpr size_t kHeaderWords = 64;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

struct Header {
  unsigned long long wv, wu;
  unsigned cursor;
};

// wedgeF / cmpWedgeCounts (butterfly_utils.h:1061-1086): 32-bit products, 64-bit sums.
__global__ void noalloc_side_wedges_kernel(const uint32_t* __restrict__ offV, int64_t nv,
                                           const uint32_t* __restrict__ offU, int64_t nu, Header* h) {
  unsigned long long sv = 0, su = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv + nu; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t d = i < nv ? offV[i + 1] - offV[i] : offU[i - nv + 1] - offU[i - nv];
    const unsigned long long w = (unsigned long long)((uint32_t)(d * (d - 1u)) / 2u);
    if (i < nv) sv += w;
    else su += w;
  }
  sv = warp_sum(sv);
  su = warp_sum(su);
  if ((threadIdx.x & 31) == 0) {
    if (sv) atomicAdd(&h->wv, sv);
    if (su) atomicAdd(&h->wu, su);
  }
}

// One warp per endpoint i of the count side; wedges (i, v, u2) with v in N(i), u2 in N(v),
// u2 < i.  Multiplicities go to the warp's dense window; a second walk reads and clears them
// (atomicExch), adding C(w, 2) once per distinct u2.
__global__ void noalloc_total_kernel(const uint32_t* __restrict__ offV, const uint32_t* __restrict__ edgV,
                                     const uint32_t* __restrict__ offU, const uint32_t* __restrict__ edgU,
                                     int64_t nv, int64_t nu, Header* h, uint32_t* windows, unsigned n_windows,
                                     int64_t* total) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= n_windows) return;
  const bool use_v = h->wv <= h->wu;  // count side U when use_v
  const uint32_t* offK = use_v ? offU : offV;
  const uint32_t* edgK = use_v ? edgU : edgV;
  const uint32_t* offC = use_v ? offV : offU;
  const uint32_t* edgC = use_v ? edgV : edgU;
  const int64_t nK = use_v ? nu : nv;
  uint32_t* cnt = windows + (size_t)wid * (size_t)(nv > nu ? nv : nu);
  long long acc = 0;
  while (true) {
    unsigned i = 0;
    if (lane == 0) i = atomicAdd(&h->cursor, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
    if ((int64_t)i >= nK) break;
    for (int pass = 0; pass < 2; ++pass) {
      for (uint32_t j0 = offK[i]; j0 < offK[i + 1]; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint32_t L = 0, sb = 0;
        if (j < offK[i + 1]) {
          const uint32_t v = edgK[j];
          sb = offC[v];
          L = lower_bound_u32(edgC, sb, offC[v + 1], i) - sb;  // u2 < i
        }
        const uint32_t incl = warp_inclusive_scan(L);
        const uint32_t excl = incl - L;
        const uint32_t T = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t t0 = 0; t0 < T; t0 += 32) {
          const uint32_t t = t0 + lane;
          uint32_t lo = 0;
#pragma unroll
          for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint32_t x = __shfl_sync(0xffffffffu, incl, lo + step - 1);
            if (x <= t) lo += step;
          }
          const uint32_t ex = __shfl_sync(0xffffffffu, excl, lo);
          const uint32_t s = __shfl_sync(0xffffffffu, sb, lo);
          if (t < T) {
            const uint32_t u2 = edgC[s + (t - ex)];
            if (pass == 0) {
              atomicAdd(&cnt[u2], 1u);
            } else {
              const long long w = atomicExch(&cnt[u2], 0u);
              if (w >= 2) acc += w * (w - 1) / 2;
            }
          }
        }
      }
      __syncwarp();
      __threadfence_block();
    }
  }
  acc = warp_sum(acc);
  if (lane == 0 && acc) atomicAdd(reinterpret_cast<unsigned long long*>(total), (unsigned long long)acc);
}

// Device address of the scratch array, resolved once per device with that device current and
// kept for the life of the process (a cudaDeviceReset on that device makes it stale; the
// header says so).
std::mutex g_addr_mu;
uint32_t* g_addr[64] = {nullptr};

cudaError_t scratch_address(int dev, uint32_t** out) {
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

pb_status fail(char* msg, size_t len, pb_status st, const std::string& s) {
  if (msg && len) {
    std::strncpy(msg, s.c_str(), len - 1);
    msg[len - 1] = '\0';
  }
  return st;
}

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" pb_status pb_count_total_noalloc(const pb_csr* g, void* stream, int64_t* total, char* msg, size_t msg_len) {
  if (msg && msg_len) msg[0] = '\0';
  if (!g || !total) return fail(msg, msg_len, PB_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(total) & 7u)
    return fail(msg, msg_len, PB_EINVAL, "pb_count_total_noalloc: total must be 8-byte aligned");
  if (g->nv < 0 || g->nu < 0 || g->m < 0) return fail(msg, msg_len, PB_EINVAL, "negative size");
  const int64_t nmax = g->nv > g->nu ? g->nv : g->nu;
  const size_t avail = kNoAllocWords - kHeaderWords;
  if ((size_t)nmax > avail)
    return fail(msg, msg_len, PB_ETOOBIG,
                "pb_count_total_noalloc: max(nv, nu) = " + std::to_string(nmax) + " exceeds the static scratch limit of " +
                    std::to_string(avail) + " vertices per side");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  uint32_t* base = nullptr;
  if (e == cudaSuccess) e = scratch_address(dev, &base);
  if (e != cudaSuccess) return fail(msg, msg_len, PB_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return fail(msg, msg_len, PB_ECUDA, cudaGetErrorString(e));
  // Windows: one per warp, as many as fit (at most 16 warps per SM).
  size_t n_windows = nmax > 0 ? avail / (size_t)nmax : 0;
  if (n_windows > (size_t)sms * 16) n_windows = (size_t)sms * 16;
  // Everything that must start at zero: the header, the output, and the windows in use (the
  // array keeps the previous call's contents).
  e = cudaMemsetAsync(base, 0, (kHeaderWords + n_windows * (size_t)nmax) * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(total, 0, sizeof(int64_t), s);
  if (e != cudaSuccess) return fail(msg, msg_len, PB_ECUDA, cudaGetErrorString(e));
  if (g->m == 0 || nmax == 0) return PB_OK;
  Header* h = reinterpret_cast<Header*>(base);
  uint32_t* windows = base + kHeaderWords;
  const int64_t n = g->nv + g->nu;
  int grid = (int)((n + 255) / 256);
  if (grid > sms * 8) grid = sms * 8;
  noalloc_side_wedges_kernel<<<grid, 256, 0, s>>>(g->offsetsV, g->nv, g->offsetsU, g->nu, h);
  const unsigned threads = 256;
  const unsigned blocks = (unsigned)((n_windows * 32 + threads - 1) / threads);
  noalloc_total_kernel<<<blocks, threads, 0, s>>>(g->offsetsV, g->edgesV, g->offsetsU, g->edgesU, g->nv, g->nu, h,
                                                  windows, (unsigned)n_windows, total);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(msg, msg_len, PB_ECUDA, cudaGetErrorString(e));
  return PB_OK;
}
