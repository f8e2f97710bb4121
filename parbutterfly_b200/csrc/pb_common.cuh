// Shared device/host helpers of libpbgpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/parbutterfly_b200.h"

namespace pb {

constexpr int kWarp = 32;

// Error carried out of internal routines; the C ABI converts it into a pb_status plus the
// context's last-error string.
struct Error {
  pb_status status;
  std::string msg;
};

#define PB_CUDA_TRY(expr)                                                                       \
  do {                                                                                          \
    cudaError_t _e = (expr);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      throw ::pb::Error{PB_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e) + " at " + \
                                      __FILE__ + ":" + std::to_string(__LINE__)};              \
  } while (0)

#define PB_REQUIRE(cond, status, msg)                  \
  do {                                                 \
    if (!(cond)) throw ::pb::Error{(status), (msg)};   \
  } while (0)

// Launch bookkeeping: every kernel launch of the library goes through PB_LAUNCH so the
// context can report how many of its own kernels ran.
extern thread_local int64_t* g_launch_counter;
#define PB_LAUNCH(kernel, grid, block, smem, stream, ...)                      \
  do {                                                                         \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                \
    PB_CUDA_TRY(cudaGetLastError());                                           \
    if (::pb::g_launch_counter) ++*::pb::g_launch_counter;                     \
  } while (0)

// Stream-ordered device buffer (cudaMallocAsync from the device's default pool, which the
// context configures to keep freed memory for reuse).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(size_t count, cudaStream_t stream) { alloc(count, stream); }
  void alloc(size_t count, cudaStream_t stream) {
    release();
    s = stream;
    n = count;
    if (count) {
      cudaError_t e = cudaMallocAsync((void**)&p, sizeof(T) * count, stream);
      if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        cudaGetLastError();
        throw Error{PB_ENOMEM, "device allocation of " + std::to_string(sizeof(T) * count) + " bytes failed"};
      }
    }
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    release();
    p = o.p; n = o.n; s = o.s;
    o.p = nullptr; o.n = 0;
    return *this;
  }
  T* get() const { return p; }
  size_t bytes() const { return n * sizeof(T); }
  // The stream the buffer is freed on.  Long-lived objects (graphs, models, batches) may outlive
  // the stream they were allocated on (a context's own stream ends with the context); their
  // destroy functions synchronise the device and rebind their buffers to the legacy default
  // stream, which is always valid.
  void rebind(cudaStream_t ns) { s = ns; }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Host readbacks between kernels (sizes, counters, status words) go through readback(), so a
// whole pipeline can be captured into a CUDA graph: during an eager recording run every value
// read is logged; while the stream is being captured the logged values are returned instead
// and no device-to-host copy or synchronisation enters the graph.  Without an active
// recorder readback() is a plain cudaMemcpyAsync + cudaStreamSynchronize.
struct Recorder {
  bool capturing = false;
  std::vector<std::vector<uint8_t>> log;
  size_t pos = 0;
  std::vector<void*> pinned;  // host memory the captured graph reads or writes (kept alive)
  unsigned* status = nullptr; // pinned {peel error bits, unpeeled items} written by the graph
  ~Recorder();
  void* pinned_alloc(size_t bytes);
};
extern thread_local Recorder* g_recorder;
void readback(void* dst, const void* src, size_t bytes, cudaStream_t s);
inline bool capturing() { return g_recorder && g_recorder->capturing; }

// Number of SMs of the current device (cached per process; one device per context).
int sm_count();

// ---- device helpers -----------------------------------------------------------------------
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T x) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if ((int)lane_id() >= o) x += y;
  }
  return x;
}

template <class T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// floor(log2(d)) + 1 for d > 0 and 0 for d == 0: the approximate-degree key of
// butterfly_utils.h:279-280, exact in integer arithmetic.
__device__ __forceinline__ uint32_t log_key(uint32_t d) { return 32u - __clz(d); }

// First index in a[lo, hi) with a[idx] >= key (a ascending).
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                                     uint32_t key) {
  while (lo < hi) {
    uint32_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void atomic_add_i64(int64_t* p, int64_t v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

}  // namespace pb
