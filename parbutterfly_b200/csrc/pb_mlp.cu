// Tensor-core GEMM (tcgen05) and the learned scheduler's MLP: forward, backward and Adam.
//
// tc_gemm_kernel: one CTA of 128 threads computes a 128 x N tile (N <= 128) of
// D = A * B^T.  Operands are staged by the threads into shared memory in the canonical
// no-swizzle K-major core-matrix layout (8 rows x 16 bytes per core matrix), one 64-wide K
// chunk at a time; thread 0 issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) with the
// accumulator in TMEM and commits to an mbarrier; after the last chunk every warp reads its 32
// TMEM lanes with tcgen05.ld and applies the epilogue.  Every wait on the mbarrier is bounded
// (2 s of globaltimer); a timeout is recorded in err[0] and the kernel releases its TMEM and
// returns.
//
// The operands are small (the scheduler's features and 64-wide hidden layers), so they are
// staged with ordinary loads rather than TMA: the staging handles any stride (transposed
// operands for the backward pass) and zero-pads partial tiles.
#include <cmath>
#include <cstring>

#include "pb_mlp.cuh"

namespace pb {

namespace {

constexpr int kTileM = 128;
constexpr int kKC = 64;
constexpr int kGemmThreads = 128;
constexpr uint64_t kWaitNs = 2000000000ull;
constexpr int kGemmPadSmem = 24 * 1024;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) of a tile with `rows` rows: core matrices of 8 rows x 8
// BF16; consecutive 8-row groups 128 bytes apart (SBO), consecutive 8-column K chunks
// rows * 16 bytes apart (LBO).
__device__ __forceinline__ uint32_t cm_off(uint32_t r, uint32_t k, uint32_t rows) {
  return (k >> 3) * (rows * 16u) + (r >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (tcgen05): start address, leading and stride byte
// offsets (all >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = gtimer();
  while (!mbar_try(bar, parity))
    if (gtimer() - t0 > limit_ns) return false;
  return true;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kGemmThreads) tc_gemm_kernel(GemmSpec g, uint32_t* err) {
  __shared__ __align__(1024) uint8_t sA[kTileM * kKC * 2];
  __shared__ __align__(1024) uint8_t sB[kGemmMaxN * kKC * 2];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * kTileM;
  const int npad = (g.N + 15) & ~15;
  uint32_t ncols = 32;
  while (ncols < (uint32_t)npad) ncols <<= 1;
  const int64_t kbeg = g.k_split > 0 ? (int64_t)blockIdx.y * g.k_split : 0;
  const int64_t kend = g.k_split > 0 ? (g.K < kbeg + g.k_split ? g.K : kbeg + g.k_split) : g.K;
  const uint32_t bar_a = smem_addr(&bar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    failed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = idesc_bf16(kTileM, (uint32_t)npad);
  uint32_t parity = 0;
  int chunks = 0;
  for (int64_t k0 = kbeg; k0 < kend; k0 += kKC, ++chunks) {
    const int kc = (int)(kend - k0 < (int64_t)kKC ? kend - k0 : (int64_t)kKC);
    const int ksteps = (kc + 15) >> 4;
    const int kcols = ksteps * 16;
    for (int idx = tid; idx < kTileM * kcols; idx += kGemmThreads) {
      const int r = idx / kcols, k = idx - r * kcols;
      const int64_t m = m0 + r;
      __nv_bfloat16 v = __float2bfloat16(0.f);
      if (m < g.M && k < kc) v = g.A[m * g.sam + (k0 + k) * g.sak];
      *reinterpret_cast<__nv_bfloat16*>(sA + cm_off(r, k, kTileM)) = v;
    }
    for (int idx = tid; idx < npad * kcols; idx += kGemmThreads) {
      const int r = idx / kcols, k = idx - r * kcols;
      __nv_bfloat16 v = __float2bfloat16(0.f);
      if (r < g.N && k < kc) v = g.B[(int64_t)r * g.sbn + (k0 + k) * g.sbk];
      *reinterpret_cast<__nv_bfloat16*>(sB + cm_off(r, k, npad)) = v;
    }
    // Make the generic-proxy stores visible to the tensor cores (async proxy).
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int s = 0; s < ksteps; ++s) {
        const uint64_t ad = smem_desc(smem_addr(sA) + (uint32_t)s * 2u * kTileM * 16u, kTileM * 16u, 128u);
        const uint64_t bd = smem_desc(smem_addr(sB) + (uint32_t)s * 2u * (uint32_t)npad * 16u, (uint32_t)npad * 16u, 128u);
        const uint32_t accumulate = (chunks > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
                tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                   : "memory");
    }
    // The next chunk overwrites the staged operands: wait until the MMAs have read them.
    const bool ok = mbar_wait(bar_a, parity, kWaitNs);
    parity ^= 1u;
    if (!ok) failed = 1;
    __syncthreads();
    if (failed) break;
  }
  if (failed) {
    if (tid == 0 && err) atomicExch(err, 1u);
    mbar_wait(bar_a, parity ^ 1u, kWaitNs);  // give an MMA still in flight the chance to land
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t m = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < npad; c0 += 16) {
      uint32_t r[16];
      if (chunks > 0) {
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = 0u;
      }
      if (m >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = c0 + j;
        if (n >= g.N) break;
        float v = __uint_as_float(r[j]);
        if (g.bias && (g.epi != GEMM_ATOMIC || blockIdx.y == 0)) v += g.bias[n];
        if (g.epi == GEMM_STORE) {
          g.D[m * g.ldd + n] = v;
        } else if (g.epi == GEMM_RELU) {
          g.H[m * g.ldh + n] = __float2bfloat16(v > 0.f ? v : 0.f);
        } else if (g.epi == GEMM_ATOMIC) {
          atomicAdd(&g.D[m * g.ldd + n], v);
        } else {
          const float mk = __bfloat162float(g.mask[m * g.ldh + n]);
          g.H[m * g.ldh + n] = __float2bfloat16(mk > 0.f ? v : 0.f);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// ---- MLP helpers ---------------------------------------------------------------------------
// Packed FP32 parameter vector: w1 [64x16] | b1 [64] | w2 [64x64] | b2 [64] | w3 [16x64] | b3 [16]
// (rows 1..15 of w3 and entries 1..15 of b3 stay zero: the output layer is an N = 16 product).
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpOutPad * kMlpHidden;
constexpr int kParams = kOffB3 + kMlpOutPad;

struct Norm {
  float mean[kMlpIn];
  float scale[kMlpIn];
};

// Xh[r] = bf16((X[idx[r]] - mean) * scale); t[r] = y[idx[r]] (idx null: identity).
__global__ void gather_standardize_kernel(const float* __restrict__ X, const float* __restrict__ y,
                                          const uint32_t* __restrict__ idx, int64_t rows, Norm nm,
                                          __nv_bfloat16* Xh, float* t) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < rows * kMlpIn;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / kMlpIn;
    const int f = (int)(e - r * kMlpIn);
    const int64_t src = idx ? (int64_t)idx[r] : r;
    Xh[e] = __float2bfloat16((X[src * kMlpIn + f] - nm.mean[f]) * nm.scale[f]);
    if (f == 0 && t) t[r] = y[src];
  }
}

// dY (padded to 16 columns, BF16) = 2 (Y - t) / B; db3 += dY; loss += (Y - t)^2 / B.
__global__ void loss_grad_kernel(const float* __restrict__ Y, const float* __restrict__ t, int64_t B,
                                 __nv_bfloat16* dYh, float* db3, float* loss) {
  float gsum = 0.f, lsum = 0.f;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
    const float d = Y[b * kMlpOutPad] - t[b];
    const float gr = 2.f * d / (float)B;
    dYh[b * kMlpOutPad] = __float2bfloat16(gr);
    for (int c = 1; c < kMlpOutPad; ++c) dYh[b * kMlpOutPad + c] = __float2bfloat16(0.f);
    gsum += gr;
    lsum += d * d / (float)B;
  }
  gsum = warp_sum(gsum);
  lsum = warp_sum(lsum);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(db3, gsum);
    atomicAdd(loss, lsum);
  }
}

// out[c] += sum over rows of Z[r][c] (Z BF16 [rows x 64]).
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ Z, int64_t rows, float* out) {
  const int c = threadIdx.x & 63;
  float acc = 0.f;
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 6) + (threadIdx.x >> 6); r < rows;
       r += (int64_t)gridDim.x * (blockDim.x >> 6))
    acc += __bfloat162float(Z[r * kMlpHidden + c]);
  atomicAdd(&out[c], acc);
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                            float c1, float c2, float eps) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ p, int n, __nv_bfloat16* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(p[i]);
}

// y[r] = Y[r][0] / y_scale + y_mean.
__global__ void destandardize_kernel(const float* __restrict__ Y, int64_t n, float mean, float inv_scale, float* y) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    y[r] = Y[r * kMlpOutPad] * inv_scale + mean;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double uniform01(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

int grid_for(int64_t n, int threads) { return std::max(1, std::min(ceil_div(n, threads), sm_count() * 4)); }

}  // namespace

void tc_gemm_bf16(const GemmSpec& g, uint32_t* err, cudaStream_t s) {
  PB_REQUIRE(g.N >= 1 && g.N <= kGemmMaxN, PB_EINVAL, "tc_gemm_bf16: N must be in [1, 128]");
  PB_REQUIRE(g.M >= 0 && g.K >= 0, PB_EINVAL, "tc_gemm_bf16: negative size");
  PB_REQUIRE(g.k_split == 0 || g.epi == GEMM_ATOMIC, PB_EINVAL, "tc_gemm_bf16: split K needs the atomic epilogue");
  PB_REQUIRE(g.k_split >= 0, PB_EINVAL, "tc_gemm_bf16: negative k_split");
  if (g.M == 0) return;
  const int gx = (int)((g.M + kTileM - 1) / kTileM);
  const int gy = g.k_split > 0 ? std::max(1, (int)((g.K + g.k_split - 1) / g.k_split)) : 1;
  // Unused dynamic shared memory caps residency at 4 CTAs per SM, so the CTAs on an SM never
  // ask for more than its 512 TMEM columns (4 x 128) and no allocation has to wait.
  static thread_local int attr_dev = -1;
  int dev = 0;
  PB_CUDA_TRY(cudaGetDevice(&dev));
  if (attr_dev != dev) {
    PB_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmPadSmem));
    attr_dev = dev;
  }
  PB_LAUNCH(tc_gemm_kernel, dim3(gx, gy), kGemmThreads, kGemmPadSmem, s, g, err);
}

void MlpModel::init(uint64_t seed, cudaStream_t stream) {
  s = stream;
  PB_CUDA_TRY(cudaGetDevice(&device));
  std::vector<float> p(kParams, 0.f);
  uint64_t st = seed;
  // He-style uniform initialisation; biases zero.
  auto fill = [&](int off, int cols, int live_rows) {  // live_rows x cols, row-major
    const double a = std::sqrt(6.0 / cols);
    for (int r = 0; r < live_rows; ++r)
      for (int c = 0; c < cols; ++c) p[off + r * cols + c] = (float)((2.0 * uniform01(st) - 1.0) * a);
  };
  fill(kOffW1, kMlpIn, kMlpHidden);
  fill(kOffW2, kMlpHidden, kMlpHidden);
  fill(kOffW3, kMlpHidden, 1);  // output layer: row 0 only
  params.alloc(kParams, s);
  grads.alloc(kParams, s);
  m_adam.alloc(kParams, s);
  v_adam.alloc(kParams, s);
  whalf.alloc(kParams, s);
  err.alloc(4, s);
  PB_CUDA_TRY(cudaMemcpyAsync(params.get(), p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemsetAsync(m_adam.get(), 0, m_adam.bytes(), s));
  PB_CUDA_TRY(cudaMemsetAsync(v_adam.get(), 0, v_adam.bytes(), s));
  PB_CUDA_TRY(cudaMemsetAsync(err.get(), 0, err.bytes(), s));
  PB_LAUNCH(to_bf16_kernel, grid_for(kParams, 256), 256, 0, s, params.get(), kParams, whalf.get());
  for (int f = 0; f < kMlpIn; ++f) {
    x_mean[f] = 0.f;
    x_scale[f] = 1.f;
  }
  y_mean = 0.f;
  y_scale = 1.f;
  steps = 0;
  trained = false;
}

namespace {

struct Act {
  DevBuf<__nv_bfloat16> Xh, H1, H2, dYh, dZ2, dZ1;
  DevBuf<float> Y, t;
  int64_t cap = 0;
  void ensure(int64_t rows, cudaStream_t s) {
    if (rows <= cap) return;
    cap = rows;
    Xh.alloc(rows * kMlpIn, s);
    H1.alloc(rows * kMlpHidden, s);
    H2.alloc(rows * kMlpHidden, s);
    dYh.alloc(rows * kMlpOutPad, s);
    dZ2.alloc(rows * kMlpHidden, s);
    dZ1.alloc(rows * kMlpHidden, s);
    Y.alloc(rows * kMlpOutPad, s);
    t.alloc(rows, s);
  }
};

// Forward pass of B standardised rows in A.Xh: A.H1, A.H2 (BF16) and A.Y (FP32, 16 columns).
void forward(const MlpModel& M, Act& A, int64_t B, cudaStream_t s) {
  const __nv_bfloat16* wh = M.whalf.get();
  const float* p = M.params.get();
  uint32_t* err = M.err.get();
  GemmSpec g;
  g.A = A.Xh.get(); g.sam = kMlpIn; g.sak = 1;
  g.B = wh + kOffW1; g.sbn = kMlpIn; g.sbk = 1;
  g.M = B; g.N = kMlpHidden; g.K = kMlpIn;
  g.epi = GEMM_RELU; g.bias = p + kOffB1; g.H = A.H1.get(); g.ldh = kMlpHidden;
  tc_gemm_bf16(g, err, s);
  g = GemmSpec();
  g.A = A.H1.get(); g.sam = kMlpHidden; g.sak = 1;
  g.B = wh + kOffW2; g.sbn = kMlpHidden; g.sbk = 1;
  g.M = B; g.N = kMlpHidden; g.K = kMlpHidden;
  g.epi = GEMM_RELU; g.bias = p + kOffB2; g.H = A.H2.get(); g.ldh = kMlpHidden;
  tc_gemm_bf16(g, err, s);
  g = GemmSpec();
  g.A = A.H2.get(); g.sam = kMlpHidden; g.sak = 1;
  g.B = wh + kOffW3; g.sbn = kMlpHidden; g.sbk = 1;
  g.M = B; g.N = kMlpOutPad; g.K = kMlpHidden;
  g.epi = GEMM_STORE; g.bias = p + kOffB3; g.D = A.Y.get(); g.ldd = kMlpOutPad;
  tc_gemm_bf16(g, err, s);
}

// Gradients of the batch loss into M.grads (zeroed here).
void backward(MlpModel& M, Act& A, int64_t B, float* loss_dev, cudaStream_t s) {
  float* gr = M.grads.get();
  const __nv_bfloat16* wh = M.whalf.get();
  uint32_t* err = M.err.get();
  PB_CUDA_TRY(cudaMemsetAsync(gr, 0, sizeof(float) * kParams, s));
  PB_LAUNCH(loss_grad_kernel, grid_for(B, 256), 256, 0, s, A.Y.get(), A.t.get(), B, A.dYh.get(), gr + kOffB3, loss_dev);
  const int64_t ks = 512;  // split of the batch dimension for the weight gradients
  // dW3[c][h] = sum_b dY[b][c] H2[b][h]
  GemmSpec g;
  g.A = A.dYh.get(); g.sam = 1; g.sak = kMlpOutPad;
  g.B = A.H2.get(); g.sbn = 1; g.sbk = kMlpHidden;
  g.M = kMlpOutPad; g.N = kMlpHidden; g.K = B; g.k_split = ks;
  g.epi = GEMM_ATOMIC; g.D = gr + kOffW3; g.ldd = kMlpHidden;
  tc_gemm_bf16(g, err, s);
  // dZ2[b][h] = (sum_c dY[b][c] W3[c][h]) * [H2[b][h] > 0]
  g = GemmSpec();
  g.A = A.dYh.get(); g.sam = kMlpOutPad; g.sak = 1;
  g.B = wh + kOffW3; g.sbn = 1; g.sbk = kMlpHidden;
  g.M = B; g.N = kMlpHidden; g.K = kMlpOutPad;
  g.epi = GEMM_MASK; g.H = A.dZ2.get(); g.ldh = kMlpHidden; g.mask = A.H2.get();
  tc_gemm_bf16(g, err, s);
  PB_LAUNCH(colsum_kernel, grid_for(B * kMlpHidden, 256), 256, 0, s, A.dZ2.get(), B, gr + kOffB2);
  // dW2[j][i] = sum_b dZ2[b][j] H1[b][i]
  g = GemmSpec();
  g.A = A.dZ2.get(); g.sam = 1; g.sak = kMlpHidden;
  g.B = A.H1.get(); g.sbn = 1; g.sbk = kMlpHidden;
  g.M = kMlpHidden; g.N = kMlpHidden; g.K = B; g.k_split = ks;
  g.epi = GEMM_ATOMIC; g.D = gr + kOffW2; g.ldd = kMlpHidden;
  tc_gemm_bf16(g, err, s);
  // dZ1[b][i] = (sum_j dZ2[b][j] W2[j][i]) * [H1[b][i] > 0]
  g = GemmSpec();
  g.A = A.dZ2.get(); g.sam = kMlpHidden; g.sak = 1;
  g.B = wh + kOffW2; g.sbn = 1; g.sbk = kMlpHidden;
  g.M = B; g.N = kMlpHidden; g.K = kMlpHidden;
  g.epi = GEMM_MASK; g.H = A.dZ1.get(); g.ldh = kMlpHidden; g.mask = A.H1.get();
  tc_gemm_bf16(g, err, s);
  PB_LAUNCH(colsum_kernel, grid_for(B * kMlpHidden, 256), 256, 0, s, A.dZ1.get(), B, gr + kOffB1);
  // dW1[j][f] = sum_b dZ1[b][j] X[b][f]
  g = GemmSpec();
  g.A = A.dZ1.get(); g.sam = 1; g.sak = kMlpHidden;
  g.B = A.Xh.get(); g.sbn = 1; g.sbk = kMlpIn;
  g.M = kMlpHidden; g.N = kMlpIn; g.K = B; g.k_split = ks;
  g.epi = GEMM_ATOMIC; g.D = gr + kOffW1; g.ldd = kMlpIn;
  tc_gemm_bf16(g, err, s);
}

Norm norm_of(const MlpModel& M) {
  Norm nm;
  for (int f = 0; f < kMlpIn; ++f) {
    nm.mean[f] = M.x_mean[f];
    nm.scale[f] = M.x_scale[f];
  }
  return nm;
}

void check_err(const MlpModel& M, cudaStream_t s) {
  uint32_t h = 0;
  PB_CUDA_TRY(cudaMemcpyAsync(&h, M.err.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  PB_REQUIRE(h == 0, PB_ETIMEOUT, "tensor-core GEMM: bounded mbarrier wait ran out");
}

}  // namespace

float MlpModel::train(const float* X, const float* y, int64_t n, int epochs, int batch, float lr, uint64_t seed) {
  PB_REQUIRE(n > 0 && epochs > 0 && batch > 0, PB_EINVAL, "train: empty data or bad schedule");
  // Normalisation from the data.
  for (int f = 0; f < kMlpIn; ++f) {
    double mu = 0, sq = 0;
    for (int64_t r = 0; r < n; ++r) mu += X[r * kMlpIn + f];
    mu /= n;
    for (int64_t r = 0; r < n; ++r) sq += (X[r * kMlpIn + f] - mu) * (X[r * kMlpIn + f] - mu);
    const double sd = std::sqrt(sq / n);
    x_mean[f] = (float)mu;
    x_scale[f] = sd > 1e-6 ? (float)(1.0 / sd) : 0.f;
  }
  {
    double mu = 0, sq = 0;
    for (int64_t r = 0; r < n; ++r) mu += y[r];
    mu /= n;
    for (int64_t r = 0; r < n; ++r) sq += (y[r] - mu) * (y[r] - mu);
    const double sd = std::sqrt(sq / n);
    y_mean = (float)mu;
    y_scale = sd > 1e-6 ? (float)(1.0 / sd) : 1.f;
  }
  std::vector<float> yn(n);
  for (int64_t r = 0; r < n; ++r) yn[r] = (y[r] - y_mean) * y_scale;
  DevBuf<float> Xd(n * kMlpIn, s), yd(n, s), loss(1, s);
  DevBuf<uint32_t> perm(n, s);
  PB_CUDA_TRY(cudaMemcpyAsync(Xd.get(), X, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(yd.get(), yn.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
  const int64_t B = std::min<int64_t>(batch, n);
  Act A;
  A.ensure(B, s);
  const Norm nm = norm_of(*this);
  std::vector<uint32_t> order(n);
  for (int64_t r = 0; r < n; ++r) order[r] = (uint32_t)r;
  uint64_t st = seed;
  float last = 0.f;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int64_t r = n - 1; r > 0; --r) std::swap(order[r], order[splitmix(st) % (uint64_t)(r + 1)]);
    PB_CUDA_TRY(cudaMemcpyAsync(perm.get(), order.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
    PB_CUDA_TRY(cudaMemsetAsync(loss.get(), 0, sizeof(float), s));
    int64_t nb = 0;
    for (int64_t b0 = 0; b0 + B <= n; b0 += B, ++nb) {
      PB_LAUNCH(gather_standardize_kernel, grid_for(B * kMlpIn, 256), 256, 0, s, Xd.get(), yd.get(), perm.get() + b0,
                B, nm, A.Xh.get(), A.t.get());
      forward(*this, A, B, s);
      backward(*this, A, B, loss.get(), s);
      ++steps;
      const float c1 = 1.f - std::pow(b1, (float)steps), c2 = 1.f - std::pow(b2, (float)steps);
      PB_LAUNCH(adam_kernel, grid_for(kParams, 256), 256, 0, s, params.get(), grads.get(), m_adam.get(), v_adam.get(),
                kParams, lr, b1, b2, c1, c2, 1e-8f);
      PB_LAUNCH(to_bf16_kernel, grid_for(kParams, 256), 256, 0, s, params.get(), kParams, whalf.get());
    }
    float h = 0.f;
    PB_CUDA_TRY(cudaMemcpyAsync(&h, loss.get(), sizeof(float), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    last = nb > 0 ? h / (float)nb : 0.f;
  }
  check_err(*this, s);
  trained = true;
  return last;
}

void MlpModel::predict_dev(const float* X_dev, int64_t n, float* y_dev, cudaStream_t stream) {
  if (n <= 0) return;
  Act A;
  A.ensure(n, stream);
  const Norm nm = norm_of(*this);
  PB_LAUNCH(gather_standardize_kernel, grid_for(n * kMlpIn, 256), 256, 0, stream, X_dev, nullptr, nullptr, n, nm,
            A.Xh.get(), nullptr);
  forward(*this, A, n, stream);
  PB_LAUNCH(destandardize_kernel, grid_for(n, 256), 256, 0, stream, A.Y.get(), n, y_mean, 1.f / y_scale, y_dev);
  check_err(*this, stream);
}

std::vector<float> MlpModel::pack() const {
  std::vector<float> blob(kParams + 2 * kMlpIn + 2);
  PB_CUDA_TRY(cudaMemcpyAsync(blob.data(), params.get(), sizeof(float) * kParams, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  std::memcpy(blob.data() + kParams, x_mean, sizeof(x_mean));
  std::memcpy(blob.data() + kParams + kMlpIn, x_scale, sizeof(x_scale));
  blob[kParams + 2 * kMlpIn] = y_mean;
  blob[kParams + 2 * kMlpIn + 1] = y_scale;
  return blob;
}

void MlpModel::unpack(const std::vector<float>& blob, cudaStream_t stream) {
  PB_REQUIRE(blob.size() == (size_t)(kParams + 2 * kMlpIn + 2), PB_EINVAL, "model blob has the wrong size");
  s = stream;
  PB_CUDA_TRY(cudaMemcpyAsync(params.get(), blob.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, s));
  std::memcpy(x_mean, blob.data() + kParams, sizeof(x_mean));
  std::memcpy(x_scale, blob.data() + kParams + kMlpIn, sizeof(x_scale));
  y_mean = blob[kParams + 2 * kMlpIn];
  y_scale = blob[kParams + 2 * kMlpIn + 1];
  PB_LAUNCH(to_bf16_kernel, grid_for(kParams, 256), 256, 0, s, params.get(), kParams, whalf.get());
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  trained = true;
}

int mlp_param_count() { return kParams; }

}  // namespace pb
