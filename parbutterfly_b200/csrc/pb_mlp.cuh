// The learned scheduler's cost model: a 3-layer MLP (BF16 operands, FP32 accumulation) whose
// every matrix product runs on the 5th-generation tensor cores (tcgen05.mma, accumulators in
// TMEM) through tc_gemm_bf16.  No counterpart in the reference, which always runs the fixed
// aggregation strategy the -countType flag names.
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "pb_common.cuh"

namespace pb {

// D(m, n) = sum_k A(m, k) * B(n, k) on the tensor cores.  A and B are BF16 and addressed by
// element strides, so transposed operands need no copy: A(m, k) = A[m * sam + k * sak],
// B(n, k) = B[n * sbn + k * sbk].  Epilogues:
//   GEMM_STORE   D[m * ldd + n] = acc + bias[n]                       (FP32)
//   GEMM_RELU    H[m * ldh + n] = bf16(max(acc + bias[n], 0))          (BF16)
//   GEMM_ATOMIC  D[m * ldd + n] += acc (+ bias[n] from the first K split) (FP32, split-K)
//   GEMM_MASK    H[m * ldh + n] = bf16(mask[m * ldh + n] > 0 ? acc : 0) (BF16, ReLU backward)
// M is unbounded (tiles of 128 rows), 1 <= N <= 128, K unbounded; k_split > 0 splits K across
// CTAs (GEMM_ATOMIC only).
enum GemmEpi { GEMM_STORE = 0, GEMM_RELU = 1, GEMM_ATOMIC = 2, GEMM_MASK = 3 };
struct GemmSpec {
  const __nv_bfloat16* A = nullptr;
  int64_t sam = 0, sak = 1;
  const __nv_bfloat16* B = nullptr;
  int64_t sbn = 0, sbk = 1;
  int64_t M = 0;
  int N = 0;
  int64_t K = 0;
  int64_t k_split = 0;
  int epi = GEMM_STORE;
  float* D = nullptr;
  int64_t ldd = 0;
  const float* bias = nullptr;
  __nv_bfloat16* H = nullptr;
  int64_t ldh = 0;
  const __nv_bfloat16* mask = nullptr;
};
constexpr int kGemmMaxN = 128;
// Launches the GEMM; err (device, 4 words) records a barrier that timed out (word 0 = 1).
void tc_gemm_bf16(const GemmSpec& g, uint32_t* err, cudaStream_t s);

// The cost model: in kMlpIn features -> kMlpHidden -> kMlpHidden -> 1, ReLU between layers.
constexpr int kMlpIn = 16;
constexpr int kMlpHidden = 64;
constexpr int kMlpOutPad = 16;  // the output layer runs as an N = 16 product (rows 1..15 zero)

struct MlpModel {
  // Packed FP32 master parameters w1 [64x16] | b1 | w2 [64x64] | b2 | w3 [16x64] (row 0 live)
  // | b3 [16] (entry 0 live), their BF16 operand copy, gradients and Adam moments.
  DevBuf<float> params, grads, m_adam, v_adam;
  DevBuf<__nv_bfloat16> whalf;
  DevBuf<uint32_t> err;
  // Feature and target normalisation (host copies; features are standardised before the
  // first layer, the output is de-standardised).
  float x_mean[kMlpIn] = {0}, x_scale[kMlpIn] = {0};
  float y_mean = 0, y_scale = 1;
  int64_t steps = 0;
  bool trained = false;
  int device = 0;
  cudaStream_t s = nullptr;
  void init(uint64_t seed, cudaStream_t stream);
  // Trains on host rows X [n x kMlpIn] with targets y [n]; returns the final training MSE in
  // normalised units.  Every product of the forward and backward passes runs through
  // tc_gemm_bf16; the optimiser is Adam on the FP32 master copy.
  float train(const float* X, const float* y, int64_t n, int epochs, int batch, float lr, uint64_t seed);
  // Predictions for n feature rows already on the device (FP32 [n x kMlpIn]) into y_dev [n].
  void predict_dev(const float* X_dev, int64_t n, float* y_dev, cudaStream_t stream);
  // Parameter blob (host) for saving / loading.
  std::vector<float> pack() const;
  void unpack(const std::vector<float>& blob, cudaStream_t stream);
};
int mlp_param_count();

}  // namespace pb
