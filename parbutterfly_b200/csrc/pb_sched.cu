// Learned scheduler, peeling side: the setting of a peel call (how the exact rounds are batched
// into partitions of the two-phase schedule, how a round's CTA-level work is cut into units,
// which items take the whole grid, how many CTAs run) is picked by the cost model from
// call-level features.  Candidates are a fixed grid of
// PeelTuning values per peel kind; candidate 0 is the plain path's setting.  The counting side
// (per-item aggregation modes) lives with the aggregator in pb_count.cu.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pb_engine.cuh"
#include "pb_mlp.cuh"
#include "pb_sched.cuh"

namespace pb {

namespace {

__global__ void count_stats_kernel(const int64_t* __restrict__ c, int64_t n, unsigned long long* out) {
  unsigned long long sum = 0, mx = 0, nz = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long v = c[i] > 0 ? (unsigned long long)c[i] : 0ull;
    sum += v;
    mx = v > mx ? v : mx;
    nz += v ? 1ull : 0ull;
  }
  sum = warp_sum(sum);
  nz = warp_sum(nz);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = y > mx ? y : mx;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], sum);
    atomicMax(&out[1], mx);
    atomicAdd(&out[2], nz);
  }
}

constexpr float kPeelMargin = 0.2016f;  // log2(1.15)
constexpr int64_t kUnits[3] = {4, 2, 8};
constexpr int64_t kTipHuge[4] = {int64_t(1) << 13, int64_t(1) << 11, int64_t(1) << 15, int64_t(1) << 40};
constexpr int kCtaDiv[4] = {1, 2, 4, 8};
// Peel-round batching: 0 runs one exact round at a time over the whole GPU; p > 0 batches the
// rounds into about p partitions per CTA (the two-phase schedule).
constexpr double kTipPpc[3] = {0, 1, 4};

}  // namespace

int peel_candidates(bool wing) { return wing ? kWingCandidates : kTipCandidates; }

PeelTuning peel_candidate(bool wing, int c, int resident_ctas) {
  PeelTuning t = plain_peel_tuning(wing);
  int div = 1;
  double ppc = 0;
  if (wing) {
    // c = units on the full grid; c = 0 is the plain setting.  Wing peels run one round at a
    // time: the two-phase schedule enumerates every butterfly twice, which made the 2^24-edge
    // wing peel 1.2-1.6x slower at every partition count measured, and a model trained on
    // smaller graphs (where it pays) picked it there.  Fewer CTAs are slower there too (1.2-1.8x),
    // and warp units are no faster, so both stay out of the grid.
    t.units_per_cta = kUnits[c % 3];
  } else {
    // c = (ppc * 4 + huge) * 4 + cta divisor; c = 0 is the plain setting.
    div = kCtaDiv[c % 4];
    t.huge_work = kTipHuge[(c / 4) % 4];
    ppc = kTipPpc[(c / 16) % 3];
  }
  t.max_ctas = div > 1 ? std::max(1, resident_ctas / div) : 0;
  t.two_phase = ppc > 0;
  t.parts_per_cta = ppc;
  return t;
}

void peel_call_features(const pb_graph& g, int use_v, bool wing, const int64_t* counts_dev, float* f, cudaStream_t s) {
  const int64_t nK = use_v ? g.nu : g.nv, nC = use_v ? g.nv : g.nu;
  const int64_t N = wing ? g.m : nK;
  int uv = 0;
  int64_t wmin = 0, wv = 0, wu = 0;
  cmp_wedge_counts(g, &uv, &wmin, &wv, &wu, s);
  unsigned long long h[3] = {0, 0, 0};
  if (N > 0) {
    DevBuf<unsigned long long> acc(3, s);
    PB_CUDA_TRY(cudaMemsetAsync(acc.get(), 0, acc.bytes(), s));
    PB_LAUNCH(count_stats_kernel, std::max(1, std::min(ceil_div(N, 256), sm_count() * 4)), 256, 0, s, counts_dev, N,
              acc.get());
    PB_CUDA_TRY(cudaMemcpyAsync(h, acc.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
  }
  const double wK = use_v ? (double)wv : (double)wu;  // wedges centred on the other side's ids
  const double wC = use_v ? (double)wu : (double)wv;
  auto lg = [](double x) { return (float)std::log2(1.0 + (x > 0 ? x : 0)); };
  f[0] = wing ? 1.f : 0.f;
  f[1] = lg((double)N);
  f[2] = lg((double)g.m);
  f[3] = lg((double)nK);
  f[4] = lg((double)nC);
  f[5] = lg((double)g.max_deg);
  f[6] = lg(wK);
  f[7] = lg(wC);
  f[8] = lg(nK ? (double)g.m / nK : 0.0);
  f[9] = lg(nC ? (double)g.m / nC : 0.0);
  f[10] = lg((double)h[1]);
  f[11] = lg(h[2] ? (double)h[0] / (double)h[2] : 0.0);
}

void peel_row(const float* call_f, bool wing, int c, float* row) {
  const PeelTuning t = peel_candidate(wing, c, 1 << 20);
  for (int k = 0; k < kPeelCallFeatures; ++k) row[k] = call_f[k];
  if (wing) {
    row[12] = (float)std::log2((double)t.units_per_cta);
    row[13] = 0.f;
  } else {
    row[12] = t.max_ctas > 0 ? (float)std::log2((double)((1 << 20) / t.max_ctas)) : 0.f;  // log2 of the CTA divisor
    row[13] = (float)std::log2((double)std::min<int64_t>(t.huge_work, int64_t(1) << 20));
  }
  row[14] = 0.f;
  row[15] = (float)std::log2(1.0 + 4.0 * (t.two_phase ? t.parts_per_cta : 0.0));
}

int choose_peel(MlpModel& model, const float* call_f, bool wing, float* pred_log2ms, cudaStream_t s) {
  const int nc = peel_candidates(wing);
  // Calls unlike the training data (a call feature more than 4 standard deviations from the
  // training mean) keep the plain setting: the model has no basis to predict them.  (Evaluating
  // them at the edge of the training range instead chose round batchings that ran 1.6x slower
  // on the 2^24-edge wing peel and 2.2x slower on the 1e9-edge tip peel.)
  bool in_range = true;
  for (int k = 0; k < kPeelCallFeatures; ++k)
    if (model.x_scale[k] > 0.f && std::fabs((call_f[k] - model.x_mean[k]) * model.x_scale[k]) > 4.f) in_range = false;
  std::vector<float> X((size_t)nc * kMlpIn), y(nc);
  for (int c = 0; c < nc; ++c) peel_row(call_f, wing, c, X.data() + (size_t)c * kMlpIn);
  DevBuf<float> Xd(X.size(), s), yd(nc, s);
  PB_CUDA_TRY(cudaMemcpyAsync(Xd.get(), X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice, s));
  model.predict_dev(Xd.get(), nc, yd.get(), s);
  PB_CUDA_TRY(cudaMemcpyAsync(y.data(), yd.get(), sizeof(float) * nc, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  int best = 0;
  for (int c = 1; c < nc; ++c)
    if (y[c] < y[best]) best = c;
  // Another setting replaces the plain one only when predicted at least 15% faster.
  if (!in_range || y[0] - y[best] < kPeelMargin) best = 0;
  if (pred_log2ms) *pred_log2ms = y[best];
  return best;
}

}  // namespace pb
