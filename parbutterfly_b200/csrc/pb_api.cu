// C ABI of libpbgpu: contexts, graphs and the Count / CountE / CountTotal / Peel / PeelE
// entry points (include/parbutterfly_b200.h).
#include <algorithm>
#include <array>
#include <map>
#include <memory>
#include <tuple>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pb_engine.cuh"
#include "pb_mlp.cuh"
#include "pb_prims.cuh"
#include "pb_sched.cuh"

struct pb_sched_model {
  int device = 0;
  pb::MlpModel count, peel;
};

// A planned batch: the disjoint union of k graphs and one CUDA graph that ranks it, counts its
// butterflies per vertex and peels its tips (pb_batch_create / pb_batch_run).
struct pb_batch {
  int device = 0;
  pb_graph U;
  std::vector<int64_t> kbase, ksize;
  pb::DevBuf<int64_t> counts, tips;  // union count side (U side of the union)
  pb::Recorder rec;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int rank_type = PB_ADEG, strategy = 0;
  std::array<int, 3> geom = {0, 0, 0};
  bool tuned = false;
  int64_t graph_launches = 0;  // kernel launches one replay performs
  pb::PeelParts parts;         // one peel instance per graph
  ~pb_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

struct pb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  pb_stats stats{};
  int64_t launches = 0;
  // Learned scheduler: attached model and trace log (index: pb_sched_target).
  pb_sched_model* model = nullptr;
  // Autotuner: block-aggregator geometry per graph signature (n, 2m, W_rank, per type).
  std::map<std::tuple<int64_t, int64_t, int64_t, int>, std::array<int, 3>> tuned;
  int trace_mode = PB_TRACE_OFF;
  uint64_t trace_seed = 0;
  uint64_t peel_sweep[2] = {0, 0};  // explore-mode position in the setting grid (tip, wing)
  std::vector<float> trace_X[2], trace_y[2];
};

namespace pb {

thread_local int64_t* g_launch_counter = nullptr;
thread_local Recorder* g_recorder = nullptr;

Recorder::~Recorder() {
  for (void* p : pinned) cudaFreeHost(p);
}

void* Recorder::pinned_alloc(size_t bytes) {
  void* p = nullptr;
  PB_CUDA_TRY(cudaMallocHost(&p, bytes));
  std::memset(p, 0, bytes);
  pinned.push_back(p);
  return p;
}

void readback(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  Recorder* r = g_recorder;
  if (r && r->capturing) {
    PB_REQUIRE(r->pos < r->log.size() && r->log[r->pos].size() == bytes, PB_ECUDA,
               "graph capture: the pipeline took a different path than its recording run");
    std::memcpy(dst, r->log[r->pos].data(), bytes);
    ++r->pos;
    return;
  }
  PB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  if (r) r->log.emplace_back((const uint8_t*)dst, (const uint8_t*)dst + bytes);
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}

namespace {

// Sets the device and the launch counter of a context for the duration of one API call.
struct CallScope {
  pb_ctx* ctx;
  int prev_dev = -1;
  explicit CallScope(pb_ctx* c) : ctx(c) {
    cudaGetDevice(&prev_dev);
    if (prev_dev != c->device) PB_CUDA_TRY(cudaSetDevice(c->device));
    g_launch_counter = &c->launches;
  }
  ~CallScope() {
    g_launch_counter = nullptr;
    if (prev_dev >= 0 && prev_dev != ctx->device) cudaSetDevice(prev_dev);
  }
};

template <class F>
pb_status guarded(pb_ctx* ctx, F&& f) {
  if (!ctx) return PB_EINVAL;
  try {
    CallScope scope(ctx);
    f();
    ctx->last_error.clear();
    return PB_OK;
  } catch (const Error& e) {
    ctx->last_error = e.msg;
    if (e.status == PB_ECUDA) cudaGetLastError();
    return e.status;
  } catch (const std::bad_alloc&) {
    ctx->last_error = "host allocation failed";
    return PB_ENOMEM;
  }
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

pb_opts resolve_opts(const pb_opts* o) {
  pb_opts r;
  pb_opts_default(&r);
  if (o) r = *o;
  PB_REQUIRE(r.count_type >= PB_SORT && r.count_type <= PB_SERIAL, PB_EINVAL, "count_type out of range");
  PB_REQUIRE(r.rank_type >= PB_SIDE && r.rank_type <= PB_ADEG, PB_EINVAL, "rank_type out of range");
  PB_REQUIRE(r.peel_type >= PB_PSORT && r.peel_type <= PB_PBATCHWA, PB_EINVAL, "peel_type out of range");
  PB_REQUIRE(r.per_type >= PB_VERT && r.per_type <= PB_TOTAL, PB_EINVAL, "per_type out of range");
  PB_REQUIRE(r.sched == PB_SCHED_PLAIN || r.sched == PB_SCHED_LEARNED, PB_EINVAL, "sched out of range");
  PB_REQUIRE(r.peel_parts >= -1, PB_EINVAL, "peel_parts out of range");
  return r;
}

__global__ void max_degree_kernel(const uint32_t* __restrict__ off, int64_t n, uint32_t* out) {
  uint32_t m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, off[i + 1] - off[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void gather_vert_kernel(const int64_t* __restrict__ rc, const uint32_t* __restrict__ rank, int64_t base,
                                   int64_t nc, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = rc[rank[base + i]];
}

// Device-side graph validation: offsets monotone, ids in range, lists strictly ascending.
__global__ void validate_side_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edg, int64_t n,
                                     int64_t other_n, uint32_t* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t b = off[i], e = off[i + 1];
    if (e < b) { atomicOr(bad, 1u); continue; }
    for (uint32_t k = b; k < e; ++k) {
      uint32_t x = edg[k];
      if ((int64_t)x >= other_n || (k > b && x <= edg[k - 1])) { atomicOr(bad, 2u); break; }
    }
  }
}

// PB_TRACE=1 in the environment: synchronise after every counting / peeling stage and print
// its wall time to stderr (diagnostics; off by default).
bool trace_on() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("PB_TRACE");
    on = (e && *e && *e != '0') ? 1 : 0;
  }
  return on == 1;
}

struct Trace {
  cudaStream_t s;
  std::chrono::steady_clock::time_point t0;
  explicit Trace(cudaStream_t st) : s(st), t0(std::chrono::steady_clock::now()) {}
  void stage(const char* name) {
    if (!trace_on()) return;
    cudaError_t e = cudaStreamSynchronize(s);
    auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "[pb] %-10s %9.3f ms  %s\n", name, std::chrono::duration<double, std::milli>(t1 - t0).count(),
            e == cudaSuccess ? "" : cudaGetErrorString(e));
    fflush(stderr);
    t0 = t1;
  }
};

struct Timer {
  cudaEvent_t ev[8];
  int k = 0;
  cudaStream_t s;
  explicit Timer(cudaStream_t st) : s(st) {
    for (auto& e : ev) PB_CUDA_TRY(cudaEventCreate(&e));
  }
  ~Timer() {
    for (auto& e : ev) cudaEventDestroy(e);
  }
  void mark() { PB_CUDA_TRY(cudaEventRecord(ev[k++], s)); }
  double ms(int a, int b) {
    float x = 0;
    PB_CUDA_TRY(cudaEventElapsedTime(&x, ev[a], ev[b]));
    return x;
  }
};

int64_t out_len_of(const pb_graph* g, int per, int use_v) {
  if (per == PB_VERT) return use_v ? g->nu : g->nv;
  if (per == PB_EDGE) return g->m;
  return 1;
}

// The whole counting pipeline; result (dense int64, length out_len_of) in out_dev.
void run_count(pb_ctx* ctx, const pb_graph* g, const pb_opts& o, int per, int use_v, int64_t* out_dev) {
  cudaStream_t s = ctx->stream;
  pb_stats& st = ctx->stats;
  std::memset(&st, 0, sizeof(st));
  int uv = 0;
  int64_t wmin = 0, wv = 0, wu = 0;
  cmp_wedge_counts(*g, &uv, &wmin, &wv, &wu, s);
  if (use_v < 0) use_v = uv;
  st.w_side = use_v ? wv : wu;
  st.use_v = use_v;
  Timer T(s);
  Trace tr(s);
  Ranked R;
  T.mark();
  vertex_order(*g, o.rank_type, use_v, R, s);
  T.mark();
  tr.stage("rank");
  build_ranked_csr(*g, R, per == PB_EDGE, s);
  T.mark();
  tr.stage("relabel");
  wedge_scan(R, s);
  T.mark();
  tr.stage("scan");
  CountConfig cfg;
  switch (o.count_type) {
    case PB_BATCHS: case PB_BATCHWA: case PB_SERIAL: cfg.strategy = STRAT_DENSE; break;
    case PB_SORT: case PB_ASORT: cfg.strategy = STRAT_SORT; break;
    case PB_HIST: case PB_AHIST: cfg.strategy = STRAT_HIST; break;
    default: cfg.strategy = STRAT_HASH; break;
  }
  // Learned scheduler / trace hooks of the block aggregator (HASH and dense count types).
  SchedHooks hooks;
  const bool fused = cfg.strategy == STRAT_DENSE || cfg.strategy == STRAT_HASH;
  if (fused && o.sched == PB_SCHED_LEARNED && ctx->model && ctx->model->count.trained)
    hooks.model = &ctx->model->count;
  if (fused && ctx->trace_mode != PB_TRACE_OFF) {
    hooks.trace_X = &ctx->trace_X[PB_SCHED_COUNT];
    hooks.trace_y = &ctx->trace_y[PB_SCHED_COUNT];
    hooks.explore = ctx->trace_mode == PB_TRACE_EXPLORE && !hooks.model;
    hooks.seed = ctx->trace_seed++;
  }
  if (hooks.model || hooks.trace_X) cfg.sched = &hooks;
  // Autotuner: the first call on a graph signature times the block aggregator under each
  // candidate geometry (shared-memory table bytes, CTAs per SM, warp/CTA boundary in wedges)
  // with the plain rule and keeps the fastest for this and later calls on the context.
  st.autotuned = 0;
  if (fused && o.autotune && R.w_rank > 0) {
    static const int kGeom[10][3] = {{48 << 10, 4, 512}, {32 << 10, 4, 512}, {48 << 10, 2, 512}, {96 << 10, 2, 512},
                                     {200 << 10, 1, 512}, {48 << 10, 4, 256}, {32 << 10, 4, 256},
                                     {48 << 10, 2, 256}, {96 << 10, 2, 256}, {200 << 10, 1, 256}};
    const auto key = std::make_tuple(R.n, R.m2, R.w_rank, per);
    auto it = ctx->tuned.find(key);
    if (it == ctx->tuned.end()) {
      DevBuf<int64_t> scratch;
      int64_t* tgt = per == PB_VERT ? nullptr : out_dev;
      if (per == PB_VERT) {
        scratch.alloc(R.n > 0 ? R.n : 1, s);
        tgt = scratch.get();
      }
      double best = 1e300;
      std::array<int, 3> bg = {kGeom[0][0], kGeom[0][1], kGeom[0][2]};
      for (const auto& gm : kGeom) {
        CountConfig t = cfg;
        t.sched = nullptr;
        t.smem_bytes = gm[0];
        t.blocks_per_sm = gm[1];
        t.small_w = gm[2];
        const CountResult r = count_ranked(R, per, tgt, t, s);
        if (r.agg_ms < best) {
          best = r.agg_ms;
          bg = {gm[0], gm[1], gm[2]};
        }
      }
      it = ctx->tuned.emplace(key, bg).first;
      st.autotuned = 1;
    }
    cfg.smem_bytes = it->second[0];
    cfg.blocks_per_sm = it->second[1];
    cfg.small_w = it->second[2];
  }
  st.count_smem_bytes = cfg.smem_bytes;
  st.count_blocks_per_sm = cfg.blocks_per_sm;
  st.count_small_w = cfg.small_w;
  DevBuf<uint32_t> chk;
  if (check_mode()) {
    chk.alloc(4, s);
    PB_CUDA_TRY(cudaMemsetAsync(chk.get(), 0, 4 * sizeof(uint32_t), s));
    validate_ranked(R, g->m, chk.get(), s);
    cfg.err = chk.get();
  }
  DevBuf<int64_t> rc;
  int64_t* target = out_dev;
  if (per == PB_VERT) {
    rc.alloc(R.n > 0 ? R.n : 1, s);
    target = rc.get();
  }
  CountResult cr = cfg.strategy == STRAT_SORT   ? count_ranked_materialized(R, per, target, false, o.max_wedges, s)
                   : cfg.strategy == STRAT_HIST ? count_ranked_materialized(R, per, target, true, o.max_wedges, s)
                                                : count_ranked(R, per, target, cfg, s);
  T.mark();
  tr.stage("count");
  if (trace_on())
    fprintf(stderr, "[pb] CTA modes (endpoints / wedges): dense %llu/%llu hash %llu/%llu global %llu/%llu hybrid %llu/%llu\n",
            cr.mode_items[0], cr.mode_wedges[0], cr.mode_items[1], cr.mode_wedges[1], cr.mode_items[2],
            cr.mode_wedges[2], cr.mode_items[3], cr.mode_wedges[3]);
  if (chk.get()) {
    uint32_t h[4];
    PB_CUDA_TRY(cudaMemcpyAsync(h, chk.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    PB_REQUIRE(h[0] == 0, PB_ECUDA,
               "checked mode: bounds violation code " + std::to_string(h[0]) + " index " +
                   std::to_string(((uint64_t)h[2] << 32) | h[1]) + " aux " + std::to_string(h[3]));
  }
  if (per == PB_VERT) {
    const int64_t nc = use_v ? g->nu : g->nv;
    const int64_t base = use_v ? g->nv : 0;
    if (nc > 0)
      PB_LAUNCH(gather_vert_kernel, std::max(1, std::min(ceil_div(nc, 256), sm_count() * 8)), 256, 0, s, rc.get(),
                R.rank.get(), base, nc, out_dev);
  }
  T.mark();
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  st.w_rank = R.w_rank;
  st.n_big = cr.n_big;
  st.ms_rank = T.ms(0, 1);
  st.ms_relabel = T.ms(1, 2);
  st.ms_scan = T.ms(2, 3);
  st.ms_count = T.ms(3, 4);
  st.ms_convert = T.ms(4, 5);
  st.ms_agg_kernel = cr.agg_ms;
  st.sched_used = hooks.model ? 1 : 0;
  st.sched_items = hooks.items;
  st.ms_sched = hooks.ms;
  st.sched_pred = hooks.pred_cycles;
  st.sched_meas = hooks.meas_cycles;
  st.sched_mae_log2 = hooks.mae_log2;
}

// The batch pipeline of pb_batch_create: rank the union (count side = U), count per vertex,
// gather the counts to union ids, peel tips.  Host readbacks go through readback(), so the same
// sequence records (eagerly) and then captures into a CUDA graph.
void batch_pipeline(pb_batch& b, cudaStream_t s) {
  const pb_graph& U = b.U;
  Ranked R;
  vertex_order(U, b.rank_type, 1, R, s);
  build_ranked_csr(U, R, false, s);
  wedge_scan(R, s);
  CountConfig cfg;
  cfg.strategy = b.strategy;
  if (b.tuned) {
    cfg.smem_bytes = b.geom[0];
    cfg.blocks_per_sm = b.geom[1];
    cfg.small_w = b.geom[2];
  }
  DevBuf<int64_t> rc(R.n > 0 ? R.n : 1, s);
  count_ranked(R, PB_VERT, rc.get(), cfg, s);
  if (U.nu > 0)
    PB_LAUNCH(gather_vert_kernel, std::max(1, std::min(ceil_div(U.nu, 256), sm_count() * 8)), 256, 0, s, rc.get(),
              R.rank.get(), U.nv, U.nu, b.counts.get());
  peel_vertices(U, 1, b.counts.get(), b.tips.get(), s, plain_peel_tuning(false), &b.parts);
}

// One peel instance per graph of a batch, weighted by its two-hop work.
PeelParts batch_parts(const std::vector<int64_t>& kbase, const std::vector<int64_t>& ksize,
                      const std::vector<double>& work) {
  PeelParts p;
  p.base = kbase;
  p.size = ksize;
  p.weight = work;
  return p;
}

// Work-unit setting of one peel call: learned (when a trained model is attached and the call
// asks for it), a random candidate (explore tracing) or the plain setting.  Fills the
// scheduler fields of the stats; *row receives the call's cost-model row for the trace.
PeelTuning peel_setting(pb_ctx* ctx, const pb_graph& g, int use_v, bool wing, const int64_t* cdev, const pb_opts& o,
                        std::vector<float>& row, float* pred) {
  pb_stats& st = ctx->stats;
  st.sched_used = 0;
  st.sched_choice = 0;
  st.ms_sched = 0;
  st.sched_pred = 0;
  if (o.peel_parts > 0) {  // the caller fixes the round batching
    PeelTuning t = plain_peel_tuning(wing);
    t.two_phase = true;
    t.parts_total = o.peel_parts;
    return t;
  }
  const bool learned = o.peel_parts == 0 && o.sched == PB_SCHED_LEARNED && ctx->model && ctx->model->peel.trained;
  if (!learned && ctx->trace_mode == PB_TRACE_OFF) return plain_peel_tuning(wing);
  auto t0 = std::chrono::steady_clock::now();
  float f[kPeelCallFeatures];
  peel_call_features(g, use_v, wing, cdev, f, ctx->stream);
  int c = 0;
  if (learned) {
    c = choose_peel(ctx->model->peel, f, wing, pred, ctx->stream);
    st.sched_used = 1;
    st.sched_pred = std::exp2((double)*pred);
  } else if (ctx->trace_mode == PB_TRACE_EXPLORE) {
    c = (int)(ctx->peel_sweep[wing ? 1 : 0]++ % (uint64_t)peel_candidates(wing));  // a cyclic sweep
  }
  st.sched_choice = c;
  row.assign(kMlpIn, 0.f);
  peel_row(f, wing, c, row.data());
  st.ms_sched = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return peel_candidate(wing, c, 2 * sm_count());
}

void log_peel_trace(pb_ctx* ctx, const std::vector<float>& row, double ms) {
  if (ctx->trace_mode == PB_TRACE_OFF || row.empty()) return;
  auto& X = ctx->trace_X[PB_SCHED_PEEL];
  X.insert(X.end(), row.begin(), row.end());
  ctx->trace_y[PB_SCHED_PEEL].push_back((float)std::log2(std::max(ms, 1e-3)));
}

// Runs fn(out_dev) with a device buffer of len int64 and delivers it to a host or device
// pointer.
template <class F>
void with_output(pb_ctx* ctx, int64_t* user_out, int64_t len, F&& fn) {
  cudaStream_t s = ctx->stream;
  if (len <= 0) { fn(nullptr); return; }
  if (is_device_ptr(user_out)) {
    fn(user_out);
    return;
  }
  DevBuf<int64_t> tmp(len, s);
  fn(tmp.get());
  PB_CUDA_TRY(cudaMemcpyAsync(user_out, tmp.get(), sizeof(int64_t) * len, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
}

void upload_graph(pb_ctx* ctx, const pb_csr* c, bool from_device, pb_graph** out) {
  PB_REQUIRE(c && out, PB_EINVAL, "null argument");
  PB_REQUIRE(c->nv >= 0 && c->nu >= 0 && c->m >= 0, PB_EINVAL, "negative size");
  PB_REQUIRE(c->nv + c->nu < (int64_t)(1u << 31), PB_ETOOBIG, "nv + nu must stay below 2^31");
  PB_REQUIRE(2 * c->m <= (int64_t)UINT32_MAX, PB_ETOOBIG, "2*m must fit 32-bit offsets");
  cudaStream_t s = ctx->stream;
  if (!from_device) {
    char msg[256];
    pb_status st = pb_csr_validate(c, msg, sizeof(msg));
    PB_REQUIRE(st == PB_OK, st, std::string("invalid CSR: ") + msg);
  }
  auto* g = new pb_graph();
  try {
    g->device = ctx->device;
    g->nv = c->nv; g->nu = c->nu; g->m = c->m;
    g->offV.alloc(c->nv + 1, s);
    g->offU.alloc(c->nu + 1, s);
    g->edgV.alloc(c->m > 0 ? c->m : 1, s);
    g->edgU.alloc(c->m > 0 ? c->m : 1, s);
    const cudaMemcpyKind kind = from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PB_CUDA_TRY(cudaMemcpyAsync(g->offV.get(), c->offsetsV, sizeof(uint32_t) * (c->nv + 1), kind, s));
    PB_CUDA_TRY(cudaMemcpyAsync(g->offU.get(), c->offsetsU, sizeof(uint32_t) * (c->nu + 1), kind, s));
    if (c->m > 0) {
      PB_CUDA_TRY(cudaMemcpyAsync(g->edgV.get(), c->edgesV, sizeof(uint32_t) * c->m, kind, s));
      PB_CUDA_TRY(cudaMemcpyAsync(g->edgU.get(), c->edgesU, sizeof(uint32_t) * c->m, kind, s));
    }
    DevBuf<uint32_t> mx(2, s);
    PB_CUDA_TRY(cudaMemsetAsync(mx.get(), 0, 2 * sizeof(uint32_t), s));
    const int grid = std::max(1, std::min(ceil_div(std::max(c->nv, c->nu) + 1, 256), sm_count() * 8));
    if (c->nv) PB_LAUNCH(max_degree_kernel, grid, 256, 0, s, g->offV.get(), c->nv, mx.get());
    if (c->nu) PB_LAUNCH(max_degree_kernel, grid, 256, 0, s, g->offU.get(), c->nu, mx.get());
    if (from_device) {
      uint32_t hoff[2];
      PB_CUDA_TRY(cudaMemcpyAsync(&hoff[0], g->offV.get() + c->nv, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      PB_CUDA_TRY(cudaMemcpyAsync(&hoff[1], g->offU.get() + c->nu, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      PB_CUDA_TRY(cudaStreamSynchronize(s));
      PB_REQUIRE(hoff[0] == (uint32_t)c->m && hoff[1] == (uint32_t)c->m, PB_EINVAL, "offsets[n] != m");
      if (c->nv) PB_LAUNCH(validate_side_kernel, grid, 256, 0, s, g->offV.get(), g->edgV.get(), c->nv, c->nu, mx.get() + 1);
      if (c->nu) PB_LAUNCH(validate_side_kernel, grid, 256, 0, s, g->offU.get(), g->edgU.get(), c->nu, c->nv, mx.get() + 1);
    }
    uint32_t h[2];
    PB_CUDA_TRY(cudaMemcpyAsync(h, mx.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    PB_REQUIRE(h[1] == 0, PB_EINVAL, "invalid CSR (unsorted list or id out of range)");
    g->max_deg = h[0];
    PB_REQUIRE(g->max_deg < (1u << 23), PB_ETOOBIG, "maximum degree must stay below 2^23");
  } catch (...) {
    delete g;
    throw;
  }
  *out = g;
}

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" {

int pb_abi_version(void) { return PB_ABI_VERSION; }

void pb_opts_default(pb_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->count_type = PB_SERIAL;
  o->rank_type = PB_ADEG;
  o->peel_type = PB_PBATCHS;
  o->per_type = PB_VERT;
  o->max_wedges = 2577500000LL;
  o->max_array_size = 23090996160LL;
  o->sched = PB_SCHED_PLAIN;
  o->autotune = 0;
  o->use_v = -1;
}

pb_status pb_ctx_create(int device, void* stream, pb_ctx** out) {
  if (!out) return PB_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PB_ECUDA;
  }
  if (device < 0 || device >= ndev) return PB_EINVAL;
  auto* c = new (std::nothrow) pb_ctx();
  if (!c) return PB_ENOMEM;
  c->device = device;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) { delete c; return PB_ECUDA; }
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      cudaSetDevice(prev);
      return PB_ECUDA;
    }
    c->own_stream = true;
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  cudaSetDevice(prev);
  *out = c;
  return PB_OK;
}

pb_status pb_ctx_destroy(pb_ctx* ctx) {
  if (!ctx) return PB_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  cudaSetDevice(prev);
  delete ctx;
  return PB_OK;
}

const char* pb_last_error(const pb_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

pb_status pb_get_stats(const pb_ctx* ctx, pb_stats* out) {
  if (!ctx || !out) return PB_EINVAL;
  *out = ctx->stats;
  return PB_OK;
}

int64_t pb_kernel_launches(const pb_ctx* ctx) { return ctx ? ctx->launches : 0; }

pb_status pb_graph_upload(pb_ctx* ctx, const pb_csr* host, pb_graph** out) {
  return guarded(ctx, [&] { upload_graph(ctx, host, false, out); });
}

pb_status pb_graph_from_device(pb_ctx* ctx, const pb_csr* dev, pb_graph** out) {
  return guarded(ctx, [&] { upload_graph(ctx, dev, true, out); });
}

pb_status pb_graph_parse_text(pb_ctx* ctx, const char* text, size_t len, pb_graph** out) {
  return guarded(ctx, [&] {
    PB_REQUIRE(text && out, PB_EINVAL, "null argument");
    ParsedCSR P;
    parse_adjacency_hypergraph(text, len, is_device_ptr(text), P, ctx->stream);
    const pb_csr c{P.nv, P.nu, P.m, P.offV.get(), P.edgV.get(), P.offU.get(), P.edgU.get()};
    upload_graph(ctx, &c, true, out);  // validated on the device (offsets, ranges, sorted lists)
  });
}

pb_status pb_gen_rmat_device(pb_ctx* ctx, int32_t log_nv, int32_t log_nu, int64_t m, double a, double b, double c,
                             double d, uint64_t seed, pb_graph** out) {
  return guarded(ctx, [&] {
    PB_REQUIRE(out, PB_EINVAL, "null argument");
    ParsedCSR P;
    gen_rmat_device(log_nv, log_nu, m, a, b, c, d, seed, P, ctx->stream);
    const pb_csr cs{P.nv, P.nu, P.m, P.offV.get(), P.edgV.get(), P.offU.get(), P.edgU.get()};
    upload_graph(ctx, &cs, true, out);  // validated on the device (offsets, ranges, sorted lists)
  });
}

pb_status pb_graph_read_text(pb_ctx* ctx, const char* path, pb_graph** out) {
  return guarded(ctx, [&] {
    PB_REQUIRE(path && out, PB_EINVAL, "null argument");
    FILE* f = fopen(path, "rb");
    PB_REQUIRE(f, PB_EIO, std::string("cannot open ") + path);
    fseek(f, 0, SEEK_END);
    const long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* buf = nullptr;
    if (len > 0 && cudaMallocHost((void**)&buf, (size_t)len) != cudaSuccess) {
      fclose(f);
      throw Error{PB_ENOMEM, "pinned host allocation for the file failed"};
    }
    const size_t got = len > 0 ? fread(buf, 1, (size_t)len, f) : 0;
    fclose(f);
    try {
      PB_REQUIRE(got == (size_t)(len > 0 ? len : 0), PB_EIO, std::string("short read of ") + path);
      ParsedCSR P;
      parse_adjacency_hypergraph(buf ? buf : "", (size_t)(len > 0 ? len : 0), false, P, ctx->stream);
      const pb_csr c{P.nv, P.nu, P.m, P.offV.get(), P.edgV.get(), P.offU.get(), P.edgU.get()};
      upload_graph(ctx, &c, true, out);
    } catch (...) {
      if (buf) cudaFreeHost(buf);
      throw;
    }
    if (buf) cudaFreeHost(buf);
  });
}

static void rebind_graph(pb_graph& g) {
  g.offV.rebind(nullptr);
  g.edgV.rebind(nullptr);
  g.offU.rebind(nullptr);
  g.edgU.rebind(nullptr);
}

static void rebind_model(pb::MlpModel& m) {
  m.params.rebind(nullptr);
  m.grads.rebind(nullptr);
  m.m_adam.rebind(nullptr);
  m.v_adam.rebind(nullptr);
  m.whalf.rebind(nullptr);
  m.err.rebind(nullptr);
}

pb_status pb_graph_destroy(pb_graph* g) {
  if (!g) return PB_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  cudaDeviceSynchronize();
  rebind_graph(*g);  // the context (and its stream) may already be gone
  delete g;
  cudaSetDevice(prev);
  return PB_OK;
}

pb_status pb_graph_download(const pb_graph* g, pb_csr_owned* out) {
  if (!g || !out) return PB_EINVAL;
  std::memset(out, 0, sizeof(*out));
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  out->nv = g->nv;
  out->nu = g->nu;
  out->m = g->m;
  out->offsetsV = (uint32_t*)malloc(sizeof(uint32_t) * (g->nv + 1));
  out->offsetsU = (uint32_t*)malloc(sizeof(uint32_t) * (g->nu + 1));
  out->edgesV = (uint32_t*)malloc(sizeof(uint32_t) * (g->m > 0 ? g->m : 1));
  out->edgesU = (uint32_t*)malloc(sizeof(uint32_t) * (g->m > 0 ? g->m : 1));
  pb_status st = PB_OK;
  if (!out->offsetsV || !out->offsetsU || !out->edgesV || !out->edgesU) {
    st = PB_ENOMEM;
  } else {
    cudaDeviceSynchronize();
    if (cudaMemcpy(out->offsetsV, g->offV.get(), sizeof(uint32_t) * (g->nv + 1), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(out->offsetsU, g->offU.get(), sizeof(uint32_t) * (g->nu + 1), cudaMemcpyDeviceToHost) != cudaSuccess ||
        (g->m > 0 && (cudaMemcpy(out->edgesV, g->edgV.get(), sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost) != cudaSuccess ||
                      cudaMemcpy(out->edgesU, g->edgU.get(), sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost) != cudaSuccess)))
      st = PB_ECUDA;
  }
  if (st != PB_OK) pb_csr_free(out);
  cudaSetDevice(prev);
  return st;
}

pb_status pb_graph_dims(const pb_graph* g, int64_t* nv, int64_t* nu, int64_t* m) {
  if (!g) return PB_EINVAL;
  if (nv) *nv = g->nv;
  if (nu) *nu = g->nu;
  if (m) *m = g->m;
  return PB_OK;
}

pb_status pb_cmp_wedge_counts(pb_ctx* ctx, const pb_graph* g, int32_t* use_v, int64_t* num_wedges) {
  return guarded(ctx, [&] {
    PB_REQUIRE(g && use_v && num_wedges, PB_EINVAL, "null argument");
    int uv = 0;
    int64_t w = 0, wv = 0, wu = 0;
    cmp_wedge_counts(*g, &uv, &w, &wv, &wu, ctx->stream);
    *use_v = uv;
    *num_wedges = w;
  });
}

pb_status pb_edge_to_idxs(pb_ctx* ctx, const pb_graph* g, int32_t use_v, uint32_t* eti) {
  return guarded(ctx, [&] {
    PB_REQUIRE(g && eti, PB_EINVAL, "null argument");
    if (g->m == 0) return;
    if (is_device_ptr(eti)) {
      edge_to_idxs(*g, use_v != 0, eti, ctx->stream);
      PB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    } else {
      DevBuf<uint32_t> tmp(g->m, ctx->stream);
      edge_to_idxs(*g, use_v != 0, tmp.get(), ctx->stream);
      PB_CUDA_TRY(cudaMemcpyAsync(eti, tmp.get(), sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, ctx->stream));
      PB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
  });
}

static pb_status count_entry(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out, int per) {
  return guarded(ctx, [&] {
    PB_REQUIRE(g && out, PB_EINVAL, "null argument");
    pb_opts o = resolve_opts(opts);
    int use_v = o.use_v;
    if (use_v >= 0) use_v = use_v != 0;
    if (use_v < 0) {
      int uv = 0;
      int64_t w = 0, wv = 0, wu = 0;
      cmp_wedge_counts(*g, &uv, &w, &wv, &wu, ctx->stream);
      use_v = uv;
    }
    const int64_t len = out_len_of(g, per, use_v);
    if (per == PB_TOTAL && len > 0 && !is_device_ptr(out)) {
      DevBuf<int64_t> tmp(1, ctx->stream);
      run_count(ctx, g, o, per, use_v, tmp.get());
      PB_CUDA_TRY(cudaMemcpyAsync(out, tmp.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
      PB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      return;
    }
    with_output(ctx, out, len, [&](int64_t* dev) {
      if (dev) run_count(ctx, g, o, per, use_v, dev);
    });
  });
}

pb_status pb_count_vert(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out) {
  return count_entry(ctx, g, opts, out, PB_VERT);
}
pb_status pb_count_edge(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out) {
  return count_entry(ctx, g, opts, out, PB_EDGE);
}
pb_status pb_count_total(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out) {
  return count_entry(ctx, g, opts, out, PB_TOTAL);
}

static pb_status peel_entry(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, const int64_t* counts, int64_t* res,
                            bool edges) {
  return guarded(ctx, [&] {
    PB_REQUIRE(g && counts && res, PB_EINVAL, "null argument");
    pb_opts o = resolve_opts(opts);
    int use_v = o.use_v;
    if (use_v >= 0) use_v = use_v != 0;
    if (use_v < 0) {
      int uv = 0;
      int64_t w = 0, wv = 0, wu = 0;
      cmp_wedge_counts(*g, &uv, &w, &wv, &wu, ctx->stream);
      use_v = uv;
    }
    cudaStream_t s = ctx->stream;
    const int64_t len = edges ? g->m : (use_v ? g->nu : g->nv);
    if (len <= 0) return;
    DevBuf<int64_t> cin;
    const int64_t* cdev = counts;
    if (!is_device_ptr(counts)) {
      cin.alloc(len, s);
      PB_CUDA_TRY(cudaMemcpyAsync(cin.get(), counts, sizeof(int64_t) * len, cudaMemcpyHostToDevice, s));
      cdev = cin.get();
    }
    Timer T(s);
    std::vector<float> row;
    float pred = 0.f;
    const PeelTuning tune = peel_setting(ctx, *g, use_v, edges, cdev, o, row, &pred);
    with_output(ctx, res, len, [&](int64_t* dev) {
      T.mark();
      PeelResult pr = edges ? peel_edges(*g, use_v, cdev, dev, s, tune) : peel_vertices(*g, use_v, cdev, dev, s, tune);
      T.mark();
      PB_CUDA_TRY(cudaStreamSynchronize(s));
      ctx->stats.ms_peel = T.ms(0, 1);
      ctx->stats.peel_rounds = pr.rounds;
      ctx->stats.peel_work = pr.work;
      ctx->stats.peel_parts = pr.parts;
      ctx->stats.peel_coarse_rounds = pr.coarse_rounds;
      ctx->stats.peel_fine_rounds_max = pr.fine_rounds_max;
      ctx->stats.sched_meas = ctx->stats.ms_peel;
      log_peel_trace(ctx, row, ctx->stats.ms_peel);
    });
  });
}

pb_status pb_count_vert_batch(pb_ctx* ctx, const pb_graph* const* gs, int32_t k, const pb_opts* opts,
                              int64_t* const* counts) {
  return guarded(ctx, [&] {
    PB_REQUIRE(gs && counts && k > 0, PB_EINVAL, "null argument or empty batch");
    pb_opts o = resolve_opts(opts);
    o.use_v = 1;
    cudaStream_t s = ctx->stream;
    pb_graph U;
    std::vector<int64_t> kbase, ksize;
    build_union(gs, k, U, kbase, ksize, s);
    DevBuf<int64_t> out(U.nu > 0 ? U.nu : 1, s);
    run_count(ctx, &U, o, PB_VERT, 1, out.get());
    for (int g = 0; g < k; ++g) {
      PB_REQUIRE(counts[g] || ksize[g] == 0, PB_EINVAL, "null output in batch");
      if (ksize[g])
        PB_CUDA_TRY(cudaMemcpyAsync(counts[g], out.get() + kbase[g], sizeof(int64_t) * ksize[g], cudaMemcpyDefault, s));
    }
    PB_CUDA_TRY(cudaStreamSynchronize(s));
  });
}

pb_status pb_peel_vert_batch(pb_ctx* ctx, const pb_graph* const* gs, int32_t k, const pb_opts* opts,
                             const int64_t* const* counts, int64_t* const* tips) {
  return guarded(ctx, [&] {
    PB_REQUIRE(gs && counts && tips && k > 0, PB_EINVAL, "null argument or empty batch");
    const pb_opts o = resolve_opts(opts);
    cudaStream_t s = ctx->stream;
    pb_graph U;
    std::vector<int64_t> kbase, ksize;
    std::vector<double> work;
    build_union(gs, k, U, kbase, ksize, s, &work);
    const int64_t n = U.nu;
    if (n == 0) return;
    DevBuf<int64_t> cin(n, s), tout(n, s);
    for (int g = 0; g < k; ++g) {
      PB_REQUIRE((counts[g] && tips[g]) || ksize[g] == 0, PB_EINVAL, "null buffer in batch");
      if (ksize[g])
        PB_CUDA_TRY(cudaMemcpyAsync(cin.get() + kbase[g], counts[g], sizeof(int64_t) * ksize[g], cudaMemcpyDefault, s));
    }
    Timer T(s);
    std::vector<float> row;
    float pred = 0.f;
    const PeelTuning tune = peel_setting(ctx, U, 1, false, cin.get(), o, row, &pred);
    T.mark();
    const PeelParts parts = batch_parts(kbase, ksize, work);
    PeelResult pr = peel_vertices(U, 1, cin.get(), tout.get(), s, tune, &parts);
    T.mark();
    for (int g = 0; g < k; ++g)
      if (ksize[g])
        PB_CUDA_TRY(cudaMemcpyAsync(tips[g], tout.get() + kbase[g], sizeof(int64_t) * ksize[g], cudaMemcpyDefault, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    ctx->stats.ms_peel = T.ms(0, 1);
    ctx->stats.peel_rounds = pr.rounds;
    ctx->stats.peel_work = pr.work;
    ctx->stats.peel_parts = pr.parts;
    ctx->stats.peel_coarse_rounds = pr.coarse_rounds;
    ctx->stats.peel_fine_rounds_max = pr.fine_rounds_max;
    ctx->stats.sched_meas = ctx->stats.ms_peel;
    log_peel_trace(ctx, row, ctx->stats.ms_peel);
  });
}

pb_status pb_batch_create(pb_ctx* ctx, const pb_graph* const* gs, int32_t k, const pb_opts* opts, pb_batch** out) {
  return guarded(ctx, [&] {
    PB_REQUIRE(gs && out && k > 0, PB_EINVAL, "null argument or empty batch");
    *out = nullptr;
    pb_opts o = resolve_opts(opts);
    PB_REQUIRE(o.count_type != PB_SORT && o.count_type != PB_ASORT && o.count_type != PB_HIST &&
                   o.count_type != PB_AHIST,
               PB_EUNSUPPORTED, "batch graphs run the fused aggregators (HASH / BATCHS / BATCHWA / SERIAL)");
    cudaStream_t s = ctx->stream;
    std::unique_ptr<pb_batch> b(new pb_batch());
    b->device = ctx->device;
    b->rank_type = o.rank_type;
    b->strategy = (o.count_type == PB_HASH || o.count_type == PB_AHASH) ? STRAT_HASH : STRAT_DENSE;
    std::vector<double> work;
    build_union(gs, k, b->U, b->kbase, b->ksize, s, &work);
    b->parts = batch_parts(b->kbase, b->ksize, work);
    const int64_t n = b->U.nu;
    b->counts.alloc(n > 0 ? n : 1, s);
    b->tips.alloc(n > 0 ? n : 1, s);
    if (o.autotune) {  // tune the aggregator geometry on the union once, eagerly
      pb_opts t = o;
      t.use_v = 1;
      t.sched = PB_SCHED_PLAIN;
      run_count(ctx, &b->U, t, PB_VERT, 1, b->counts.get());
      b->geom = {ctx->stats.count_smem_bytes, ctx->stats.count_blocks_per_sm, ctx->stats.count_small_w};
      b->tuned = true;
    }
    b->rec.status = (unsigned*)b->rec.pinned_alloc(2 * sizeof(unsigned));
    // 1. Recording run (eager): every host readback is logged.
    g_recorder = &b->rec;
    try {
      batch_pipeline(*b, s);
      PB_CUDA_TRY(cudaStreamSynchronize(s));
      // 2. Capture: the same sequence, readbacks served from the log.
      b->rec.capturing = true;
      b->rec.pos = 0;
      PB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
      const int64_t l0 = ctx->launches;
      try {
        batch_pipeline(*b, s);
        b->graph_launches = ctx->launches - l0;
      } catch (...) {
        cudaGraph_t broken = nullptr;
        cudaStreamEndCapture(s, &broken);
        if (broken) cudaGraphDestroy(broken);
        throw;
      }
      PB_CUDA_TRY(cudaStreamEndCapture(s, &b->graph));
    } catch (...) {
      g_recorder = nullptr;
      b->rec.capturing = false;
      throw;
    }
    g_recorder = nullptr;
    b->rec.capturing = false;
    PB_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    *out = b.release();
  });
}

pb_status pb_batch_run(pb_ctx* ctx, pb_batch* b, int64_t* const* counts, int64_t* const* tips) {
  return guarded(ctx, [&] {
    PB_REQUIRE(b && b->exec, PB_EINVAL, "null batch");
    PB_REQUIRE(b->device == ctx->device, PB_EINVAL, "batch and context are on different devices");
    cudaStream_t s = ctx->stream;
    Timer T(s);
    b->rec.status[0] = 0xFFFFFFFFu;
    T.mark();
    PB_CUDA_TRY(cudaGraphLaunch(b->exec, s));
    T.mark();
    ctx->launches += b->graph_launches;
    const int k = (int)b->kbase.size();
    for (int g = 0; g < k; ++g) {
      if (!b->ksize[g]) continue;
      const size_t bytes = sizeof(int64_t) * b->ksize[g];
      if (counts && counts[g])
        PB_CUDA_TRY(cudaMemcpyAsync(counts[g], b->counts.get() + b->kbase[g], bytes, cudaMemcpyDefault, s));
      if (tips && tips[g])
        PB_CUDA_TRY(cudaMemcpyAsync(tips[g], b->tips.get() + b->kbase[g], bytes, cudaMemcpyDefault, s));
    }
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    if (b->U.nu > 0) {
      const unsigned err = b->rec.status[0], alive = b->rec.status[1];
      PB_REQUIRE(err != 0xFFFFFFFFu, PB_ECUDA, "batch graph: the peel reported no status");
      PB_REQUIRE(!(err & 1u), PB_ETIMEOUT, "batch graph: a grid barrier wait of the peel ran out of time");
      PB_REQUIRE(err == 0 && alive == 0, PB_ECUDA, "batch graph: peeling did not complete");
    }
    std::memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.ms_count = T.ms(0, 1);  // the whole replay: ranking, counting and peeling
    ctx->stats.count_smem_bytes = b->geom[0];
    ctx->stats.count_blocks_per_sm = b->geom[1];
    ctx->stats.count_small_w = b->geom[2];
  });
}

pb_status pb_batch_destroy(pb_batch* b) {
  if (!b) return PB_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  rebind_graph(b->U);
  b->counts.rebind(nullptr);
  b->tips.rebind(nullptr);
  delete b;
  cudaSetDevice(prev);
  return PB_OK;
}

pb_status pb_peel_vert(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, const int64_t* counts, int64_t* tip) {
  return peel_entry(ctx, g, opts, counts, tip, false);
}
pb_status pb_peel_edge(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, const int64_t* ecounts, int64_t* wing) {
  return peel_entry(ctx, g, opts, ecounts, wing, true);
}

// ---- learned scheduler ---------------------------------------------------------------------
static pb::MlpModel* model_of(pb_sched_model* m, int32_t target) {
  PB_REQUIRE(m, PB_EINVAL, "null model");
  PB_REQUIRE(target == PB_SCHED_COUNT || target == PB_SCHED_PEEL, PB_EINVAL, "target must be COUNT or PEEL");
  return target == PB_SCHED_COUNT ? &m->count : &m->peel;
}

pb_status pb_sched_model_create(pb_ctx* ctx, uint64_t seed, pb_sched_model** out) {
  return guarded(ctx, [&] {
    PB_REQUIRE(out, PB_EINVAL, "null argument");
    auto* m = new pb_sched_model();
    try {
      m->device = ctx->device;
      m->count.init(seed, ctx->stream);
      m->peel.init(seed ^ 0x5bd1e995ull, ctx->stream);
      PB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
  });
}

pb_status pb_sched_model_destroy(pb_sched_model* model) {
  if (!model) return PB_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(model->device);
  cudaDeviceSynchronize();
  rebind_model(model->count);
  rebind_model(model->peel);
  delete model;
  cudaSetDevice(prev);
  return PB_OK;
}

pb_status pb_sched_train(pb_ctx* ctx, pb_sched_model* model, int32_t target, const float* X, const float* y, int64_t n,
                         int32_t epochs, int32_t batch, float lr, float* final_mse) {
  return guarded(ctx, [&] {
    pb::MlpModel* m = model_of(model, target);
    PB_REQUIRE(X && y && n > 0, PB_EINVAL, "empty training set");
    PB_REQUIRE(model->device == ctx->device, PB_EINVAL, "model and context are on different devices");
    m->s = ctx->stream;
    const float mse = m->train(X, y, n, epochs, batch, lr, 0x2545F4914F6CDD1Dull ^ (uint64_t)n);
    if (final_mse) *final_mse = mse;
  });
}

pb_status pb_sched_predict(pb_ctx* ctx, pb_sched_model* model, int32_t target, const float* X, int64_t n, float* y) {
  return guarded(ctx, [&] {
    pb::MlpModel* m = model_of(model, target);
    PB_REQUIRE(X && y, PB_EINVAL, "null argument");
    if (n <= 0) return;
    cudaStream_t s = ctx->stream;
    DevBuf<float> Xd((size_t)n * pb::kMlpIn, s), yd(n, s);
    PB_CUDA_TRY(cudaMemcpyAsync(Xd.get(), X, Xd.bytes(), cudaMemcpyHostToDevice, s));
    m->predict_dev(Xd.get(), n, yd.get(), s);
    PB_CUDA_TRY(cudaMemcpyAsync(y, yd.get(), yd.bytes(), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
  });
}

pb_status pb_sched_save(pb_ctx* ctx, const pb_sched_model* model, const char* path) {
  return guarded(ctx, [&] {
    PB_REQUIRE(model && path, PB_EINVAL, "null argument");
    FILE* f = fopen(path, "wb");
    PB_REQUIRE(f, PB_EIO, std::string("cannot write ") + path);
    const char magic[8] = {'P', 'B', 'S', 'C', 'H', 'E', 'D', '1'};
    bool ok = fwrite(magic, 1, 8, f) == 8;
    for (const pb::MlpModel* m : {&model->count, &model->peel}) {
      const std::vector<float> blob = m->pack();
      const int32_t trained = m->trained ? 1 : 0;
      const int64_t len = (int64_t)blob.size();
      ok = ok && fwrite(&trained, 4, 1, f) == 1 && fwrite(&len, 8, 1, f) == 1 &&
           fwrite(blob.data(), sizeof(float), blob.size(), f) == blob.size();
    }
    fclose(f);
    PB_REQUIRE(ok, PB_EIO, std::string("short write to ") + path);
  });
}

pb_status pb_sched_load(pb_ctx* ctx, pb_sched_model* model, const char* path) {
  return guarded(ctx, [&] {
    PB_REQUIRE(model && path, PB_EINVAL, "null argument");
    FILE* f = fopen(path, "rb");
    PB_REQUIRE(f, PB_EIO, std::string("cannot read ") + path);
    char magic[8];
    bool ok = fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PBSCHED1", 8) == 0;
    for (pb::MlpModel* m : {&model->count, &model->peel}) {
      int32_t trained = 0;
      int64_t len = 0;
      ok = ok && fread(&trained, 4, 1, f) == 1 && fread(&len, 8, 1, f) == 1 && len == pb::mlp_param_count() + 34;
      if (!ok) break;
      std::vector<float> blob((size_t)len);
      ok = fread(blob.data(), sizeof(float), blob.size(), f) == blob.size();
      if (!ok) break;
      m->unpack(blob, ctx->stream);
      m->trained = trained != 0;
    }
    fclose(f);
    PB_REQUIRE(ok, PB_EIO, std::string("not a scheduler model file: ") + path);
  });
}

pb_status pb_ctx_set_sched_model(pb_ctx* ctx, pb_sched_model* model) {
  if (!ctx) return PB_EINVAL;
  if (model && model->device != ctx->device) return PB_EINVAL;
  ctx->model = model;
  return PB_OK;
}

pb_status pb_trace_set(pb_ctx* ctx, int32_t mode, uint64_t seed) {
  if (!ctx) return PB_EINVAL;
  if (mode < PB_TRACE_OFF || mode > PB_TRACE_EXPLORE) return PB_EINVAL;
  ctx->trace_mode = mode;
  ctx->trace_seed = seed;
  ctx->peel_sweep[0] = ctx->peel_sweep[1] = seed;
  return PB_OK;
}

pb_status pb_trace_rows(pb_ctx* ctx, int32_t target, float* X, float* y, int64_t cap, int64_t* n) {
  if (!ctx || !n || (target != PB_SCHED_COUNT && target != PB_SCHED_PEEL)) return PB_EINVAL;
  const int64_t rows = (int64_t)ctx->trace_y[target].size();
  *n = rows;
  if (X && y) {
    const int64_t k = std::min(rows, cap);
    std::memcpy(X, ctx->trace_X[target].data(), sizeof(float) * (size_t)k * pb::kMlpIn);
    std::memcpy(y, ctx->trace_y[target].data(), sizeof(float) * (size_t)k);
  }
  return PB_OK;
}

pb_status pb_trace_clear(pb_ctx* ctx) {
  if (!ctx) return PB_EINVAL;
  for (int t = 0; t < 2; ++t) {
    ctx->trace_X[t].clear();
    ctx->trace_y[t].clear();
  }
  return PB_OK;
}

pb_status pb_tc_gemm_bf16(pb_ctx* ctx, int64_t M, int32_t N, int64_t K, const void* A, int64_t sam, int64_t sak,
                          const void* B, int64_t sbn, int64_t sbk, float* D, int64_t ldd) {
  return guarded(ctx, [&] {
    PB_REQUIRE(A && B && D, PB_EINVAL, "null argument");
    PB_REQUIRE(is_device_ptr(A) && is_device_ptr(B) && is_device_ptr(D), PB_EINVAL, "operands must be device memory");
    cudaStream_t s = ctx->stream;
    DevBuf<uint32_t> err(4, s);
    PB_CUDA_TRY(cudaMemsetAsync(err.get(), 0, err.bytes(), s));
    pb::GemmSpec g;
    g.A = (const __nv_bfloat16*)A; g.sam = sam; g.sak = sak;
    g.B = (const __nv_bfloat16*)B; g.sbn = sbn; g.sbk = sbk;
    g.M = M; g.N = N; g.K = K;
    g.epi = pb::GEMM_STORE; g.D = D; g.ldd = ldd;
    pb::tc_gemm_bf16(g, err.get(), s);
    uint32_t h = 0;
    PB_CUDA_TRY(cudaMemcpyAsync(&h, err.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    PB_REQUIRE(h == 0, PB_ETIMEOUT, "tensor-core GEMM: bounded mbarrier wait ran out");
  });
}

}  // extern "C"
