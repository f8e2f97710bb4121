// Many graphs in one pass: per-vertex counts and tip numbers of k independent graphs.
//
// Butterflies never span two connected pieces, so the disjoint union of the k graphs has, for
// every vertex, exactly the count it has in its own graph, and tip peeling of the union gives
// every vertex the tip number it gets alone (a graph is untouched by rounds below its own
// minimum and peels exactly its own frontier at each of its own levels).  The union is built
// on the device with each graph's count side (chosen per graph as cmpWedgeCounts does,
// butterfly_utils.h:1080-1086) placed on the union's U side, so the whole batch runs as one
// ranking, one aggregation launch pair and one persistent peeling launch.
#include <algorithm>
#include <vector>

#include "pb_engine.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

struct GraphRef {
  const uint32_t* offK;  // count side of the graph (after its own count-side choice)
  const uint32_t* edgK;
  const uint32_t* offC;
  const uint32_t* edgC;
  int64_t nK, nC;
  int64_t kbase, cbase, ebase;  // first union id on each side, first union edge
};

// Side wedge sums of every graph (wedgeF, butterfly_utils.h:1061-1070: 32-bit products).
__global__ void batch_side_wedges_kernel(const uint32_t* const* offV, const uint32_t* const* offU,
                                         const int64_t* __restrict__ nv, const int64_t* __restrict__ nu, int k,
                                         unsigned long long* sums /* [2k] */) {
  for (int g = blockIdx.y; g < k; g += gridDim.y) {
    unsigned long long sv = 0, su = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv[g] + nu[g];
         i += (int64_t)gridDim.x * blockDim.x) {
      const uint32_t d = i < nv[g] ? offV[g][i + 1] - offV[g][i] : offU[g][i - nv[g] + 1] - offU[g][i - nv[g]];
      const unsigned long long w = (unsigned long long)((uint32_t)(d * (d - 1u)) / 2u);
      if (i < nv[g]) sv += w;
      else su += w;
    }
    sv = warp_sum(sv);
    su = warp_sum(su);
    if ((threadIdx.x & 31) == 0) {
      if (sv) atomicAdd(&sums[2 * g], sv);
      if (su) atomicAdd(&sums[2 * g + 1], su);
    }
  }
}

// Union offsets and edges.  Offsets: one thread per union vertex (both sides); edges: one warp
// per union vertex copies its list with the id shift of the other side.
__global__ void batch_union_kernel(const GraphRef* __restrict__ G, int k, const int64_t* __restrict__ kstart,
                                   const int64_t* __restrict__ cstart, int64_t nK, int64_t nC, uint32_t* uoffU,
                                   uint32_t* uedgU, uint32_t* uoffV, uint32_t* uedgV) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t x = warp; x < nK + nC; x += nwarps) {
    const bool countside = x < nK;
    const int64_t ux = countside ? x : x - nK;
    const int64_t* starts = countside ? kstart : cstart;
    int lo = 0, hi = k;  // graph of ux: last g with starts[g] <= ux
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (starts[mid] <= ux) lo = mid;
      else hi = mid;
    }
    const GraphRef& R = G[lo];
    const int64_t local = ux - (countside ? R.kbase : R.cbase);
    const uint32_t* off = countside ? R.offK : R.offC;
    const uint32_t* edg = countside ? R.edgK : R.edgC;
    const int64_t shift = countside ? R.cbase : R.kbase;
    const uint32_t b = off[local], e = off[local + 1];
    const uint32_t ub = (uint32_t)(R.ebase + b);
    if (lane == 0) {
      (countside ? uoffU : uoffV)[ux] = ub;
    }
    uint32_t* dst = countside ? uedgU : uedgV;
    for (uint32_t j = b + lane; j < e; j += 32) dst[ub + (j - b)] = (uint32_t)(edg[j] + shift);
  }
}

int grid_for(int64_t n) { return std::max(1, std::min(ceil_div(n, 256), sm_count() * 16)); }

}  // namespace

// Builds the union graph; returns per-graph count-side bases and sizes, and (when work is not
// null) each graph's two-hop wedges from its count side, sum over centres of deg (deg - 1).
void build_union(const pb_graph* const* gs, int k, pb_graph& U, std::vector<int64_t>& kbase,
                 std::vector<int64_t>& ksize, cudaStream_t s, std::vector<double>* work) {
  PB_REQUIRE(k > 0, PB_EINVAL, "empty batch");
  std::vector<const uint32_t*> hoffV(k), hoffU(k);
  std::vector<int64_t> hnv(k), hnu(k);
  int64_t maxn = 0;
  for (int g = 0; g < k; ++g) {
    PB_REQUIRE(gs[g], PB_EINVAL, "null graph in batch");
    hoffV[g] = gs[g]->offV.get();
    hoffU[g] = gs[g]->offU.get();
    hnv[g] = gs[g]->nv;
    hnu[g] = gs[g]->nu;
    maxn = std::max(maxn, hnv[g] + hnu[g]);
  }
  DevBuf<const uint32_t*> doffV(k, s), doffU(k, s);
  DevBuf<int64_t> dnv(k, s), dnu(k, s);
  DevBuf<unsigned long long> sums(2 * k, s);
  PB_CUDA_TRY(cudaMemcpyAsync(doffV.get(), hoffV.data(), sizeof(void*) * k, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(doffU.get(), hoffU.data(), sizeof(void*) * k, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(dnv.get(), hnv.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(dnu.get(), hnu.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemsetAsync(sums.get(), 0, sizeof(unsigned long long) * 2 * k, s));
  dim3 grid((unsigned)std::max(1, std::min(ceil_div(maxn, 256), 64)), (unsigned)std::min(k, 1024));
  batch_side_wedges_kernel<<<grid, 256, 0, s>>>(doffV.get(), doffU.get(), dnv.get(), dnu.get(), k, sums.get());
  PB_CUDA_TRY(cudaGetLastError());
  if (g_launch_counter) ++*g_launch_counter;
  std::vector<unsigned long long> hs(2 * k);
  PB_CUDA_TRY(cudaMemcpyAsync(hs.data(), sums.get(), sizeof(unsigned long long) * 2 * k, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));

  std::vector<GraphRef> refs(k);
  std::vector<int64_t> kst(k), cst(k);
  kbase.assign(k, 0);
  ksize.assign(k, 0);
  if (work) work->assign(k, 0.0);
  int64_t nK = 0, nC = 0, m = 0;
  uint32_t maxdeg = 0;
  for (int g = 0; g < k; ++g) {
    const pb_graph* G = gs[g];
    const bool use_v = hs[2 * g] <= hs[2 * g + 1];  // count side U when use_v
    if (work) (*work)[g] = 2.0 * (double)(use_v ? hs[2 * g] : hs[2 * g + 1]) + (double)G->m;
    GraphRef& R = refs[g];
    R.offK = use_v ? G->offU.get() : G->offV.get();
    R.edgK = use_v ? G->edgU.get() : G->edgV.get();
    R.offC = use_v ? G->offV.get() : G->offU.get();
    R.edgC = use_v ? G->edgV.get() : G->edgU.get();
    R.nK = use_v ? G->nu : G->nv;
    R.nC = use_v ? G->nv : G->nu;
    R.kbase = nK;
    R.cbase = nC;
    R.ebase = m;
    kst[g] = nK;
    cst[g] = nC;
    kbase[g] = nK;
    ksize[g] = R.nK;
    nK += R.nK;
    nC += R.nC;
    m += G->m;
    maxdeg = std::max(maxdeg, G->max_deg);
  }
  PB_REQUIRE(nK + nC < (int64_t)(1u << 31), PB_ETOOBIG, "batch too large: nv + nu of the union must stay below 2^31");
  PB_REQUIRE(2 * m <= (int64_t)UINT32_MAX, PB_ETOOBIG, "batch too large: 2 m of the union must fit 32 bits");
  U.device = gs[0]->device;
  U.nv = nC;  // union V = centre sides
  U.nu = nK;  // union U = count sides
  U.m = m;
  U.max_deg = maxdeg;
  U.offV.alloc(nC + 1, s);
  U.offU.alloc(nK + 1, s);
  U.edgV.alloc(m > 0 ? m : 1, s);
  U.edgU.alloc(m > 0 ? m : 1, s);
  DevBuf<GraphRef> drefs(k, s);
  DevBuf<int64_t> dk(k, s), dc(k, s);
  PB_CUDA_TRY(cudaMemcpyAsync(drefs.get(), refs.data(), sizeof(GraphRef) * k, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(dk.get(), kst.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(dc.get(), cst.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, s));
  if (nK + nC > 0)
    PB_LAUNCH(batch_union_kernel, grid_for((nK + nC) * 32), 256, 0, s, drefs.get(), k, dk.get(), dc.get(), nK, nC,
              U.offU.get(), U.edgU.get(), U.offV.get(), U.edgV.get());
  const uint32_t mm = (uint32_t)m;
  PB_CUDA_TRY(cudaMemcpyAsync(U.offU.get() + nK, &mm, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaMemcpyAsync(U.offV.get() + nC, &mm, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
}

}  // namespace pb
