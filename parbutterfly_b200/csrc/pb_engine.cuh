// Internal structures shared by the ranking, counting and peeling stages.
#pragma once

#include <vector>

#include "pb_common.cuh"

struct pb_graph {
  int device = 0;
  int64_t nv = 0, nu = 0, m = 0;
  // Device copy of the two-sided CSR (never modified after upload).
  pb::DevBuf<uint32_t> offV, edgV, offU, edgU;
  uint32_t max_deg = 0;
};

namespace pb {

// Timing of one counting call (milliseconds, CUDA events on the context stream).
struct StageTimes {
  double rank = 0, relabel = 0, scan = 0, count = 0, convert = 0, agg_kernel = 0;
};

// Ranked single CSR of n = nv + nu vertices (rankGraph / rankGraphEdges,
// butterfly_utils.h:579-700): row r holds (rank << 1 | on_count_side) of the neighbours of the
// vertex of rank r, ascending.
struct Ranked {
  int64_t n = 0, m2 = 0;
  int use_v = 1;
  DevBuf<uint32_t> order;  // order[r] = combined id (V ids 0..nv-1, then nv + U id)
  DevBuf<uint32_t> rank;   // rank[combined id]
  DevBuf<uint32_t> off;    // n+1
  DevBuf<uint32_t> adj;    // 2m tagged ranks
  DevBuf<uint32_t> eout;   // 2m output edge index (per-edge counting only)
  DevBuf<uint32_t> pref;   // 2m: wedges of slot (i,j) = #{u2 in N(v): u2 < min(i,v)}
  DevBuf<int64_t> wsum;    // n+1: exclusive prefix of per-endpoint wedge counts
  int64_t w_rank = 0;
  uint32_t max_deg = 0;
};

// Ranking stage (pb_rank.cu).
void degrees_combined(const pb_graph& g, uint32_t* deg, cudaStream_t s);
void cmp_wedge_counts(const pb_graph& g, int* use_v, int64_t* w_min, int64_t* wv, int64_t* wu, cudaStream_t s);
void vertex_order(const pb_graph& g, int rank_type, int use_v, Ranked& R, cudaStream_t s);
void build_ranked_csr(const pb_graph& g, Ranked& R, bool with_eout, cudaStream_t s);
void wedge_scan(Ranked& R, cudaStream_t s);
void edge_to_idxs(const pb_graph& g, int use_v, uint32_t* eti, cudaStream_t s);

// Counting stage (pb_count.cu).  per: 0 VERT (out: rank-space counts [n]), 1 EDGE (out: [m]
// in output edge order), 2 TOTAL (out: [1]).  `strategy` selects the aggregator.
enum Strategy { STRAT_HASH = 0, STRAT_DENSE = 1, STRAT_SORT = 2, STRAT_HIST = 3, STRAT_AUTO = 4 };
struct MlpModel;
// Scheduler hooks of one counting call.  Each endpoint the block aggregator takes is one
// scheduling item; its features (12 numbers) plus a one-hot of the aggregation mode (dense,
// hash, global, hybrid) form one cost-model row, and the item's measured SM cycles its target.
struct SchedHooks {
  MlpModel* model = nullptr;  // learned: the valid shared-memory mode with the least predicted
                              // cycles (global scratch when none can hold the item)
  bool explore = false;       // a seeded random valid mode per item (trace collection)
  uint64_t seed = 0;
  std::vector<float>* trace_X = nullptr;  // when set, rows are appended (16 floats per row)
  std::vector<float>* trace_y = nullptr;  // with log2(cycles) targets
  // Filled by the call.
  int64_t items = 0;
  double pred_cycles = 0, meas_cycles = 0, mae_log2 = 0, ms = 0;
};
struct CountConfig {
  int strategy = STRAT_AUTO;
  int small_w = 512;          // endpoints with W_i <= small_w go to the warp aggregator
  int block_threads = 512;    // threads of the block aggregator
  int smem_bytes = 48 * 1024;   // dynamic shared memory of the block aggregator
  int blocks_per_sm = 4;
  int split_w = 0;            // endpoints above this many wedges are split across CTAs (0: auto)
  uint32_t* err = nullptr;    // checked mode: device record of the first bounds violation
  SchedHooks* sched = nullptr;
};

// Checked mode (PB_CHECK=1): kernels bounds-check indices read from memory and record the
// first violation instead of accessing out of bounds; the ranked CSR is validated after the
// relabel.  Off by default.
bool check_mode();
void validate_ranked(const Ranked& R, int64_t m, uint32_t* err, cudaStream_t s);
struct CountResult {
  int n_big = 0;
  double agg_ms = 0;
  // CTA aggregator modes (dense, hash, global scratch, hybrid): endpoints and wedges.
  unsigned long long mode_items[4] = {0, 0, 0, 0};
  unsigned long long mode_wedges[4] = {0, 0, 0, 0};
};
CountResult count_ranked(const Ranked& R, int per, int64_t* out, const CountConfig& cfg, cudaStream_t s);
// SORT (hist = false) and HIST (hist = true) aggregators over materialised wedge batches of at
// most max_wedges wedges (pb_agg_sort.cu).
CountResult count_ranked_materialized(const Ranked& R, int per, int64_t* out, bool hist, int64_t max_wedges,
                                      cudaStream_t s);

// Device parsing of the AdjacencyHypergraph text (pb_parse.cu): the four CSR arrays of the
// file in `text` (len bytes, host or device memory), offsets including the final m.
struct ParsedCSR {
  int64_t nv = 0, nu = 0, m = 0;
  DevBuf<uint32_t> offV, edgV, offU, edgU;
};
void parse_adjacency_hypergraph(const char* text, size_t len, bool on_device, ParsedCSR& out, cudaStream_t s);
// The graph of the host R-MAT generator (pb_gen.cpp), generated on the device (pb_gen_dev.cu).
void gen_rmat_device(int log_nv, int log_nu, int64_t m, double a, double b, double c, double d, uint64_t seed,
                     ParsedCSR& out, cudaStream_t s);

// Batches (pb_batch.cu): the disjoint union of k graphs, each graph's count side on the union's
// U side (count with use_v = 1); kbase/ksize locate each graph's count side in the union.
void build_union(const pb_graph* const* gs, int k, pb_graph& U, std::vector<int64_t>& kbase,
                 std::vector<int64_t>& ksize, cudaStream_t s, std::vector<double>* work = nullptr);

// Peeling stage (pb_peel.cu).
struct PeelResult {
  int64_t rounds = 0;           // exact bucket rounds (summed over the partitions of a two-phase peel)
  int64_t work = 0;
  int64_t coarse_rounds = 0;    // two-phase: rounds of the coarse pass
  int64_t parts = 0;            // two-phase: partitions
  int64_t fine_rounds_max = 0;  // two-phase: rounds of the longest partition
};
// Work-unit sizing of the persistent peel kernel (the defaults are the plain path's).
struct PeelTuning {
  int64_t small_work = 512;               // items up to this work run on one warp
  int64_t huge_work = int64_t(1) << 40;   // items above this run on the whole grid
  int64_t chunk_work = 512;               // probes per warp unit, minimum per CTA work unit (wing)
  bool warp_units = false;                // wing: items with warp-sized probe sets run as warp units
  int64_t units_per_cta = 4;              // CTA work units per CTA and round (wing)
  int64_t near_min = 32768;               // the near window holds at least this many items
  int64_t near_div = 64;                  // ... or alive / near_div
  int64_t max_ctas = 0;                   // CTAs of the persistent kernel (0: all resident)
  // Two-phase schedule: a coarse pass cuts the items into partitions (ranges of their final
  // numbers, about parts_per_cta per CTA or parts_total in all, of equal estimated work), then
  // every partition runs its exact rounds as an independent instance of one launch.  Same
  // results as one instance running every round over the whole GPU.
  bool two_phase = false;
  double parts_per_cta = 2.0;
  int64_t parts_total = 0;
};
// The plain path's settings: wing items never take the whole grid; tip items above 2^13
// wedges do (one CTA per heavy vertex leaves the rest of the GPU idle in most rounds).
inline PeelTuning plain_peel_tuning(bool wing) {
  PeelTuning t;
  if (!wing) t.huge_work = int64_t(1) << 13;
  return t;
}
// Independent peel instances of one launch (the graphs of a batch): items base[i] ..
// base[i] + size[i] - 1 form instance i, which gets a share of the CTAs in proportion to
// weight[i] and runs its own rounds.
struct PeelParts {
  std::vector<int64_t> base, size;
  std::vector<double> weight;
};
PeelResult peel_vertices(const pb_graph& g, int use_v, const int64_t* counts_dev, int64_t* tip_dev, cudaStream_t s,
                         const PeelTuning& tune = plain_peel_tuning(false), const PeelParts* parts = nullptr);
PeelResult peel_edges(const pb_graph& g, int use_v, const int64_t* ecounts_dev, int64_t* wing_dev, cudaStream_t s,
                      const PeelTuning& tune = plain_peel_tuning(true));

}  // namespace pb
