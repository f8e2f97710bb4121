/*
 * parbutterfly_b200 — C ABI of the B200-native butterfly counting / peeling library.
 *
 * The reference (ParButterfly, apps/hyper/) has no FFI: its boundary is the
 * BipartiteButterflies CLI and the C++ entry points that Compute() calls
 * (apps/hyper/BipartiteButterflies.C:75-277).  Every entry point below replaces one of
 * those calls; the comment on each one cites the reference function it stands in for.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Graph arrays use the reference's default integer
 *    widths: offsets are uintT (uint32_t) and vertex ids are uintE (uint32_t)
 *    (ligra/parallel.h:102-125, no -DLONG / -DEDGELONG).  Counts are int64_t ("long").
 *  - Outputs are DENSE int64 arrays (the reference strides them by 8 longs, one per cache
 *    line, e.g. BipartiteButterflies.C:228-232; the stride carries no information and is
 *    dropped).  Output pointers may be host or device memory; the library detects which.
 *  - Every call returns a pb_status and never exits the process (the reference prints and
 *    calls exit(0)/abort(), e.g. butterfly_utils.h:1014-1016,1040,1050).  On error,
 *    pb_last_error() returns a message for the calling context.
 *  - All calls are synchronous with respect to the context's CUDA stream on return.
 *  - One pb_ctx per host thread; distinct contexts are independent.
 */
#ifndef PARBUTTERFLY_B200_H
#define PARBUTTERFLY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB_ABI_VERSION 2

typedef enum {
  PB_OK = 0,
  PB_EINVAL = 1,       /* bad argument or malformed CSR (unsorted list, id out of range, mv != mu) */
  PB_ENOMEM = 2,       /* device or host allocation failed */
  PB_ETOOBIG = 3,      /* a size exceeds a documented limit */
  PB_ETIMEOUT = 4,     /* a bounded device wait ran out; the context stays usable */
  PB_ECUDA = 5,        /* a CUDA runtime call failed */
  PB_EUNSUPPORTED = 6, /* option outside the supported surface (e.g. sparsification) */
  PB_EIO = 7           /* file could not be read / parsed */
} pb_status;

/* Enum values and order follow apps/hyper/butterfly_utils.h:24-28 exactly. */
typedef enum { PB_SORT = 0, PB_ASORT, PB_HASH, PB_AHASH, PB_HIST, PB_AHIST, PB_BATCHS, PB_BATCHWA, PB_SERIAL } pb_count_type;
typedef enum { PB_SIDE = 0, PB_COCORE, PB_ACOCORE, PB_DEG, PB_ADEG } pb_rank_type;
typedef enum { PB_PSORT = 0, PB_PHASH, PB_PHIST, PB_PBATCHS, PB_PBATCHWA } pb_peel_type;
typedef enum { PB_VERT = 0, PB_EDGE, PB_TOTAL } pb_per_type;
/* SparseType, butterfly_utils.h:28 (same values). */
typedef enum { PB_NOSPARSE = 0, PB_SPARSE_COLOR, PB_SPARSE_EDGE } pb_sparse_type;

/* Strategy scheduler: PLAIN = the fixed strategy named by count_type; LEARNED = per-block
 * strategy picked by the learned scheduler (results are identical either way). */
typedef enum { PB_SCHED_PLAIN = 0, PB_SCHED_LEARNED = 1 } pb_sched;

/* Options.  Field meanings and defaults follow the CLI of BipartiteButterflies.C:79-194. */
typedef struct {
  int32_t count_type;     /* pb_count_type, default PB_SERIAL (BipartiteButterflies.C:92) */
  int32_t rank_type;      /* pb_rank_type, default PB_ADEG (BipartiteButterflies.C:118) */
  int32_t peel_type;      /* pb_peel_type, default PB_PBATCHS */
  int32_t per_type;       /* pb_per_type, default PB_VERT */
  int64_t max_wedges;     /* -m, default 2577500000 (BipartiteButterflies.C:172) */
  int64_t max_array_size; /* -a, default 23090996160 (BipartiteButterflies.C:173) */
  int32_t sched;          /* pb_sched, default PB_SCHED_PLAIN */
  int32_t autotune;       /* 0/1: the autotuner picks the block aggregator's table size, CTAs
                             per SM and warp/CTA boundary per graph: the first call on a graph
                             signature times every candidate, later calls on the context reuse
                             the fastest (results are identical either way) */
  int32_t use_v;          /* -1 = choose as cmpWedgeCounts does; 0/1 forces the count side */
  int32_t peel_parts;     /* batching of the peel's exact rounds (no counterpart in the reference;
                             results are identical either way): 0 = the scheduler's choice when
                             sched = LEARNED, else one round at a time over the whole GPU;
                             n > 0 = the two-phase schedule with about n partitions (a coarse
                             pass cuts the items by ranges of their final numbers, then every
                             partition runs its exact rounds independently, all in one launch);
                             -1 = one round at a time even when sched = LEARNED */
} pb_opts;

/* Host-side two-sided CSR, the layout of struct bipartiteCSR (butterfly_utils.h:184-197).
 * offsetsV[nv+1], edgesV[m] (U ids), offsetsU[nu+1], edgesU[m] (V ids); every adjacency
 * list sorted ascending without duplicates (the contract of utils/graphIO.h:378-420). */
typedef struct {
  int64_t nv, nu, m;
  const uint32_t* offsetsV;
  const uint32_t* edgesV;
  const uint32_t* offsetsU;
  const uint32_t* edgesU;
} pb_csr;

/* Owned host CSR returned by the generators and the file reader; release with pb_csr_free. */
typedef struct {
  int64_t nv, nu, m;
  uint32_t* offsetsV;
  uint32_t* edgesV;
  uint32_t* offsetsU;
  uint32_t* edgesU;
} pb_csr_owned;

/* Per-call statistics of the last count/peel call on a context. */
typedef struct {
  int64_t w_side;         /* get<1>(cmpWedgeCounts(G)) (butterfly_utils.h:1080-1086) */
  int64_t w_rank;         /* wedges the ranked traversal enumerates (countWedgesScan total) */
  int32_t use_v;          /* count side actually used */
  int32_t n_big;          /* endpoints handled by the block-cooperative aggregator */
  double ms_rank;         /* ranking: vertex order (ADEG/DEG/COCORE/ACOCORE/SIDE) */
  double ms_relabel;      /* ranked CSR build (rankGraph / rankGraphEdges) */
  double ms_scan;         /* wedge scan (countWedgesScan) */
  double ms_count;        /* wedge aggregation + butterfly accumulation */
  double ms_convert;      /* rank -> original index conversion */
  double ms_peel;         /* peeling (tip or wing) */
  int64_t peel_rounds;    /* bucket rounds executed by the last peel call */
  int64_t peel_work;      /* wedges (tip) or intersection probes (wing) processed while peeling */
  double ms_agg_kernel;   /* device time of the aggregation kernels alone */
  /* Learned scheduler (no counterpart in the reference): */
  int32_t sched_used;     /* 1 when the learned scheduler made this call's choices, else 0 */
  int32_t sched_choice;   /* peel calls: index of the work-unit setting that ran (0 = plain) */
  int64_t sched_items;    /* count calls: block-aggregator items the scheduler decided */
  double ms_sched;        /* scheduler time inside the call (features, inference, ordering) */
  double sched_pred;      /* predicted time: SM cycles summed over items (count), ms (peel) */
  double sched_meas;      /* measured time in the same unit */
  double sched_mae_log2;  /* count calls: mean |log2(predicted / measured)| over the items */
  /* Block-aggregator geometry of the last count call (opts.autotune picks it per graph): */
  int32_t count_smem_bytes;    /* shared-memory table bytes per CTA */
  int32_t count_blocks_per_sm; /* CTAs per SM */
  int32_t count_small_w;       /* endpoints with at most this many wedges go to a warp */
  int32_t autotuned;           /* 1 when this call ran the autotuner's sweep */
  /* Round batching of the last peel call (two-phase schedule; zeros when it ran one round at a
   * time): partitions, rounds of the coarse pass, rounds of the longest partition. */
  int64_t peel_parts;
  int64_t peel_coarse_rounds;
  int64_t peel_fine_rounds_max;
} pb_stats;

typedef struct pb_ctx pb_ctx;
typedef struct pb_graph pb_graph;

/* ---- library / context ---------------------------------------------------------------- */
int pb_abi_version(void);
void pb_opts_default(pb_opts* opts);
/* Creates a context on CUDA device `device`.  `stream` is a cudaStream_t or NULL (the context
 * then creates its own non-blocking stream). */
pb_status pb_ctx_create(int device, void* stream, pb_ctx** out);
pb_status pb_ctx_destroy(pb_ctx* ctx);
const char* pb_last_error(const pb_ctx* ctx);
pb_status pb_get_stats(const pb_ctx* ctx, pb_stats* out);
/* Counts of this library's kernel launches on the context since creation (for reporting). */
int64_t pb_kernel_launches(const pb_ctx* ctx);

/* ---- graph ----------------------------------------------------------------------------- */
/* Copies a host CSR to the device and validates it (sortedness, ranges, mv == mu); replaces
 * the in-memory result of readBipartite (butterfly_utils.h:1008-1058). */
pb_status pb_graph_upload(pb_ctx* ctx, const pb_csr* host, pb_graph** out);
/* Same contract, for arrays already resident in device memory (copied, not adopted). */
pb_status pb_graph_from_device(pb_ctx* ctx, const pb_csr* dev, pb_graph** out);
/* readBipartite (butterfly_utils.h:1008-1058) on the device: the AdjacencyHypergraph text of
 * `len` bytes at `text` (host or device memory) is tokenised and parsed by GPU threads, its sizes
 * and token count checked as readBipartite does (PB_EIO instead of abort), ids range-checked and
 * the CSR validated (sorted lists) on the device. */
pb_status pb_graph_parse_text(pb_ctx* ctx, const char* text, size_t len, pb_graph** out);
/* The same for a file: read into pinned host memory, parsed on the device. */
pb_status pb_graph_read_text(pb_ctx* ctx, const char* path, pb_graph** out);
/* The graph of pb_gen_rmat (same arguments, same graph) generated on the device of ctx, for
 * sizes whose host generation does not fit host memory (no counterpart in the reference, whose
 * generators run on the CPU: utils/rMatGraph.C). */
pb_status pb_gen_rmat_device(pb_ctx* ctx, int32_t log_nv, int32_t log_nu, int64_t m, double a, double b, double c,
                             double d, uint64_t seed, pb_graph** out);
pb_status pb_graph_destroy(pb_graph* g);
pb_status pb_graph_dims(const pb_graph* g, int64_t* nv, int64_t* nu, int64_t* m);
/* Copies a device graph back to host memory (release with pb_csr_free). */
pb_status pb_graph_download(const pb_graph* g, pb_csr_owned* out);

/* cmpWedgeCounts (butterfly_utils.h:1080-1086): *use_v = (W_V <= W_U), *num_wedges = min. */
pb_status pb_cmp_wedge_counts(pb_ctx* ctx, const pb_graph* g, int32_t* use_v, int64_t* num_wedges);

/* edgeToIdxs (butterfly_utils.h:2034-2062): eti[m], for the orientation given by use_v.
 * idxsToEdge (:2065-2067) is the same call with use_v inverted. */
pb_status pb_edge_to_idxs(pb_ctx* ctx, const pb_graph* g, int32_t use_v, uint32_t* eti);

/* ---- counting -------------------------------------------------------------------------- */
/* Count (butterfly_count.h:1634-1731): out[nCount] per count-side vertex, original ids;
 * nCount = nu if use_v else nv. */
pb_status pb_count_vert(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out);
/* CountE (butterfly_ecount.h:1766-1899): out[m] per edge, indexed like the reference's
 * result: by position in edgesV when use_v, else by position in edgesU. */
pb_status pb_count_edge(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out);
/* CountTotal (butterfly_count_total.h:1014-1102): total number of butterflies. */
pb_status pb_count_total(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, int64_t* out);

/* ---- peeling --------------------------------------------------------------------------- */
/* Peel (butterfly_peel.h:896-934): tip numbers tip[nCount] from per-vertex counts (as from
 * pb_count_vert with the same use_v).  64-bit buckets throughout. */
pb_status pb_peel_vert(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, const int64_t* counts,
                       int64_t* tip);
/* PeelE (butterfly_epeel.h:519-569): wing numbers wing[m] from per-edge counts (edge order of
 * pb_count_edge).  The graph is not modified (the reference tombstones its input). */
pb_status pb_peel_edge(pb_ctx* ctx, const pb_graph* g, const pb_opts* opts, const int64_t* ecounts,
                       int64_t* wing);

/* ---- many graphs at once --------------------------------------------------------------- */
/* Count (butterfly_count.h:1634-1731) for k graphs in one pass: counts[g] receives nCount(g)
 * per-vertex counts, each graph using its own count side as cmpWedgeCounts decides for it.
 * The batch runs as one disjoint union on the device (one ranking, one aggregation, no
 * per-graph launches); results equal k separate pb_count_vert calls. */
pb_status pb_count_vert_batch(pb_ctx* ctx, const pb_graph* const* gs, int32_t k, const pb_opts* opts,
                              int64_t* const* counts);
/* Peel (butterfly_peel.h:896-934) for k graphs in one persistent launch: tips[g] receives the
 * tip numbers of graph g from its per-vertex counts counts[g] (as from pb_count_vert_batch). */
pb_status pb_peel_vert_batch(pb_ctx* ctx, const pb_graph* const* gs, int32_t k, const pb_opts* opts,
                             const int64_t* const* counts, int64_t* const* tips);

/* ---- learned scheduler (no counterpart in the reference) -------------------------------- */
/* The reference always runs the fixed strategy its flags name.  Here a cost model — a 3-layer
 * MLP (16 -> 64 -> 64 -> 1, BF16 operands, FP32 accumulation, every product on the tensor
 * cores) — predicts log2 of the time of each candidate choice and the call takes the least:
 *   counting (opts.sched = PB_SCHED_LEARNED, HASH/BATCHS/BATCHWA/SERIAL count types): the
 *     aggregation mode of every endpoint the block aggregator takes, among the shared-memory
 *     modes that can hold its table (dense window, hash table, dense window + hash table); the
 *     global-scratch mode remains the fallback of endpoints none of them can hold;
 *   peeling (opts.sched = PB_SCHED_LEARNED): the setting of the persistent peel kernel — how
 *     many CTAs it runs on (tip), how a round's CTA work is cut into units (wing), which items run
 *     on a warp and which take the whole grid (tip) — from a grid of PB_SCHED_WING_CANDIDATES (wing)
 *     or PB_SCHED_TIP_CANDIDATES (tip) settings (0 = the plain setting).
 * Results are identical to the plain path's (every choice is exact).  Without an attached,
 * trained model a LEARNED call runs the plain path (stats.sched_used = 0).
 * The model learns from traces the plain path logs: with tracing on, every count call appends
 * one row per block-aggregator item (12 features + one-hot mode, target log2 SM cycles) and
 * every peel call one row (12 call features + 4 setting features, target log2 ms).  In explore
 * mode count calls draw each item's mode at random among the valid ones (seeded) and peel calls
 * sweep the setting grid cyclically (tip and wing calls each from setting seed mod
 * the kind's number of candidates, one step per call), so that the traces cover every choice. */
#define PB_SCHED_FEATURES 16
#define PB_SCHED_WING_CANDIDATES 6
#define PB_SCHED_TIP_CANDIDATES 32
typedef enum { PB_SCHED_COUNT = 0, PB_SCHED_PEEL = 1 } pb_sched_target;
typedef enum { PB_TRACE_OFF = 0, PB_TRACE_PLAIN = 1, PB_TRACE_EXPLORE = 2 } pb_trace_mode;
typedef struct pb_sched_model pb_sched_model;
/* A model with both cost models (count, peel) initialised from `seed`, on ctx's device. */
pb_status pb_sched_model_create(pb_ctx* ctx, uint64_t seed, pb_sched_model** out);
pb_status pb_sched_model_destroy(pb_sched_model* model);
/* Trains one cost model on host rows X[n][PB_SCHED_FEATURES], targets y[n] (log2 time) with
 * Adam for `epochs` passes of mini-batches of `batch` rows; *final_mse (may be NULL) receives the
 * last epoch's mean squared error in standardised units. */
pb_status pb_sched_train(pb_ctx* ctx, pb_sched_model* model, int32_t target, const float* X, const float* y, int64_t n,
                         int32_t epochs, int32_t batch, float lr, float* final_mse);
/* Predicted log2 time for host rows X[n][PB_SCHED_FEATURES] into y[n] (host). */
pb_status pb_sched_predict(pb_ctx* ctx, pb_sched_model* model, int32_t target, const float* X, int64_t n, float* y);
pb_status pb_sched_save(pb_ctx* ctx, const pb_sched_model* model, const char* path);
pb_status pb_sched_load(pb_ctx* ctx, pb_sched_model* model, const char* path);
/* Attaches a model to the context (NULL detaches); LEARNED calls on ctx use it. */
pb_status pb_ctx_set_sched_model(pb_ctx* ctx, pb_sched_model* model);
/* Trace logging on ctx: mode pb_trace_mode; seed drives explore-mode choices. */
pb_status pb_trace_set(pb_ctx* ctx, int32_t mode, uint64_t seed);
/* Number of rows logged for `target`; with X and y non-NULL copies up to cap rows out. */
pb_status pb_trace_rows(pb_ctx* ctx, int32_t target, float* X, float* y, int64_t cap, int64_t* n);
pb_status pb_trace_clear(pb_ctx* ctx);
/* The tensor-core product the cost model runs on, exposed for testing: D[m][n] (FP32, row
 * stride ldd) = sum_k A(m,k) B(n,k) with BF16 operands in device memory addressed by element
 * strides, A(m,k) = A[m*sam + k*sak], B(n,k) = B[n*sbn + k*sbk]; 1 <= N <= 128. */
pb_status pb_tc_gemm_bf16(pb_ctx* ctx, int64_t M, int32_t N, int64_t K, const void* A, int64_t sam, int64_t sak,
                          const void* B, int64_t sbn, int64_t sbk, float* D, int64_t ldd);

/* ---- a batch as one CUDA graph (no counterpart in the reference) ----------------------------
 * Count (butterfly_count.h:1634-1731) and Peel (butterfly_peel.h:896-934) of k graphs, planned
 * once and replayed as one CUDA graph: pb_batch_create builds the disjoint union on the device
 * (each graph's count side as cmpWedgeCounts decides for it), runs the whole pipeline once
 * eagerly (ranking, per-vertex counting, tip peeling as one persistent launch) while logging
 * every host readback, then captures the same sequence with the logged values, so the graph
 * holds no host synchronisation.  opts.autotune tunes the aggregator geometry on the union
 * first.  pb_batch_run replays the graph (the full ranking + counting + peeling work every
 * time) and copies counts[g] / tips[g] (nCount(g) each, host or device; either may be NULL) out;
 * stats.ms_count is the replay's device time.  Count types HASH/AHASH/BATCHS/BATCHWA/SERIAL
 * (SORT / HIST return PB_EUNSUPPORTED).  The graphs may be destroyed after pb_batch_create. */
typedef struct pb_batch pb_batch;
pb_status pb_batch_create(pb_ctx* ctx, const pb_graph* const* gs, int32_t k, const pb_opts* opts, pb_batch** out);
pb_status pb_batch_run(pb_ctx* ctx, pb_batch* batch, int64_t* const* counts, int64_t* const* tips);
pb_status pb_batch_destroy(pb_batch* batch);

/* ---- counting without device allocation ------------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc where they need a
 * count (code running inside another framework's memory pool, paths that must not synchronise
 * the device, callers close to the memory limit): total butterflies of a graph whose four CSR
 * arrays are already in device memory, written to *total (device memory), on `stream` (a
 * cudaStream_t, NULL = legacy default stream).  Nothing is allocated: all scratch lives in one
 * file-scope device array of PB_NOALLOC_SCRATCH_BYTES, reserved on every GPU that loads the
 * library until the process exits.  Limit: max(nv, nu) <= PB_NOALLOC_MAX_SIDE, else PB_ETOOBIG
 * (message in msg when msg_len > 0).  The graph must satisfy pb_graph_upload's contract; it is
 * not validated.  *total must be 8-byte-aligned device memory (else PB_EINVAL).  The first
 * call on a device resolves the array's device address with that device current and keeps it
 * for the life of the process; make that first call before any stream capture, and do not call
 * the entry point on a device after cudaDeviceReset there (the kept address is then stale).
 * Calls share the array:
 * calls that overlap on the GPU (other streams, other host threads) race and give wrong
 * results.  Asynchronous: *total is ready when `stream` reaches this point. */
#define PB_NOALLOC_SCRATCH_BYTES (16u << 20)
#define PB_NOALLOC_MAX_SIDE ((1u << 22) - 64u)
pb_status pb_count_total_noalloc(const pb_csr* dev_graph, void* stream, int64_t* total, char* msg, size_t msg_len);

/* ---- host utilities (no GPU needed) ---------------------------------------------------- */
void pb_csr_free(pb_csr_owned* g);
/* readBipartite (butterfly_utils.h:1008-1058): Ligra "AdjacencyHypergraph" text file. */
pb_status pb_read_adjacency_hypergraph(const char* path, pb_csr_owned* out);
/* Writer for the same format (utils/graphIO.h:752-779 layout). */
pb_status pb_write_adjacency_hypergraph(const char* path, const pb_csr* g);
/* The binary variant written by utils/hyperAdjToBinary.C: <base>.config ("nv mv nh mh") and
 * <base>.vidx / .vadj / .hidx / .hadj (32-bit offsets without the final m, 32-bit ids). */
pb_status pb_read_binary_hypergraph(const char* base, pb_csr_owned* out);
/* KONECT edge list (utils/KONECTtoHyperAdj.C, readKONECT utils/graphIO.h:1033-1100): leading
 * '%' lines skipped, first column V ids, second column U ids (other columns ignored), ids of
 * each side compacted in increasing order, lists sorted, repeated pairs dropped. */
pb_status pb_read_konect(const char* path, pb_csr_owned* out);
/* Sparsification for approximate total counts (-sparseType / -s, -d of BipartiteButterflies.C:
 * 175-193, 333-340), host preprocessing before the GPU count.  PB_SPARSE_EDGE keeps each edge
 * whose hash of (v, u, seed) is 0 mod denom (eSparseBipartite, butterfly_utils.h:790-890);
 * PB_SPARSE_COLOR colours every vertex by a hash of (id, seed) mod denom and keeps the edges
 * whose endpoints share a colour (clrSparseBipartite, :900-996).  Both then drop the vertices
 * left without edges and renumber each side in increasing order (delZeroDeg, :744-786).  The
 * reference's driver uses seed 0.  Release the result with pb_csr_free. */
pb_status pb_sparsify_bipartite(const pb_csr* g, int32_t sparse_type, int64_t denom, int64_t seed,
                                pb_csr_owned* out);
/* The estimate printed for a sparsified graph's total count (BipartiteButterflies.C:213-214):
 * count * denom^3 (colour) or count * denom^4 (edge), computed in double precision and
 * truncated to an integer, as the reference does. */
int64_t pb_sparse_estimate(int64_t sparse_count, int32_t sparse_type, int64_t denom);
pb_status pb_write_binary_hypergraph(const char* base, const pb_csr* g);
/* Host validation of a CSR (same checks as pb_graph_upload). */
pb_status pb_csr_validate(const pb_csr* g, char* msg, size_t msg_len);

/* Seeded generators (SplitMix64 counter RNG).  Each draws edges until m distinct (v,u) pairs
 * exist and returns both adjacency sides sorted. */
pb_status pb_gen_uniform(int64_t nv, int64_t nu, int64_t m, uint64_t seed, pb_csr_owned* out);
/* Bipartite R-MAT on a 2^log_nv x 2^log_nu grid with quadrant probabilities a,b,c,d. */
pb_status pb_gen_rmat(int32_t log_nv, int32_t log_nu, int64_t m, double a, double b, double c, double d,
                      uint64_t seed, pb_csr_owned* out);
/* U side with discrete power-law degrees p(k) ~ k^-alpha on [dmin, dmax] (sum trimmed to m),
 * each U vertex joined to distinct uniform V vertices. */
pb_status pb_gen_powerlaw_u(int64_t nv, int64_t nu, int64_t m, double alpha, int64_t dmax, uint64_t seed,
                            pb_csr_owned* out);
/* Endpoints drawn with Zipf(s) over ids on both sides (s = 0 gives uniform). */
pb_status pb_gen_zipf(int64_t nv, int64_t nu, int64_t m, double s, uint64_t seed, pb_csr_owned* out);
/* Graph g of the 256-graph batch workload (sizes log-uniform; seed 4000+g). */
pb_status pb_gen_batch_member(int32_t g, pb_csr_owned* out);

#ifdef __cplusplus
}
#endif
#endif /* PARBUTTERFLY_B200_H */
