/*
 * pb_oracle.c — CPU restatement of ParButterfly's counting and peeling semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load it.  The
 * product path never calls it and fails loudly when its CUDA library is missing.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here against golden
 * vectors produced by the reference itself (oracle/ref_harness.cpp compiled from the
 * reference sources by oracle/Makefile; fixtures in tests/golden/).
 *
 * What is restated (reference paths are relative to the ParButterfly tree):
 *  - wedge counts per side and the choice of count side: cmpWedgeCounts / wedgeF
 *    (apps/hyper/butterfly_utils.h:1061-1086), including wedgeF's 32-bit product
 *    v_deg*(v_deg-1) (uintE arithmetic, :1066-1067);
 *  - vertex orders: getApproxDegRanks (:275-284), getDegRanks (:294-301),
 *    getApproxCoCoreRanks (:448-503), getCoCoreRanks (:514-559); ties are broken by the
 *    combined id (V ids first, then nv+U ids); the reference's sample sort breaks them
 *    arbitrarily, and counts/tip/wing numbers do not depend on the tie order;
 *  - SIDE is expressed as the order "count side by id, then the other side", which gives
 *    exactly the wedge set of the side algorithms (u2 < i over count-side endpoints,
 *    butterfly_count.h:1335-1397);
 *  - the ranked graph: rankGraph / rankGraphEdges (:579-700) with the tag bit
 *    (rank<<1 | on-count-side) and ascending lists (INVERSE);
 *  - counting: CountWorkEfficientSerial (butterfly_count.h:1402-1497),
 *    CountEWorkEfficientSerial (butterfly_ecount.h:1438-1529),
 *    CountWorkEfficientSerialTotal (butterfly_count_total.h:761-835) and the rank->original
 *    conversions (butterfly_count.h:1600-1608, butterfly_ecount.h:1723-1738);
 *  - countWedgesScan on the ranked graph (butterfly_utils.h:1192-1239) for W_rank;
 *  - edgeToIdxs (butterfly_utils.h:2034-2062);
 *  - tip peeling: Peel / PeelOrigParallel / updateBuckets (butterfly_peel.h:647-711,896-934,
 *    butterfly_putils.h:1027-1115) with 64-bit bucket keys;
 *  - wing peeling: PeelE / PeelEOrigParallel (butterfly_epeel.h:339-443,519-569) with the
 *    same-round tie rule (a butterfly is removed by its active edge of smallest index).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int64_t nv, nu, m;
  const uint32_t* offV;
  const uint32_t* edgV;
  const uint32_t* offU;
  const uint32_t* edgU;
} pbo_graph;

enum { R_SIDE = 0, R_COCORE = 1, R_ACOCORE = 2, R_DEG = 3, R_ADEG = 4 };
enum { P_VERT = 0, P_EDGE = 1, P_TOTAL = 2 };

static uint32_t deg_of(const pbo_graph* g, int64_t x) {
  if (x < g->nv) return g->offV[x + 1] - g->offV[x];
  return g->offU[x - g->nv + 1] - g->offU[x - g->nv];
}

/* floor(log2(d)) + 1 for d > 0, else 0 (butterfly_utils.h:279-280); exact in integers. */
static uint32_t log_key(uint32_t d) {
  uint32_t k = 0;
  while (d) { ++k; d >>= 1; }
  return k;
}

/* cmpWedgeCounts (butterfly_utils.h:1080-1086).  wedgeF computes v_deg*(v_deg-1) in uintE
 * (32-bit unsigned) before dividing by 2 (:1066-1067); the same wraparound is kept so the
 * count side matches the reference for every input. */
int64_t pbo_cmp_wedge_counts(const pbo_graph* g, int32_t* use_v, int64_t* wv_out, int64_t* wu_out) {
  int64_t wv = 0, wu = 0;
  for (int64_t i = 0; i < g->nv; ++i) {
    uint32_t d = g->offV[i + 1] - g->offV[i];
    wv += (int64_t)((uint32_t)(d * (d - 1u)) / 2u);
  }
  for (int64_t i = 0; i < g->nu; ++i) {
    uint32_t d = g->offU[i + 1] - g->offU[i];
    wu += (int64_t)((uint32_t)(d * (d - 1u)) / 2u);
  }
  if (wv_out) *wv_out = wv;
  if (wu_out) *wu_out = wu;
  *use_v = wv <= wu;
  return wv <= wu ? wv : wu;
}

/* Neighbours of combined id x as combined ids. */
static void nbrs(const pbo_graph* g, int64_t x, const uint32_t** p, uint32_t* d, int64_t* shift) {
  if (x < g->nv) { *p = g->edgV + g->offV[x]; *d = g->offV[x + 1] - g->offV[x]; *shift = g->nv; }
  else { *p = g->edgU + g->offU[x - g->nv]; *d = g->offU[x - g->nv + 1] - g->offU[x - g->nv]; *shift = 0; }
}

/* Co-core orders: getCoCoreRanks (butterfly_utils.h:514-559) when approx == 0 and
 * getApproxCoCoreRanks (:448-503) when approx == 1.  Buckets are processed in decreasing
 * order; every vertex of the current bucket k is finished together, and each unfinished
 * neighbour with key < k loses one degree per finished neighbour; its key becomes
 * min(new key, k).  The final key orders the vertices (larger first). */
static void cocore_keys(const pbo_graph* g, int approx, uint32_t* key) {
  const int64_t n = g->nv + g->nu;
  uint32_t* dact = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* removed = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
  char* done = (char*)calloc(n ? n : 1, 1);
  int64_t* act = (int64_t*)malloc(sizeof(int64_t) * (n ? n : 1));
  for (int64_t x = 0; x < n; ++x) {
    dact[x] = deg_of(g, x);
    key[x] = approx ? log_key(dact[x]) : dact[x];
  }
  int64_t finished = 0;
  while (finished < n) {
    uint32_t k = 0;
    int first = 1;
    for (int64_t x = 0; x < n; ++x) if (!done[x] && (first || key[x] > k)) { k = key[x]; first = 0; }
    int64_t na = 0;
    for (int64_t x = 0; x < n; ++x) if (!done[x] && key[x] == k) act[na++] = x;
    for (int64_t a = 0; a < na; ++a) done[act[a]] = 1;
    finished += na;
    for (int64_t a = 0; a < na; ++a) {
      const uint32_t* p; uint32_t d; int64_t sh;
      nbrs(g, act[a], &p, &d, &sh);
      for (uint32_t j = 0; j < d; ++j) removed[p[j] + sh]++;
    }
    for (int64_t a = 0; a < na; ++a) {
      const uint32_t* p; uint32_t d; int64_t sh;
      nbrs(g, act[a], &p, &d, &sh);
      for (uint32_t j = 0; j < d; ++j) {
        int64_t y = p[j] + sh;
        if (!removed[y]) continue;
        if (key[y] < k) {
          dact[y] -= removed[y];
          uint32_t nk = approx ? log_key(dact[y]) : dact[y];
          key[y] = nk < k ? nk : k;
        }
        removed[y] = 0;
      }
    }
  }
  free(dact); free(removed); free(done); free(act);
}

/* order[r] = combined id of rank r; rank[x] = rank of combined id x. */
void pbo_vertex_order(const pbo_graph* g, int32_t rank_type, int32_t use_v, uint32_t* order, uint32_t* rank) {
  const int64_t n = g->nv + g->nu;
  uint32_t* key = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  if (rank_type == R_SIDE) {
    /* count side first (by id), then the other side */
    for (int64_t x = 0; x < n; ++x) {
      int on_count = use_v ? (x >= g->nv) : (x < g->nv);
      key[x] = on_count ? 1 : 0;
    }
  } else if (rank_type == R_DEG) {
    for (int64_t x = 0; x < n; ++x) key[x] = deg_of(g, x);
  } else if (rank_type == R_ADEG) {
    for (int64_t x = 0; x < n; ++x) key[x] = log_key(deg_of(g, x));
  } else {
    cocore_keys(g, rank_type == R_ACOCORE, key);
  }
  /* stable counting sort by key descending */
  uint32_t kmax = 0;
  for (int64_t x = 0; x < n; ++x) if (key[x] > kmax) kmax = key[x];
  int64_t* cnt = (int64_t*)calloc((size_t)kmax + 2, sizeof(int64_t));
  for (int64_t x = 0; x < n; ++x) cnt[kmax - key[x] + 1]++;
  for (uint32_t k = 0; k <= kmax; ++k) cnt[k + 1] += cnt[k];
  if (rank_type == R_SIDE && use_v) {
    /* count side is U: ids nv.. come first; within a class keep id order */
  }
  for (int64_t x = 0; x < n; ++x) {
    int64_t r = cnt[kmax - key[x]]++;
    order[r] = (uint32_t)x;
    rank[x] = (uint32_t)r;
  }
  free(cnt);
  free(key);
}

typedef struct {
  int64_t n;
  uint32_t* off;  /* n+1 */
  uint32_t* adj;  /* 2m tagged ranks */
  uint32_t* eout; /* 2m output edge index (EDGE) */
} pbo_ranked;

static int cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : x > y;
}

/* eti (edgeToIdxs, butterfly_utils.h:2034-2062): for the orientation chosen by use_v,
 * maps an index into the count-side lists to the index of the same edge in the other
 * side's lists (binary search for i in N(v)). */
void pbo_edge_to_idxs(const pbo_graph* g, int32_t use_v, uint32_t* eti) {
  const int64_t nu = use_v ? g->nu : g->nv;
  const uint32_t* offsetsV = use_v ? g->offV : g->offU;
  const uint32_t* offsetsU = use_v ? g->offU : g->offV;
  const uint32_t* edgesV = use_v ? g->edgV : g->edgU;
  const uint32_t* edgesU = use_v ? g->edgU : g->edgV;
  for (int64_t i = 0; i < nu; ++i) {
    for (uint32_t e = offsetsU[i]; e < offsetsU[i + 1]; ++e) {
      uint32_t v = edgesU[e];
      uint32_t lo = offsetsV[v], hi = offsetsV[v + 1];
      while (lo < hi) { uint32_t mid = lo + (hi - lo) / 2; if (edgesV[mid] < (uint32_t)i) lo = mid + 1; else hi = mid; }
      eti[e] = lo;
    }
  }
}

/* rankGraph / rankGraphEdges (butterfly_utils.h:579-700).  eout maps each ranked slot to the
 * output edge index of CountERank's conversion (butterfly_ecount.h:1728-1738): slots whose
 * neighbour is on the count side index the center side's lists directly; the others go
 * through eti. */
static pbo_ranked build_ranked(const pbo_graph* g, int32_t use_v, const uint32_t* order, const uint32_t* rank,
                               int want_eout) {
  pbo_ranked R;
  const int64_t n = g->nv + g->nu;
  R.n = n;
  R.off = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  R.adj = (uint32_t*)malloc(sizeof(uint32_t) * (2 * g->m + 1));
  R.eout = want_eout ? (uint32_t*)malloc(sizeof(uint32_t) * (2 * g->m + 1)) : NULL;
  uint32_t* eti = NULL;
  if (want_eout) {
    eti = (uint32_t*)malloc(sizeof(uint32_t) * (g->m + 1));
    pbo_edge_to_idxs(g, use_v, eti);
  }
  R.off[0] = 0;
  for (int64_t r = 0; r < n; ++r) R.off[r + 1] = R.off[r] + deg_of(g, order[r]);
  uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (g->m + 1));
  for (int64_t r = 0; r < n; ++r) {
    int64_t x = order[r];
    int x_is_v = x < g->nv;
    const uint32_t* p; uint32_t d; int64_t sh;
    nbrs(g, x, &p, &d, &sh);
    uint32_t base = x_is_v ? g->offV[x] : g->offU[x - g->nv];
    for (uint32_t j = 0; j < d; ++j) {
      int64_t y = p[j] + sh;
      int y_on_count = use_v ? (y >= g->nv) : (y < g->nv);
      uint32_t t = (rank[y] << 1) | (uint32_t)y_on_count;
      uint32_t e = base + j; /* index into x's side lists */
      uint32_t eo = 0;
      if (want_eout) eo = y_on_count ? e : eti[e];
      tmp[j] = ((uint64_t)t << 32) | eo;
    }
    qsort(tmp, d, sizeof(uint64_t), cmp_u64);
    for (uint32_t j = 0; j < d; ++j) {
      R.adj[R.off[r] + j] = (uint32_t)(tmp[j] >> 32);
      if (want_eout) R.eout[R.off[r] + j] = (uint32_t)tmp[j];
    }
  }
  free(tmp);
  free(eti);
  return R;
}

static void free_ranked(pbo_ranked* R) { free(R->off); free(R->adj); free(R->eout); }

/* countWedgesScan total on the ranked graph (butterfly_utils.h:1192-1239, INVERSE): the
 * number of (i, v, u2) with u2 < min(i, v). */
static int64_t ranked_wedges(const pbo_ranked* R) {
  int64_t w = 0;
  for (int64_t i = 0; i < R->n; ++i)
    for (uint32_t j = R->off[i]; j < R->off[i + 1]; ++j) {
      uint32_t v = R->adj[j] >> 1;
      uint32_t lim = (uint32_t)i < v ? (uint32_t)i : v;
      for (uint32_t k = R->off[v]; k < R->off[v + 1] && (R->adj[k] >> 1) < lim; ++k) ++w;
    }
  return w;
}

/* The serial work-efficient count over the ranked graph.  per = VERT: rank-indexed vertex
 * counts (CountWorkEfficientSerial, butterfly_count.h:1402-1497): endpoints credited with
 * C(w,2) when tagged, centres with w-1 per wedge when tagged.  per = EDGE: slot counts,
 * w-1 to (i,v) and (v,u2) (CountEWorkEfficientSerial, butterfly_ecount.h:1438-1529).
 * per = TOTAL: sum of C(w,2) over all endpoint pairs (butterfly_count_total.h:761-835). */
static int64_t ranked_count(const pbo_ranked* R, int per, int64_t* rc) {
  const int64_t n = R->n;
  uint32_t* w = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
  uint32_t* used = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) {
    int64_t nused = 0;
    for (uint32_t j = R->off[i]; j < R->off[i + 1]; ++j) {
      uint32_t v = R->adj[j] >> 1;
      uint32_t lim = (uint32_t)i < v ? (uint32_t)i : v;
      for (uint32_t k = R->off[v]; k < R->off[v + 1] && (R->adj[k] >> 1) < lim; ++k) {
        uint32_t u2 = R->adj[k] >> 1;
        if (w[u2]++ == 0) used[nused++] = R->adj[k];
      }
    }
    if (per == P_VERT || per == P_EDGE) {
      for (uint32_t j = R->off[i]; j < R->off[i + 1]; ++j) {
        uint32_t vt = R->adj[j], v = vt >> 1;
        uint32_t lim = (uint32_t)i < v ? (uint32_t)i : v;
        for (uint32_t k = R->off[v]; k < R->off[v + 1] && (R->adj[k] >> 1) < lim; ++k) {
          uint32_t c = w[R->adj[k] >> 1];
          if (c <= 1) continue;
          if (per == P_VERT) { if (vt & 1u) rc[v] += (int64_t)(c - 1); }
          else { rc[j] += (int64_t)(c - 1); rc[k] += (int64_t)(c - 1); }
        }
      }
    }
    for (int64_t t = 0; t < nused; ++t) {
      uint32_t u2t = used[t], u2 = u2t >> 1;
      int64_t c = w[u2];
      int64_t b = c * (c - 1) / 2;
      total += b;
      if (per == P_VERT && (u2t & 1u)) { rc[i] += b; rc[u2] += b; }
      w[u2] = 0;
    }
  }
  free(w);
  free(used);
  return total;
}

/* Count / CountE / CountTotal with the chosen order.  out: VERT -> nCount counts by original
 * id; EDGE -> m counts in the reference's edge order; TOTAL -> out[0].  Returns W_rank. */
int64_t pbo_count(const pbo_graph* g, int32_t rank_type, int32_t per, int32_t use_v, int64_t* out) {
  const int64_t n = g->nv + g->nu;
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* rank = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  pbo_vertex_order(g, rank_type, use_v, order, rank);
  pbo_ranked R = build_ranked(g, use_v, order, rank, per == P_EDGE);
  int64_t wr = ranked_wedges(&R);
  if (per == P_TOTAL) {
    out[0] = ranked_count(&R, P_TOTAL, NULL);
  } else if (per == P_VERT) {
    int64_t* rc = (int64_t*)calloc(n ? n : 1, sizeof(int64_t));
    ranked_count(&R, P_VERT, rc);
    /* butterfly_count.h:1600-1608: out[i] = rank_butterflies[rank_converter[i]] */
    const int64_t nc = use_v ? g->nu : g->nv;
    const int64_t base = use_v ? g->nv : 0;
    for (int64_t i = 0; i < nc; ++i) out[i] = rc[rank[base + i]];
    free(rc);
  } else {
    int64_t* rc = (int64_t*)calloc(2 * g->m + 1, sizeof(int64_t));
    ranked_count(&R, P_EDGE, rc);
    memset(out, 0, sizeof(int64_t) * (size_t)g->m);
    for (int64_t s = 0; s < 2 * g->m; ++s) out[R.eout[s]] += rc[s];
    free(rc);
  }
  free_ranked(&R);
  free(order);
  free(rank);
  return wr;
}

/* Tip decomposition (Peel, butterfly_peel.h:896-934, with PeelOrigParallel :647-711 and
 * updateBuckets, butterfly_putils.h:1027-1115).  Each round takes every unpeeled vertex whose
 * bucket equals the current minimum k; for each such u and each two-hop neighbour u2 != u,
 * the shared butterflies C(w(u,u2),2) leave u2's count; every touched u2 with bucket > k
 * moves to max(count, k).  Buckets are 64-bit (the reference squeezes them to 32 bits,
 * ligra/bucket.h:15-16, which is exact only below 2^32-1).  Returns the number of rounds. */
int64_t pbo_peel_vert(const pbo_graph* g, int32_t use_v, const int64_t* counts, int64_t* D) {
  const int64_t nu = use_v ? g->nu : g->nv;
  const uint32_t* offsetsV = use_v ? g->offV : g->offU;
  const uint32_t* offsetsU = use_v ? g->offU : g->offV;
  const uint32_t* edgesV = use_v ? g->edgV : g->edgU;
  const uint32_t* edgesU = use_v ? g->edgU : g->edgV;
  int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * (nu ? nu : 1));
  char* peeled = (char*)calloc(nu ? nu : 1, 1);
  char* touched = (char*)calloc(nu ? nu : 1, 1);
  uint32_t* w = (uint32_t*)calloc(nu ? nu : 1, sizeof(uint32_t));
  uint32_t* used = (uint32_t*)malloc(sizeof(uint32_t) * (nu ? nu : 1));
  int64_t* act = (int64_t*)malloc(sizeof(int64_t) * (nu ? nu : 1));
  for (int64_t i = 0; i < nu; ++i) { cnt[i] = counts[i]; D[i] = counts[i]; }
  int64_t left = nu, rounds = 0;
  while (left > 0) {
    int64_t k = 0;
    int first = 1;
    for (int64_t i = 0; i < nu; ++i) if (!peeled[i] && (first || D[i] < k)) { k = D[i]; first = 0; }
    int64_t na = 0;
    for (int64_t i = 0; i < nu; ++i) if (!peeled[i] && D[i] == k) act[na++] = i;
    for (int64_t a = 0; a < na; ++a) peeled[act[a]] = 1;
    left -= na;
    ++rounds;
    for (int64_t a = 0; a < na; ++a) {
      uint32_t u = (uint32_t)act[a];
      int64_t nused = 0;
      for (uint32_t e = offsetsU[u]; e < offsetsU[u + 1]; ++e) {
        uint32_t v = edgesU[e];
        for (uint32_t f = offsetsV[v]; f < offsetsV[v + 1]; ++f) {
          uint32_t u2 = edgesV[f];
          if (u2 == u) continue;
          cnt[u2] -= (int64_t)w[u2];
          if (w[u2]++ == 0) { used[nused++] = u2; touched[u2] = 1; }
        }
      }
      for (int64_t t = 0; t < nused; ++t) w[used[t]] = 0;
    }
    for (int64_t i = 0; i < nu; ++i) {
      if (!touched[i]) continue;
      touched[i] = 0;
      if (!peeled[i] && D[i] > k) D[i] = cnt[i] > k ? cnt[i] : k;
    }
  }
  free(cnt); free(peeled); free(touched); free(w); free(used); free(act);
  return rounds;
}

/* Wing decomposition (PeelE, butterfly_epeel.h:519-569, with PeelEOrigParallel :339-443).
 * Edges are indexed in the output order of CountE (the center side's lists, i.e. edgesV
 * when use_v).  Each round takes every unpeeled edge whose bucket equals the minimum k; each
 * butterfly that contains an active edge and no edge peeled in an earlier round is removed
 * once, by its active edge of smallest index, and each of its other edges loses one.
 * Touched edges with bucket > k move to max(count, k).  Returns the number of rounds. */
int64_t pbo_peel_edge(const pbo_graph* g, int32_t use_v, const int64_t* ecounts, int64_t* D) {
  const int64_t nv = use_v ? g->nv : g->nu;  /* center side */
  const int64_t nu = use_v ? g->nu : g->nv;  /* count side */
  const int64_t m = g->m;
  const uint32_t* offsetsV = use_v ? g->offV : g->offU;
  const uint32_t* offsetsU = use_v ? g->offU : g->offV;
  const uint32_t* edgesV = use_v ? g->edgV : g->edgU;
  const uint32_t* edgesU = use_v ? g->edgU : g->edgV;
  uint32_t* eti = (uint32_t*)malloc(sizeof(uint32_t) * (m + 1));
  pbo_edge_to_idxs(g, use_v, eti);          /* count-side list index -> output index */
  uint32_t* center_of = (uint32_t*)malloc(sizeof(uint32_t) * (m + 1));
  for (int64_t v = 0; v < nv; ++v)
    for (uint32_t e = offsetsV[v]; e < offsetsV[v + 1]; ++e) center_of[e] = (uint32_t)v;
  int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * (m + 1));
  char* state = (char*)calloc(m + 1, 1);   /* 0 live, 1 active this round, 2 peeled */
  char* touched = (char*)calloc(m + 1, 1);
  int64_t* act = (int64_t*)malloc(sizeof(int64_t) * (m + 1));
  int64_t* mark = (int64_t*)malloc(sizeof(int64_t) * (nv ? nv : 1)); /* center -> output idx of (u,center) + 1 */
  for (int64_t v = 0; v < nv; ++v) mark[v] = 0;
  for (int64_t e = 0; e < m; ++e) { cnt[e] = ecounts[e]; D[e] = ecounts[e]; }
  int64_t left = m, rounds = 0;
  (void)nu;
  while (left > 0) {
    int64_t k = 0;
    int first = 1;
    for (int64_t e = 0; e < m; ++e) if (state[e] == 0 && (first || D[e] < k)) { k = D[e]; first = 0; }
    int64_t na = 0;
    for (int64_t e = 0; e < m; ++e) if (state[e] == 0 && D[e] == k) { act[na++] = e; state[e] = 1; }
    left -= na;
    ++rounds;
    for (int64_t a = 0; a < na; ++a) {
      const int64_t e1 = act[a];
      const uint32_t v = center_of[e1], u = edgesV[e1];
      for (uint32_t f = offsetsU[u]; f < offsetsU[u + 1]; ++f) {
        uint32_t eo = eti[f];
        if (state[eo] != 2) mark[edgesU[f]] = (int64_t)eo + 1;
      }
      for (uint32_t f2 = offsetsV[v]; f2 < offsetsV[v + 1]; ++f2) {
        const uint32_t u2 = edgesV[f2];
        const int64_t e2 = f2;                 /* (v,u2) */
        if (u2 == u || state[e2] == 2) continue;
        if (state[e2] == 1 && e2 < e1) continue;
        for (uint32_t f3 = offsetsU[u2]; f3 < offsetsU[u2 + 1]; ++f3) {
          const uint32_t v2 = edgesU[f3];
          const int64_t e3 = eti[f3];           /* (v2,u2) */
          if (v2 == v || state[e3] == 2) continue;
          if (state[e3] == 1 && e3 < e1) continue;
          if (!mark[v2]) continue;
          const int64_t e4 = mark[v2] - 1;      /* (v2,u) */
          if (state[e4] == 1 && e4 < e1) continue;
          cnt[e2] -= 1; cnt[e3] -= 1; cnt[e4] -= 1;
          touched[e2] = touched[e3] = touched[e4] = 1;
        }
      }
      for (uint32_t f = offsetsU[u]; f < offsetsU[u + 1]; ++f) mark[edgesU[f]] = 0;
    }
    for (int64_t a = 0; a < na; ++a) state[act[a]] = 2;
    for (int64_t e = 0; e < m; ++e) {
      if (!touched[e]) continue;
      touched[e] = 0;
      if (state[e] == 0 && D[e] > k) D[e] = cnt[e] > k ? cnt[e] : k;
    }
  }
  free(eti); free(center_of); free(cnt); free(state); free(touched); free(act); free(mark);
  return rounds;
}

/* W_side of a ranking by side = countWedgesScan(GA, use_v, half=true) total
 * (butterfly_utils.h:1254-1304); exposed for the wedge-count checks. */
int64_t pbo_ranked_wedges(const pbo_graph* g, int32_t rank_type, int32_t use_v) {
  const int64_t n = g->nv + g->nu;
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* rank = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  pbo_vertex_order(g, rank_type, use_v, order, rank);
  pbo_ranked R = build_ranked(g, use_v, order, rank, 0);
  int64_t w = ranked_wedges(&R);
  free_ranked(&R);
  free(order);
  free(rank);
  return w;
}
