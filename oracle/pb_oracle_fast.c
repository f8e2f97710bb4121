/*
 * pb_oracle_fast.c — the wing-peeling restatement of pb_oracle.c (pbo_peel_edge), organised to
 * finish on the benchmark's 2^24-edge graph on a multi-core host.
 *
 * TEST INFRASTRUCTURE ONLY (see pb_oracle.c).  Semantics are those of PeelE /
 * PeelEOrigParallel (apps/hyper/butterfly_epeel.h:339-443,519-569) with updateBuckets
 * (apps/hyper/butterfly_putils.h:1027-1115) and 64-bit buckets:
 *   - every round takes the unpeeled edges whose bucket equals the minimum k;
 *   - each butterfly that contains an edge of the round and no edge of an earlier round is
 *     removed once, by its round edge of smallest index; each of its other edges loses 1;
 *   - every touched unpeeled edge moves to bucket max(count, k).
 * What differs from pbo_peel_edge is only how the work is organised, never the result
 * (tests/test_oracle_golden.py checks both on every golden graph):
 *   - the minimum bucket comes from a bucket queue (a window of exact buckets over
 *     [base, base + kWin), lazily filled, rebuilt from the unpeeled edges when it runs dry)
 *     instead of a scan over all edges per round;
 *   - the round's edges are processed by OpenMP threads (counts change by atomic adds);
 *   - each butterfly of a round edge (u, v) is enumerated from the side whose two-hop list is
 *     shorter: u2 in N(v) then v2 in N(u2) probed against N(u), or v2 in N(u) then u2 in N(v2)
 *     probed against N(v); both find the same butterflies.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int64_t nv, nu, m;
  const uint32_t* offV;
  const uint32_t* edgV;
  const uint32_t* offU;
  const uint32_t* edgU;
} pbo_graph;

void pbo_edge_to_idxs(const pbo_graph* g, int32_t use_v, uint32_t* eti);

enum { kWin = 1 << 16 };

typedef struct {
  uint32_t* a;
  int64_t n, cap;
} vec_u32;

static void vpush(vec_u32* v, uint32_t x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 16;
    v->a = (uint32_t*)realloc(v->a, sizeof(uint32_t) * (size_t)v->cap);
  }
  v->a[v->n++] = x;
}

static int nthreads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static int tid(void) {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

/* Removes butterfly {e2, e3, e4} + the round edge from the counts of its other edges. */
static void hit(int64_t* cnt, uint8_t* touched, vec_u32* tl, int64_t e2, int64_t e3, int64_t e4) {
  const int64_t es[3] = {e2, e3, e4};
  for (int i = 0; i < 3; ++i) {
    __atomic_fetch_sub(&cnt[es[i]], 1, __ATOMIC_RELAXED);
    if (!__atomic_exchange_n(&touched[es[i]], 1, __ATOMIC_RELAXED)) vpush(tl, (uint32_t)es[i]);
  }
}

int64_t pbo_peel_edge_fast(const pbo_graph* g, int32_t use_v, const int64_t* ecounts, int64_t* D) {
  const int64_t nC = use_v ? g->nv : g->nu; /* centre side */
  const int64_t nK = use_v ? g->nu : g->nv; /* count side */
  const int64_t m = g->m;
  const uint32_t* offC = use_v ? g->offV : g->offU;
  const uint32_t* offK = use_v ? g->offU : g->offV;
  const uint32_t* edgC = use_v ? g->edgV : g->edgU; /* centre v -> count-side u; position = edge id */
  const uint32_t* edgK = use_v ? g->edgU : g->edgV; /* count-side u -> centre v */
  if (m == 0) return 0;
  uint32_t* eti = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)m); /* count-side position -> edge id */
  pbo_edge_to_idxs(g, use_v, eti);
  uint32_t* center_of = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)m);
  for (int64_t v = 0; v < nC; ++v)
    for (uint32_t e = offC[v]; e < offC[v + 1]; ++e) center_of[e] = (uint32_t)v;
  int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * (size_t)m);
  uint8_t* state = (uint8_t*)calloc((size_t)m, 1); /* 0 unpeeled, 1 in this round, 2 peeled */
  uint8_t* touched = (uint8_t*)calloc((size_t)m, 1);
  for (int64_t e = 0; e < m; ++e) { cnt[e] = ecounts[e]; D[e] = ecounts[e]; }
  const int T = nthreads();
  /* Per-thread probe marks: centre id -> edge id + 1 (walk from v) and count-side id ->
   * edge id + 1 (walk from u); cleared after each edge. */
  int64_t** markC = (int64_t**)malloc(sizeof(int64_t*) * (size_t)T);
  int64_t** markK = (int64_t**)malloc(sizeof(int64_t*) * (size_t)T);
  vec_u32* tl = (vec_u32*)calloc((size_t)T, sizeof(vec_u32));
  for (int t = 0; t < T; ++t) {
    markC[t] = (int64_t*)calloc((size_t)(nC ? nC : 1), sizeof(int64_t));
    markK[t] = (int64_t*)calloc((size_t)(nK ? nK : 1), sizeof(int64_t));
  }
  /* Two-hop list sizes for the choice of side. */
  int64_t* SC = (int64_t*)calloc((size_t)(nC ? nC : 1), sizeof(int64_t));
  int64_t* SK = (int64_t*)calloc((size_t)(nK ? nK : 1), sizeof(int64_t));
  for (int64_t v = 0; v < nC; ++v)
    for (uint32_t p = offC[v]; p < offC[v + 1]; ++p) SC[v] += offK[edgC[p] + 1] - offK[edgC[p]];
  for (int64_t u = 0; u < nK; ++u)
    for (uint32_t p = offK[u]; p < offK[u + 1]; ++p) SK[u] += offC[edgK[p] + 1] - offC[edgK[p]];

  vec_u32* bucket = (vec_u32*)calloc(kWin, sizeof(vec_u32));
  uint32_t* alive = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)m);
  int64_t nalive = m;
  for (int64_t e = 0; e < m; ++e) alive[e] = (uint32_t)e;
  int64_t base = 0, cur = kWin; /* cur == kWin: the window must be rebuilt */
  vec_u32 act = {0, 0, 0};
  int64_t rounds = 0, left = m;

  while (left > 0) {
    /* ---- next round: the smallest bucket with a valid entry ---- */
    act.n = 0;
    int64_t k = -1;
    while (k < 0) {
      if (cur >= kWin) {
        /* Rebuild: compact the unpeeled list, take its minimum, fill the window. */
        int64_t w = 0;
        int64_t mn = INT64_MAX;
        for (int64_t q = 0; q < nalive; ++q) {
          const uint32_t e = alive[q];
          if (state[e] != 0) continue;
          alive[w++] = e;
          if (D[e] < mn) mn = D[e];
        }
        nalive = w;
        for (int64_t b = 0; b < kWin; ++b) bucket[b].n = 0;
        base = mn;
        for (int64_t q = 0; q < nalive; ++q) {
          const uint32_t e = alive[q];
          if (D[e] - base < kWin) vpush(&bucket[D[e] - base], e);
        }
        cur = 0;
      }
      for (; cur < kWin && k < 0; ++cur) {
        vec_u32* b = &bucket[cur];
        for (int64_t q = 0; q < b->n; ++q) {
          const uint32_t e = b->a[q];
          if (state[e] == 0 && D[e] == base + cur) {
            state[e] = 1;
            vpush(&act, e);
          }
        }
        b->n = 0;
        if (act.n) k = base + cur;
      }
      if (k >= 0) --cur; /* the next round may take this bucket again (bucket = max(count, k)) */
    }
    left -= act.n;
    ++rounds;
    /* ---- process the round's edges ---- */
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < act.n; ++a) {
      const int t = tid();
      const int64_t e1 = act.a[a];
      const uint32_t v = center_of[e1], u = edgC[e1];
      if (SC[v] <= SK[u]) {
        /* probe set N(u): centre v2 -> edge (v2, u) */
        int64_t* mk = markC[t];
        for (uint32_t f = offK[u]; f < offK[u + 1]; ++f) {
          const uint32_t eo = eti[f];
          if (state[eo] != 2) mk[edgK[f]] = (int64_t)eo + 1;
        }
        for (uint32_t f2 = offC[v]; f2 < offC[v + 1]; ++f2) {
          const uint32_t u2 = edgC[f2];
          const int64_t e2 = f2; /* (v, u2) */
          if (u2 == u || state[e2] == 2 || (state[e2] == 1 && e2 < e1)) continue;
          for (uint32_t f3 = offK[u2]; f3 < offK[u2 + 1]; ++f3) {
            const uint32_t v2 = edgK[f3];
            if (v2 == v || !mk[v2]) continue;
            const int64_t e3 = eti[f3]; /* (v2, u2) */
            if (state[e3] == 2 || (state[e3] == 1 && e3 < e1)) continue;
            const int64_t e4 = mk[v2] - 1; /* (v2, u) */
            if (state[e4] == 1 && e4 < e1) continue;
            hit(cnt, touched, &tl[t], e2, e3, e4);
          }
        }
        for (uint32_t f = offK[u]; f < offK[u + 1]; ++f) mk[edgK[f]] = 0;
      } else {
        /* probe set N(v): count-side u2 -> edge (v, u2) */
        int64_t* mk = markK[t];
        for (uint32_t f = offC[v]; f < offC[v + 1]; ++f)
          if (state[f] != 2) mk[edgC[f]] = (int64_t)f + 1;
        for (uint32_t f4 = offK[u]; f4 < offK[u + 1]; ++f4) {
          const uint32_t v2 = edgK[f4];
          const int64_t e4 = eti[f4]; /* (v2, u) */
          if (v2 == v || state[e4] == 2 || (state[e4] == 1 && e4 < e1)) continue;
          for (uint32_t f3 = offC[v2]; f3 < offC[v2 + 1]; ++f3) {
            const uint32_t u2 = edgC[f3];
            if (u2 == u || !mk[u2]) continue;
            const int64_t e3 = f3; /* (v2, u2) */
            if (state[e3] == 2 || (state[e3] == 1 && e3 < e1)) continue;
            const int64_t e2 = mk[u2] - 1; /* (v, u2) */
            if (state[e2] == 1 && e2 < e1) continue;
            hit(cnt, touched, &tl[t], e2, e3, e4);
          }
        }
        for (uint32_t f = offC[v]; f < offC[v + 1]; ++f) mk[edgC[f]] = 0;
      }
    }
    for (int64_t a = 0; a < act.n; ++a) state[act.a[a]] = 2;
    /* ---- touched unpeeled edges move to bucket max(count, k) ---- */
    for (int t = 0; t < T; ++t) {
      for (int64_t q = 0; q < tl[t].n; ++q) {
        const uint32_t e = tl[t].a[q];
        touched[e] = 0;
        if (state[e] != 0 || D[e] <= k) continue;
        const int64_t nd = cnt[e] > k ? cnt[e] : k;
        if (nd == D[e]) continue;
        D[e] = nd;
        if (nd - base < kWin) vpush(&bucket[nd - base], e);
      }
      tl[t].n = 0;
    }
  }
  for (int t = 0; t < T; ++t) { free(markC[t]); free(markK[t]); free(tl[t].a); }
  for (int64_t b = 0; b < kWin; ++b) free(bucket[b].a);
  free(markC); free(markK); free(tl); free(bucket); free(alive); free(act.a);
  free(SC); free(SK); free(eti); free(center_of); free(cnt); free(state); free(touched);
  return rounds;
}
