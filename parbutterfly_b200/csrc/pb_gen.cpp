// Seeded synthetic bipartite graph generators (host side).
//
// The reference ships its own generators (utils/randHypergraph.C:44-92,
// utils/zipfHypergraph.C:111-171, utils/rMatGraph.C:31-91) whose builder sorts and dedups
// each adjacency list (utils/graphIO.h:378-420).  These generators are written for the
// benchmark workloads: every one draws (v,u) pairs from a SplitMix64 counter stream until m
// DISTINCT pairs exist ("dedup and refill"), then emits both CSR sides sorted ascending,
// which is the input contract of readBipartite (butterfly_utils.h:1008-1058).
//
// All arithmetic that decides an edge is integer (32-bit fixed-point thresholds), so a
// seed gives the same graph on every x86-64 host.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/parbutterfly_b200.h"

namespace {

// SplitMix64 (Steele, Lea, Flood 2014; constants as published by Vigna).
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  inline uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // Uniform integer in [0, n) by 64x64->128 multiply-shift (Lemire).
  inline uint64_t below(uint64_t n) {
    return (uint64_t)(((unsigned __int128)next() * n) >> 64);
  }
  // Uniform double in [0,1) with 53 random bits.
  inline double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Open-addressing set of 64-bit keys (linear probing).  Keys never equal kEmpty because
// they are v*nu+u < 2^63.
struct KeySet {
  static constexpr uint64_t kEmpty = ~0ull;
  std::vector<uint64_t> slots;
  uint64_t mask = 0;
  int64_t size = 0;
  explicit KeySet(int64_t expected) {
    uint64_t cap = 16;
    while (cap < (uint64_t)expected * 2) cap <<= 1;
    slots.assign(cap, kEmpty);
    mask = cap - 1;
  }
  inline bool insert(uint64_t key) {
    uint64_t h = key * 0x9E3779B97F4A7C15ull;
    uint64_t i = (h ^ (h >> 29)) & mask;
    while (true) {
      uint64_t cur = slots[i];
      if (cur == key) return false;
      if (cur == kEmpty) { slots[i] = key; ++size; return true; }
      i = (i + 1) & mask;
    }
  }
};

// Builds both sorted CSR sides from a set of distinct keys v*nu+u.
pb_status build_csr(int64_t nv, int64_t nu, std::vector<uint64_t>& keys, pb_csr_owned* out) {
  const int64_t m = (int64_t)keys.size();
  if (m > (int64_t)UINT32_MAX || nv > (int64_t)UINT32_MAX || nu > (int64_t)UINT32_MAX) return PB_ETOOBIG;
  std::sort(keys.begin(), keys.end());
  uint32_t* offV = (uint32_t*)malloc(sizeof(uint32_t) * (nv + 1));
  uint32_t* offU = (uint32_t*)malloc(sizeof(uint32_t) * (nu + 1));
  uint32_t* edgV = (uint32_t*)malloc(sizeof(uint32_t) * (m > 0 ? m : 1));
  uint32_t* edgU = (uint32_t*)malloc(sizeof(uint32_t) * (m > 0 ? m : 1));
  if (!offV || !offU || !edgV || !edgU) {
    free(offV); free(offU); free(edgV); free(edgU);
    return PB_ENOMEM;
  }
  std::memset(offV, 0, sizeof(uint32_t) * (nv + 1));
  std::memset(offU, 0, sizeof(uint32_t) * (nu + 1));
  for (int64_t e = 0; e < m; ++e) {
    uint64_t v = keys[e] / (uint64_t)nu, u = keys[e] % (uint64_t)nu;
    offV[v + 1]++;
    offU[u + 1]++;
    edgV[e] = (uint32_t)u;  // keys sorted => lists of V sorted by u
  }
  for (int64_t i = 0; i < nv; ++i) offV[i + 1] += offV[i];
  for (int64_t i = 0; i < nu; ++i) offU[i + 1] += offU[i];
  std::vector<uint32_t> cur(offU, offU + nu);
  for (int64_t e = 0; e < m; ++e) {  // stable scatter in v order => lists of U sorted by v
    uint64_t v = keys[e] / (uint64_t)nu, u = keys[e] % (uint64_t)nu;
    edgU[cur[u]++] = (uint32_t)v;
  }
  out->nv = nv; out->nu = nu; out->m = m;
  out->offsetsV = offV; out->offsetsU = offU; out->edgesV = edgV; out->edgesU = edgU;
  return PB_OK;
}

// Draws pairs from `draw` until m distinct ones exist, then builds the CSR.
template <class Draw>
pb_status draw_distinct(int64_t nv, int64_t nu, int64_t m, Draw draw, pb_csr_owned* out, bool allow_short = false) {
  if (nv <= 0 || nu <= 0 || m < 0) return PB_EINVAL;
  if ((double)m > (double)nv * (double)nu) return PB_EINVAL;
  try {
    KeySet set(m);
    std::vector<uint64_t> keys;
    keys.reserve(m);
    // Bound on draws: guards against a degenerate distribution that cannot reach m.
    const int64_t max_draws = 64 * m + 1000000;
    int64_t draws = 0;
    while ((int64_t)keys.size() < m) {
      if (++draws > max_draws) {
        if (allow_short) break;  // keep the distinct pairs drawn so far
        return PB_EINVAL;
      }
      uint64_t v, u;
      draw(v, u);
      uint64_t key = v * (uint64_t)nu + u;
      if (set.insert(key)) keys.push_back(key);
    }
    return build_csr(nv, nu, keys, out);
  } catch (const std::bad_alloc&) {
    return PB_ENOMEM;
  }
}

inline uint32_t prob_threshold(double p) {
  if (p <= 0) return 0;
  if (p >= 1) return UINT32_MAX;
  return (uint32_t)std::llround(p * 4294967296.0);
}

// Zipf(s) sampler over [0, n): p(k) ~ (k+1)^-s, inverse CDF by binary search.
struct ZipfTable {
  std::vector<double> cdf;
  ZipfTable(int64_t n, double s) : cdf(n) {
    double acc = 0;
    for (int64_t k = 0; k < n; ++k) { acc += std::pow((double)(k + 1), -s); cdf[k] = acc; }
    for (int64_t k = 0; k < n; ++k) cdf[k] /= acc;
    cdf[n - 1] = 1.0;
  }
  inline uint64_t sample(SplitMix64& r) const {
    double x = r.unit();
    return (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
  }
};

}  // namespace

extern "C" {

void pb_csr_free(pb_csr_owned* g) {
  if (!g) return;
  free(g->offsetsV); free(g->offsetsU); free(g->edgesV); free(g->edgesU);
  std::memset(g, 0, sizeof(*g));
}

pb_status pb_gen_uniform(int64_t nv, int64_t nu, int64_t m, uint64_t seed, pb_csr_owned* out) {
  if (!out) return PB_EINVAL;
  SplitMix64 r(seed);
  return draw_distinct(nv, nu, m, [&](uint64_t& v, uint64_t& u) {
    v = r.below((uint64_t)nv);
    u = r.below((uint64_t)nu);
  }, out);
}

pb_status pb_gen_rmat(int32_t log_nv, int32_t log_nu, int64_t m, double a, double b, double c, double d,
                      uint64_t seed, pb_csr_owned* out) {
  if (!out || log_nv < 0 || log_nu < 0 || log_nv > 31 || log_nu > 31) return PB_EINVAL;
  const double tot = a + b + c + d;
  if (!(tot > 0)) return PB_EINVAL;
  a /= tot; b /= tot; c /= tot; d /= tot;
  // Quadrant thresholds: a -> (row 0, col 0), b -> (0,1), c -> (1,0), d -> (1,1).
  const uint32_t ta = prob_threshold(a), tab = prob_threshold(a + b), tabc = prob_threshold(a + b + c);
  // Once one side's bits are used up, the other continues with its marginal.
  const uint32_t t_row1 = prob_threshold(c + d);  // P(row bit = 1)
  const uint32_t t_col1 = prob_threshold(b + d);  // P(col bit = 1)
  const int levels = std::max(log_nv, log_nu);
  SplitMix64 r(seed);
  return draw_distinct((int64_t)1 << log_nv, (int64_t)1 << log_nu, m, [&](uint64_t& v, uint64_t& u) {
    uint64_t row = 0, col = 0, bits = 0;
    int have = 0;
    for (int lvl = 0; lvl < levels; ++lvl) {
      if (have == 0) { bits = r.next(); have = 2; }
      uint32_t x = (uint32_t)bits;
      bits >>= 32;
      --have;
      const bool row_live = lvl < log_nv, col_live = lvl < log_nu;
      uint32_t rb, cb;
      if (row_live && col_live) {
        rb = x >= tab;
        cb = (x >= ta && x < tab) || x >= tabc;
      } else if (row_live) {
        rb = x < t_row1; cb = 0;
      } else {
        rb = 0; cb = x < t_col1;
      }
      if (row_live) row = (row << 1) | rb;
      if (col_live) col = (col << 1) | cb;
    }
    v = row;
    u = col;
  }, out);
}

static pb_status gen_zipf_impl(int64_t nv, int64_t nu, int64_t m, double s, uint64_t seed, pb_csr_owned* out,
                               bool allow_short);

pb_status pb_gen_zipf(int64_t nv, int64_t nu, int64_t m, double s, uint64_t seed, pb_csr_owned* out) {
  return gen_zipf_impl(nv, nu, m, s, seed, out, false);
}

static pb_status gen_zipf_impl(int64_t nv, int64_t nu, int64_t m, double s, uint64_t seed, pb_csr_owned* out,
                               bool allow_short) {
  if (!out || nv <= 0 || nu <= 0) return PB_EINVAL;
  if (s <= 0) return pb_gen_uniform(nv, nu, m, seed, out);
  try {
    ZipfTable zv(nv, s), zu(nu, s);
    SplitMix64 r(seed);
    // Scatter Zipf ranks over ids with a seeded permutation so hubs are not the low ids.
    std::vector<uint32_t> pv(nv), pu(nu);
    for (int64_t i = 0; i < nv; ++i) pv[i] = (uint32_t)i;
    for (int64_t i = 0; i < nu; ++i) pu[i] = (uint32_t)i;
    for (int64_t i = nv - 1; i > 0; --i) std::swap(pv[i], pv[r.below((uint64_t)i + 1)]);
    for (int64_t i = nu - 1; i > 0; --i) std::swap(pu[i], pu[r.below((uint64_t)i + 1)]);
    return draw_distinct(nv, nu, m, [&](uint64_t& v, uint64_t& u) {
      v = pv[zv.sample(r)];
      u = pu[zu.sample(r)];
    }, out, allow_short);
  } catch (const std::bad_alloc&) {
    return PB_ENOMEM;
  }
}

pb_status pb_gen_powerlaw_u(int64_t nv, int64_t nu, int64_t m, double alpha, int64_t dmax, uint64_t seed,
                            pb_csr_owned* out) {
  if (!out || nv <= 0 || nu <= 0 || m < nu || alpha <= 1.0) return PB_EINVAL;
  if (dmax > nv) dmax = nv;
  if ((double)m > (double)nu * (double)dmax) return PB_EINVAL;
  try {
    // Pick dmin so the expected sum of the truncated power law is closest to m.
    auto mean_for = [&](int64_t dmin) {
      double z = 0, s1 = 0;
      for (int64_t k = dmin; k <= dmax; ++k) { double p = std::pow((double)k, -alpha); z += p; s1 += p * k; }
      return s1 / z;
    };
    const double target = (double)m / (double)nu;
    int64_t dmin = 1;
    while (dmin < dmax && mean_for(dmin + 1) <= target) ++dmin;
    // Deterministic quantile degree sequence: deg_k = F^-1((k + 0.5) / nu).
    std::vector<double> cdf;
    cdf.reserve(dmax - dmin + 1);
    double z = 0;
    for (int64_t k = dmin; k <= dmax; ++k) { z += std::pow((double)k, -alpha); cdf.push_back(z); }
    for (auto& x : cdf) x /= z;
    std::vector<int64_t> deg(nu);
    int64_t sum = 0;
    for (int64_t k = 0; k < nu; ++k) {
      double q = ((double)k + 0.5) / (double)nu;
      int64_t d = dmin + (int64_t)(std::lower_bound(cdf.begin(), cdf.end(), q) - cdf.begin());
      deg[k] = std::min<int64_t>(d, dmax);
      sum += deg[k];
    }
    // Trim or pad to exactly m, one unit at a time over the sequence (largest first when
    // trimming, smallest first when padding).
    int64_t k = 0;
    while (sum > m) { int64_t idx = k % nu; if (deg[idx] > 1) { deg[idx]--; sum--; } ++k; }
    k = nu - 1;
    while (sum < m) { int64_t idx = ((k % nu) + nu) % nu; if (deg[idx] < dmax) { deg[idx]++; sum++; } --k; }
    SplitMix64 r(seed);
    // Assign the degree sequence to U ids by a seeded permutation.
    for (int64_t i = nu - 1; i > 0; --i) std::swap(deg[i], deg[r.below((uint64_t)i + 1)]);
    std::vector<uint64_t> keys;
    keys.reserve(m);
    std::vector<uint32_t> mark(nv, 0);
    std::vector<uint32_t> pick;
    uint32_t epoch = 0;
    for (int64_t u = 0; u < nu; ++u) {
      const int64_t d = deg[u];
      ++epoch;
      if (epoch == 0) { std::fill(mark.begin(), mark.end(), 0); epoch = 1; }
      pick.clear();
      if (2 * d <= nv) {
        while ((int64_t)pick.size() < d) {
          uint32_t v = (uint32_t)r.below((uint64_t)nv);
          if (mark[v] != epoch) { mark[v] = epoch; pick.push_back(v); }
        }
      } else {  // dense: choose the complement
        int64_t skip = nv - d;
        int64_t got = 0;
        while (got < skip) {
          uint32_t v = (uint32_t)r.below((uint64_t)nv);
          if (mark[v] != epoch) { mark[v] = epoch; ++got; }
        }
        for (int64_t v = 0; v < nv; ++v) if (mark[v] != epoch) pick.push_back((uint32_t)v);
      }
      for (uint32_t v : pick) keys.push_back((uint64_t)v * (uint64_t)nu + (uint64_t)u);
    }
    return build_csr(nv, nu, keys, out);
  } catch (const std::bad_alloc&) {
    return PB_ENOMEM;
  }
}

pb_status pb_gen_batch_member(int32_t g, pb_csr_owned* out) {
  if (!out || g < 0) return PB_EINVAL;
  SplitMix64 r(4000ull + (uint64_t)g);
  auto log_uniform = [&](double lo, double hi) { return std::exp(std::log(lo) + r.unit() * (std::log(hi) - std::log(lo))); };
  int64_t nu = (int64_t)std::llround(log_uniform(64, 65536));
  int64_t nv = (int64_t)std::llround(log_uniform(64, 65536));
  double factor = log_uniform(4, 64);
  int64_t m = (int64_t)std::llround(factor * (double)std::min(nu, nv));
  m = std::min<int64_t>(m, nu * nv);
  const bool zipf = (r.next() >> 63) != 0;
  uint64_t seed = r.next();
  // A Zipf graph whose heavy ids saturate cannot reach m distinct pairs quickly: cap m at half
  // the grid, and keep the distinct pairs drawn so far if 64 m + 10^6 draws do not reach it.
  if (zipf) m = std::min<int64_t>(m, nu * nv / 2);
  return zipf ? gen_zipf_impl(nv, nu, m, 1.5, seed, out, true) : pb_gen_uniform(nv, nu, m, seed, out);
}

}  // extern "C"
