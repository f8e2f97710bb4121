// Host-side input/output for the Ligra AdjacencyHypergraph format and CSR validation.
//
// Format (readBipartite, butterfly_utils.h:1008-1058; writer layout utils/graphIO.h:752-779):
//   AdjacencyHypergraph
//   nv  mv  nu  mu
//   offsetsV[0..nv)   edgesV[0..mv)   offsetsU[0..nu)   edgesU[0..mu)
// whitespace separated.  The reference aborts with "Bad input file" when the header word is
// wrong, the token count is not nv+mv+nu+mu+5, or mv != mu (:1013-1027), and exits when an
// edge id is out of range (:1039-1051).  Here each of those is a PB_EINVAL/PB_EIO status.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/parbutterfly_b200.h"

namespace {

struct Tokenizer {
  const char* p;
  const char* end;
  bool next_word(const char*& s, size_t& len) {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    if (p >= end) return false;
    s = p;
    while (p < end && !(*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    len = (size_t)(p - s);
    return true;
  }
  bool next_u64(uint64_t& x) {
    const char* s;
    size_t len;
    if (!next_word(s, len)) return false;
    uint64_t v = 0;
    for (size_t i = 0; i < len; ++i) {
      unsigned c = (unsigned)(s[i] - '0');
      if (c > 9) return false;
      v = v * 10 + c;
    }
    x = v;
    return true;
  }
};

pb_status fill_msg(char* msg, size_t msg_len, pb_status st, const std::string& s) {
  if (msg && msg_len) {
    std::snprintf(msg, msg_len, "%s", s.c_str());
  }
  return st;
}

// Checks one side: offsets monotone, ends at m, each list strictly ascending, ids < other_n.
pb_status check_side(const uint32_t* off, const uint32_t* edg, int64_t n, int64_t m, int64_t other_n,
                     const char* side, char* msg, size_t msg_len) {
  if (off[0] != 0) return fill_msg(msg, msg_len, PB_EINVAL, std::string("offsets") + side + "[0] != 0");
  if ((int64_t)off[n] != m) return fill_msg(msg, msg_len, PB_EINVAL, std::string("offsets") + side + "[n] != m");
  for (int64_t i = 0; i < n; ++i) {
    if (off[i + 1] < off[i])
      return fill_msg(msg, msg_len, PB_EINVAL, std::string("offsets") + side + " not monotone at " + std::to_string(i));
    for (uint32_t e = off[i]; e < off[i + 1]; ++e) {
      if ((int64_t)edg[e] >= other_n)
        return fill_msg(msg, msg_len, PB_EINVAL,
                        std::string("edges") + side + " out of range: id " + std::to_string(edg[e]) + " at " + std::to_string(e));
      if (e > off[i] && edg[e] <= edg[e - 1])
        return fill_msg(msg, msg_len, PB_EINVAL,
                        std::string("edges") + side + " list of vertex " + std::to_string(i) + " not strictly ascending");
    }
  }
  return PB_OK;
}

}  // namespace

extern "C" {

pb_status pb_csr_validate(const pb_csr* g, char* msg, size_t msg_len) {
  if (!g) return fill_msg(msg, msg_len, PB_EINVAL, "null graph");
  if (g->nv < 0 || g->nu < 0 || g->m < 0) return fill_msg(msg, msg_len, PB_EINVAL, "negative size");
  if (g->nv > (int64_t)UINT32_MAX / 2 || g->nu > (int64_t)UINT32_MAX / 2 || g->nv + g->nu >= (int64_t)(1u << 31))
    return fill_msg(msg, msg_len, PB_ETOOBIG, "nv + nu must stay below 2^31 (ranked ids carry a tag bit)");
  if (2 * g->m > (int64_t)UINT32_MAX) return fill_msg(msg, msg_len, PB_ETOOBIG, "2*m must fit 32-bit offsets");
  if (!g->offsetsV || !g->offsetsU || (g->m > 0 && (!g->edgesV || !g->edgesU)))
    return fill_msg(msg, msg_len, PB_EINVAL, "null array");
  pb_status st = check_side(g->offsetsV, g->edgesV, g->nv, g->m, g->nu, "V", msg, msg_len);
  if (st != PB_OK) return st;
  st = check_side(g->offsetsU, g->edgesU, g->nu, g->m, g->nv, "U", msg, msg_len);
  if (st != PB_OK) return st;
  // Both sides must describe the same edge set: per-vertex degree agreement is implied by
  // the transpose check below (count of each (v,u) in V lists equals that in U lists).
  std::vector<uint32_t> cur(g->offsetsU, g->offsetsU + g->nu);
  for (int64_t v = 0; v < g->nv; ++v) {
    for (uint32_t e = g->offsetsV[v]; e < g->offsetsV[v + 1]; ++e) {
      uint32_t u = g->edgesV[e];
      if (cur[u] >= g->offsetsU[u + 1] || g->edgesU[cur[u]] != (uint32_t)v)
        return fill_msg(msg, msg_len, PB_EINVAL, "edgesV and edgesU describe different edge sets");
      cur[u]++;
    }
  }
  return fill_msg(msg, msg_len, PB_OK, "");
}

pb_status pb_read_adjacency_hypergraph(const char* path, pb_csr_owned* out) {
  if (!path || !out) return PB_EINVAL;
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return PB_EIO;
  std::vector<char> buf;
  if (std::fseek(f, 0, SEEK_END) != 0) { std::fclose(f); return PB_EIO; }
  long size = std::ftell(f);
  if (size < 0) { std::fclose(f); return PB_EIO; }
  std::rewind(f);
  buf.resize((size_t)size);
  if (size > 0 && std::fread(buf.data(), 1, (size_t)size, f) != (size_t)size) { std::fclose(f); return PB_EIO; }
  std::fclose(f);
  Tokenizer t{buf.data(), buf.data() + buf.size()};
  const char* w;
  size_t len;
  if (!t.next_word(w, len) || std::string(w, len) != "AdjacencyHypergraph") return PB_EINVAL;
  uint64_t nv, mv, nu, mu;
  if (!t.next_u64(nv) || !t.next_u64(mv) || !t.next_u64(nu) || !t.next_u64(mu)) return PB_EINVAL;
  if (mv != mu) return PB_EINVAL;
  if (nv >= (1ull << 31) || nu >= (1ull << 31) || mv >= (1ull << 32)) return PB_ETOOBIG;
  pb_csr_owned g;
  g.nv = (int64_t)nv; g.nu = (int64_t)nu; g.m = (int64_t)mv;
  g.offsetsV = (uint32_t*)malloc(sizeof(uint32_t) * (nv + 1));
  g.offsetsU = (uint32_t*)malloc(sizeof(uint32_t) * (nu + 1));
  g.edgesV = (uint32_t*)malloc(sizeof(uint32_t) * (mv ? mv : 1));
  g.edgesU = (uint32_t*)malloc(sizeof(uint32_t) * (mu ? mu : 1));
  if (!g.offsetsV || !g.offsetsU || !g.edgesV || !g.edgesU) { pb_csr_free(&g); return PB_ENOMEM; }
  auto read_arr = [&](uint32_t* a, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
      uint64_t x;
      if (!t.next_u64(x) || x > UINT32_MAX) return false;
      a[i] = (uint32_t)x;
    }
    return true;
  };
  if (!read_arr(g.offsetsV, nv) || !read_arr(g.edgesV, mv) || !read_arr(g.offsetsU, nu) || !read_arr(g.edgesU, mu)) {
    pb_csr_free(&g);
    return PB_EINVAL;
  }
  uint64_t extra;
  if (t.next_u64(extra)) { pb_csr_free(&g); return PB_EINVAL; }  // token count mismatch
  g.offsetsV[nv] = (uint32_t)mv;
  g.offsetsU[nu] = (uint32_t)mu;
  for (uint64_t i = 0; i < mv; ++i) if (g.edgesV[i] >= nu) { pb_csr_free(&g); return PB_EINVAL; }
  for (uint64_t i = 0; i < mu; ++i) if (g.edgesU[i] >= nv) { pb_csr_free(&g); return PB_EINVAL; }
  *out = g;
  return PB_OK;
}

pb_status pb_write_adjacency_hypergraph(const char* path, const pb_csr* g) {
  if (!path || !g) return PB_EINVAL;
  FILE* f = std::fopen(path, "wb");
  if (!f) return PB_EIO;
  std::fprintf(f, "AdjacencyHypergraph\n%lld\n%lld\n%lld\n%lld\n", (long long)g->nv, (long long)g->m,
               (long long)g->nu, (long long)g->m);
  for (int64_t i = 0; i < g->nv; ++i) std::fprintf(f, "%u\n", g->offsetsV[i]);
  for (int64_t i = 0; i < g->m; ++i) std::fprintf(f, "%u\n", g->edgesV[i]);
  for (int64_t i = 0; i < g->nu; ++i) std::fprintf(f, "%u\n", g->offsetsU[i]);
  for (int64_t i = 0; i < g->m; ++i) std::fprintf(f, "%u\n", g->edgesU[i]);
  return std::fclose(f) == 0 ? PB_OK : PB_EIO;
}


// hyperAdjToBinary's output (utils/hyperAdjToBinary.C): <base>.config holds "nv mv nh mh" as
// text; <base>.vidx / .vadj / .hidx / .hadj hold offsetsV[nv], edgesV[mv], offsetsH[nh],
// edgesH[mh] as raw 32-bit words (uintT / uintE of the default build).
pb_status pb_read_binary_hypergraph(const char* base, pb_csr_owned* out) {
  if (!base || !out) return PB_EINVAL;
  std::memset(out, 0, sizeof(*out));
  const std::string b(base);
  FILE* cf = std::fopen((b + ".config").c_str(), "r");
  if (!cf) return PB_EIO;
  unsigned long long nv = 0, mv = 0, nh = 0, mh = 0;
  const int got = std::fscanf(cf, "%llu %llu %llu %llu", &nv, &mv, &nh, &mh);
  std::fclose(cf);
  if (got != 4 || mv != mh) return PB_EIO;
  if (nv + nh >= (1ull << 31) || 2 * mv > 0xFFFFFFFFull) return PB_ETOOBIG;
  auto read_words = [&](const char* ext, uint32_t* dst, unsigned long long n) -> bool {
    FILE* f = std::fopen((b + ext).c_str(), "rb");
    if (!f) return false;
    const size_t r = n ? std::fread(dst, sizeof(uint32_t), (size_t)n, f) : 0;
    std::fclose(f);
    return r == (size_t)n;
  };
  out->nv = (int64_t)nv;
  out->nu = (int64_t)nh;
  out->m = (int64_t)mv;
  out->offsetsV = (uint32_t*)std::malloc(sizeof(uint32_t) * (nv + 1));
  out->offsetsU = (uint32_t*)std::malloc(sizeof(uint32_t) * (nh + 1));
  out->edgesV = (uint32_t*)std::malloc(sizeof(uint32_t) * (mv ? mv : 1));
  out->edgesU = (uint32_t*)std::malloc(sizeof(uint32_t) * (mv ? mv : 1));
  if (!out->offsetsV || !out->offsetsU || !out->edgesV || !out->edgesU) {
    pb_csr_free(out);
    return PB_ENOMEM;
  }
  if (!read_words(".vidx", out->offsetsV, nv) || !read_words(".vadj", out->edgesV, mv) ||
      !read_words(".hidx", out->offsetsU, nh) || !read_words(".hadj", out->edgesU, mv)) {
    pb_csr_free(out);
    return PB_EIO;
  }
  out->offsetsV[nv] = (uint32_t)mv;
  out->offsetsU[nh] = (uint32_t)mv;
  return PB_OK;
}

// Writes the same five files.
pb_status pb_write_binary_hypergraph(const char* base, const pb_csr* g) {
  if (!base || !g) return PB_EINVAL;
  const std::string b(base);
  FILE* cf = std::fopen((b + ".config").c_str(), "w");
  if (!cf) return PB_EIO;
  std::fprintf(cf, "%lld %lld %lld %lld", (long long)g->nv, (long long)g->m, (long long)g->nu, (long long)g->m);
  std::fclose(cf);
  auto write_words = [&](const char* ext, const uint32_t* src, int64_t n) -> bool {
    FILE* f = std::fopen((b + ext).c_str(), "wb");
    if (!f) return false;
    const size_t w = n ? std::fwrite(src, sizeof(uint32_t), (size_t)n, f) : 0;
    std::fclose(f);
    return w == (size_t)n;
  };
  if (!write_words(".vidx", g->offsetsV, g->nv) || !write_words(".vadj", g->edgesV, g->m) ||
      !write_words(".hidx", g->offsetsU, g->nu) || !write_words(".hadj", g->edgesU, g->m))
    return PB_EIO;
  return PB_OK;
}

}  // extern "C"

// KONECT edge lists (utils/KONECTtoHyperAdj.C -> readKONECT, utils/graphIO.h:1033-1100, then
// hypergraphFromHyperedges, :378-440): leading lines starting with '%' are skipped; the first
// data line fixes the number of columns; every line's first column is a V id and its second a
// U id (further columns, weights and times, are ignored); the ids of each side are compacted to
// 0..n-1 in increasing order of the ids that occur; every adjacency list is sorted and repeated
// pairs are dropped.
pb_status pb_read_konect(const char* path, pb_csr_owned* out) {
  if (!path || !out) return PB_EINVAL;
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return PB_EIO;
  std::vector<char> buf;
  if (std::fseek(f, 0, SEEK_END) != 0) { std::fclose(f); return PB_EIO; }
  long size = std::ftell(f);
  if (size < 0) { std::fclose(f); return PB_EIO; }
  std::rewind(f);
  buf.resize((size_t)size);
  if (size > 0 && std::fread(buf.data(), 1, (size_t)size, f) != (size_t)size) { std::fclose(f); return PB_EIO; }
  std::fclose(f);
  size_t k = 0;
  while (k < buf.size() && buf[k] == '%') {  // comment lines at the start
    while (k < buf.size() && buf[k] != '\n') ++k;
    if (k < buf.size()) ++k;
  }
  // Columns: the words of the first data line.
  size_t cols = 0;
  {
    bool prev_space = true;
    for (size_t t = k; t < buf.size() && buf[t] != '\n'; ++t) {
      const bool sp = buf[t] == ' ' || buf[t] == '\t' || buf[t] == '\r';
      if (!sp && prev_space) ++cols;
      prev_space = sp;
    }
  }
  if (cols < 2) return PB_EINVAL;
  Tokenizer t{buf.data() + k, buf.data() + buf.size()};
  std::vector<uint64_t> vid, uid;
  for (size_t col = 0;; col = (col + 1) % cols) {
    const char* w;
    size_t len;
    if (!t.next_word(w, len)) {
      if (col != 0) return PB_EINVAL;  // a short last line
      break;
    }
    if (col >= 2) continue;  // weight / time columns
    uint64_t x = 0;
    for (size_t i = 0; i < len; ++i) {
      const unsigned c = (unsigned)(w[i] - '0');
      if (c > 9) return PB_EINVAL;
      x = x * 10 + c;
    }
    (col == 0 ? vid : uid).push_back(x);
  }
  const size_t m = vid.size();
  auto compact = [](std::vector<uint64_t>& ids, int64_t& n) {
    std::vector<uint64_t> u(ids);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    n = (int64_t)u.size();
    for (auto& x : ids) x = (uint64_t)(std::lower_bound(u.begin(), u.end(), x) - u.begin());
  };
  int64_t nv = 0, nu = 0;
  compact(vid, nv);
  compact(uid, nu);
  if (nv >= (int64_t(1) << 31) || nu >= (int64_t(1) << 31)) return PB_ETOOBIG;
  std::vector<uint64_t> keys(m);
  for (size_t e = 0; e < m; ++e) keys[e] = (vid[e] << 32) | uid[e];
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  const int64_t mm = (int64_t)keys.size();
  if (mm > (int64_t)UINT32_MAX / 2) return PB_ETOOBIG;
  pb_csr_owned g;
  g.nv = nv; g.nu = nu; g.m = mm;
  g.offsetsV = (uint32_t*)calloc((size_t)nv + 1, sizeof(uint32_t));
  g.offsetsU = (uint32_t*)calloc((size_t)nu + 1, sizeof(uint32_t));
  g.edgesV = (uint32_t*)malloc(sizeof(uint32_t) * (mm ? mm : 1));
  g.edgesU = (uint32_t*)malloc(sizeof(uint32_t) * (mm ? mm : 1));
  if (!g.offsetsV || !g.offsetsU || !g.edgesV || !g.edgesU) { pb_csr_free(&g); return PB_ENOMEM; }
  for (int64_t e = 0; e < mm; ++e) {
    const uint32_t v = (uint32_t)(keys[e] >> 32), u = (uint32_t)keys[e];
    g.offsetsV[v + 1]++;
    g.offsetsU[u + 1]++;
    g.edgesV[e] = u;  // keys sorted by (v, u)
  }
  for (int64_t i = 0; i < nv; ++i) g.offsetsV[i + 1] += g.offsetsV[i];
  for (int64_t i = 0; i < nu; ++i) g.offsetsU[i + 1] += g.offsetsU[i];
  std::vector<uint32_t> cur(g.offsetsU, g.offsetsU + nu);
  for (int64_t e = 0; e < mm; ++e) g.edgesU[cur[(uint32_t)keys[e]]++] = (uint32_t)(keys[e] >> 32);  // v ascending
  *out = g;
  return PB_OK;
}

// ---- sparsification (approximate counting) -------------------------------------------------
// Host preprocessing, like the readers: the sparsified graph is then counted on the GPU.
namespace {

// The 64-bit integer mixer of ligra/utils.h:389-397 (hashInt(ulong)).  Its constants decide which
// edges a sparsification keeps, so they have to be the reference's for the same sample.
inline uint64_t mix64_ligra(uint64_t a) {
  a = (a + 0x7ed55d166bef7a1dull) + (a << 12);
  a = (a ^ 0xc761c23c510fa2ddull) ^ (a >> 9);
  a = (a + 0x165667b183a9c0e1ull) + (a << 59);
  a = (a + 0xd3a2646cab3487e3ull) ^ (a << 49);
  a = (a + 0xfd7046c5ef9ab54cull) + (a << 3);
  a = (a ^ 0xb55a4f090dd4a67bull) ^ (a >> 32);
  return a;
}

// Keeps the edges for which keep(v, u) holds, in list order on both sides, then drops the
// vertices left without edges and renumbers each side in increasing order
// (eSparseBipartite / clrSparseBipartite + delZeroDeg, butterfly_utils.h:744-996).
template <class Keep>
pb_status filter_graph(const pb_csr* g, Keep&& keep, pb_csr_owned* out) {
  const int64_t nv = g->nv, nu = g->nu;
  std::vector<uint32_t> offV(nv + 1, 0), offU(nu + 1, 0), eV, eU;
  eV.reserve((size_t)g->m);
  eU.reserve((size_t)g->m);
  for (int64_t v = 0; v < nv; ++v) {
    for (uint32_t j = g->offsetsV[v]; j < g->offsetsV[v + 1]; ++j)
      if (keep((uint32_t)v, g->edgesV[j])) eV.push_back(g->edgesV[j]);
    offV[v + 1] = (uint32_t)eV.size();
  }
  for (int64_t u = 0; u < nu; ++u) {
    for (uint32_t j = g->offsetsU[u]; j < g->offsetsU[u + 1]; ++j)
      if (keep(g->edgesU[j], (uint32_t)u)) eU.push_back(g->edgesU[j]);
    offU[u + 1] = (uint32_t)eU.size();
  }
  if (eV.size() != eU.size()) return PB_EINVAL;  // the two sides of the input disagree
  // New ids of the vertices that keep an edge.
  std::vector<uint32_t> idV(nv), idU(nu);
  int64_t kv = 0, ku = 0;
  for (int64_t v = 0; v < nv; ++v) idV[v] = offV[v + 1] > offV[v] ? (uint32_t)kv++ : UINT32_MAX;
  for (int64_t u = 0; u < nu; ++u) idU[u] = offU[u + 1] > offU[u] ? (uint32_t)ku++ : UINT32_MAX;
  const int64_t m = (int64_t)eV.size();
  std::memset(out, 0, sizeof(*out));
  out->nv = kv;
  out->nu = ku;
  out->m = m;
  out->offsetsV = (uint32_t*)std::malloc(sizeof(uint32_t) * (kv + 1));
  out->offsetsU = (uint32_t*)std::malloc(sizeof(uint32_t) * (ku + 1));
  out->edgesV = (uint32_t*)std::malloc(sizeof(uint32_t) * (m ? m : 1));
  out->edgesU = (uint32_t*)std::malloc(sizeof(uint32_t) * (m ? m : 1));
  if (!out->offsetsV || !out->offsetsU || !out->edgesV || !out->edgesU) {
    pb_csr_free(out);
    return PB_ENOMEM;
  }
  for (int64_t v = 0; v < nv; ++v)
    if (idV[v] != UINT32_MAX) out->offsetsV[idV[v]] = offV[v];
  out->offsetsV[kv] = (uint32_t)m;
  for (int64_t u = 0; u < nu; ++u)
    if (idU[u] != UINT32_MAX) out->offsetsU[idU[u]] = offU[u];
  out->offsetsU[ku] = (uint32_t)m;
  for (int64_t k = 0; k < m; ++k) {
    out->edgesV[k] = idU[eV[k]];
    out->edgesU[k] = idV[eU[k]];
  }
  return PB_OK;
}

}  // namespace

extern "C" pb_status pb_sparsify_bipartite(const pb_csr* g, int32_t sparse_type, int64_t denom, int64_t seed,
                                           pb_csr_owned* out) {
  if (!g || !out) return PB_EINVAL;
  std::memset(out, 0, sizeof(*out));
  if (g->nv < 0 || g->nu < 0 || g->m < 0) return PB_EINVAL;
  const uint64_t colors = denom > 1 ? (uint64_t)denom : 1u;
  if (sparse_type == PB_SPARSE_EDGE) {
    // eSparseBipartite (butterfly_utils.h:798-809): edge (v, u) keeps colour 0 of a hash of both
    // ids and the seed.  v + 0x9e3779b9 is computed in 64 bits, u + 0x9e3779b9 in 32 bits (the
    // reference's operand types), the rest in 64 bits.
    const int64_t sh = (seed << 6) + (seed >> 2);
    return filter_graph(g, [&](uint32_t v, uint32_t u) {
      int64_t concat = (int64_t)v + (int64_t)0x9e3779b9u + sh;
      concat ^= (int64_t)(uint32_t)(u + 0x9e3779b9u) + sh;
      return mix64_ligra((uint64_t)seed + (uint64_t)concat) % colors == 0;
    }, out);
  }
  if (sparse_type == PB_SPARSE_COLOR) {
    // clrSparseBipartite (:919-925): every vertex gets a colour from its id and the seed (the same
    // function on both sides); an edge stays when its endpoints share a colour.
    return filter_graph(g, [&](uint32_t v, uint32_t u) {
      return mix64_ligra((uint64_t)seed + v) % colors == mix64_ligra((uint64_t)seed + u) % colors;
    }, out);
  }
  return PB_EINVAL;
}

extern "C" int64_t pb_sparse_estimate(int64_t sparse_count, int32_t sparse_type, int64_t denom) {
  // BipartiteButterflies.C:213-214: the long count is multiplied by pow(denom, 3) (colour) or
  // pow(denom, 4) (edge) in double precision and truncated back.
  long long x = sparse_count;
  if (sparse_type == PB_SPARSE_COLOR) x = (long long)((double)x * std::pow((double)denom, 3.0));
  else if (sparse_type == PB_SPARSE_EDGE) x = (long long)((double)x * std::pow((double)denom, 4.0));
  return (int64_t)x;
}
