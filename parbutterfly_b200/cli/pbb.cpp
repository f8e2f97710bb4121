// pbb — command-line drop-in for ParButterfly's BipartiteButterflies driver, running the
// B200 path through the C ABI (include/parbutterfly_b200.h).
//
// Flags, aliases, defaults and stdout lines follow apps/hyper/BipartiteButterflies.C:
//   -countType/-t, -rankType/-w, -peelType/-tp (+ -nopeel), -per/-e/-total, -m, -a, -d,
//   -sparseType/-s, -r; Compute() at :75-277 and parallel_main() at :283-355.  Timer lines use
//   the reference's "<name> : <seconds>" format (ligra/gettime.h:87-96, setprecision(3)).
// Additions: -sched {plain,learned}, -schedModel <file>, -autotune, -device N.
// Sparsification (-sparseType EDGE/COLOR, -s, -d) sparsifies each round's graph on the host
// (pb_sparsify_bipartite, seed 0 as the reference's driver) and prints the scaled estimate.
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/parbutterfly_b200.h"

namespace {

struct Args {
  int argc;
  char** argv;
  // parseCommandLine.h:72-116 semantics: an option's value is the next argument; the last
  // argument (the input file) is never read as a value.
  const char* value(const std::string& opt) const {
    for (int i = 1; i < argc - 1; ++i)
      if (opt == argv[i]) return argv[i + 1];
    return nullptr;
  }
  std::string str(const std::string& opt, const std::string& def) const {
    const char* v = value(opt);
    return v ? std::string(v) : def;
  }
  long lng(const std::string& opt, long def) const {
    const char* v = value(opt);
    return v ? atol(v) : def;
  }
};

const char* count_name(int ty) {  // CountTypeToStr, BipartiteButterflies.C:41-55
  switch (ty) {
    case PB_ASORT: return "Sort";
    case PB_SORT: return "SortCE";
    case PB_AHASH: return "Hash";
    case PB_HASH: return "HashCE";
    case PB_AHIST: return "Hist";
    case PB_HIST: return "HistCE";
    case PB_BATCHS: return "Par";
    case PB_SERIAL: return "Serial";
    case PB_BATCHWA: return "WedgePar";
  }
  return "";
}

const char* peel_name(int tp) {  // PeelTypeToStr, BipartiteButterflies.C:57-67
  switch (tp) {
    case PB_PSORT: return "SortCE Peel";
    case PB_PHASH: return "HashCE Peel";
    case PB_PHIST: return "HistCE Peel";
    case PB_PBATCHS: return "Par Peel";
    case PB_PBATCHWA: return "WedgePar Peel";
  }
  return "";
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void report(const std::string& name, double secs) {
  std::cout << name << " : " << std::setprecision(3) << secs << std::endl;
}

int fail(pb_ctx* ctx, pb_status st, const char* what) {
  std::cerr << what << " failed (status " << st << "): " << (ctx ? pb_last_error(ctx) : "") << std::endl;
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: " << argv[0] << " [options] <inFile>" << std::endl;
    return 2;
  }
  Args P{argc, argv};
  const char* file = argv[argc - 1];
  pb_opts o;
  pb_opts_default(&o);

  // Count type (BipartiteButterflies.C:79-106)
  long t = P.lng("-t", LONG_MAX);
  std::string cts = P.str("-countType", "");
  if (t == LONG_MAX) {
    if (cts == "ASORT") o.count_type = PB_ASORT;
    else if (cts == "SORT") o.count_type = PB_SORT;
    else if (cts == "AHASH") o.count_type = PB_AHASH;
    else if (cts == "HASH") o.count_type = PB_HASH;
    else if (cts == "AHIST") o.count_type = PB_AHIST;
    else if (cts == "HIST") o.count_type = PB_HIST;
    else if (cts == "BATCHS") o.count_type = PB_BATCHS;
    else if (cts == "BATCHWA") o.count_type = PB_BATCHWA;
    else o.count_type = PB_SERIAL;
  } else {
    switch (t) {
      case 0: o.count_type = PB_ASORT; break;
      case 1: o.count_type = PB_SORT; break;
      case 2: o.count_type = PB_AHASH; break;
      case 3: o.count_type = PB_HASH; break;
      case 4: o.count_type = PB_AHIST; break;
      case 6: o.count_type = PB_HIST; break;
      case 5: case 7: case 11: o.count_type = PB_BATCHS; break;
      case 9: case 12: o.count_type = PB_SERIAL; break;
      case 8: o.count_type = PB_BATCHWA; break;
      default: break;
    }
  }
  // Rank type (:108-128)
  long w = P.lng("-w", LONG_MAX);
  std::string rts = P.str("-rankType", "");
  if (w == LONG_MAX) {
    if (rts == "SIDE") o.rank_type = PB_SIDE;
    else if (rts == "COCORE") o.rank_type = PB_COCORE;
    else if (rts == "ACOCORE") o.rank_type = PB_ACOCORE;
    else if (rts == "DEG") o.rank_type = PB_DEG;
    else o.rank_type = PB_ADEG;
  } else if (w >= 0 && w <= 4) {
    o.rank_type = (int)w;
  }
  // Peel type (:130-153)
  long tp = P.lng("-tp", LONG_MAX);
  std::string pts = P.str("-peelType", "");
  bool nopeel = false;
  if (tp == LONG_MAX) {
    if (pts == "SORT") o.peel_type = PB_PSORT;
    else if (pts == "HASH") o.peel_type = PB_PHASH;
    else if (pts == "HIST") o.peel_type = PB_PHIST;
    else if (pts == "BATCHS") o.peel_type = PB_PBATCHS;
    else if (pts == "BATCHWA") o.peel_type = PB_PBATCHWA;
    else nopeel = true;
  } else {
    nopeel = P.value("-nopeel") != nullptr;
    switch (tp) {
      case 0: o.peel_type = PB_PHASH; break;
      case 1: o.peel_type = PB_PSORT; break;
      case 2: o.peel_type = PB_PHIST; break;
      case 3: case 4: o.peel_type = PB_PBATCHS; break;
      case 5: o.peel_type = PB_PBATCHWA; break;
      default: nopeel = true; break;
    }
  }
  // Per type (:155-170)
  std::string pers = P.str("-per", "");
  long te = P.lng("-e", LONG_MAX);
  bool total = P.value("-total") != nullptr;
  if (te == LONG_MAX) {
    if (pers == "EDGE") o.per_type = PB_EDGE;
    else if (pers == "TOTAL") o.per_type = PB_TOTAL;
    else o.per_type = PB_VERT;
  } else {
    o.per_type = total ? PB_TOTAL : (te == 0 ? PB_VERT : PB_EDGE);
  }
  o.max_wedges = P.lng("-m", 2577500000L);
  o.max_array_size = P.lng("-a", 23090996160L);
  // Sparsification (:175-193): -d denom, -s 0/1/2 or -sparseType COLOR/EDGE; forces TOTAL.
  const long denom = P.lng("-d", 25);
  const long sparse_num = P.lng("-s", LONG_MAX);
  const std::string ss = P.str("-sparseType", "");
  int32_t sparse = PB_NOSPARSE;
  if (sparse_num == LONG_MAX) sparse = ss == "EDGE" ? PB_SPARSE_EDGE : (ss == "COLOR" ? PB_SPARSE_COLOR : PB_NOSPARSE);
  else sparse = sparse_num == 1 ? PB_SPARSE_COLOR : (sparse_num == 2 ? PB_SPARSE_EDGE : PB_NOSPARSE);
  if (sparse != PB_NOSPARSE) o.per_type = PB_TOTAL;
  if (o.per_type == PB_TOTAL) nopeel = true;
  o.sched = P.str("-sched", "plain") == "learned" ? PB_SCHED_LEARNED : PB_SCHED_PLAIN;
  for (int i = 1; i < argc - 1; ++i)
    if (std::string(argv[i]) == "-autotune") o.autotune = 1;
  const long rounds = P.lng("-r", 3);
  const int device = (int)P.lng("-device", 0);

  pb_ctx* ctx = nullptr;
  pb_status st = pb_ctx_create(device, nullptr, &ctx);
  if (st != PB_OK) return fail(nullptr, st, "pb_ctx_create");
  // -sched learned: the cost models of -schedModel <file> (default: the trained models that
  // ship beside the library, ../models/sched_b200.bin relative to this binary).
  pb_sched_model* model = nullptr;
  if (o.sched == PB_SCHED_LEARNED) {
    std::string path = P.str("-schedModel", "");
    if (path.empty()) {
      std::string self = argv[0];
      const size_t slash = self.find_last_of('/');
      path = (slash == std::string::npos ? std::string(".") : self.substr(0, slash)) + "/../models/sched_b200.bin";
    }
    if (pb_sched_model_create(ctx, 1, &model) != PB_OK || pb_sched_load(ctx, model, path.c_str()) != PB_OK ||
        pb_ctx_set_sched_model(ctx, model) != PB_OK) {
      std::cerr << "no scheduler model at " << path << " (" << pb_last_error(ctx) << "); running the plain path"
                << std::endl;
      if (model) pb_sched_model_destroy(model);
      model = nullptr;
    }
  }

  for (long r = 0; r < rounds + 1; ++r) {  // parallel_main re-reads the file each round (:331-341)
    pb_csr_owned h;
    st = pb_read_adjacency_hypergraph(file, &h);
    if (st != PB_OK) {
      std::cerr << "Bad input file" << std::endl;
      pb_ctx_destroy(ctx);
      return 1;
    }
    if (sparse != PB_NOSPARSE) {  // the reference sparsifies each round's graph with seed 0 (:333-340)
      pb_csr full{h.nv, h.nu, h.m, h.offsetsV, h.edgesV, h.offsetsU, h.edgesU};
      pb_csr_owned hs;
      st = pb_sparsify_bipartite(&full, sparse, denom, 0, &hs);
      pb_csr_free(&h);
      if (st != PB_OK) return fail(ctx, st, "pb_sparsify_bipartite");
      h = hs;
    }
    pb_csr c{h.nv, h.nu, h.m, h.offsetsV, h.edgesV, h.offsetsU, h.edgesU};
    pb_graph* g = nullptr;
    double t0 = now();
    st = pb_graph_upload(ctx, &c, &g);
    if (st != PB_OK) { pb_csr_free(&h); return fail(ctx, st, "pb_graph_upload"); }
    int32_t use_v = 0;
    int64_t num_wedges = 0;
    st = pb_cmp_wedge_counts(ctx, g, &use_v, &num_wedges);
    if (st != PB_OK) return fail(ctx, st, "pb_cmp_wedge_counts");
    report("preprocess (wedge counts)", now() - t0);
    o.use_v = use_v;
    if (o.per_type == PB_TOTAL) {
      int64_t nb = 0;
      double t1 = now();
      st = pb_count_total(ctx, g, &o, &nb);
      if (st != PB_OK) return fail(ctx, st, "pb_count_total");
      report(count_name(o.count_type), now() - t1);
      if (sparse != PB_NOSPARSE) nb = pb_sparse_estimate(nb, sparse, denom);
      std::cout << "number of butterflies: " << nb << "\n";
    } else if (o.per_type == PB_VERT) {
      const int64_t nc = use_v ? h.nu : h.nv;
      std::vector<int64_t> b(nc > 0 ? nc : 1);
      double t1 = now();
      st = pb_count_vert(ctx, g, &o, b.data());
      if (st != PB_OK) return fail(ctx, st, "pb_count_vert");
      report(count_name(o.count_type), now() - t1);
      int64_t tot = 0;
      for (int64_t i = 0; i < nc; ++i) tot += b[i];
      std::cout << "number of butterflies: " << tot / 2 << "\n";
      if (!nopeel) {
        std::vector<int64_t> tip(b.size());
        double t2 = now();
        st = pb_peel_vert(ctx, g, &o, b.data(), tip.data());
        if (st != PB_OK) return fail(ctx, st, "pb_peel_vert");
        report(peel_name(o.peel_type), now() - t2);
      }
    } else {
      std::vector<int64_t> b(h.m > 0 ? h.m : 1);
      double t1 = now();
      st = pb_count_edge(ctx, g, &o, b.data());
      if (st != PB_OK) return fail(ctx, st, "pb_count_edge");
      report(count_name(o.count_type), now() - t1);
      int64_t tot = 0;
      for (int64_t i = 0; i < h.m; ++i) tot += b[i];
      std::cout << "number of edge butterflies: " << tot / 4 << "\n";
      if (!nopeel) {
        std::vector<int64_t> wing(b.size());
        double t2 = now();
        st = pb_peel_edge(ctx, g, &o, b.data(), wing.data());
        if (st != PB_OK) return fail(ctx, st, "pb_peel_edge");
        report(peel_name(o.peel_type), now() - t2);
      }
    }
    pb_graph_destroy(g);
    pb_csr_free(&h);
  }
  if (model) pb_sched_model_destroy(model);
  pb_ctx_destroy(ctx);
  return 0;
}
