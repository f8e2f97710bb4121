// ref_harness.cpp — drives the UNMODIFIED ParButterfly sources and dumps dense results.
//
// TEST / BASELINE INFRASTRUCTURE ONLY (built by oracle/Makefile into oracle/_ref/).  It is
// compiled against the reference's own headers where they lie, with the macro set of
// apps/hyper/BipartiteButterflies.C:7-10 (VERBOSE off) and the same include list (:12-35).
// Compute() never prints tip or wing numbers (BipartiteButterflies.C:239,268), so this
// harness calls Count / CountE / CountTotal / Peel / PeelE directly and writes the dense
// arrays (the reference's results are strided by 8 longs; the stride is removed here).
//
// Usage:
//   ref_harness GRAPH.bin PER COUNT RANK PEEL OUTPREFIX [ROUNDS] [CSV]
//     PER   : VERT | EDGE | TOTAL
//     COUNT : SORT ASORT HASH AHASH HIST AHIST BATCHS BATCHWA SERIAL
//     RANK  : SIDE COCORE ACOCORE DEG ADEG
//     PEEL  : NONE SORT HASH HIST BATCHS BATCHWA
//   Writes OUTPREFIX.count (int64 little endian) and, when PEEL != NONE, OUTPREFIX.peel.
//   Prints one line: use_v=<0|1> w_side=<W> total=<N> count_s=<median> peel_s=<median>
//   ROUNDS (default 1) repeats count (+peel) on a fresh copy of the graph each round, as
//   parallel_main does (BipartiteButterflies.C:331-341), and reports the median time.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define HYPER 1
#define MCX16 1
// BipartiteButterflies.C:10 defines INVERSE (the direction its driver ships with); the
// PB_REF_FORWARD build leaves it undefined to run the reference's other wedge direction.
#ifndef PB_REF_FORWARD
#define INVERSE 1
#endif

#include "hypergraphIO.h"
#include "index_map.h"
#include "bucket.h"
#include "edgeMapReduce.h"

#include "parallel.h"
#include "gettime.h"
#include "utils.h"
#include "graph.h"
#include "parseCommandLine.h"
#include "vertex.h"
#include "sequence.h"
#include "sparseSet.h"
#include "sampleSort.h"
#ifndef OPENMP
#include "../../lib/histogram.h"
#endif

#include "butterfly_count.h"
#include "butterfly_ecount.h"
#include "butterfly_peel.h"
#include "butterfly_epeel.h"
#include "butterfly_count_total.h"

using namespace std;

// Binary graph file written by parbutterfly_b200.graphio.save_bin:
//   char magic[8] = "PBBGRAPH"; int64 nv, nu, m;
//   uint32 offsetsV[nv+1], edgesV[m], offsetsU[nu+1], edgesU[m]
static bipartiteCSR load_bin(const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  char magic[8];
  int64_t hdr[3];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "PBBGRAPH", 8) != 0 || fread(hdr, 8, 3, f) != 3) {
    fprintf(stderr, "bad graph file %s\n", path);
    exit(2);
  }
  long nv = hdr[0], nu = hdr[1], m = hdr[2];
  uintT* offV = newA(uintT, nv + 1);
  uintT* offU = newA(uintT, nu + 1);
  uintE* edgV = newA(uintE, m + 1);
  uintE* edgU = newA(uintE, m + 1);
  bool ok = fread(offV, 4, nv + 1, f) == (size_t)(nv + 1) && fread(edgV, 4, m, f) == (size_t)m &&
            fread(offU, 4, nu + 1, f) == (size_t)(nu + 1) && fread(edgU, 4, m, f) == (size_t)m;
  fclose(f);
  if (!ok) { fprintf(stderr, "truncated graph file %s\n", path); exit(2); }
  return bipartiteCSR(offV, offU, edgV, edgU, nv, nu, m);
}

static bipartiteCSR copy_graph(const bipartiteCSR& g) {
  uintT* offV = newA(uintT, g.nv + 1);
  uintT* offU = newA(uintT, g.nu + 1);
  uintE* edgV = newA(uintE, g.numEdges + 1);
  uintE* edgU = newA(uintE, g.numEdges + 1);
  memcpy(offV, g.offsetsV, sizeof(uintT) * (g.nv + 1));
  memcpy(offU, g.offsetsU, sizeof(uintT) * (g.nu + 1));
  memcpy(edgV, g.edgesV, sizeof(uintE) * g.numEdges);
  memcpy(edgU, g.edgesU, sizeof(uintE) * g.numEdges);
  return bipartiteCSR(offV, offU, edgV, edgU, g.nv, g.nu, g.numEdges);
}

static CountType parse_count(const string& s) {
  if (s == "SORT") return SORT;
  if (s == "ASORT") return ASORT;
  if (s == "HASH") return HASH;
  if (s == "AHASH") return AHASH;
  if (s == "HIST") return HIST;
  if (s == "AHIST") return AHIST;
  if (s == "BATCHS") return BATCHS;
  if (s == "BATCHWA") return BATCHWA;
  return SERIAL;
}
static RankType parse_rank(const string& s) {
  if (s == "SIDE") return SIDE;
  if (s == "COCORE") return COCORE;
  if (s == "ACOCORE") return ACOCORE;
  if (s == "DEG") return DEG;
  return ADEG;
}
static bool parse_peel(const string& s, PeelType* p) {
  if (s == "SORT") { *p = PSORT; return true; }
  if (s == "HASH") { *p = PHASH; return true; }
  if (s == "HIST") { *p = PHIST; return true; }
  if (s == "BATCHS") { *p = PBATCHS; return true; }
  if (s == "BATCHWA") { *p = PBATCHWA; return true; }
  return false;
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void write_longs(const string& path, const vector<long>& a) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  if (!a.empty()) fwrite(a.data(), sizeof(long), a.size(), f);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s GRAPH.bin PER COUNT RANK PEEL OUTPREFIX [ROUNDS]\n", argv[0]);
    return 2;
  }
  const string per = argv[2];
  const CountType ty = parse_count(argv[3]);
  const RankType tw = parse_rank(argv[4]);
  PeelType tp = PBATCHS;
  const bool peel = parse_peel(argv[5], &tp);
  const string outp = argv[6];
  const int rounds = argc > 7 ? atoi(argv[7]) : 1;
  const long max_wedges = 2577500000L, max_array_size = 23090996160L;
  const size_t stride = 64 / sizeof(long);

  bipartiteCSR G0 = load_bin(argv[1]);
  vector<double> tc, tpl;
  long total = 0;
  int use_v_out = 0;
  long w_side = 0;
  for (int r = 0; r < rounds; ++r) {
    bipartiteCSR GA = copy_graph(G0);
    tuple<bool, long> uv = cmpWedgeCounts(GA);
    bool use_v = get<0>(uv);
    long num_wedges = get<1>(uv);
    use_v_out = use_v;
    w_side = num_wedges;
    if (per == "TOTAL") {
      double t0 = now_s();
      total = CountTotal(GA, use_v, num_wedges, max_wedges, max_array_size, ty, tw);
      tc.push_back(now_s() - t0);
      if (r == rounds - 1) write_longs(outp + ".count", vector<long>{total});
    } else if (per == "VERT") {
      double t0 = now_s();
      long* b = Count(GA, use_v, num_wedges, max_wedges, max_array_size, ty, tw);
      tc.push_back(now_s() - t0);
      long nc = use_v ? GA.nu : GA.nv;
      vector<long> dense(nc);
      long s = 0;
      for (long i = 0; i < nc; ++i) { dense[i] = b[stride * i]; s += dense[i]; }
      total = s / 2;
      if (r == rounds - 1) write_longs(outp + ".count", dense);
      if (peel) {
        double t1 = now_s();
        auto D = Peel(GA, use_v, b, max_wedges, tp, max_array_size);
        tpl.push_back(now_s() - t1);
        if (r == rounds - 1) {
          vector<long> tip(nc);
          for (long i = 0; i < nc; ++i) tip[i] = D.s[i];
          write_longs(outp + ".peel", tip);
        }
      }
      free(b);
    } else {
      uintE* eti = edgeToIdxs(GA, use_v);
      double t0 = now_s();
      long* b = CountE(eti, GA, use_v, num_wedges, max_wedges, max_array_size, ty, tw);
      tc.push_back(now_s() - t0);
      vector<long> dense(GA.numEdges);
      long s = 0;
      for (long i = 0; i < GA.numEdges; ++i) { dense[i] = b[stride * i]; s += dense[i]; }
      total = s / 4;
      if (r == rounds - 1) write_longs(outp + ".count", dense);
      if (peel) {
        double t1 = now_s();
        uintE* ite = idxsToEdge(GA, use_v);
        auto D = PeelE(eti, ite, GA, use_v, b, max_wedges, tp);
        free(ite);
        tpl.push_back(now_s() - t1);
        if (r == rounds - 1) {
          vector<long> wing(GA.numEdges);
          for (long i = 0; i < GA.numEdges; ++i) wing[i] = D.s[i];
          write_longs(outp + ".peel", wing);
        }
      }
      free(b);
      free(eti);
    }
    GA.del();
  }
  auto median = [](vector<double> v) {
    if (v.empty()) return 0.0;
    sort(v.begin(), v.end());
    return v[v.size() / 2];
  };
  printf("use_v=%d w_side=%ld total=%ld count_s=%.6f peel_s=%.6f\n", use_v_out, w_side, total, median(tc), median(tpl));
  G0.del();
  return 0;
}
