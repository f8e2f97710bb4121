// Device-side parsing of the AdjacencyHypergraph text format (readBipartite's input,
// butterfly_utils.h:1008-1058: the word "AdjacencyHypergraph", then nv mv nu mu, offsetsV[nv],
// edgesV[mv], offsetsU[nu], edgesU[mu], whitespace separated).
//
// The bytes after the header word are split into 64-byte chunks, one per thread.  Pass 1 counts
// the tokens that start in each chunk (a digit preceded by a non-digit) and flags bytes that are
// neither digits nor whitespace; an exclusive scan gives every chunk its first token index; pass 2
// parses each token that starts in a chunk (reading past the chunk end when the token does) into
// a 64-bit value.  The host then checks the four sizes and the token count as readBipartite does
// (:1013-1027) and a conversion kernel builds the two CSR sides, checking that every value fits
// and every id is in range (:1039-1051).  Sortedness is checked when the graph is adopted.
#include <cstring>

#include "pb_engine.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

constexpr int kChunk = 64;

__device__ __forceinline__ bool is_digit(unsigned char c) { return c >= '0' && c <= '9'; }
__device__ __forceinline__ bool is_space(unsigned char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

__global__ void count_tokens_kernel(const unsigned char* __restrict__ t, int64_t len, int64_t nchunks,
                                    int64_t* counts, uint32_t* bad) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = c * kChunk, e = min(len, b + kChunk);
    uint32_t n = 0, badc = 0;
    bool prev_digit = b > 0 && is_digit(t[b - 1]);
    for (int64_t i = b; i < e; ++i) {
      const unsigned char ch = t[i];
      const bool d = is_digit(ch);
      if (d && !prev_digit) ++n;
      if (!d && !is_space(ch)) badc = 1;
      prev_digit = d;
    }
    counts[c] = n;
    if (badc) atomicOr(bad, 1u);
  }
}

__global__ void parse_tokens_kernel(const unsigned char* __restrict__ t, int64_t len, int64_t nchunks,
                                    const int64_t* __restrict__ first, uint64_t* vals, int64_t cap, uint32_t* bad) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = c * kChunk, e = min(len, b + kChunk);
    int64_t k = first[c];
    bool prev_digit = b > 0 && is_digit(t[b - 1]);
    for (int64_t i = b; i < e; ++i) {
      const bool d = is_digit(t[i]);
      if (d && !prev_digit) {
        uint64_t v = 0;
        int digits = 0;
        for (int64_t j = i; j < len && is_digit(t[j]); ++j, ++digits) v = v * 10 + (uint64_t)(t[j] - '0');
        if (digits > 19) atomicOr(bad, 2u);  // beyond 64 bits
        if (k < cap) vals[k] = v;
        ++k;
      }
      prev_digit = d;
    }
  }
}

// Builds one CSR side from its token ranges: off[i] = offsets token i (off[n] = m), edg[j] =
// edges token j; flags values beyond 32 bits, offsets beyond m and ids >= other_n.
__global__ void build_side_kernel(const uint64_t* __restrict__ offs, const uint64_t* __restrict__ edges, int64_t n,
                                  int64_t m, int64_t other_n, uint32_t* off, uint32_t* edg, uint32_t* bad) {
  const int64_t total = n + m;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
    if (x < n) {
      const uint64_t v = offs[x];
      if (v > (uint64_t)m) atomicOr(bad, 4u);
      off[x] = (uint32_t)v;
    } else {
      const uint64_t v = edges[x - n];
      if (v >= (uint64_t)other_n) atomicOr(bad, 8u);
      edg[x - n] = (uint32_t)v;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) off[n] = (uint32_t)m;
}

int grid_for(int64_t n) { return std::max(1, std::min(ceil_div(n, 256), sm_count() * 16)); }

}  // namespace

void parse_adjacency_hypergraph(const char* text, size_t len, bool on_device, ParsedCSR& out, cudaStream_t s) {
  static const char kHeader[] = "AdjacencyHypergraph";
  const size_t hl = sizeof(kHeader) - 1;
  // The header word (readBipartite compares the first token with it, :1013-1016).
  char head[64] = {0};
  const size_t hn = std::min(len, sizeof(head) - 1);
  if (on_device) PB_CUDA_TRY(cudaMemcpyAsync(head, text, hn, cudaMemcpyDeviceToHost, s));
  else std::memcpy(head, text, hn);
  if (on_device) PB_CUDA_TRY(cudaStreamSynchronize(s));
  size_t p = 0;
  while (p < hn && (head[p] == ' ' || head[p] == '\n' || head[p] == '\r' || head[p] == '\t')) ++p;
  PB_REQUIRE(hn >= p + hl && std::memcmp(head + p, kHeader, hl) == 0 &&
                 (p + hl == len || head[p + hl] == ' ' || head[p + hl] == '\n' || head[p + hl] == '\r' ||
                  head[p + hl] == '\t'),
             PB_EIO, "Bad input file: the first word is not AdjacencyHypergraph");
  const size_t body = p + hl;
  const int64_t blen = (int64_t)(len - body);
  DevBuf<unsigned char> dtext;
  const unsigned char* t;
  if (on_device) {
    t = reinterpret_cast<const unsigned char*>(text) + body;
  } else {
    dtext.alloc(blen > 0 ? blen : 1, s);
    if (blen > 0) PB_CUDA_TRY(cudaMemcpyAsync(dtext.get(), text + body, blen, cudaMemcpyHostToDevice, s));
    t = dtext.get();
  }
  const int64_t nchunks = (blen + kChunk - 1) / kChunk;
  PB_REQUIRE(nchunks > 0, PB_EIO, "Bad input file: nothing after the header");
  // Token counts per chunk and their prefix are 64-bit: a valid file near the 32-bit edge limit
  // has more than 2^32 tokens.
  DevBuf<int64_t> counts(nchunks + 1, s);
  DevBuf<uint32_t> bad(1, s);
  PB_CUDA_TRY(cudaMemsetAsync(bad.get(), 0, sizeof(uint32_t), s));
  PB_CUDA_TRY(cudaMemsetAsync(counts.get(), 0, counts.bytes(), s));
  PB_LAUNCH(count_tokens_kernel, grid_for(nchunks), 256, 0, s, t, blen, nchunks, counts.get(), bad.get());
  exclusive_scan_i64(counts.get(), counts.get(), nchunks, s);
  int64_t ntok = 0;
  uint32_t hb[2];
  readback(&ntok, counts.get() + nchunks, sizeof(int64_t), s);
  readback(&hb[1], bad.get(), sizeof(uint32_t), s);
  PB_REQUIRE(hb[1] == 0, PB_EIO, "Bad input file: a character that is neither a digit nor whitespace");
  PB_REQUIRE(ntok >= 4, PB_EIO, "Bad input file: fewer than four sizes after the header");
  DevBuf<uint64_t> vals(ntok, s);
  PB_LAUNCH(parse_tokens_kernel, grid_for(nchunks), 256, 0, s, t, blen, nchunks, counts.get(), vals.get(), ntok,
            bad.get());
  uint64_t sz[4];
  readback(sz, vals.get(), sizeof(sz), s);
  readback(&hb[1], bad.get(), sizeof(uint32_t), s);
  PB_REQUIRE(hb[1] == 0, PB_EIO, "Bad input file: a number beyond 64 bits");
  const uint64_t nv = sz[0], mv = sz[1], nu = sz[2], mu = sz[3];
  PB_REQUIRE(nv < (1ull << 40) && mv < (1ull << 40) && nu < (1ull << 40) && mu < (1ull << 40), PB_EIO,
             "Bad input file: a size is implausibly large");
  PB_REQUIRE((uint64_t)ntok == nv + mv + nu + mu + 4, PB_EIO,
             "Bad input file: the token count is not nv + mv + nu + mu + 4");
  PB_REQUIRE(mv == mu, PB_EIO, "Bad input file: mv != mu");
  PB_REQUIRE(nv + nu < (1ull << 31) && 2 * mv <= 0xFFFFFFFFull, PB_ETOOBIG,
             "graph too large for 32-bit ids and offsets");
  out.nv = (int64_t)nv;
  out.nu = (int64_t)nu;
  out.m = (int64_t)mv;
  out.offV.alloc(nv + 1, s);
  out.offU.alloc(nu + 1, s);
  out.edgV.alloc(mv > 0 ? mv : 1, s);
  out.edgU.alloc(mv > 0 ? mv : 1, s);
  PB_CUDA_TRY(cudaMemsetAsync(bad.get(), 0, sizeof(uint32_t), s));
  const uint64_t* v = vals.get() + 4;
  PB_LAUNCH(build_side_kernel, grid_for(nv + mv + 1), 256, 0, s, v, v + nv, (int64_t)nv, (int64_t)mv, (int64_t)nu,
            out.offV.get(), out.edgV.get(), bad.get());
  PB_LAUNCH(build_side_kernel, grid_for(nu + mv + 1), 256, 0, s, v + nv + mv, v + nv + mv + nu, (int64_t)nu,
            (int64_t)mv, (int64_t)nv, out.offU.get(), out.edgU.get(), bad.get());
  readback(&hb[1], bad.get(), sizeof(uint32_t), s);
  PB_REQUIRE(!(hb[1] & 8u), PB_EINVAL, "Bad input file: an edge id is out of range");
  PB_REQUIRE(!(hb[1] & 4u), PB_EINVAL, "Bad input file: an offset exceeds the edge count");
}

}  // namespace pb
