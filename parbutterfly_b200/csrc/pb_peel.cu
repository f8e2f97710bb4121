// Tip (vertex) and wing (edge) peeling on the device.
//
// Semantics (Peel / PeelOrigParallel, butterfly_peel.h:647-711,896-934; PeelE /
// PeelEOrigParallel, butterfly_epeel.h:339-443,519-569; updateBuckets,
// butterfly_putils.h:1027-1115): items start in bucket D = their butterfly count.  Each round
// takes every unpeeled item whose bucket equals the current minimum k (the frontier):
//   tip : for each frontier vertex u and each two-hop neighbour u2 != u, the C(w(u,u2), 2)
//         shared butterflies leave u2's count;
//   wing: each butterfly that contains a frontier edge and no edge peeled in an earlier round
//         is removed once, by its frontier edge of smallest index, and its other edges lose 1.
// Every touched unpeeled item moves to bucket max(count, k).  Buckets are 64-bit (the
// reference's are 32-bit, ligra/bucket.h:15-16, exact only below 2^32 - 1).
//
// Device design: one cooperative persistent kernel runs all rounds.  Phases are separated by
// a grid barrier whose wait is bounded in time (on expiry the kernel records PB_ETIMEOUT and
// returns; the context stays usable).  Buckets are kept as a near/far split: the near list
// holds the unpeeled items whose bucket lies below a window bound; each round scans only the
// near list (frontier extraction fused with the next minimum), and the window advances (one
// pass over the alive list, a log2 histogram of distances to the minimum) when the near list
// runs dry.  Frontier items with little work run one per warp; heavy ones one per CTA.
#include <algorithm>
#include <functional>
#include <memory>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pb_engine.cuh"
#include "pb_prims.cuh"

namespace pb {

namespace {

constexpr int kPT = 512;
constexpr int kWarpSlots = 512;    // per-warp table slots (keys, values, hit counters: 6 KiB)
constexpr int kBlockSlots = 8192;  // per-CTA table slots (96 KiB), shares memory with warp tables
constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr unsigned long long kInf = ~0ull;
constexpr uint8_t ALIVE = 0, ACTIVE = 1, PEELED = 2;
constexpr unsigned ERR_TIMEOUT = 1u;
constexpr unsigned long long kBarrierTimeoutNs = 60ull * 1000000000ull;  // 60 s per wait

struct Ctl {
  unsigned long long nm[2];       // next minimum per round parity
  unsigned long long k_lo, win_hi;
  unsigned long long rounds, work;
  unsigned flen_small[2], flen_big[2], flen_huge[2];
  unsigned tlen[2];
  unsigned cur_small[2], cur_big[2];
  unsigned units;  // work units (chunks of CTA-level items) of the current round
  unsigned long long round_cost[2];  // summed cost estimate of the round's CTA-level items
  unsigned near_len;
  unsigned alive;                 // unpeeled items
  unsigned alen[2];               // alive list lengths
  unsigned hist[66];
  unsigned bar_count, bar_gen, err;
  unsigned long long round;   // next round to run (kept across launches)
  unsigned alist_cur;         // current alive list (kept across launches)
  unsigned started;           // alive list initialised
  unsigned alive_at_compact;  // unpeeled items when the lists were last compacted
  unsigned min_gain;          // pause for compaction once this many more items are peeled
  // Instrumentation (CTA 0): device time per phase and work counters.
  unsigned long long t_last, phase_ns[4];  // advance, F, P, U
  unsigned long long barrier_timeout_ns;   // bound of every grid-barrier wait
  unsigned test_skip_arrival;              // test hook: CTA 0 never arrives at grid barriers
  unsigned long long scanned, touched_total, n_small, n_big, n_huge, advances;
  // Phase-P time of the rounds binned by log2 of their estimated work (frontier cost sum).
  unsigned long long round_est[2];
  unsigned long long pbin_ns[42], pbin_rounds[42], pbin_est[42];
  // Near-window size: at least near_min items, or alive / near_div.
  unsigned near_min, near_div;
  // Barriers of CTA groups that process heavy tip items concurrently.
  unsigned gbar_count[32], gbar_gen[32];
  // Range mode (the coarse pass of the two-phase peel): each window is one partition, its
  // frontier every unpeeled item whose count is below the window bound, repeated until no
  // unpeeled item is below it.  The bound is chosen so that the window holds about
  // part_target of estimated work.  npart counts the partitions opened so far.
  unsigned range_mode, npart;
  unsigned long long part_target;  // base target per partition
  // Partitions grow past their opening bound (items fall below it while the partition peels):
  // part_done sums the estimated work actually peeled, part_used the target the partition was
  // opened with, part_ratio_q (x256, smoothed) their ratio, which scales the next target down.
  unsigned long long part_done, part_used, part_ratio_q;
  unsigned long long whist[66];    // estimated work per log2 distance bin
  unsigned long long wsub[256];    // estimated work per linear sub-bin of the chosen octave
  // Wing items per probe structure (warp table, CTA table, dense markers, grid) and their probes;
  // probes that walked the probe set against a binary search (the reverse direction).
  unsigned long long mode_items[4], mode_work[4], rev_work;
  unsigned prev_items;  // frontier items of the previous round
  unsigned wunits;      // warp units of the current round (global prefix only)
};
constexpr unsigned kMaxGroups = 32;
// Device memory for grid-shared dense counters (one n-sized slice per concurrent heavy tip
// item group or per fine-pass instance with a CTA range of its own).
constexpr int64_t kGsharedBudget = int64_t(2) << 30;


// Live adjacency of both sides.  Lists are compacted to their live entries between launches
// of the peeling kernel, so list positions are not edge ids: eidK / eidC carry the output
// edge index of every entry.
struct Lists {
  const uint32_t* offK;  // count side: vertex -> centre ids
  const uint32_t* edgK;
  const uint32_t* eidK;  // count-side entry -> output edge index (wing only)
  const uint32_t* offC;  // centre side: vertex -> count-side ids
  const uint32_t* edgC;
  const uint32_t* eidC;  // centre-side entry -> output edge index (wing only)
  const uint32_t* center_of;  // output edge index -> centre vertex (wing only)
  const uint32_t* u_of;       // output edge index -> count-side vertex (wing only)
  const int64_t* S;      // per count-side vertex then per centre vertex: sum of neighbour degrees (wing)
  const int64_t* wk;     // per count-side vertex: two-hop wedges sum(deg(v) - 1) (tip)
  int64_t nK, nC;
};

struct Work {
  int64_t* D;        // buckets (final: tip / wing numbers)
  int64_t* cnt;      // butterfly counts
  uint8_t* state;
  uint8_t* in_near;
  uint32_t* touched;
  uint32_t* alist[2];
  uint32_t* near;
  uint32_t* fsmall[2];
  uint32_t* fbig[2];
  uint32_t* fchunks[2];  // work units of each CTA-level item (parallel to fbig)
  uint32_t* uprefix;     // exclusive prefix of fchunks for the current round (N + 1)
  uint32_t* fwchunks[2]; // warp units of each warp-level wing item (parallel to fsmall)
  uint32_t* wprefix;     // exclusive prefix of fwchunks (N + 1)
  uint32_t* fhuge[2];
  uint32_t* tlist[2];
  uint32_t* gshared;   // grid-shared dense counters / probe markers for huge items (zeroed);
                       // tip: ngroups slices of gshared_stride counters, one per CTA group
  int64_t gshared_stride;
  unsigned ngroups;
  uint32_t* gscratch;  // per-CTA dense scratch (dense counters / probe markers)
  int64_t gscratch_len;
  int64_t N;           // items of this instance
  uint32_t item0;      // first item of this instance: its items are items[item0 .. item0 + N)
                       // (item0 .. item0 + N - 1 themselves when items is null)
  const uint32_t* items;
  // Two-phase peel.  Fine pass: every instance is one partition of the coarse pass; part[x]
  // is the partition of item x and my_part this instance's.  Items of lower partitions are
  // peeled, items of higher partitions stay unpeeled for the whole pass (and are never
  // charged), items of my_part follow the exact rounds.  Coarse pass: part_out receives the
  // partition of every item as it is peeled.  level: the live-list version the instance reads.
  const uint32_t* part;
  uint32_t my_part;
  uint32_t* part_out;
  uint32_t level;
  const uint32_t* wgt;  // coarse pass: every item's estimated work (item_weight, capped at 2^32 - 1)
};

// Every CTA belongs to one peel instance (the whole input, or one graph of a batch, each with
// its own control block, lists and rounds): its index within the instance and the instance's
// CTA count, set at kernel start.
__shared__ unsigned s_vb, s_vg;
__device__ __forceinline__ unsigned vblock() { return s_vb; }
__device__ __forceinline__ unsigned vgrid() { return s_vg; }

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// CTA 0 charges the time since its previous mark to phase `ph` (called right after barriers).
// Phase P is also binned by log2 of the round's estimated work (est).
__device__ __forceinline__ void phase_mark(Ctl* ctl, int ph, unsigned long long est = 0) {
  if (vblock() == 0 && threadIdx.x == 0) {
    const unsigned long long now = globaltimer_ns();
    if (ctl->t_last) {
      ctl->phase_ns[ph] += now - ctl->t_last;
      if (ph == 2) {
        const int b = est ? min(41, 64 - __clzll(est)) : 0;
        ctl->pbin_ns[b] += now - ctl->t_last;
        ctl->pbin_rounds[b] += 1;
        ctl->pbin_est[b] += est;
      }
    }
    ctl->t_last = now;
  }
}

// Barrier over the CTAs of one peel instance (a cooperative launch keeps every CTA co-resident).
// Bounded: a wait longer than the control block's timeout sets ERR_TIMEOUT and returns false.
__device__ bool grid_barrier(Ctl* ctl) {
  __shared__ int ok;
  if (vgrid() == 1) {  // one CTA: a block barrier orders its global memory accesses too
    __syncthreads();
    return *(volatile unsigned*)&ctl->err == 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &ctl->bar_gen;
    const unsigned gen = *vgen;
    __threadfence();
    // (test hook) without CTA 0's arrival no CTA is last, so every wait runs out.
    const unsigned arrived =
        (vblock() == 0 && *(volatile unsigned*)&ctl->test_skip_arrival) ? 0xFFFFFFFFu : atomicAdd(&ctl->bar_count, 1u);
    ok = 1;
    if (arrived == vgrid() - 1) {
      atomicExch(&ctl->bar_count, 0u);
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      while (*vgen == gen) {
        if (*(volatile unsigned*)&ctl->err) { ok = 0; break; }
        if (globaltimer_ns() - t0 > ctl->barrier_timeout_ns) {
          atomicOr(&ctl->err, ERR_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    if (*(volatile unsigned*)&ctl->err) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

// Barrier over `size` CTAs of a group (slot: the group's counters).  Bounded like grid_barrier.
__device__ bool group_barrier(Ctl* ctl, unsigned slot, unsigned size) {
  __shared__ int gok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &ctl->gbar_gen[slot];
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(&ctl->gbar_count[slot], 1u);
    gok = 1;
    if (arrived == size - 1) {
      atomicExch(&ctl->gbar_count[slot], 0u);
      __threadfence();
      atomicAdd(&ctl->gbar_gen[slot], 1u);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      while (*vgen == gen) {
        if (*(volatile unsigned*)&ctl->err) { gok = 0; break; }
        if (globaltimer_ns() - t0 > ctl->barrier_timeout_ns) {
          atomicOr(&ctl->err, ERR_TIMEOUT);
          gok = 0;
          break;
        }
      }
    }
    __threadfence();
    if (*(volatile unsigned*)&ctl->err) gok = 0;
  }
  __syncthreads();
  return gok != 0;
}

// Fibonacci hashing: the high bits of key * 2^32/phi, folded into the table size.
__device__ __forceinline__ uint32_t hslot(uint32_t key, uint32_t mask) {
  return __umulhi(key * 0x9E3779B1u, mask + 1u) & mask;
}

// Tables are sized to at least twice their key count, so probe sequences stay shorter than
// the table; the bounds turn a broken invariant into a recorded error, not an endless loop.
constexpr unsigned ERR_TABLE = 2u;

__device__ __forceinline__ void t_add(uint32_t* keys, uint32_t* vals, uint32_t mask, uint32_t key, Ctl* ctl) {
  uint32_t h = hslot(key, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    uint32_t k = keys[h];
    if (k == key) { atomicAdd(&vals[h], 1u); return; }
    if (k == kEmpty) {
      uint32_t prev = atomicCAS(&keys[h], kEmpty, key);
      if (prev == kEmpty || prev == key) { atomicAdd(&vals[h], 1u); return; }
    }
    h = (h + 1) & mask;
  }
  atomicOr(&ctl->err, ERR_TABLE);
}

// Unique-key insert of (key, val).
__device__ __forceinline__ void t_put(uint32_t* keys, uint32_t* vals, uint32_t mask, uint32_t key, uint32_t val,
                                      Ctl* ctl) {
  uint32_t h = hslot(key, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    uint32_t prev = atomicCAS(&keys[h], kEmpty, key);
    if (prev == kEmpty) { vals[h] = val; return; }
    h = (h + 1) & mask;
  }
  atomicOr(&ctl->err, ERR_TABLE);
}

// Slot of key, or kEmpty when absent.
__device__ __forceinline__ uint32_t t_slot(const uint32_t* keys, uint32_t mask, uint32_t key) {
  uint32_t h = hslot(key, mask);
  for (uint32_t probes = 0; probes <= mask; ++probes) {
    const uint32_t k = keys[h];
    if (k == key) return h;
    if (k == kEmpty) return kEmpty;
    h = (h + 1) & mask;
  }
  return kEmpty;
}

__device__ __forceinline__ uint32_t np2(uint32_t x) { return x <= 1 ? 1u : 1u << (32 - __clz(x - 1)); }

constexpr uint32_t kLocalUnits = 2048;  // rounds with at most this many CTA-level items lay
                                        // out their work units in every CTA's shared memory
struct Shared {
  uint32_t incl[kPT];
  uint32_t sb[kPT];
  uint32_t len[kPT];
  uint32_t cursor;
  uint32_t scan[32];
  unsigned long long red[32];
  uint32_t item;
  unsigned hist[66];
  uint32_t uprefix[kLocalUnits + 1];
};

// A second-level position with this bit set walks the probe set instead (the reverse direction of
// a wing intersection); list positions stay below 2^31 (2m <= 2^32).
constexpr uint32_t kRevFlag = 0x80000000u;

// Flattened two-level iteration by one warp: first(j, L, sb) gives the second-level range
// [sb, sb + L) of first-level position j in [b, e); f(j, q) is called once per pair.
template <class First, class F>
__device__ __forceinline__ void warp_iter(uint32_t b, uint32_t e, First&& first, F&& f, const uint32_t* __restrict__ arr) {
  const unsigned lane = lane_id();
  for (uint32_t j0 = b; j0 < e; j0 += 32) {
    const uint32_t j = j0 + lane;
    uint32_t L = 0, sb = 0;
    if (j < e) first(j, L, sb);
    const uint32_t incl = warp_inclusive_scan(L);
    const uint32_t excl = incl - L;
    const uint32_t T = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t t0 = 0; t0 < T; t0 += 32) {
      const uint32_t t = t0 + lane;
      uint32_t lo = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        uint32_t x = __shfl_sync(0xffffffffu, incl, lo + step - 1);
        if (x <= t) lo += step;
      }
      const uint32_t ex = __shfl_sync(0xffffffffu, excl, lo);
      const uint32_t s = __shfl_sync(0xffffffffu, sb, lo);
      if (t < T) {
        const uint32_t q = s + (t - ex);
        f(j0 + lo, q, arr[q & ~kRevFlag]);
      }
    }
  }
}

__device__ __forceinline__ uint32_t block_incl_scan(uint32_t x, uint32_t* smem, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t incl = warp_inclusive_scan(x);
  if (lane == 31) smem[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t v = lane < nwarps ? smem[lane] : 0u;
    v = warp_inclusive_scan(v);
    smem[lane] = v;
  }
  __syncthreads();
  incl += warp > 0 ? smem[warp - 1] : 0u;
  total = smem[nwarps - 1];
  __syncthreads();
  return incl;
}

// Same iteration by the whole CTA.  Each chunk of kPT first-level positions has its second-level
// ranges cut into pieces of at most kPiece entries; warps claim pieces from a shared-memory
// counter, locate a piece's position once (binary search over the chunk's inclusive piece
// counts) and walk it with 32 lanes, so consecutive lanes read consecutive entries and no
// per-entry search is needed.
constexpr uint32_t kPiece = 128;

template <class First, class F>
__device__ __forceinline__ void block_iter(uint32_t b, uint32_t e, Shared& S, First&& first, F&& f,
                                           const uint32_t* __restrict__ arr) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  for (uint32_t j0 = b; j0 < e; j0 += kPT) {
    const uint32_t j = j0 + tid;
    uint32_t L = 0, sb = 0;
    if (j < e) first(j, L, sb);
    uint32_t T;
    const uint32_t incl = block_incl_scan((L + kPiece - 1) / kPiece, S.scan, T);
    S.incl[tid] = incl;
    S.sb[tid] = sb;
    S.len[tid] = L;
    if (tid == 0) S.cursor = 0;
    __syncthreads();
    while (true) {
      uint32_t p = 0;
      if (lane == 0) p = atomicAdd(&S.cursor, 1u);
      p = __shfl_sync(0xffffffffu, p, 0);
      if (p >= T) break;
      uint32_t lo = 0;
#pragma unroll
      for (uint32_t step = kPT / 2; step > 0; step >>= 1)
        if (S.incl[lo + step - 1] <= p) lo += step;
      const uint32_t k0 = (p - (lo ? S.incl[lo - 1] : 0u)) * kPiece;
      const uint32_t kend = min(k0 + kPiece, S.len[lo]);
      const uint32_t sbj = S.sb[lo], base = sbj & ~kRevFlag;
      // A piece is 4 x 32 entries: every lane issues its 4 loads before it uses any of them.
      uint32_t x[kPiece / 32];
#pragma unroll
      for (uint32_t r = 0; r < kPiece / 32; ++r) {
        const uint32_t k = k0 + lane + 32 * r;
        x[r] = k < kend ? arr[base + k] : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < kPiece / 32; ++r) {
        const uint32_t k = k0 + lane + 32 * r;
        if (k < kend) f(j0 + lo, sbj + k, x[r]);
      }
    }
    __syncthreads();
  }
}

// The same iteration restricted to flattened pair indices [lo, hi) (counted from the first
// pair of [b, e)); every CTA of the grid takes one slice of a huge item.
template <class First, class F>
__device__ __forceinline__ void block_iter_range(uint32_t b, uint32_t e, Shared& S, First&& first, F&& f,
                                                 uint64_t lo, uint64_t hi, const uint32_t* __restrict__ arr) {
  const uint32_t tid = threadIdx.x;
  uint64_t base = 0;
  for (uint32_t j0 = b; j0 < e && base < hi; j0 += kPT) {
    const uint32_t j = j0 + tid;
    uint32_t L = 0, sb = 0;
    if (j < e) first(j, L, sb);
    uint32_t T;
    const uint32_t incl = block_incl_scan(L, S.scan, T);
    S.incl[tid] = incl;
    S.sb[tid] = sb;
    __syncthreads();
    const uint64_t tb = lo > base ? lo - base : 0;
    const uint64_t te = (hi - base) < (uint64_t)T ? (hi - base) : (uint64_t)T;
    for (uint64_t t0 = tb; t0 < te; t0 += kPT) {
      const uint64_t tt = t0 + tid;
      if (tt < te) {
        const uint32_t t = (uint32_t)tt;
        uint32_t lo2 = 0;
#pragma unroll
        for (uint32_t step = kPT / 2; step > 0; step >>= 1)
          if (S.incl[lo2 + step - 1] <= t) lo2 += step;
        const uint32_t ex = lo2 ? S.incl[lo2 - 1] : 0u;
        const uint32_t q = S.sb[lo2] + (t - ex);
        f(j0 + lo2, q, arr[q & ~kRevFlag]);
      }
    }
    __syncthreads();
    base += T;
  }
}

// Sum of the second-level lengths of [b, e) (valid in every thread).
template <class First>
__device__ __forceinline__ uint64_t block_total(uint32_t b, uint32_t e, Shared& S, First&& first) {
  unsigned long long sum = 0;
  for (uint32_t j = b + threadIdx.x; j < e; j += kPT) {
    uint32_t L = 0, sb = 0;
    first(j, L, sb);
    sum += L;
  }
  sum = warp_sum(sum);
  if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = sum;
  __syncthreads();
  unsigned long long t = 0;
  for (int w = 0; w < kPT / 32; ++w) t += S.red[w];
  __syncthreads();
  return t;
}

__device__ __forceinline__ void touch(const Work& W, Ctl* ctl, unsigned par, uint32_t x) {
  if (W.touched[x] == 0 && atomicExch(&W.touched[x], 1u) == 0u) W.tlist[par][atomicAdd(&ctl->tlen[par], 1u)] = x;
}

// Window bound of the current round, per CTA (set at the start of every round).
__shared__ unsigned long long s_win_hi;

// Removes `amount` butterflies from an unpeeled item.  Only an item whose count falls below
// the window bound can reach the frontier before the next window advance, so only those are
// queued for re-bucketing; items that stay above it keep bucket == count implicitly (the
// advance resynchronises buckets from counts, when no unpeeled item is in the near list).
__device__ __forceinline__ bool mine(const Work& W, uint32_t x) { return !W.part || W.part[x] == W.my_part; }

__device__ __forceinline__ void dec(const Work& W, Ctl* ctl, unsigned par, uint32_t x, int64_t amount) {
  if (mine(W, x) && W.state[x] == ALIVE) {
    const long long old = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(&W.cnt[x]),
                                               (unsigned long long)(-amount));
    if ((unsigned long long)(old - amount) < s_win_hi) touch(W, ctl, par, x);
  }
}

// Per-thread accumulator keyed by the first-level position.
struct PosAcc {
  uint32_t j = kEmpty;
  int64_t acc = 0;
};

// ---- tip: process one frontier vertex -------------------------------------------------------
__device__ void tip_item_warp(const Lists& G, const Work& W, Ctl* ctl, unsigned par, uint32_t u, uint32_t* keys,
                              uint32_t* vals, unsigned long long& work) {
  const unsigned lane = lane_id();
  const int64_t wk = G.wk[u];
  const uint32_t tsize = max(64u, np2(2u * (uint32_t)wk));
  const uint32_t mask = tsize - 1;
  for (uint32_t s = lane; s < tsize; s += 32) { keys[s] = kEmpty; vals[s] = 0; }
  __syncwarp();
  warp_iter(G.offK[u], G.offK[u + 1],
            [&](uint32_t j, uint32_t& L, uint32_t& sb) {
              const uint32_t v = G.edgK[j];
              sb = G.offC[v];
              L = G.offC[v + 1] - sb;
            },
            [&](uint32_t, uint32_t, uint32_t u2) {
              if (u2 != u) t_add(keys, vals, mask, u2, ctl);
            },
            G.edgC);
  __syncwarp();
  for (uint32_t s = lane; s < tsize; s += 32) {
    const uint32_t k = keys[s];
    if (k == kEmpty) continue;
    const int64_t w = vals[s];
    if (w >= 2) dec(W, ctl, par, k, w * (w - 1) / 2);
  }
  if (lane == 0) work += (unsigned long long)wk;
  __syncwarp();
}

__device__ void tip_item_block(const Lists& G, const Work& W, Ctl* ctl, unsigned par, uint32_t u, uint32_t* table,
                               Shared& S, unsigned long long& work) {
  const int64_t wk = G.wk[u];
  const bool hash = (uint64_t)2 * (uint64_t)wk <= (uint64_t)kBlockSlots;
  uint32_t* keys = table;
  uint32_t* vals = table + kBlockSlots;
  uint32_t* gcnt = W.gscratch + (size_t)blockIdx.x * (size_t)W.gscratch_len;
  const uint32_t tsize = hash ? max(64u, np2(2u * (uint32_t)wk)) : 0u;
  const uint32_t mask = tsize - 1;
  if (hash)
    for (uint32_t s = threadIdx.x; s < tsize; s += kPT) { keys[s] = kEmpty; vals[s] = 0; }
  __syncthreads();
  auto first = [&](uint32_t j, uint32_t& L, uint32_t& sb) {
    const uint32_t v = G.edgK[j];
    sb = G.offC[v];
    L = G.offC[v + 1] - sb;
  };
  block_iter(G.offK[u], G.offK[u + 1], S, first, [&](uint32_t, uint32_t, uint32_t u2) {
    if (u2 == u) return;
    if (hash) t_add(keys, vals, mask, u2, ctl);
    else atomicAdd(&gcnt[u2], 1u);
  }, G.edgC);
  __syncthreads();
  if (hash) {
    for (uint32_t s = threadIdx.x; s < tsize; s += kPT) {
      const uint32_t k = keys[s];
      if (k == kEmpty) continue;
      const int64_t w = vals[s];
      if (w >= 2) dec(W, ctl, par, k, w * (w - 1) / 2);
    }
  } else {
    block_iter(G.offK[u], G.offK[u + 1], S, first, [&](uint32_t, uint32_t, uint32_t u2) {
      if (u2 == u) return;
      const int64_t w = atomicExch(&gcnt[u2], 0u);
      if (w >= 2) dec(W, ctl, par, u2, w * (w - 1) / 2);
    }, G.edgC);
  }
  if (threadIdx.x == 0) work += (unsigned long long)wk;
  __syncthreads();
}

// ---- wing: process one frontier edge --------------------------------------------------------
// Orientation A (walk from the centre v): probe set N(u) (centre -> edge), first level N(v)
// (u2, edge e2), second level N(u2) (v2, edge e3), probe v2 -> e4.
// Orientation B (walk from u): probe set N(v) (count-side vertex -> edge), first level N(u)
// (v2, e4), second level N(v2) (u2, e3), probe u2 -> e2.  Both find the same butterflies.

// Binary-searching a list of length dbig for each of dsmall keys beats scanning it.
__device__ __forceinline__ bool reverse_cheaper(uint32_t dsmall, uint32_t dbig) {
  return (uint64_t)dsmall * (uint64_t)(33u - __clz(dbig | 1u)) < (uint64_t)dbig;
}

struct WingEdge {
  uint32_t e1, u, v;
  bool from_v;
};

// An edge of a lower partition is gone; one of a higher partition is present and unpeeled.
__device__ __forceinline__ bool skip_edge(const Work& W, uint32_t e, uint32_t e1) {
  if (W.part) {
    const uint32_t p = W.part[e];
    if (p != W.my_part) return p < W.my_part;
  }
  const uint8_t s = W.state[e];
  return s == PEELED || (s == ACTIVE && e < e1);
}

__device__ __forceinline__ bool edge_gone(const Work& W, uint32_t e) {
  if (W.part) {
    const uint32_t p = W.part[e];
    if (p != W.my_part) return p < W.my_part;
  }
  return W.state[e] == PEELED;
}

// In this round's frontier with a smaller index than e1 (the tie rule).
__device__ __forceinline__ bool active_before(const Work& W, uint32_t e, uint32_t e1) {
  return e < e1 && mine(W, e) && W.state[e] == ACTIVE;
}

// Item granularity: one warp, one CTA, or the whole grid (huge items; all CTAs call it).
enum Level { LV_WARP = 0, LV_BLOCK = 1, LV_GRID = 2 };

template <int kLevel>
__device__ bool wing_item(const Lists& G, const Work& W, Ctl* ctl, unsigned par, const WingEdge& E, uint32_t* keys,
                          uint32_t* vals, uint32_t slots, Shared* S, unsigned long long& work, uint32_t chunk = 0,
                          uint32_t nchunks = 1, uint32_t chunk_end = 0) {
  // First-level slice: units [chunk, chunk_end) of nchunks (chunk_end 0: chunk + 1).
  if (chunk_end == 0) chunk_end = chunk + 1;
  const uint32_t rank = kLevel == LV_WARP ? lane_id() : (kLevel == LV_GRID ? vblock() * kPT + threadIdx.x : threadIdx.x);
  const uint32_t gsize = kLevel == LV_WARP ? 32 : (kLevel == LV_GRID ? vgrid() * kPT : kPT);
  auto sync = [&]() -> bool {
    if (kLevel == LV_WARP) { __syncwarp(); return true; }
    if (kLevel == LV_BLOCK) { __syncthreads(); return true; }
    return grid_barrier(ctl);
  };
  // Probe set: N(u) (keys: centres) when walking from v, else N(v) (keys: count-side ids).
  uint32_t pb, pe;
  if (E.from_v) { pb = G.offK[E.u]; pe = G.offK[E.u + 1]; }
  else { pb = G.offC[E.v]; pe = G.offC[E.v + 1]; }
  const uint32_t psize = pe - pb;
  const bool hash = kLevel != LV_GRID && 2 * psize <= slots;
  uint32_t* mark = kLevel == LV_GRID ? W.gshared : W.gscratch + (size_t)blockIdx.x * (size_t)W.gscratch_len;
  const uint32_t tsize = hash ? max(64u, np2(2u * psize)) : 0u;
  const uint32_t mask = tsize - 1;
  // hits[slot]: butterflies found through a probe-set edge, charged to it in one decrement once
  // the intersections are done (the table area holds keys, edges and hits).
  uint32_t* hits = vals + slots;
  if (hash)
    for (uint32_t s = rank; s < tsize; s += gsize) {
      keys[s] = kEmpty;
      hits[s] = 0;
    }
  if (!sync()) return false;
  for (uint32_t p = pb + rank; p < pe; p += gsize) {
    uint32_t key, e;
    if (E.from_v) { key = G.edgK[p]; e = G.eidK[p]; }
    else { key = G.edgC[p]; e = G.eidC[p]; }
    if (edge_gone(W, e)) continue;
    if (hash) t_put(keys, vals, mask, key, e, ctl);
    else mark[key] = e + 1;
  }
  if (!sync()) return false;
  // e: the probe-set edge of key; slot: its table slot (kEmpty for the dense markers).
  auto probe = [&](uint32_t key, uint32_t& e, uint32_t& slot) -> bool {
    if (hash) {
      slot = t_slot(keys, mask, key);
      if (slot == kEmpty) return false;
      e = vals[slot];
      return true;
    }
    slot = kEmpty;
    const uint32_t x = mark[key];
    if (!x) return false;
    e = x - 1;
    return true;
  };
  PosAcc acc;
  unsigned long long my_work = 0, my_rev = 0;
  auto flush = [&]() {
    if (acc.j != kEmpty && acc.acc) dec(W, ctl, par, E.from_v ? G.eidC[acc.j] : G.eidK[acc.j], acc.acc);
    acc.acc = 0;
  };
  // Each (first-level vertex x, probe set) intersection runs in one of two directions: scan
  // N(x) and probe the probe-set table, or (when the probe set is much shorter than N(x))
  // walk the probe set and binary-search N(x), which is sorted.  The direction rides in the
  // top bit of the second-level position.
  // One butterfly: e_list (unique to it) loses 1 now; the probe-set edge e_set loses 1 through
  // its hit counter when it has a table slot; the first-level edge through the accumulator.
  auto found = [&](uint32_t j, uint32_t e_list, uint32_t e_set, uint32_t slot) {
    dec(W, ctl, par, e_list, 1);
    if (slot != kEmpty) atomicAdd(&hits[slot], 1u);
    else dec(W, ctl, par, e_set, 1);
    if (j != acc.j) { flush(); acc.j = j; }
    acc.acc += 1;
  };
  // Second-level entries (and the probe set walked in the reverse direction) come from one list
  // array per orientation: N(u2) / N(u) in the count side's lists when walking from v, N(v2) /
  // N(v) in the centre side's lists when walking from u.
  const uint32_t* arr = E.from_v ? G.edgK : G.edgC;
  auto run = [&](uint32_t b, uint32_t e, auto&& first, auto&& f) {
    if (kLevel == LV_WARP) {
      warp_iter(b, e, first, f, arr);
    } else if (kLevel == LV_BLOCK) {
      block_iter(b, e, *S, first, f, arr);
    } else {
      const uint64_t T = block_total(b, e, *S, first);
      const uint64_t lo = T * vblock() / vgrid(), hi = T * (vblock() + 1) / vgrid();
      block_iter_range(b, e, *S, first, f, lo, hi, arr);
    }
  };
  if (E.from_v) {
    auto first = [&](uint32_t p, uint32_t& L, uint32_t& sb) {
      const uint32_t u2 = G.edgC[p];
      if (u2 == E.u || skip_edge(W, G.eidC[p], E.e1)) { L = 0; sb = 0; return; }
      const uint32_t b2 = G.offK[u2], d2 = G.offK[u2 + 1] - b2;
      if (reverse_cheaper(psize, d2)) { sb = pb | kRevFlag; L = psize; }
      else { sb = b2; L = d2; }
    };
    auto f = [&](uint32_t p, uint32_t q, uint32_t v2) {  // v2 = G.edgK[q without the flag]
      ++my_work;
      if (q & kRevFlag) {  // walk N(u), binary-search N(u2)
        ++my_rev;
        const uint32_t pos = q & ~kRevFlag;
        if (v2 == E.v) return;
        const uint32_t e4 = G.eidK[pos];
        if (skip_edge(W, e4, E.e1)) return;
        const uint32_t u2 = G.edgC[p];
        const uint32_t hi = G.offK[u2 + 1];
        const uint32_t at = lower_bound_u32(G.edgK, G.offK[u2], hi, v2);
        if (at == hi || G.edgK[at] != v2) return;
        const uint32_t e3 = G.eidK[at];
        if (skip_edge(W, e3, E.e1)) return;
        found(p, e3, e4, kEmpty);
        return;
      }
      if (v2 == E.v) return;
      uint32_t e4, slot;
      if (!probe(v2, e4, slot)) return;  // most probes miss: test the table before any global read
      const uint32_t e3 = G.eidK[q];
      if (skip_edge(W, e3, E.e1) || active_before(W, e4, E.e1)) return;
      found(p, e3, e4, slot);
    };
    const uint32_t b1 = G.offC[E.v], d1 = G.offC[E.v + 1] - b1;
    run(b1 + (uint32_t)((uint64_t)d1 * chunk / nchunks), b1 + (uint32_t)((uint64_t)d1 * chunk_end / nchunks), first, f);
  } else {
    auto first = [&](uint32_t q, uint32_t& L, uint32_t& sb) {
      const uint32_t v2 = G.edgK[q];
      if (v2 == E.v || skip_edge(W, G.eidK[q], E.e1)) { L = 0; sb = 0; return; }
      const uint32_t b2 = G.offC[v2], d2 = G.offC[v2 + 1] - b2;
      if (reverse_cheaper(psize, d2)) { sb = pb | kRevFlag; L = psize; }
      else { sb = b2; L = d2; }
    };
    auto f = [&](uint32_t q, uint32_t p3, uint32_t u2) {  // u2 = G.edgC[p3 without the flag]
      ++my_work;
      if (p3 & kRevFlag) {  // walk N(v), binary-search N(v2)
        ++my_rev;
        const uint32_t pos = p3 & ~kRevFlag;
        if (u2 == E.u) return;
        const uint32_t e2 = G.eidC[pos];
        if (skip_edge(W, e2, E.e1)) return;
        const uint32_t v2 = G.edgK[q];
        const uint32_t hi = G.offC[v2 + 1];
        const uint32_t at = lower_bound_u32(G.edgC, G.offC[v2], hi, u2);
        if (at == hi || G.edgC[at] != u2) return;
        const uint32_t e3 = G.eidC[at];
        if (skip_edge(W, e3, E.e1)) return;
        found(q, e3, e2, kEmpty);
        return;
      }
      if (u2 == E.u) return;
      uint32_t e2, slot;
      if (!probe(u2, e2, slot)) return;
      const uint32_t e3 = G.eidC[p3];
      if (skip_edge(W, e3, E.e1) || active_before(W, e2, E.e1)) return;
      found(q, e3, e2, slot);
    };
    const uint32_t b1 = G.offK[E.u], d1 = G.offK[E.u + 1] - b1;
    run(b1 + (uint32_t)((uint64_t)d1 * chunk / nchunks), b1 + (uint32_t)((uint64_t)d1 * chunk_end / nchunks), first, f);
  }
  flush();
  work += my_work;
  if (hash) {  // the probe-set edges' decrements, one per edge
    if (!sync()) return false;
    for (uint32_t s = rank; s < tsize; s += gsize) {
      const uint32_t h = hits[s];
      if (h && keys[s] != kEmpty) dec(W, ctl, par, vals[s], (int64_t)h);
    }
  }
  {
    const int mode = kLevel == LV_WARP ? 0 : (kLevel == LV_GRID ? 3 : (hash ? 1 : 2));
    const unsigned long long w = warp_sum((unsigned long long)my_work);
    const unsigned long long rw = warp_sum((unsigned long long)my_rev);
    if (lane_id() == 0) {
      if (w) atomicAdd(&ctl->mode_work[mode], w);
      if (rw) atomicAdd(&ctl->rev_work, rw);
    }
    if (rank == 0) atomicAdd(&ctl->mode_items[mode], 1ull);
  }
  if (!sync()) return false;
  if (!hash) {  // clear the dense markers
    for (uint32_t p = pb + rank; p < pe; p += gsize) mark[E.from_v ? G.edgK[p] : G.edgC[p]] = 0;
  }
  return sync();
}

// Huge tip item: every CTA aggregates one slice of u's two-hop list into grid-shared dense
// counters; a second pass reads and clears them (atomicExch), crediting each distinct u2 once.
__device__ bool tip_item_grid(const Lists& G, const Work& W, Ctl* ctl, unsigned par, uint32_t u, Shared& S,
                              unsigned long long& work) {
  auto first = [&](uint32_t j, uint32_t& L, uint32_t& sb) {
    const uint32_t v = G.edgK[j];
    sb = G.offC[v];
    L = G.offC[v + 1] - sb;
  };
  const uint64_t T = (uint64_t)G.wk[u] + (G.offK[u + 1] - G.offK[u]);
  const uint64_t lo = T * vblock() / vgrid(), hi = T * (vblock() + 1) / vgrid();
  uint32_t* cnt = W.gshared;
  block_iter_range(G.offK[u], G.offK[u + 1], S, first, [&](uint32_t, uint32_t, uint32_t u2) {
    if (u2 != u) atomicAdd(&cnt[u2], 1u);
  }, lo, hi, G.edgC);
  if (!grid_barrier(ctl)) return false;
  block_iter_range(G.offK[u], G.offK[u + 1], S, first, [&](uint32_t, uint32_t, uint32_t u2) {
    if (u2 == u) return;
    const int64_t w = atomicExch(&cnt[u2], 0u);
    if (w >= 2) dec(W, ctl, par, u2, w * (w - 1) / 2);
  }, lo, hi, G.edgC);
  if (vblock() == 0 && threadIdx.x == 0) work += T;
  return grid_barrier(ctl);
}

// The same for a group of gs CTAs (this CTA is number lb in it) with its own counter slice and
// barrier: several heavy tip items of a round run at once, one per group.  The caller's grid
// barrier after the group's item separates it from the next use of the slice.
__device__ bool tip_item_group(const Lists& G, const Work& W, Ctl* ctl, unsigned par, uint32_t u, Shared& S,
                               unsigned long long& work, unsigned lb, unsigned gs, unsigned slot, uint32_t* cnt) {
  auto first = [&](uint32_t j, uint32_t& L, uint32_t& sb) {
    const uint32_t v = G.edgK[j];
    sb = G.offC[v];
    L = G.offC[v + 1] - sb;
  };
  const uint64_t T = (uint64_t)G.wk[u] + (G.offK[u + 1] - G.offK[u]);
  const uint64_t lo = T * lb / gs, hi = T * (lb + 1) / gs;
  block_iter_range(G.offK[u], G.offK[u + 1], S, first, [&](uint32_t, uint32_t, uint32_t u2) {
    if (u2 != u) atomicAdd(&cnt[u2], 1u);
  }, lo, hi, G.edgC);
  if (!group_barrier(ctl, slot, gs)) return false;
  block_iter_range(G.offK[u], G.offK[u + 1], S, first, [&](uint32_t, uint32_t, uint32_t u2) {
    if (u2 == u) return;
    const int64_t w = atomicExch(&cnt[u2], 0u);
    if (w >= 2) dec(W, ctl, par, u2, w * (w - 1) / 2);
  }, lo, hi, G.edgC);
  if (lb == 0 && threadIdx.x == 0) work += T;
  return true;
}

// ---- the persistent kernel ------------------------------------------------------------------
// Wing items run on one warp when their work is small and their probe set fits a warp table.
struct Classify {
  int64_t small_work;
  int64_t huge_work;   // items above this run on the whole grid
  int64_t chunk_work;  // target probes per work unit of a CTA-level wing item
  int64_t units_per_cta;  // work units per CTA a round's CTA-level wing work is cut into
  int64_t warp_units;     // wing: every item with a warp-sized probe set runs as warp units

  __device__ __forceinline__ bool tip_small(const Lists& G, uint32_t u) const {
    return G.wk[u] <= kWarpSlots / 2 && G.wk[u] <= small_work;
  }
  // Estimated probes from each side: the two-hop list sizes, capped by deg(u)*deg(v) times a
  // binary-search factor (the reverse-direction intersections).
  __device__ __forceinline__ int64_t cost_v(const Lists& G, uint32_t v, uint32_t u) const {
    const int64_t du = G.offK[u + 1] - G.offK[u], dv = G.offC[v + 1] - G.offC[v];
    return min(G.S[G.nK + v], du * dv * 16);
  }
  __device__ __forceinline__ int64_t cost_u(const Lists& G, uint32_t v, uint32_t u) const {
    const int64_t du = G.offK[u + 1] - G.offK[u], dv = G.offC[v + 1] - G.offC[v];
    return min(G.S[u], du * dv * 16);
  }
  __device__ __forceinline__ bool wing_from_v(const Lists& G, uint32_t v, uint32_t u) const {
    return cost_v(G, v, u) <= cost_u(G, v, u);
  }
  __device__ __forceinline__ bool tip_huge(const Lists& G, uint32_t u) const { return G.wk[u] > huge_work; }
};

// Estimated work of peeling item x (plus one, so that items without work still count): the
// cheaper side's two-hop probes of a wing item, the two-hop wedges of a tip item.
template <bool kWing>
__device__ __forceinline__ unsigned long long item_weight(const Lists& G, const Classify& cls, uint32_t x) {
  if (kWing) {
    const uint32_t v = G.center_of[x], u = G.u_of[x];
    const int64_t c = min(cls.cost_v(G, v, u), cls.cost_u(G, v, u));
    return 1ull + (unsigned long long)(c > 0 ? c : 0);
  }
  return 1ull + (unsigned long long)(G.wk[x] > 0 ? G.wk[x] : 0);
}

// The peel instances of one launch.  n == 1: the whole grid runs instance 0.  Otherwise CTA b
// runs instances cta_beg[b] .. cta_end[b] - 1 one after another; instance i spans the ncta[i]
// CTAs from first[i] (heavy graphs get many CTAs, light graphs share one CTA in turn).
struct Instances {
  const Work* W;
  const uint32_t* first;
  const uint32_t* ncta;
  const uint32_t* cta_beg;
  const uint32_t* cta_end;
  uint32_t n;
};

// All rounds of one peel instance, run by its CTAs; false when a bounded wait ran out or an
// invariant broke (recorded in ctl->err).
template <bool kWing>
__device__ bool peel_instance(const Lists& G, const Work& W, Ctl* ctl, const Classify& cls) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Shared& S = *reinterpret_cast<Shared*>(smem_raw);
  uint32_t* pool = reinterpret_cast<uint32_t*>(smem_raw + ((sizeof(Shared) + 15) & ~size_t(15)));
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* wkeys = pool + warp * (3 * kWarpSlots);  // keys, values, hit counters
  uint32_t* wvals = wkeys + kWarpSlots;
  const unsigned gtid = vblock() * kPT + threadIdx.x;
  const unsigned gthreads = vgrid() * kPT;
  unsigned alist_cur = *(volatile unsigned*)&ctl->alist_cur;
  const bool range = *(volatile unsigned*)&ctl->range_mode != 0;
  unsigned part_idx = *(volatile unsigned*)&ctl->npart;  // partitions opened (range mode)
  unsigned long long work = 0;
  if (!*(volatile unsigned*)&ctl->started) {
    for (int64_t x = gtid; x < W.N; x += gthreads)
      W.alist[0][x] = W.items ? W.items[W.item0 + x] : W.item0 + (uint32_t)x;
    if (!grid_barrier(ctl)) return false;
    if (vblock() == 0 && threadIdx.x == 0) ctl->started = 1;
  }

  for (unsigned long long r = *(volatile unsigned long long*)&ctl->round;; ++r) {
    const unsigned par = (unsigned)(r & 1ull), npar = par ^ 1u;
    const unsigned alive = *(volatile unsigned*)&ctl->alive;
    if (alive == 0) break;
    // Pause at a round boundary once enough items have been peeled since the lists were last
    // compacted; the host compacts them and relaunches (all CTAs see the same values here).
    const unsigned at_compact = *(volatile unsigned*)&ctl->alive_at_compact;
    if (2u * alive < at_compact && at_compact - alive >= *(volatile unsigned*)&ctl->min_gain) {
      if (vblock() == 0 && threadIdx.x == 0) {
        ctl->round = r;
        ctl->alist_cur = alist_cur;
      }
      break;
    }
    unsigned long long k = *(volatile unsigned long long*)&ctl->nm[par];
    if (k == kInf) {
      unsigned long long part_target_next = 0, part_ratio_next = 0;  // range mode
      // ---- window advance (no unpeeled item left in the near list): compact the alive list
      // and take its minimum; a log2 histogram of distances to the minimum picks the window
      // bound; the near list is rebuilt from the alive list.
      const unsigned na = alist_cur ^ 1u;
      const unsigned alen = *(volatile unsigned*)&ctl->alen[alist_cur];
      unsigned long long mn = kInf;
      for (unsigned q = gtid; q < alen; q += gthreads) {
        const uint32_t x = W.alist[alist_cur][q];
        if (W.state[x] != ALIVE) continue;
        W.alist[na][atomicAdd(&ctl->alen[na], 1u)] = x;
        // No unpeeled item is in the near list here, and items outside it were queued only
        // when they fell below the bound: their bucket is their count.
        const int64_t c = W.cnt[x];
        W.D[x] = c;
        mn = min(mn, (unsigned long long)c);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      if (lane == 0 && mn != kInf) atomicMin(&ctl->k_lo, mn);
      if (threadIdx.x < 66) S.hist[threadIdx.x] = 0;
      if (vblock() == 0) {
        // The previous advance's histograms were last read before two barriers ago.
        if (threadIdx.x < 66) {
          ctl->hist[threadIdx.x] = 0;
          ctl->whist[threadIdx.x] = 0;
        }
        if (range && threadIdx.x < 256) ctl->wsub[threadIdx.x] = 0;
        if (threadIdx.x == 0) ctl->near_len = 0;
      }
      if (!grid_barrier(ctl)) return false;
      if (range) {
        ++part_idx;  // the window opened here is partition part_idx - 1
        if (vblock() == 0 && threadIdx.x == 0) ctl->npart = part_idx;
      }
      const unsigned long long klo = *(volatile unsigned long long*)&ctl->k_lo;
      const unsigned alen2 = *(volatile unsigned*)&ctl->alen[na];
      unsigned long long hi = kInf;
      if (!range) {
        for (unsigned q = gtid; q < alen2; q += gthreads) {
          const unsigned long long d = (unsigned long long)W.D[W.alist[na][q]] - klo;
          atomicAdd(&S.hist[d ? 64 - __clzll(d) : 0], 1u);
        }
        __syncthreads();
        if (threadIdx.x < 66 && S.hist[threadIdx.x]) atomicAdd(&ctl->hist[threadIdx.x], S.hist[threadIdx.x]);
        if (!grid_barrier(ctl)) return false;
        // Every CTA derives the same bound: the smallest B with >= target items at distance < 2^B.
        const unsigned target = max(ctl->near_min, alen2 / max(1u, ctl->near_div));
        unsigned cum = 0;
        int B = 0;
        for (; B < 65; ++B) {
          cum += *(volatile unsigned*)&ctl->hist[B];
          if (cum >= target) break;
        }
        if (B < 63) {
          const unsigned long long span = 1ull << B;
          if (klo <= kInf - span) hi = klo + span;
        }
      } else {
        // Partition bound: about part_target of estimated work below it.  A log2 histogram of
        // distances to the minimum (weighted by work) picks the octave, a 256-bin linear
        // histogram inside it the bound.  The bins live in the (idle) table pool.
        unsigned long long* wh = reinterpret_cast<unsigned long long*>(pool);
        if (threadIdx.x < 66) wh[threadIdx.x] = 0;
        __syncthreads();
        for (unsigned q = gtid; q < alen2; q += gthreads) {
          const uint32_t x = W.alist[na][q];
          const unsigned long long d = (unsigned long long)W.D[x] - klo;
          atomicAdd(&wh[d ? 64 - __clzll(d) : 0], (unsigned long long)W.wgt[x]);
        }
        __syncthreads();
        if (threadIdx.x < 66 && wh[threadIdx.x]) atomicAdd(&ctl->whist[threadIdx.x], wh[threadIdx.x]);
        if (!grid_barrier(ctl)) return false;
        const unsigned long long base = *(volatile unsigned long long*)&ctl->part_target;
        const unsigned long long done = *(volatile unsigned long long*)&ctl->part_done;
        const unsigned long long used = *(volatile unsigned long long*)&ctl->part_used;
        unsigned long long ratio_q = *(volatile unsigned long long*)&ctl->part_ratio_q;
        if (used > 0 && done > 0) {
          const unsigned long long r = min(done * 256ull / used, 256ull * 4096ull);
          ratio_q = ratio_q ? (ratio_q + r) / 2 : r;
        }
        const unsigned long long target = max(1ull, ratio_q > 256 ? base * 256ull / ratio_q : base);
        part_target_next = target;
        part_ratio_next = ratio_q;
        unsigned long long cum = 0;
        int B = 0;
        for (; B < 65; ++B) {
          const unsigned long long w = *(volatile unsigned long long*)&ctl->whist[B];
          if (cum + w >= target) break;
          cum += w;
        }
        if (B == 0) {
          hi = klo + 1;
        } else if (B < 63) {
          const unsigned long long lo_d = 1ull << (B - 1), width = lo_d;  // distances [2^(B-1), 2^B)
          __syncthreads();
          if (threadIdx.x < 256) wh[threadIdx.x] = 0;
          __syncthreads();
          for (unsigned q = gtid; q < alen2; q += gthreads) {
            const uint32_t x = W.alist[na][q];
            const unsigned long long d = (unsigned long long)W.D[x] - klo;
            if (d >= lo_d && d < lo_d + width)
              atomicAdd(&wh[(unsigned)((d - lo_d) * 256ull / width)], (unsigned long long)W.wgt[x]);
          }
          __syncthreads();
          if (threadIdx.x < 256 && wh[threadIdx.x]) atomicAdd(&ctl->wsub[threadIdx.x], wh[threadIdx.x]);
          if (!grid_barrier(ctl)) return false;
          unsigned j = 0;
          for (; j < 255; ++j) {
            cum += *(volatile unsigned long long*)&ctl->wsub[j];
            if (cum >= target) break;
          }
          // Bin j covers distances [lo_d + ceil(j w / 256), lo_d + ceil((j + 1) w / 256)).
          const unsigned long long end_d = lo_d + ((unsigned long long)(j + 1) * width + 255ull) / 256ull;
          if (klo <= kInf - end_d) hi = klo + end_d;
        }
      }
      for (unsigned q = gtid; q < alen2; q += gthreads) {
        const uint32_t x = W.alist[na][q];
        if (hi == kInf || (unsigned long long)W.D[x] < hi) {
          W.in_near[x] = 1;
          W.near[atomicAdd(&ctl->near_len, 1u)] = x;
        }
      }
      if (vblock() == 0 && threadIdx.x == 0) {
        ctl->win_hi = hi;
        ctl->alen[alist_cur] = 0;  // read by every CTA before the first barrier
        ctl->k_lo = kInf;          // read by every CTA right after the first barrier
      }
      alist_cur = na;
      if (!grid_barrier(ctl)) return false;
      phase_mark(ctl, 0);
      if (vblock() == 0 && threadIdx.x == 0) {
        ctl->advances += 1;
        if (range) {  // every CTA read the previous values before this barrier
          ctl->part_used = part_target_next;
          ctl->part_ratio_q = part_ratio_next;
          ctl->part_done = 0;
        }
      }
      k = klo;
    }
    const unsigned long long win_hi = *(volatile unsigned long long*)&ctl->win_hi;
    if (threadIdx.x == 0) s_win_hi = win_hi;
    __syncthreads();
    // ---- phase F: the frontier is every near item in bucket k; the minimum of the other near
    // items is the first part of the next round's minimum.
    {
      const unsigned nl = *(volatile unsigned*)&ctl->near_len;
      unsigned long long mn = kInf;
      for (unsigned q = gtid; q < nl; q += gthreads) {
        const uint32_t x = W.near[q];
        if (W.state[x] != ALIVE) continue;
        const unsigned long long d = (unsigned long long)W.D[x];
        if (range || d == k) {
          W.state[x] = ACTIVE;
          bool small, huge;
          int64_t cost;
          uint32_t wunits_of = 1;
          if (kWing) {
            const uint32_t v = G.center_of[x], u = G.u_of[x];
            const int64_t cv = cls.cost_v(G, v, u), cu = cls.cost_u(G, v, u);
            const bool fv = cv <= cu;
            cost = fv ? cv : cu;
            const uint32_t psize = fv ? G.offK[u + 1] - G.offK[u] : G.offC[v + 1] - G.offC[v];
            // Warp-unit setting: every item whose probe set fits a warp table runs on warps, cut
            // into warp units of about chunk_work probes (first-level slices).  Otherwise only
            // items of at most small_work probes run on warps, whole.
            small = 2 * psize <= (uint32_t)kWarpSlots && (cls.warp_units || cost <= cls.small_work);
            huge = !small && cost > cls.huge_work && W.gshared != nullptr;
            if (small && cls.warp_units) {
              const int64_t d1 = fv ? G.offC[v + 1] - G.offC[v] : G.offK[u + 1] - G.offK[u];
              int64_t units = (cost + cls.chunk_work - 1) / cls.chunk_work;
              units = min(units, min(d1, (int64_t)4096));
              wunits_of = (uint32_t)max(units, (int64_t)1);
            }
          } else {
            cost = G.wk[x];
            small = cls.tip_small(G, x);
            huge = !small && cls.tip_huge(G, x) && W.gshared != nullptr;
          }
          atomicAdd(&ctl->round_est[par], (unsigned long long)(cost > 0 ? cost : 0));
          if (small) {
            const unsigned at = atomicAdd(&ctl->flen_small[par], 1u);
            W.fsmall[par][at] = x;
            if (kWing) W.fwchunks[par][at] = wunits_of;
          }
          else if (huge) W.fhuge[par][atomicAdd(&ctl->flen_huge[par], 1u)] = x;
          else {
            const unsigned at = atomicAdd(&ctl->flen_big[par], 1u);
            W.fbig[par][at] = x;
            const int64_t c = cost < 1 ? 1 : (cost > 0x7fffffff ? 0x7fffffff : cost);
            W.fchunks[par][at] = (uint32_t)c;  // cost for now; CTA 0 turns it into a unit count
            atomicAdd(&ctl->round_cost[par], (unsigned long long)c);
          }
        } else {
          mn = min(mn, d);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      if (lane == 0 && mn != kInf) atomicMin(&ctl->nm[npar], mn);
      if (vblock() == 0 && threadIdx.x == 0) {  // slots of the previous round, no longer read
        ctl->flen_small[npar] = 0;
        ctl->flen_big[npar] = 0;
        ctl->flen_huge[npar] = 0;
        ctl->round_cost[npar] = 0;
        ctl->round_est[npar] = 0;
        ctl->tlen[npar] = 0;
        ctl->cur_small[npar] = 0;
        ctl->cur_big[npar] = 0;
        ctl->scanned += nl;
      }
    }
    if (!grid_barrier(ctl)) return false;
    phase_mark(ctl, 1);
    // ---- phase P: process the frontier (small items per warp, then heavy items per CTA).
    {
      if (vblock() == 0 && threadIdx.x == 0) ctl->nm[par] = kInf;  // every CTA has read it
      const unsigned ns = *(volatile unsigned*)&ctl->flen_small[par];
      if (!kWing) {
        while (true) {
          unsigned q = 0;
          if (lane == 0) q = atomicAdd(&ctl->cur_small[par], 1u);
          q = __shfl_sync(0xffffffffu, q, 0);
          if (q >= ns) break;
          const uint32_t x = W.fsmall[par][q];
          if (W.cnt[x] == 0) continue;  // no live butterfly contains x: nothing to remove
          tip_item_warp(G, W, ctl, par, x, wkeys, wvals, work);
        }
      } else if (ns) {
        // Warp units: the exclusive prefix of the warp items' unit counts (every CTA computes it
        // in shared memory up to kLocalUnits items, else CTA 0 in global memory behind a
        // barrier); warps claim runs of consecutive units and process an item's units of a
        // run as one first-level slice, independently of the other warps.
        const bool wlocal = ns <= kLocalUnits;
        if (wlocal || vblock() == 0) {
          uint32_t carry = 0;
          for (uint32_t j0 = 0; j0 < ns; j0 += kPT) {
            const uint32_t j = j0 + threadIdx.x;
            const uint32_t c = j < ns ? W.fwchunks[par][j] : 0u;
            uint32_t T;
            const uint32_t incl = block_incl_scan(c, S.scan, T);
            if (j < ns) {
              if (wlocal) S.uprefix[j] = carry + incl - c;
              else W.wprefix[j] = carry + incl - c;
            }
            carry += T;
          }
          if (threadIdx.x == 0) {
            if (wlocal) S.uprefix[ns] = carry;
            else {
              W.wprefix[ns] = carry;
              ctl->wunits = carry;
            }
          }
        }
        if (wlocal) __syncthreads();
        else if (!grid_barrier(ctl)) return false;
        const uint32_t* wpre = wlocal ? S.uprefix : W.wprefix;
        const unsigned nwu = wlocal ? S.uprefix[ns] : *(volatile unsigned*)&ctl->wunits;
        const unsigned Kw = max(1u, nwu / (4u * vgrid() * (kPT / 32)));
        while (true) {
          unsigned u = 0;
          if (lane == 0) u = atomicAdd(&ctl->cur_small[par], Kw);
          u = __shfl_sync(0xffffffffu, u, 0);
          if (u >= nwu) break;
          uint32_t lo = 0, hi = ns;  // the last item whose prefix <= u, 32-way search
          while (hi - lo > 1) {
            const uint32_t step = (hi - lo + 31) / 32;
            const uint32_t idx = lo + lane * step;
            const bool le = idx < hi && wpre[idx] <= u;
            const unsigned bal = __ballot_sync(0xffffffffu, le);
            lo = lo + (31 - __clz(bal)) * step;
            hi = min(lo + step, hi);
          }
          const unsigned uend = min(u + Kw, nwu);
          for (unsigned uu = u, q = lo; uu < uend; ++q) {  // uniform across the warp
            const uint32_t base = wpre[q], next = wpre[q + 1];
            const uint32_t c1 = min(uend, next);
            const uint32_t x = W.fsmall[par][q];
            if (W.cnt[x] != 0) {  // no live butterfly contains x: nothing to remove
              WingEdge E;
              E.e1 = x;
              E.v = G.center_of[x];
              E.u = G.u_of[x];
              E.from_v = cls.wing_from_v(G, E.v, E.u);
              wing_item<LV_WARP>(G, W, ctl, par, E, wkeys, wvals, kWarpSlots, nullptr, work, uu - base, next - base,
                                 c1 - base);
            }
            uu = c1;
          }
        }
      }
      __syncthreads();  // warp tables and the CTA table share memory
      const unsigned nb = *(volatile unsigned*)&ctl->flen_big[par];
      if (nb) {
        // Units: the exclusive prefix of the items' unit counts; every CTA then pulls units
        // (item, slice) from a shared cursor.  Up to kLocalUnits items every CTA computes the
        // same prefix in its shared memory (from the costs phase F froze), so no grid barrier
        // is needed; beyond that CTA 0 lays it out in global memory behind a barrier.
        const bool local = nb <= kLocalUnits;
        if (local || vblock() == 0) {
          uint32_t carry = 0;
          // Unit size: about cls.units_per_cta units per CTA over the round's CTA-level work,
          // never below cls.chunk_work probes or four probe-set sizes (each unit rebuilds its
          // probe table).
          const unsigned long long rc = *(volatile unsigned long long*)&ctl->round_cost[par];
          const int64_t target =
              max((int64_t)cls.chunk_work, (int64_t)(rc / ((unsigned long long)cls.units_per_cta * vgrid())));
          for (uint32_t j0 = 0; j0 < nb; j0 += kPT) {
            const uint32_t j = j0 + threadIdx.x;
            uint32_t c = 0;
            if (j < nb) {
              if (kWing) {
                const uint32_t x = W.fbig[par][j];
                const uint32_t v = G.center_of[x], u = G.u_of[x];
                const bool fv = cls.wing_from_v(G, v, u);
                const int64_t psize = fv ? G.offK[u + 1] - G.offK[u] : G.offC[v + 1] - G.offC[v];
                const int64_t d1 = fv ? G.offC[v + 1] - G.offC[v] : G.offK[u + 1] - G.offK[u];
                const int64_t unit = max(target, 4 * psize);
                int64_t k = ((int64_t)W.fchunks[par][j] + unit - 1) / unit;
                k = min(k, min(d1, (int64_t)4096));
                c = (uint32_t)max(k, (int64_t)1);
              } else {
                c = 1;
              }
              if (!local) W.fchunks[par][j] = c;
            }
            uint32_t T;
            const uint32_t incl = block_incl_scan(c, S.scan, T);
            if (j < nb) {
              if (local) S.uprefix[j] = carry + incl - c;
              else W.uprefix[j] = carry + incl - c;
            }
            carry += T;
          }
          if (threadIdx.x == 0) {
            if (local) {
              S.uprefix[nb] = carry;
            } else {
              W.uprefix[nb] = carry;
              ctl->units = carry;
            }
          }
        }
        if (local) __syncthreads();
        else if (!grid_barrier(ctl)) return false;
        const uint32_t* upre = local ? S.uprefix : W.uprefix;
        const unsigned nu = local ? S.uprefix[nb] : *(volatile unsigned*)&ctl->units;
        // CTAs claim runs of K consecutive units (wing: about a quarter of a CTA's share; tip: one
        // unit, which is one item); the units of one item inside a run are processed as one
        // slice, so the item's probe table is built once per run, not once per unit.
        const unsigned K = kWing ? max(1u, nu / (4u * vgrid())) : 1u;
        while (true) {
          if (threadIdx.x < 32) {  // warp 0: take a run, find the item of its first unit, 32-way
            unsigned u = 0;
            if (lane == 0) u = atomicAdd(&ctl->cur_big[par], K);
            u = __shfl_sync(0xffffffffu, u, 0);
            uint32_t lo = 0, hi = nb;  // answer in [lo, hi): the last item whose prefix <= u
            if (u < nu) {
              while (hi - lo > 1) {
                const uint32_t step = (hi - lo + 31) / 32;
                const uint32_t idx = lo + lane * step;
                const bool le = idx < hi && upre[idx] <= u;
                const unsigned bal = __ballot_sync(0xffffffffu, le);
                const uint32_t last = 31 - __clz(bal);  // lane 0 always qualifies (prefix[lo] <= u)
                lo = lo + last * step;
                hi = min(lo + step, hi);
              }
            }
            if (lane == 0) {
              S.item = u;
              S.hist[0] = lo;
            }
          }
          __syncthreads();
          const unsigned u0 = S.item, q0 = S.hist[0];
          __syncthreads();
          if (u0 >= nu) break;
          const unsigned uend = min(u0 + K, nu);
          for (unsigned uu = u0, q = q0; uu < uend; ++q) {  // uniform across the CTA
            const uint32_t base = upre[q], next = upre[q + 1];
            const uint32_t c1 = min(uend, next);
            const uint32_t x = W.fbig[par][q];
            if (W.cnt[x] != 0) {  // no live butterfly contains x: nothing to remove
              if (kWing) {
                WingEdge E;
                E.e1 = x;
                E.v = G.center_of[x];
                E.u = G.u_of[x];
                E.from_v = cls.wing_from_v(G, E.v, E.u);
                wing_item<LV_BLOCK>(G, W, ctl, par, E, pool, pool + kBlockSlots, kBlockSlots, &S, work, uu - base,
                                    next - base, c1 - base);
              } else {
                tip_item_block(G, W, ctl, par, x, pool, S, work);
              }
            }
            uu = c1;
          }
        }
      }
      // Huge items: tip items in waves of up to ngroups at once, one per CTA group (equal
      // splits of the instance's CTAs); otherwise one at a time over every CTA.
      const unsigned nh = *(volatile unsigned*)&ctl->flen_huge[par];
      const unsigned ng = kWing ? 1u : min(W.ngroups, vgrid());
      if (!kWing && nh > 1 && ng > 1) {
        const unsigned vg = vgrid(), vb = vblock();
        for (unsigned w0 = 0; w0 < nh; w0 += ng) {
          const unsigned gn = min(ng, nh - w0);
          const unsigned grp = vb * gn / vg;
          const unsigned g0 = (grp * vg + gn - 1) / gn, g1 = ((grp + 1) * vg + gn - 1) / gn;
          const uint32_t x = W.fhuge[par][w0 + grp];
          if (W.cnt[x] != 0 &&  // uniform across the group
              !tip_item_group(G, W, ctl, par, x, S, work, vb - g0, g1 - g0, grp,
                              W.gshared + (size_t)grp * (size_t)W.gshared_stride))
            return false;
          if (w0 + ng < nh && !grid_barrier(ctl)) return false;  // the slices are reused next wave
        }
      }
      for (unsigned q = 0; q < nh && (kWing || nh == 1 || ng <= 1); ++q) {
        const uint32_t x = W.fhuge[par][q];
        if (W.cnt[x] == 0) continue;  // frontier counts do not change during the phase
        bool ok;
        if (kWing) {
          WingEdge E;
          E.e1 = x;
          E.v = G.center_of[x];
          E.u = G.u_of[x];
          E.from_v = cls.wing_from_v(G, E.v, E.u);
          ok = wing_item<LV_GRID>(G, W, ctl, par, E, nullptr, nullptr, 0, &S, work);
        } else {
          ok = tip_item_grid(G, W, ctl, par, x, S, work);
        }
        if (!ok) return false;
      }
    }
    if (!grid_barrier(ctl)) return false;
    phase_mark(ctl, 2, vblock() == 0 && threadIdx.x == 0 ? *(volatile unsigned long long*)&ctl->round_est[par] : 0);
    // ---- phase U: touched items move to bucket max(count, k) (all unpeeled items are above
    // k here); those entering the window join the near list and feed the next minimum.
    {
      const unsigned nt = *(volatile unsigned*)&ctl->tlen[par];
      unsigned long long mn = kInf;
      for (unsigned q = gtid; q < nt; q += gthreads) {
        const uint32_t x = W.tlist[par][q];
        W.touched[x] = 0;
        if (W.state[x] != ALIVE) continue;
        const int64_t c = W.cnt[x];
        // Range mode keeps D (the count at the partition's start) and queues by count.
        const int64_t nd = range ? c : (c > (int64_t)k ? c : (int64_t)k);
        if (!range) W.D[x] = nd;
        if ((unsigned long long)nd < win_hi) {
          mn = min(mn, (unsigned long long)nd);
          if (!W.in_near[x]) {
            W.in_near[x] = 1;
            W.near[atomicAdd(&ctl->near_len, 1u)] = x;
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      if (lane == 0 && mn != kInf) atomicMin(&ctl->nm[npar], mn);
      const unsigned ns = *(volatile unsigned*)&ctl->flen_small[par];
      const unsigned nb = *(volatile unsigned*)&ctl->flen_big[par];
      const unsigned nh = *(volatile unsigned*)&ctl->flen_huge[par];
      for (unsigned q = gtid; q < ns + nb + nh; q += gthreads) {
        const uint32_t x = q < ns ? W.fsmall[par][q] : (q < ns + nb ? W.fbig[par][q - ns] : W.fhuge[par][q - ns - nb]);
        W.state[x] = PEELED;
        if (range) W.part_out[x] = part_idx - 1;
      }
      if (vblock() == 0 && threadIdx.x == 0) {
        ctl->alive -= ns + nb + nh;
        ctl->rounds += 1;
        ctl->touched_total += nt;
        ctl->n_small += ns;
        ctl->n_big += nb;
        ctl->n_huge += nh;
        ctl->prev_items = ns + nb + nh;  // read by the next round's phase F after two barriers
        if (range) ctl->part_done += *(volatile unsigned long long*)&ctl->round_est[par];
      }
    }
    if (!grid_barrier(ctl)) return false;
    phase_mark(ctl, 3);
  }
  unsigned long long w = work;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
  if (lane == 0 && w) atomicAdd(&ctl->work, w);
  return true;
}

// kMinBlocks: CTAs per SM the register allocation must allow.  2 caps a thread at 64 registers
// (some spill); 1 leaves about 108 and no spills, at half the resident warps.  The single-
// instance tip peel runs faster on the latter (fewer CTAs also shorten its grid barriers: R-MAT
// 2^24, one round at a time, 2.36 s -> 1.60 s); wing peeling and batches keep two CTAs per SM
// (the wing peel's intersections need the warps: 18.5 s against 19.6 s).
template <bool kWing, int kMinBlocks>
__global__ void __launch_bounds__(kPT, kMinBlocks) peel_kernel(Lists G, const Lists* levels, Instances I, Ctl* ctls,
                                                               Classify cls) {
  // levels: the live-list versions of a two-phase fine pass (an instance reads
  // levels[W.level]); null: every instance reads G.
  __shared__ Work sW;
  __shared__ Lists sG;
  const unsigned ib = I.n > 1 ? I.cta_beg[blockIdx.x] : 0u, ie = I.n > 1 ? I.cta_end[blockIdx.x] : 1u;
  for (unsigned inst = ib; inst < ie; ++inst) {
    if (threadIdx.x == 0) {
      s_vb = I.n > 1 ? blockIdx.x - I.first[inst] : blockIdx.x;
      s_vg = I.n > 1 ? I.ncta[inst] : gridDim.x;
      sW = I.W[inst];
      sG = levels ? levels[sW.level] : G;
    }
    __syncthreads();
    if (!peel_instance<kWing>(sG, sW, ctls + inst, cls)) return;
    __syncthreads();
  }
}

// ---- set-up kernels -------------------------------------------------------------------------
__global__ void peel_init_kernel(const int64_t* __restrict__ counts, int64_t N, int64_t* D, int64_t* cnt,
                                 uint8_t* state, uint8_t* in_near, uint32_t* touched) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < N; x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = counts[x];
    D[x] = c;
    cnt[x] = c;
    state[x] = ALIVE;
    in_near[x] = 0;
    touched[x] = 0;
  }
}

// wk[u] = sum over v in N(u) of (deg(v) - 1): the two-hop wedges of a count-side vertex.
__global__ void tip_work_kernel(const uint32_t* __restrict__ offK, const uint32_t* __restrict__ edgK,
                                const uint32_t* __restrict__ offC, int64_t nK, int64_t* wk) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t u = warp; u < nK; u += nwarps) {
    int64_t s = 0;
    for (uint32_t j = offK[u] + lane; j < offK[u + 1]; j += 32) {
      const uint32_t v = edgK[j];
      s += (int64_t)(offC[v + 1] - offC[v]) - 1;
    }
    s = warp_sum(s);
    if (lane == 0) wk[u] = s;
  }
}

// S[x] = sum over neighbours y of deg(y), for both sides (count side first).
__global__ void nbr_degree_sum_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ edg,
                                      const uint32_t* __restrict__ off_other, int64_t n, int64_t* S) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t x = warp; x < n; x += nwarps) {
    int64_t s = 0;
    for (uint32_t j = off[x] + lane; j < off[x + 1]; j += 32) {
      const uint32_t y = edg[j];
      s += (int64_t)(off_other[y + 1] - off_other[y]);
    }
    s = warp_sum(s);
    if (lane == 0) S[x] = s;
  }
}

__global__ void center_of_kernel(const uint32_t* __restrict__ offC, int64_t nC, uint32_t* center_of) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t v = warp; v < nC; v += nwarps)
    for (uint32_t j = offC[v] + lane; j < offC[v + 1]; j += 32) center_of[j] = (uint32_t)v;
}

__global__ void max_i64_kernel(const int64_t* __restrict__ a, int64_t n, unsigned long long* out) {
  unsigned long long m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (unsigned long long)a[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Live-entry count per vertex.  kByEdge: an entry is live when its edge is not peeled
// (wing); otherwise when its neighbour (a count-side vertex) is not peeled (tip, centre lists).
template <bool kByEdge>
__global__ void live_degree_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr,
                                   const uint32_t* __restrict__ eid, int64_t n, const uint8_t* __restrict__ state,
                                   uint32_t* deg) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t x = warp; x < n; x += nwarps) {
    uint32_t c = 0;
    for (uint32_t p = off[x] + lane; p < off[x + 1]; p += 32)
      c += state[kByEdge ? eid[p] : nbr[p]] != PEELED;
    c = warp_sum(c);
    if (lane == 0) deg[x] = c;
  }
}

// Stable filter of every list to its live entries (order kept, so lists stay ascending).
template <bool kByEdge>
__global__ void compact_lists_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr,
                                     const uint32_t* __restrict__ eid, int64_t n, const uint8_t* __restrict__ state,
                                     const uint32_t* __restrict__ noff, uint32_t* nnbr, uint32_t* neid) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (int64_t x = warp; x < n; x += nwarps) {
    uint32_t dst = noff[x];
    const uint32_t e = off[x + 1];
    for (uint32_t p0 = off[x]; p0 < e; p0 += 32) {
      const uint32_t p = p0 + lane;
      bool live = false;
      uint32_t y = 0, id = 0;
      if (p < e) {
        y = nbr[p];
        id = eid ? eid[p] : 0u;
        live = state[kByEdge ? id : y] != PEELED;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, live);
      if (live) {
        const uint32_t at = dst + __popc(bal & ((1u << lane) - 1u));
        nnbr[at] = y;
        if (neid) neid[at] = id;
      }
      dst += __popc(bal);
    }
  }
}

__global__ void iota_kernel(uint32_t* a, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

int grid_for(int64_t n, int per_block = 256) { return std::max(1, std::min(ceil_div(n, per_block), sm_count() * 16)); }

// One version of one side's live lists.
struct ListVersion {
  DevBuf<uint32_t> off, nbr, eid;
};

// One side's live lists: every compaction makes a new version from the current one.  With
// keep_all (two-phase peel) every version stays: the fine pass reads, for each partition, the
// newest version that still holds all of its items.  Otherwise only the newest stays.
struct LiveSide {
  std::vector<std::unique_ptr<ListVersion>> ver;
  int64_t n = 0;
  bool keep_all = false;
};

template <bool kByEdge>
void compact_side(LiveSide& L, const uint32_t* off, const uint32_t* nbr, const uint32_t* eid, const uint8_t* state,
                  bool with_eid, cudaStream_t s) {
  auto nv = std::make_unique<ListVersion>();
  DevBuf<uint32_t> deg(L.n > 0 ? L.n : 1, s);
  if (L.n) PB_LAUNCH(live_degree_kernel<kByEdge>, grid_for(L.n * 32), 256, 0, s, off, nbr, eid, L.n, state, deg.get());
  nv->off.alloc(L.n + 1, s);
  exclusive_scan_u32(deg.get(), nv->off.get(), L.n, s);
  uint32_t live = 0;
  PB_CUDA_TRY(cudaMemcpyAsync(&live, nv->off.get() + L.n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  nv->nbr.alloc(live + 1, s);
  if (with_eid) nv->eid.alloc(live + 1, s);
  if (L.n)
    PB_LAUNCH(compact_lists_kernel<kByEdge>, grid_for(L.n * 32), 256, 0, s, off, nbr, with_eid ? eid : nullptr, L.n,
              state, nv->off.get(), nv->nbr.get(), with_eid ? nv->eid.get() : nullptr);
  if (!L.keep_all) L.ver.clear();  // stream-ordered frees, after the compaction has read them
  L.ver.push_back(std::move(nv));
}

// {error bits OR-ed, unpeeled items summed} over the control blocks of one launch.
__global__ void ctl_status_kernel(const Ctl* __restrict__ ctls, unsigned n, unsigned* out) {
  unsigned err = 0, alive = 0;
  for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
    err |= ctls[i].err;
    alive += ctls[i].alive;
  }
  err = __reduce_or_sync(0xffffffffu, err);
  alive = __reduce_add_sync(0xffffffffu, alive);
  if (threadIdx.x == 0) {
    out[0] = err;
    out[1] = alive;
  }
}

// Per partition of the coarse pass: items and summed estimated work (the fine pass's CTA
// shares); with part null, the totals over all items (partition 0).
template <bool kWing>
__global__ void part_stats_kernel(Lists G, Classify cls, const uint32_t* __restrict__ part, int64_t N,
                                  unsigned* cnt, unsigned long long* work) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < N; x += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t p = part ? part[x] : 0u;
    atomicAdd(&cnt[p], 1u);
    atomicAdd(&work[p], item_weight<kWing>(G, cls, (uint32_t)x));
  }
}

template <bool kWing>
__global__ void item_weight_kernel(Lists G, Classify cls, int64_t N, uint32_t* wgt) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < N; x += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long w = item_weight<kWing>(G, cls, (uint32_t)x);
    wgt[x] = (uint32_t)min(w, 0xFFFFFFFFull);
  }
}

// gid[x] = i for the items x in [base[i], base[i + 1]) (one CTA per range).
__global__ void range_ids_kernel(const uint32_t* __restrict__ base, uint32_t n, const uint32_t* unused, uint32_t* gid) {
  const uint32_t i = blockIdx.x;
  if (i >= n) return;
  for (uint32_t x = base[i] + threadIdx.x; x < base[i + 1]; x += blockDim.x) gid[x] = i;
}

// key[x] = pbase[gid[x]] + part[x]: graph-major global partition ids of a batch.
__global__ void global_part_kernel(const uint32_t* __restrict__ gid, const uint32_t* __restrict__ part,
                                   const uint32_t* __restrict__ pbase, int64_t N, uint32_t* key) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < N; x += (int64_t)gridDim.x * blockDim.x)
    key[x] = pbase[gid[x]] + part[x];
}

// Splits `grid` CTAs among instances by weight: an instance whose share is at least one CTA
// gets a CTA range of its own (its barriers span only that range); the light ones are packed,
// longest first onto the least-loaded CTA, into the CTAs left over, where they run one after
// another.  Fills the launch order (slot -> instance), each slot's first CTA and CTA count,
// and each CTA's slot range.
void assign_ctas(const std::vector<double>& pweight, int grid, std::vector<int>& inst_of, std::vector<uint32_t>& first,
                 std::vector<uint32_t>& cnt, std::vector<uint32_t>& cbeg, std::vector<uint32_t>& cend) {
  const int ninst = (int)pweight.size();
  std::vector<int> ord(ninst);
  for (int i = 0; i < ninst; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return pweight[a] > pweight[b]; });
  double wsum = 0;
  for (double w : pweight) wsum += w;
  int nheavy = 0;
  while (nheavy < ninst && pweight[ord[nheavy]] / wsum * grid >= 1.0) ++nheavy;
  double lw = 0;
  for (int j = nheavy; j < ninst; ++j) lw += pweight[ord[j]];
  int light_ctas = 0;
  if (nheavy < ninst) light_ctas = std::min(ninst - nheavy, std::max(1, (int)std::ceil(lw / wsum * grid)));
  // Heavy instances share the rest; demote the lightest ones while they outnumber it.
  while (nheavy > grid - light_ctas) {
    --nheavy;
    if (!light_ctas) light_ctas = 1;
  }
  if (!nheavy) light_ctas = std::min(grid, ninst);
  const int hbudget = grid - light_ctas;
  std::vector<int> ncta(ninst, 0);
  if (nheavy) {
    double hw = 0;
    for (int j = 0; j < nheavy; ++j) hw += pweight[ord[j]];
    int total = 0;
    for (int j = 0; j < nheavy; ++j) {
      ncta[ord[j]] = std::max(1, (int)(pweight[ord[j]] / hw * hbudget));
      total += ncta[ord[j]];
    }
    for (int j = 0; total < hbudget; j = (j + 1) % nheavy, ++total) ++ncta[ord[j]];
    while (total > hbudget) {  // some instance has more than one CTA here (hbudget >= nheavy)
      int k = ord[0];
      for (int j = 1; j < nheavy; ++j)
        if (ncta[ord[j]] > ncta[k]) k = ord[j];
      --ncta[k];
      --total;
    }
  }
  inst_of.clear();
  first.clear();
  cnt.clear();
  cbeg.assign(grid, 0);
  cend.assign(grid, 0);
  uint32_t cta = 0;
  for (int j = 0; j < nheavy; ++j) {
    const int i = ord[j];
    for (int c = 0; c < ncta[i]; ++c) {
      cbeg[cta + c] = (uint32_t)inst_of.size();
      cend[cta + c] = (uint32_t)inst_of.size() + 1;
    }
    inst_of.push_back(i);
    first.push_back(cta);
    cnt.push_back((uint32_t)ncta[i]);
    cta += (uint32_t)ncta[i];
  }
  if (nheavy < ninst) {
    std::vector<std::vector<int>> bins(light_ctas);
    std::vector<double> load(light_ctas, 0.0);
    for (int j = nheavy; j < ninst; ++j) {
      const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      bins[b].push_back(ord[j]);
      load[b] += pweight[ord[j]];
    }
    for (int b = 0; b < light_ctas; ++b, ++cta) {
      cbeg[cta] = (uint32_t)inst_of.size();
      for (int i : bins[b]) {
        inst_of.push_back(i);
        first.push_back(cta);
        cnt.push_back(1u);
      }
      cend[cta] = (uint32_t)inst_of.size();
    }
  }
}

template <bool kWing>
PeelResult run_peel(const pb_graph& g, int use_v, const int64_t* counts, int64_t* out, cudaStream_t s,
                    const PeelTuning& tune, const PeelParts* parts) {
  PeelResult res;
  Lists G{};
  const uint32_t* offK0 = use_v ? g.offU.get() : g.offV.get();
  const uint32_t* edgK0 = use_v ? g.edgU.get() : g.edgV.get();
  const uint32_t* offC0 = use_v ? g.offV.get() : g.offU.get();
  const uint32_t* edgC0 = use_v ? g.edgV.get() : g.edgU.get();
  G.nK = use_v ? g.nu : g.nv;
  G.nC = use_v ? g.nv : g.nu;
  const int64_t N = kWing ? g.m : G.nK;
  if (N == 0) return res;
  PB_REQUIRE(N < (int64_t)UINT32_MAX, PB_ETOOBIG, "too many items to peel");
  G.offK = offK0;
  G.edgK = edgK0;
  G.offC = offC0;
  G.edgC = edgC0;
  const bool batch = parts && parts->base.size() > 1;
  // Two-phase peel (a schedule of the same rounds, never a different result): a coarse pass
  // cuts the items into partitions of about equal estimated work by ranges of their final
  // numbers, then every partition runs its exact rounds as an independent instance.
  bool two_phase_req = tune.two_phase;
  double parts_per_cta = tune.parts_per_cta;
  int64_t parts_total = tune.parts_total;
  if (const char* e = getenv("PB_PEEL_TWO_PHASE")) {  // diagnostic hook: partitions per CTA, 0 = off
    parts_per_cta = atof(e);
    parts_total = 0;
    two_phase_req = parts_per_cta > 0;
  }
  const bool two_phase = !batch && two_phase_req && g_recorder == nullptr;
  const bool two_phase_batch = batch && two_phase_req && g_recorder == nullptr;

  DevBuf<int64_t> cnt(N, s);
  DevBuf<uint32_t> eti, iota, center_of, touched(N, s), alist0(N, s), alist1(N, s), nearl(N, s);
  DevBuf<uint32_t> fs0(N, s), fs1(N, s), fb0(N, s), fb1(N, s), fh0(N, s), fh1(N, s), tl0(N, s), tl1(N, s);
  // Independent instances (the graphs of a batch) or the whole input as one.
  std::vector<int64_t> pbase{0}, psize{N};
  std::vector<double> pweight{1.0};
  if (batch) {
    pbase.clear();
    psize.clear();
    pweight.clear();
    for (size_t i = 0; i < parts->base.size(); ++i) {
      if (parts->size[i] <= 0) continue;
      pbase.push_back(parts->base[i]);
      psize.push_back(parts->size[i]);
      pweight.push_back(std::max(parts->weight[i], 1.0));
    }
    if (pbase.empty()) return res;
  }
  // Grid-shared dense counters: tip peeling keeps one slice per CTA group (heavy items of a round
  // run concurrently), up to 32 slices within kGsharedBudget.
  const int64_t gstride = std::max(G.nK, G.nC) + 1;
  const unsigned ngroups =
      kWing ? 1u : (unsigned)std::max<int64_t>(1, std::min<int64_t>(kMaxGroups, kGsharedBudget / (4 * gstride)));
  DevBuf<uint32_t> gshared((size_t)gstride * ngroups, s);
  PB_CUDA_TRY(cudaMemsetAsync(gshared.get(), 0, gshared.bytes(), s));
  DevBuf<uint8_t> state(N, s), in_near(N, s);
  LiveSide liveK, liveC;
  liveK.n = G.nK;
  liveC.n = G.nC;
  liveK.keep_all = liveC.keep_all = two_phase;
  DevBuf<int64_t> snap;  // two-phase: every item's count when its partition opens
  DevBuf<uint32_t> part;
  if (two_phase || two_phase_batch) {
    snap.alloc(N, s);
    part.alloc(N, s);
  }
  PB_LAUNCH(peel_init_kernel, grid_for(N), 256, 0, s, counts, N, (two_phase || two_phase_batch) ? snap.get() : out,
            cnt.get(), state.get(), in_near.get(), touched.get());
  // Work estimates of the lists a version holds: neighbour-degree sums (wing) or two-hop wedges
  // (tip).
  std::vector<std::unique_ptr<DevBuf<int64_t>>> work_bufs;
  auto refresh_work = [&](Lists& L) {
    auto buf = std::make_unique<DevBuf<int64_t>>(kWing ? L.nK + L.nC : L.nK, s);
    if (kWing) {
      if (L.nK) PB_LAUNCH(nbr_degree_sum_kernel, grid_for(L.nK * 32), 256, 0, s, L.offK, L.edgK, L.offC, L.nK, buf->get());
      if (L.nC)
        PB_LAUNCH(nbr_degree_sum_kernel, grid_for(L.nC * 32), 256, 0, s, L.offC, L.edgC, L.offK, L.nC, buf->get() + L.nK);
      L.S = buf->get();
    } else {
      PB_LAUNCH(tip_work_kernel, grid_for(L.nK * 32), 256, 0, s, L.offK, L.edgK, L.offC, L.nK, buf->get());
      L.wk = buf->get();
    }
    if (!two_phase) work_bufs.clear();
    work_bufs.push_back(std::move(buf));
  };
  bool need_scratch = false;
  int64_t scratch_len = 0;
  if (kWing) {
    eti.alloc(g.m, s);
    iota.alloc(g.m, s);
    center_of.alloc(g.m, s);
    edge_to_idxs(g, use_v, eti.get(), s);
    PB_LAUNCH(iota_kernel, grid_for(g.m), 256, 0, s, iota.get(), g.m);
    PB_LAUNCH(center_of_kernel, grid_for(G.nC * 32), 256, 0, s, G.offC, G.nC, center_of.get());
    G.eidK = eti.get();
    G.eidC = iota.get();
    G.center_of = center_of.get();
    G.u_of = edgC0;  // edge ids are positions in the centre side's original lists
    refresh_work(G);
    need_scratch = 2ull * g.max_deg > (uint64_t)kBlockSlots;
    scratch_len = std::max(G.nK, G.nC);
  } else {
    refresh_work(G);
    DevBuf<unsigned long long> mx(1, s);
    PB_CUDA_TRY(cudaMemsetAsync(mx.get(), 0, sizeof(unsigned long long), s));
    PB_LAUNCH(max_i64_kernel, grid_for(G.nK), 256, 0, s, G.wk, G.nK, mx.get());
    unsigned long long hmx = 0;
    readback(&hmx, mx.get(), sizeof(hmx), s);
    need_scratch = 2ull * hmx > (uint64_t)kBlockSlots;
    scratch_len = G.nK;
  }
  const Lists G0 = G;  // the full lists (version 0)

  const size_t smem = ((sizeof(Shared) + 15) & ~size_t(15)) + (size_t)kBlockSlots * 3 * sizeof(uint32_t);
  void (*kern)(Lists, const Lists*, Instances, Ctl*, Classify) = peel_kernel<kWing, 2>;
  if constexpr (!kWing) {
    if (!batch) kern = peel_kernel<false, 1>;
  }
  PB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  PB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPT, smem));
  PB_REQUIRE(per_sm >= 1, PB_ECUDA, "peeling kernel does not fit on an SM");
  int grid = sm_count() * per_sm;
  // A single instance may run on fewer CTAs: its barriers and grid-stride phases then span
  // fewer CTAs, which shortens light rounds.
  int64_t cap = batch ? 0 : tune.max_ctas;
  if (const char* e = getenv("PB_PEEL_CTAS")) cap = atoll(e);  // diagnostic hook
  if (cap > 0) grid = (int)std::max<int64_t>(1, std::min<int64_t>(grid, cap));

  DevBuf<uint32_t> gscratch;
  if (need_scratch) {
    gscratch.alloc((size_t)grid * (size_t)scratch_len, s);
    PB_CUDA_TRY(cudaMemsetAsync(gscratch.get(), 0, gscratch.bytes(), s));
  }
  DevBuf<uint32_t> fc0(N, s), fc1(N, s), upre(N + (int64_t)pbase.size() + 1, s);
  DevBuf<uint32_t> fw0, fw1, wpre;  // warp units of wing items
  if (kWing) {
    fw0.alloc(N, s);
    fw1.alloc(N, s);
    wpre.alloc(N + (int64_t)pbase.size() + 1, s);
  }
  Work W{};
  W.D = (two_phase || two_phase_batch) ? snap.get() : out;
  W.cnt = cnt.get();
  W.state = state.get();
  W.in_near = in_near.get();
  W.touched = touched.get();
  W.alist[0] = alist0.get();
  W.alist[1] = alist1.get();
  W.near = nearl.get();
  W.fsmall[0] = fs0.get();
  W.fsmall[1] = fs1.get();
  W.fbig[0] = fb0.get();
  W.fbig[1] = fb1.get();
  W.fchunks[0] = fc0.get();
  W.fchunks[1] = fc1.get();
  W.uprefix = upre.get();
  W.fwchunks[0] = fw0.get();
  W.fwchunks[1] = fw1.get();
  W.wprefix = wpre.get();
  W.fhuge[0] = fh0.get();
  W.fhuge[1] = fh1.get();
  W.gshared = gshared.get();
  W.gshared_stride = gstride;
  W.ngroups = ngroups;
  W.tlist[0] = tl0.get();
  W.tlist[1] = tl1.get();
  W.gscratch = gscratch.get();
  W.gscratch_len = scratch_len;
  W.N = N;
  W.item0 = 0;
  W.part_out = two_phase ? part.get() : nullptr;

  Ctl hctl;
  std::memset(&hctl, 0, sizeof(hctl));
  hctl.nm[0] = kInf;
  hctl.nm[1] = kInf;
  hctl.k_lo = kInf;
  hctl.alive = (unsigned)N;
  hctl.alen[0] = (unsigned)N;
  hctl.alive_at_compact = (unsigned)N;
  hctl.min_gain = (unsigned)std::max<int64_t>(1 << 16, N / 64);
  // A recorded / captured pipeline runs the peel as one launch without list compaction (the
  // host cannot step in between launches of a CUDA graph); so do per-graph instances.
  if (g_recorder != nullptr || batch) hctl.min_gain = 0xFFFFFFFFu;
  hctl.barrier_timeout_ns = kBarrierTimeoutNs;
  hctl.near_min = (unsigned)tune.near_min;
  hctl.near_div = (unsigned)tune.near_div;
  // Diagnostic hooks for the window size.
  if (const char* e = getenv("PB_PEEL_NEAR_MIN")) hctl.near_min = (unsigned)strtoul(e, nullptr, 10);
  if (const char* e = getenv("PB_PEEL_NEAR_DIV")) hctl.near_div = (unsigned)strtoul(e, nullptr, 10);
  if (const char* e = getenv("PB_PEEL_BARRIER_TIMEOUT_MS")) hctl.barrier_timeout_ns = 1000000ull * strtoull(e, nullptr, 10);
  // Test hook: CTA 0 skips its arrivals, so the first grid barrier cannot complete and every
  // wait runs out; checks that a timeout comes back as PB_ETIMEOUT with the context usable.
  if (const char* e = getenv("PB_PEEL_TEST_STUCK_BARRIER"))
    if (*e && *e != '0') hctl.test_skip_arrival = 1;
  Classify cls{tune.small_work, tune.huge_work, tune.chunk_work, std::max<int64_t>(1, tune.units_per_cta),
               tune.warp_units ? 1 : 0};
  if (const char* e = getenv("PB_PEEL_WARP_UNITS")) cls.warp_units = atoi(e) != 0;  // diagnostic hook
  // Thresholds may be lowered through the environment (tests use this to drive small graphs
  // through the CTA- and grid-level paths).
  if (const char* e = getenv("PB_PEEL_SMALL_WORK")) cls.small_work = atoll(e);
  if (const char* e = getenv("PB_PEEL_HUGE_WORK")) cls.huge_work = atoll(e);
  if (const char* e = getenv("PB_PEEL_CHUNK_WORK")) cls.chunk_work = atoll(e);
  DevBuf<unsigned> status(2, s);
  DevBuf<uint32_t> wgt;  // coarse passes: static per-item work estimates
  if (two_phase || two_phase_batch) {
    wgt.alloc(N, s);
    PB_LAUNCH(item_weight_kernel<kWing>, grid_for(N), 256, 0, s, G0, cls, N, wgt.get());
    W.wgt = wgt.get();
  }

  // One cooperative launch of independent instances with CTA shares by weight (no compaction
  // pauses: every instance runs to its end).  per_slot may adjust each launch slot's Work.
  auto launch_instances = [&](const std::vector<Work>& wproto, const std::vector<Ctl>& cproto,
                              const std::vector<double>& weights, const Lists* levels_dev,
                              const std::function<void(Work&, uint32_t)>& per_slot,
                              std::vector<Ctl>* inst_out = nullptr) {
    std::vector<int> inst_of;
    std::vector<uint32_t> first, ncta, cbeg, cend;
    assign_ctas(weights, grid, inst_of, first, ncta, cbeg, cend);
    const int n_slots = (int)inst_of.size();
    std::vector<Work> ws(n_slots);
    std::vector<Ctl> hctls(n_slots);
    for (int q = 0; q < n_slots; ++q) {
      ws[q] = wproto[inst_of[q]];
      hctls[q] = cproto[inst_of[q]];
      if (per_slot) per_slot(ws[q], ncta[q]);
    }
    DevBuf<Ctl> ctls(n_slots, s);
    DevBuf<Work> dws(n_slots, s);
    DevBuf<uint32_t> meta(2 * (size_t)n_slots + 2 * (size_t)grid, s);
    std::vector<uint32_t> hmeta;
    hmeta.insert(hmeta.end(), first.begin(), first.end());
    hmeta.insert(hmeta.end(), ncta.begin(), ncta.end());
    hmeta.insert(hmeta.end(), cbeg.begin(), cbeg.end());
    hmeta.insert(hmeta.end(), cend.begin(), cend.end());
    const void* src_c = hctls.data();
    const void* src_w = ws.data();
    const void* src_m = hmeta.data();
    if (capturing()) {  // the graph copies from host memory that outlives it
      void* pc = g_recorder->pinned_alloc(sizeof(Ctl) * n_slots);
      void* pw = g_recorder->pinned_alloc(sizeof(Work) * n_slots);
      void* pm = g_recorder->pinned_alloc(sizeof(uint32_t) * hmeta.size());
      std::memcpy(pc, src_c, sizeof(Ctl) * n_slots);
      std::memcpy(pw, src_w, sizeof(Work) * n_slots);
      std::memcpy(pm, src_m, sizeof(uint32_t) * hmeta.size());
      src_c = pc;
      src_w = pw;
      src_m = pm;
    }
    PB_CUDA_TRY(cudaMemcpyAsync(ctls.get(), src_c, sizeof(Ctl) * n_slots, cudaMemcpyHostToDevice, s));
    PB_CUDA_TRY(cudaMemcpyAsync(dws.get(), src_w, sizeof(Work) * n_slots, cudaMemcpyHostToDevice, s));
    PB_CUDA_TRY(cudaMemcpyAsync(meta.get(), src_m, sizeof(uint32_t) * hmeta.size(), cudaMemcpyHostToDevice, s));
    Instances I{dws.get(), meta.get(), meta.get() + n_slots, meta.get() + 2 * n_slots,
                meta.get() + 2 * n_slots + grid, (uint32_t)n_slots};
    Ctl* cp = ctls.get();
    Lists Gk = G0;
    const Lists* lv = levels_dev;
    void* args[] = {&Gk, &lv, &I, &cp, &cls};
    PB_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(kPT), args, smem, s));
    if (g_launch_counter) ++*g_launch_counter;
    PB_LAUNCH(ctl_status_kernel, 1, 32, 0, s, cp, (unsigned)n_slots, status.get());
    if (capturing()) {
      PB_CUDA_TRY(cudaMemcpyAsync(g_recorder->status, status.get(), 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
      return;
    }
    PB_CUDA_TRY(cudaMemcpyAsync(hctls.data(), cp, sizeof(Ctl) * n_slots, cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    if (inst_out) inst_out->assign(wproto.size(), Ctl{});
    for (int q = 0; q < n_slots; ++q) {
      const Ctl& c = hctls[q];
      PB_REQUIRE(!(c.err & ERR_TIMEOUT), PB_ETIMEOUT, "peeling: a grid barrier wait ran out of time");
      PB_REQUIRE(c.err == 0, PB_ECUDA, "peeling: a table invariant was violated");
      PB_REQUIRE(c.alive == 0, PB_ECUDA, "peeling: an instance stopped with unpeeled items");
      res.rounds += (int64_t)c.rounds;
      res.fine_rounds_max = std::max<int64_t>(res.fine_rounds_max, (int64_t)c.rounds);
      res.work += (int64_t)c.work;
      if (inst_out) (*inst_out)[inst_of[q]] = c;
    }
  };

  if (batch) {
    const int ninst = (int)pbase.size();
    std::vector<Work> ws(ninst, W);
    std::vector<Ctl> cs(ninst, hctl);
    for (int i = 0; i < ninst; ++i) {
      const int64_t b = pbase[i], n = psize[i];
      Work& x = ws[i];
      x.alist[0] = alist0.get() + b;
      x.alist[1] = alist1.get() + b;
      x.near = nearl.get() + b;
      x.fsmall[0] = fs0.get() + b;
      x.fsmall[1] = fs1.get() + b;
      x.fbig[0] = fb0.get() + b;
      x.fbig[1] = fb1.get() + b;
      x.fchunks[0] = fc0.get() + b;
      x.fchunks[1] = fc1.get() + b;
      x.uprefix = upre.get() + b + i;
      if (kWing) {
        x.fwchunks[0] = fw0.get() + b;
        x.fwchunks[1] = fw1.get() + b;
        x.wprefix = wpre.get() + b + i;
      }
      x.fhuge[0] = fh0.get() + b;
      x.fhuge[1] = fh1.get() + b;
      x.tlist[0] = tl0.get() + b;
      x.tlist[1] = tl1.get() + b;
      x.N = n;
      x.item0 = (uint32_t)b;
      Ctl& c = cs[i];
      c.alive = (unsigned)n;
      c.alen[0] = (unsigned)n;
      c.alive_at_compact = (unsigned)n;
    }
    if (!two_phase_batch) {
      launch_instances(ws, cs, pweight, nullptr, nullptr);
      res.rounds = res.fine_rounds_max;  // a batch reports the rounds of its longest graph
      res.fine_rounds_max = 0;
      return res;
    }
    // Two-phase schedule per graph: a coarse pass with one range-mode instance per graph (about
    // parts_per_cta partitions per CTA, split by the graphs' work), then one fine instance per
    // (graph, partition).  Partition ids are local to a graph: items of different graphs never
    // meet in a list.
    DevBuf<uint32_t> gid(N, s);
    DevBuf<uint32_t> dbase(ninst + 1, s);
    std::vector<uint32_t> hb(ninst + 1);
    for (int i = 0; i < ninst; ++i) hb[i] = (uint32_t)pbase[i];
    hb[ninst] = (uint32_t)(pbase[ninst - 1] + psize[ninst - 1]);
    PB_CUDA_TRY(cudaMemcpyAsync(dbase.get(), hb.data(), sizeof(uint32_t) * (ninst + 1), cudaMemcpyHostToDevice, s));
    PB_LAUNCH(range_ids_kernel, ninst, 256, 0, s, dbase.get(), (uint32_t)ninst, (const uint32_t*)nullptr, gid.get());
    DevBuf<unsigned> icnt(ninst, s);
    DevBuf<unsigned long long> iwork(ninst, s);
    PB_CUDA_TRY(cudaMemsetAsync(icnt.get(), 0, sizeof(unsigned) * ninst, s));
    PB_CUDA_TRY(cudaMemsetAsync(iwork.get(), 0, sizeof(unsigned long long) * ninst, s));
    PB_LAUNCH(part_stats_kernel<kWing>, grid_for(N), 256, 0, s, G, cls, (const uint32_t*)gid.get(), N, icnt.get(),
              iwork.get());
    std::vector<unsigned long long> hiw(ninst);
    PB_CUDA_TRY(cudaMemcpyAsync(hiw.data(), iwork.get(), sizeof(unsigned long long) * ninst, cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    double wsum = 0;
    for (unsigned long long w : hiw) wsum += (double)w;
    const double want = std::max(1.0, parts_total > 0 ? (double)parts_total : parts_per_cta * grid);
    for (int i = 0; i < ninst; ++i) {
      const double parts_i = std::max(1.0, std::round(want * (double)hiw[i] / std::max(1.0, wsum)));
      cs[i].range_mode = 1;
      cs[i].part_target = std::max<unsigned long long>(1, (unsigned long long)((double)hiw[i] / parts_i));
      ws[i].part_out = part.get();
    }
    std::vector<Ctl> coarse;
    launch_instances(ws, cs, pweight, nullptr, nullptr, &coarse);
    res.coarse_rounds = res.fine_rounds_max;
    res.rounds = 0;
    res.fine_rounds_max = 0;
    // Global partition keys (graph-major) and the fine instances in that order.
    std::vector<uint32_t> pb0(ninst + 1, 0);
    for (int i = 0; i < ninst; ++i) pb0[i + 1] = pb0[i] + std::max(1u, coarse[i].npart);
    const uint32_t ntot = pb0[ninst];
    DevBuf<uint32_t> dpb(ninst + 1, s), key(N, s);
    PB_CUDA_TRY(cudaMemcpyAsync(dpb.get(), pb0.data(), sizeof(uint32_t) * (ninst + 1), cudaMemcpyHostToDevice, s));
    PB_LAUNCH(global_part_kernel, grid_for(N), 256, 0, s, (const uint32_t*)gid.get(), (const uint32_t*)part.get(),
              (const uint32_t*)dpb.get(), N, key.get());
    int bits = 1;
    while (bits < 32 && (1ull << bits) < ntot) ++bits;
    DevBuf<uint32_t> key2(N, s), perm(N, s), perm2(N, s);
    PB_LAUNCH(iota_kernel, grid_for(N), 256, 0, s, perm.get(), N);
    const bool alt = radix_sort_pairs_u32(key.get(), perm.get(), key2.get(), perm2.get(), N, 0, bits, s);
    const uint32_t* items = alt ? perm2.get() : perm.get();
    // key still holds each item's global partition (radix_sort_pairs_u32 sorts into key / key2).
    PB_LAUNCH(global_part_kernel, grid_for(N), 256, 0, s, (const uint32_t*)gid.get(), (const uint32_t*)part.get(),
              (const uint32_t*)dpb.get(), N, key2.get());
    DevBuf<unsigned> pcnt(ntot, s);
    DevBuf<unsigned long long> pwork(ntot, s);
    PB_CUDA_TRY(cudaMemsetAsync(pcnt.get(), 0, sizeof(unsigned) * ntot, s));
    PB_CUDA_TRY(cudaMemsetAsync(pwork.get(), 0, sizeof(unsigned long long) * ntot, s));
    PB_LAUNCH(part_stats_kernel<kWing>, grid_for(N), 256, 0, s, G, cls, (const uint32_t*)key2.get(), N, pcnt.get(),
              pwork.get());
    std::vector<unsigned> hcnt(ntot);
    std::vector<unsigned long long> hwork(ntot);
    PB_CUDA_TRY(cudaMemcpyAsync(hcnt.data(), pcnt.get(), sizeof(unsigned) * ntot, cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaMemcpyAsync(hwork.data(), pwork.get(), sizeof(unsigned long long) * ntot, cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    PB_LAUNCH(peel_init_kernel, grid_for(N), 256, 0, s, (const int64_t*)snap.get(), N, out, cnt.get(), state.get(),
              in_near.get(), touched.get());
    std::vector<Work> fws;
    std::vector<Ctl> fcs;
    std::vector<double> fw;
    std::vector<int> graph_of;
    int64_t b = 0;
    for (int i = 0; i < ninst; ++i) {
      for (uint32_t p = 0; p + pb0[i] < pb0[i + 1]; ++p) {
        const int64_t n = hcnt[pb0[i] + p];
        if (n == 0) continue;
        Work x = ws[i];
        x.D = out;
        x.part_out = nullptr;
        x.items = items;
        x.part = part.get();
        x.my_part = p;
        x.alist[0] = alist0.get() + b;
        x.alist[1] = alist1.get() + b;
        x.near = nearl.get() + b;
        x.fsmall[0] = fs0.get() + b;
        x.fsmall[1] = fs1.get() + b;
        x.fbig[0] = fb0.get() + b;
        x.fbig[1] = fb1.get() + b;
        x.fchunks[0] = fc0.get() + b;
        x.fchunks[1] = fc1.get() + b;
        x.fhuge[0] = fh0.get() + b;
        x.fhuge[1] = fh1.get() + b;
        x.tlist[0] = tl0.get() + b;
        x.tlist[1] = tl1.get() + b;
        x.N = n;
        x.item0 = (uint32_t)b;
        fws.push_back(x);
        Ctl c = hctl;
        c.alive = (unsigned)n;
        c.alen[0] = (unsigned)n;
        c.alive_at_compact = (unsigned)n;
        fcs.push_back(c);
        fw.push_back(std::max(1.0, (double)hwork[pb0[i] + p]));
        graph_of.push_back(i);
        b += n;
      }
    }
    PB_REQUIRE(b == N, PB_ECUDA, "two-phase peel: partition sizes do not add up");
    DevBuf<uint32_t> upre2(N + (int64_t)fws.size() + 1, s), wpre2;
    if (kWing) wpre2.alloc(N + (int64_t)fws.size() + 1, s);
    for (size_t i = 0; i < fws.size(); ++i) {
      fws[i].uprefix = upre2.get() + fws[i].item0 + i;
      if (kWing) {
        fws[i].fwchunks[0] = fw0.get() + fws[i].item0;
        fws[i].fwchunks[1] = fw1.get() + fws[i].item0;
        fws[i].wprefix = wpre2.get() + fws[i].item0 + i;
      }
    }
    const int64_t gstride_b = gstride;
    const int64_t slices = std::max<int64_t>(1, kGsharedBudget / (4 * gstride_b));
    std::vector<std::unique_ptr<DevBuf<uint32_t>>> gsl;
    auto per_slot = [&](Work& x, uint32_t ncta) {
      x.gshared = nullptr;
      x.ngroups = 1;
      if (ncta >= 2 && (int64_t)gsl.size() < slices) {
        gsl.push_back(std::make_unique<DevBuf<uint32_t>>((size_t)gstride_b, s));
        PB_CUDA_TRY(cudaMemsetAsync(gsl.back()->get(), 0, gsl.back()->bytes(), s));
        x.gshared = gsl.back()->get();
      }
    };
    std::vector<Ctl> fine;
    const int64_t coarse_work = res.work;
    res.work = 0;
    launch_instances(fws, fcs, fw, nullptr, per_slot, &fine);
    std::vector<int64_t> per_graph(ninst, 0);
    for (size_t q = 0; q < fine.size(); ++q) per_graph[graph_of[q]] += (int64_t)fine[q].rounds;
    res.rounds = *std::max_element(per_graph.begin(), per_graph.end());  // the longest graph, as above
    res.work += coarse_work;
    res.parts = (int64_t)fws.size();
    return res;
  }

  if (two_phase) {
    // Coarse pass: partitions of equal estimated work, about parts_per_cta per CTA (or
    // parts_total in all).
    DevBuf<unsigned long long> wtot(1, s);
    DevBuf<unsigned> ctot(1, s);
    PB_CUDA_TRY(cudaMemsetAsync(wtot.get(), 0, sizeof(unsigned long long), s));
    PB_CUDA_TRY(cudaMemsetAsync(ctot.get(), 0, sizeof(unsigned), s));
    PB_LAUNCH(part_stats_kernel<kWing>, grid_for(N), 256, 0, s, G, cls, (const uint32_t*)nullptr, N, ctot.get(),
              wtot.get());
    unsigned long long total_w = 0;
    readback(&total_w, wtot.get(), sizeof(total_w), s);
    const double nparts_target = std::max(1.0, parts_total > 0 ? (double)parts_total : parts_per_cta * grid);
    hctl.range_mode = 1;
    hctl.part_target = std::max<unsigned long long>(1, (unsigned long long)((double)total_w / nparts_target));
  }

  // Single instance over the whole grid: launch, and between launches compact the lists to
  // their live entries (every version is kept for the fine pass of a two-phase peel).
  std::vector<Lists> levels{G0};
  std::vector<unsigned> level_from{0};  // version j holds every item of partitions >= level_from[j]
  DevBuf<Work> dW(1, s);
  DevBuf<Ctl> ctl(1, s);
  if (capturing()) {
    // The graph copies from host memory that outlives it; the status words come back to a
    // pinned buffer the caller checks after every replay.
    Ctl* h0 = (Ctl*)g_recorder->pinned_alloc(sizeof(Ctl));
    std::memcpy(h0, &hctl, sizeof(Ctl));
    Work* w0 = (Work*)g_recorder->pinned_alloc(sizeof(Work));
    std::memcpy(w0, &W, sizeof(Work));
    PB_CUDA_TRY(cudaMemcpyAsync(ctl.get(), h0, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    PB_CUDA_TRY(cudaMemcpyAsync(dW.get(), w0, sizeof(Work), cudaMemcpyHostToDevice, s));
  } else {
    PB_CUDA_TRY(cudaMemcpyAsync(ctl.get(), &hctl, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    PB_CUDA_TRY(cudaMemcpyAsync(dW.get(), &W, sizeof(Work), cudaMemcpyHostToDevice, s));
  }
  Instances I1{dW.get(), nullptr, nullptr, nullptr, nullptr, 1u};
  Ctl* ctl_ptr = ctl.get();
  const Lists* no_levels = nullptr;
  int launches = 0;
  if (capturing()) {
    void* args[] = {&G, &no_levels, &I1, &ctl_ptr, &cls};
    PB_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(kPT), args, smem, s));
    if (g_launch_counter) ++*g_launch_counter;
    // {err, alive} of the control block into the recorder's status slot (pinned).
    PB_LAUNCH(ctl_status_kernel, 1, 32, 0, s, ctl_ptr, 1u, status.get());
    PB_CUDA_TRY(cudaMemcpyAsync(g_recorder->status, status.get(), 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    return res;
  }
  while (true) {
    void* args[] = {&G, &no_levels, &I1, &ctl_ptr, &cls};
    PB_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(kPT), args, smem, s));
    if (g_launch_counter) ++*g_launch_counter;
    ++launches;
    PB_CUDA_TRY(cudaMemcpyAsync(&hctl, ctl.get(), sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    PB_CUDA_TRY(cudaStreamSynchronize(s));
    PB_REQUIRE(!(hctl.err & ERR_TIMEOUT), PB_ETIMEOUT, "peeling: a grid barrier wait ran out of time");
    PB_REQUIRE(hctl.err == 0, PB_ECUDA, "peeling: a table invariant was violated");
    if (hctl.alive == 0) break;
    PB_REQUIRE(launches < 4096, PB_ECUDA, "peeling: too many relaunches");
    // Compact the lists to their live entries and resume.
    if (kWing) {
      compact_side<true>(liveK, G.offK, G.edgK, G.eidK, state.get(), true, s);
      compact_side<true>(liveC, G.offC, G.edgC, G.eidC, state.get(), true, s);
      G.offK = liveK.ver.back()->off.get();
      G.edgK = liveK.ver.back()->nbr.get();
      G.eidK = liveK.ver.back()->eid.get();
      G.offC = liveC.ver.back()->off.get();
      G.edgC = liveC.ver.back()->nbr.get();
      G.eidC = liveC.ver.back()->eid.get();
    } else {
      compact_side<false>(liveC, G.offC, G.edgC, nullptr, state.get(), false, s);
      G.offC = liveC.ver.back()->off.get();
      G.edgC = liveC.ver.back()->nbr.get();
    }
    refresh_work(G);
    if (two_phase) {
      // Partitions not opened yet (npart and later) have all their items in the new version.
      levels.push_back(G);
      level_from.push_back(hctl.npart);
    }
    const unsigned alive = hctl.alive;
    PB_CUDA_TRY(cudaMemcpyAsync(&ctl.get()->alive_at_compact, &alive, sizeof(unsigned), cudaMemcpyHostToDevice, s));
  }
  res.rounds = (int64_t)hctl.rounds;
  res.work = (int64_t)hctl.work;
  const bool trace = [] {
    const char* tr = getenv("PB_TRACE");
    return tr && *tr && *tr != '0';
  }();
  if (trace) {
    fprintf(stderr,
            "[pb] peel %s%s: rounds %llu launches %d advances %llu | ms advance %.1f F %.1f P %.1f U %.1f | "
            "near scanned %llu touched %llu items small %llu big %llu huge %llu work %llu\n",
            kWing ? "wing" : "tip", two_phase ? " (coarse pass)" : "", hctl.rounds, launches, hctl.advances,
            hctl.phase_ns[0] / 1e6, hctl.phase_ns[1] / 1e6, hctl.phase_ns[2] / 1e6, hctl.phase_ns[3] / 1e6,
            hctl.scanned, hctl.touched_total, hctl.n_small, hctl.n_big, hctl.n_huge, hctl.work);
    if (kWing)
      fprintf(stderr,
              "[pb]   wing items / probes: warp %llu / %llu, CTA table %llu / %llu, dense markers %llu / %llu, "
              "grid %llu / %llu; reverse-direction probes %llu\n",
              hctl.mode_items[0], hctl.mode_work[0], hctl.mode_items[1], hctl.mode_work[1], hctl.mode_items[2],
              hctl.mode_work[2], hctl.mode_items[3], hctl.mode_work[3], hctl.rev_work);
    for (int b = 0; b < 42; ++b)
      if (hctl.pbin_rounds[b])
        fprintf(stderr, "[pb]   P rounds with est work in [2^%d, 2^%d): %llu rounds, %.1f ms, est %.3g (%.3g/s)\n",
                b ? b - 1 : 0, b, hctl.pbin_rounds[b], hctl.pbin_ns[b] / 1e6, (double)hctl.pbin_est[b],
                hctl.pbin_ns[b] ? hctl.pbin_est[b] / (hctl.pbin_ns[b] / 1e9) : 0.0);
  }
  if (!two_phase) return res;

  // ---- fine pass: one instance per partition, all in one launch ----------------------------
  res.coarse_rounds = res.rounds;
  const unsigned nparts = hctl.npart;
  PB_REQUIRE(nparts >= 1, PB_ECUDA, "two-phase peel: the coarse pass opened no partition");
  // Items sorted by partition (stable: ascending ids inside a partition).
  int bits = 1;
  while (bits < 32 && (1ull << bits) < nparts) ++bits;
  DevBuf<uint32_t> pkeys(N, s), pkeys2(N, s), perm(N, s), perm2(N, s);
  PB_CUDA_TRY(cudaMemcpyAsync(pkeys.get(), part.get(), sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, s));
  PB_LAUNCH(iota_kernel, grid_for(N), 256, 0, s, perm.get(), N);
  const bool alt = radix_sort_pairs_u32(pkeys.get(), perm.get(), pkeys2.get(), perm2.get(), N, 0, bits, s);
  const uint32_t* items = alt ? perm2.get() : perm.get();
  DevBuf<unsigned> pcnt(nparts, s);
  DevBuf<unsigned long long> pwork(nparts, s);
  PB_CUDA_TRY(cudaMemsetAsync(pcnt.get(), 0, sizeof(unsigned) * nparts, s));
  PB_CUDA_TRY(cudaMemsetAsync(pwork.get(), 0, sizeof(unsigned long long) * nparts, s));
  PB_LAUNCH(part_stats_kernel<kWing>, grid_for(N), 256, 0, s, G0, cls, (const uint32_t*)part.get(), N, pcnt.get(),
            pwork.get());
  std::vector<unsigned> hcnt(nparts);
  std::vector<unsigned long long> hwork(nparts);
  PB_CUDA_TRY(cudaMemcpyAsync(hcnt.data(), pcnt.get(), sizeof(unsigned) * nparts, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaMemcpyAsync(hwork.data(), pwork.get(), sizeof(unsigned long long) * nparts, cudaMemcpyDeviceToHost, s));
  PB_CUDA_TRY(cudaStreamSynchronize(s));
  // Fresh per-item state: every partition starts from the counts its items had when it opened.
  PB_LAUNCH(peel_init_kernel, grid_for(N), 256, 0, s, (const int64_t*)snap.get(), N, out, cnt.get(), state.get(),
            in_near.get(), touched.get());
  DevBuf<Lists> dlevels(levels.size(), s);
  PB_CUDA_TRY(cudaMemcpyAsync(dlevels.get(), levels.data(), sizeof(Lists) * levels.size(), cudaMemcpyHostToDevice, s));
  Ctl c0;
  std::memset(&c0, 0, sizeof(c0));
  c0.nm[0] = c0.nm[1] = kInf;
  c0.k_lo = kInf;
  c0.min_gain = 0xFFFFFFFFu;
  c0.barrier_timeout_ns = hctl.barrier_timeout_ns;
  c0.near_min = hctl.near_min;
  c0.near_div = hctl.near_div;
  std::vector<Work> ws;
  std::vector<Ctl> cs;
  std::vector<double> weights;
  int64_t b = 0;
  for (unsigned p = 0; p < nparts; ++p) {
    const int64_t n = hcnt[p];
    if (n == 0) continue;
    Work x = W;
    x.D = out;
    x.part_out = nullptr;
    x.items = items;
    x.part = part.get();
    x.my_part = p;
    unsigned lv = 0;
    for (unsigned j = 0; j < level_from.size(); ++j)
      if (level_from[j] <= p) lv = j;
    x.level = lv;
    x.alist[0] = alist0.get() + b;
    x.alist[1] = alist1.get() + b;
    x.near = nearl.get() + b;
    x.fsmall[0] = fs0.get() + b;
    x.fsmall[1] = fs1.get() + b;
    x.fbig[0] = fb0.get() + b;
    x.fbig[1] = fb1.get() + b;
    x.fchunks[0] = fc0.get() + b;
    x.fchunks[1] = fc1.get() + b;
    x.fhuge[0] = fh0.get() + b;
    x.fhuge[1] = fh1.get() + b;
    x.tlist[0] = tl0.get() + b;
    x.tlist[1] = tl1.get() + b;
    x.N = n;
    x.item0 = (uint32_t)b;
    ws.push_back(x);
    Ctl c = c0;
    c.alive = (unsigned)n;
    c.alen[0] = (unsigned)n;
    c.alive_at_compact = (unsigned)n;
    cs.push_back(c);
    weights.push_back(std::max(1.0, (double)hwork[p]));
    b += n;
  }
  PB_REQUIRE(b == N, PB_ECUDA, "two-phase peel: partition sizes do not add up");
  // Unit prefixes: N + 1 slots per instance (n + 1 each).
  DevBuf<uint32_t> upre2(N + (int64_t)ws.size() + 1, s), wpre2;
  if (kWing) wpre2.alloc(N + (int64_t)ws.size() + 1, s);
  for (size_t i = 0; i < ws.size(); ++i) {
    ws[i].uprefix = upre2.get() + ws[i].item0 + i;
    if (kWing) {
      ws[i].fwchunks[0] = fw0.get() + ws[i].item0;
      ws[i].fwchunks[1] = fw1.get() + ws[i].item0;
      ws[i].wprefix = wpre2.get() + ws[i].item0 + i;
    }
  }
  const int64_t coarse_work = res.work;
  res.rounds = 0;
  res.work = 0;
  // Grid-shared counters (grid-level items) must be per instance here, since partitions share
  // item ids: instances with a CTA range of their own get one slice each while the 256 MB
  // budget lasts; the others never take the grid-level path.
  const int64_t slices = std::max<int64_t>(1, kGsharedBudget / (4 * gstride));
  std::vector<std::unique_ptr<DevBuf<uint32_t>>> gsl;
  auto per_slot = [&](Work& x, uint32_t ncta) {
    x.gshared = nullptr;
    x.ngroups = 1;
    if (ncta >= 2 && (int64_t)gsl.size() < slices) {
      gsl.push_back(std::make_unique<DevBuf<uint32_t>>((size_t)gstride, s));
      PB_CUDA_TRY(cudaMemsetAsync(gsl.back()->get(), 0, gsl.back()->bytes(), s));
      x.gshared = gsl.back()->get();
    }
  };
  launch_instances(ws, cs, weights, dlevels.get(), per_slot);
  res.work += coarse_work;
  res.parts = (int64_t)ws.size();
  if (trace)
    fprintf(stderr, "[pb] peel %s fine pass: %zu partitions, %d list versions, %lld rounds, longest %lld\n",
            kWing ? "wing" : "tip", ws.size(), (int)levels.size(), (long long)res.rounds,
            (long long)res.fine_rounds_max);
  return res;
}

}  // namespace

PeelResult peel_vertices(const pb_graph& g, int use_v, const int64_t* counts_dev, int64_t* tip_dev, cudaStream_t s,
                         const PeelTuning& tune, const PeelParts* parts) {
  return run_peel<false>(g, use_v, counts_dev, tip_dev, s, tune, parts);
}

PeelResult peel_edges(const pb_graph& g, int use_v, const int64_t* ecounts_dev, int64_t* wing_dev, cudaStream_t s,
                      const PeelTuning& tune) {
  return run_peel<true>(g, use_v, ecounts_dev, wing_dev, s, tune, nullptr);
}

}  // namespace pb
