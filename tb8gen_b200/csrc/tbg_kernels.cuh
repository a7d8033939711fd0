// The ply-step device code (sm_100a).  All arithmetic is integer and bitwise.
//
//  mark_unmoves_inc, mark_king_unmoves, mark_piece_unmoves
//                        predecessors_worker      tb8gen.c:484-527   (W step / L candidates)
//                        predecessors_sub_worker  tb8gen.c:346-414   (uncaptures)
//  survives_quick, refute
//                        check_successors_worker  tb8gen.c:607-661   (L-step verify)
//  k_calc_sub            calc_sub_worker          tb8gen.c:280-342   (capture classes, seeded stub)
//  k_calc_illegal        calc_illegal_worker      tb8gen.c:664-684
//  k_calc_mate           calc_mate_worker         tb8gen.c:686-727
//  k_epilogue_W          kslice_and_not + kslice_count + kslice_or  (tb8gen.c:1072-1077)
//
// The per-position work of the sparse steps (the first three lines) is
// driven by two schemes: warp-wide (tbg_warp.cuh: the per-call kernel k_op_w
// and the persistent k_batch_w) and block-wide (the tile_* functions below,
// run by the persistent k_batch of tbg_batch.cuh): each thread loads 16 B of
// a tile of kTileWords 32-bit words (coalesced), the block compacts the set
// bits of the tile into a shared-memory list, and the threads then take list
// entries; the list is drained in rounds, so any density is handled.
#pragma once

#include "tbg_device.cuh"

namespace tbg {

// Threads per block of every kernel (a sparse tile is 4 words per thread)
// and blocks per SM the sparse kernels are compiled for: 1,024 resident
// threads at 64 registers each.
#ifndef TBG_THREADS
#define TBG_THREADS 256
#endif
#ifndef TBG_MINB_VERIFY
#define TBG_MINB_VERIFY (1024 / TBG_THREADS)
#endif
#ifndef TBG_MINB_SCATTER
#define TBG_MINB_SCATTER (1024 / TBG_THREADS)
#endif

constexpr int kThreads = TBG_THREADS;
constexpr int kTileWords = kThreads * 4;      // 1024 words = 32768 positions at 256
constexpr int kListCap = kThreads * 16;

// Materials and stub parameters, uniform across a launch: constant memory.
// Every translation unit that includes this header (tbg_api.cu and the two
// persistent-kernel units, tbg_persist_block.cu and tbg_persist_warp.cu)
// holds its own copy; the host writes all of them (tbg_persist.h).
static __constant__ DMat c_mats[TBG_MAX_MATS];
static __constant__ uint64_t c_stub_seed;
static __constant__ int c_stub_mod;

// ------------------------------------------------------------------ ranks
// Rank of a position given as kings + sets, with up to two per-set bit
// toggles applied first (a move is a toggle of two bits; a capture removes
// one; an uncapture adds one), then the normalisation transform.  Sets
// below kfrom keep the contribution idx0 and the occupancy occ0.
template <int NS>
__device__ __forceinline__ uint64_t rank_mod(const DIdx &X, const uint32_t *bin, int k0,
                                            int k1, const bb *set, int ka, bb xa, int kb,
                                            bb xb, int mirror, int flip, int kfrom = 0,
                                            bb occ0 = 0, uint64_t idx0 = 0) {
  bb occ = kfrom == 0 ? (bit(k0) | bit(k1)) : occ0;
  uint64_t idx = kfrom == 0 ? 0 : idx0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    if (k >= kfrom) {
      bb b = set[k];
      if (k == ka) b ^= xa;
      if (k == kb) b ^= xb;
      b = xform(b, mirror, flip);
      bb occ2 = occ | b;
      uint32_t s = 0;
      int j = 1;
      while (b) {
        int x = pop_lsb(b);
        s += bin[j * 64 + x - __popcll(occ & (bit(x) - 1))];
        j++;
      }
      idx += (uint64_t)s * X.factor[k];
      occ = occ2;
    }
  }
  return idx;
}

// Code that few positions reach is compiled out of line (TBG_COLD, on by
// default), so that the hot loops of the persistent kernel -- whose warps
// run different ops at once -- stay within the instruction cache.  The sets
// travel by value (a struct), which keeps the caller's set[] in registers.
#ifndef TBG_COLD
#define TBG_COLD 1
#endif
#if TBG_COLD
#define TBG_COLD_FN __noinline__
#else
#define TBG_COLD_FN __forceinline__
#endif

template <int NS>
struct SetsV {
  bb s[NS];
};

template <int NS>
__device__ __forceinline__ SetsV<NS> sets_v(const bb *set) {
  SetsV<NS> v;
#pragma unroll
  for (int k = 0; k < NS; k++) v.s[k] = set[k];
  return v;
}

// rank_mod for the rare paths: king steps into a transformed slice, the
// diagonal double mark, sets of more than four pieces.
template <int NS>
__device__ TBG_COLD_FN uint64_t rank_mod_cold(const DIdx &X, const uint32_t *bin, int k0, int k1,
                                              SetsV<NS> v, int ka, bb xa, int kb, bb xb,
                                              int mirror, int flip) {
  return rank_mod<NS>(X, bin, k0, k1, v.s, ka, xa, kb, xb, mirror, flip);
}

// ------------------------------------------------------- incremental ranks
// A position's index is the sum over its sets of each set's combinatorial
// rank among the squares left free by the kings and the sets before it,
// times the set's factor (sq_to_idx_helper, tb8gen.c:129-149).  When one
// piece moves from a to b (or a king does, with no normalising transform),
// a later set's rank changes only if one of its squares lies strictly
// between a and b: only those squares change their count of occupied
// squares below them.  The kernels keep each set's share and recompute
// only the shares that change.

// Squares strictly between a and b (a != b).
__device__ __forceinline__ bb between(int a, int b) {
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return (bit(hi) - 1) & ~((bit(lo) << 1) - 1);
}

// Rank of one set's squares among the squares not in occ.
__device__ __forceinline__ uint32_t rank_one(bb b, bb occ, const uint32_t *bin) {
  uint32_t s = 0;
  int j = 1;
  while (b) {
    const int x = pop_lsb(b);
    s += bin[j * 64 + x - __popcll(occ & (bit(x) - 1))];
    j++;
  }
  return s;
}

template <int NS>
struct RankCtx {
  bb pre_occ[NS];        // kings + sets before k
  uint64_t pre_idx[NS];  // the shares of the sets before k
  uint64_t share[NS];    // set k's share of the index
};

template <int NS>
__device__ __forceinline__ void rank_ctx(RankCtx<NS> &c, const DIdx &X, const uint32_t *bin,
                                         int k0, int k1, const bb *set) {
  bb occ = bit(k0) | bit(k1);
  uint64_t idx = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    c.pre_occ[k] = occ;
    c.pre_idx[k] = idx;
    c.share[k] = (uint64_t)rank_one(set[k], occ, bin) * X.factor[k];
    idx += c.share[k];
    occ |= set[k];
  }
}

// Index after a piece of set k moves from x to `to` (same kings, no
// transform).
template <int NS>
__device__ __forceinline__ uint64_t rank_move(const RankCtx<NS> &c, const DIdx &X,
                                              const uint32_t *bin, const bb *set, int k, int x,
                                              int to) {
  uint64_t idx = 0;
  bb occ = 0;
  const bb betw = between(x, to);
#pragma unroll
  for (int j = 0; j < NS; j++) {
    if (j < k) continue;
    if (j == k) {
      idx = c.pre_idx[j];
      const bb b = set[j] ^ (bit(x) | bit(to));
      idx += (uint64_t)rank_one(b, c.pre_occ[j], bin) * X.factor[j];
      occ = c.pre_occ[j] | b;
    } else {
      idx += (set[j] & betw) ? (uint64_t)rank_one(set[j], occ, bin) * X.factor[j] : c.share[j];
      occ |= set[j];
    }
  }
  return idx;
}

// Index after a king moves from `from` to `to` with no normalising
// transform; nk0, nk1 are the kings after the move.
template <int NS>
__device__ __forceinline__ uint64_t rank_king_move(const RankCtx<NS> &c, const DIdx &X,
                                                   const uint32_t *bin, const bb *set, int nk0,
                                                   int nk1, int from, int to) {
  const bb betw = between(from, to);
  bb occ = bit(nk0) | bit(nk1);
  uint64_t idx = 0;
#pragma unroll
  for (int j = 0; j < NS; j++) {
    idx += (set[j] & betw) ? (uint64_t)rank_one(set[j], occ, bin) * X.factor[j] : c.share[j];
    occ |= set[j];
  }
  return idx;
}

// The set holding square sq (-1 if none), and set[l] for a run-time l,
// without indexing the register array at run time.
template <int NS>
__device__ __forceinline__ int set_of(const bb *set, int sq) {
  int l = -1;
#pragma unroll
  for (int q = 0; q < NS; q++)
    if ((set[q] >> sq) & 1) l = q;
  return l;
}

template <int NS>
__device__ __forceinline__ bb set_at(const bb *set, int l) {
  bb v = 0;
#pragma unroll
  for (int q = 0; q < NS; q++)
    if (q == l) v = set[q];
  return v;
}

__device__ __forceinline__ void report(DevStatus *st, unsigned code, unsigned where,
                                       unsigned long long info) {
  if (atomicCAS(&st->err, 0u, code) == 0u) {
    st->where = where;
    st->info = info;
  }
}

// Bit set / test in a slice bitmap of n positions; an index outside the
// slice is reported and skipped (it would mean a broken position).
__device__ __forceinline__ void mark(uint32_t *bits, uint64_t idx, uint64_t n, DevStatus *st) {
  if (idx >= n) {
    report(st, 1, 2, idx);
    return;
  }
  // a fire-and-forget reduction (RED): the old value is never needed
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(
                   __cvta_generic_to_global(bits + (idx >> 5))),
               "r"(1u << (idx & 31))
               : "memory");
}

__device__ __forceinline__ bool test(const uint32_t *bits, uint64_t idx, uint64_t n,
                                     DevStatus *st) {
  if (idx >= n) {
    report(st, 1, 3, idx);
    return false;
  }
  return (__ldg(bits + (idx >> 5)) >> (idx & 31)) & 1u;
}

// Test a bit of a sub bitmap (kslice_sub_get_address(s, l), kslice.h:63-73),
// refusing reads outside the bound buffer.
__device__ __forceinline__ bool test_sub(const uint8_t *sub, uint64_t len, uint64_t off,
                                         uint64_t idx, DevStatus *st) {
  uint64_t byte = off + (idx >> 3);
  if (sub == nullptr || byte >= len) {
    report(st, 2, 1, byte);
    return false;
  }
  return (__ldg(sub + byte) >> (idx & 7)) & 1u;
}

// ------------------------------------------------------ tile compaction
// Calls f(idx) for every set bit idx < nbits of bits[].  If kClear, f
// returns true to clear the bit and the tile is written back in place, or,
// with out != nullptr, the surviving bits of every word of the scanned range
// go to out (out = in & ~cleared) and bits[] is left untouched.
// With kContig each thread takes a contiguous run of the tile's list (in
// index order within each warp's segment) so that consecutive positions of
// one thread share their leading index digits; otherwise entries go
// round-robin.  begin(t) runs (block-wide) before the tile's entries,
// end(t) after them.
struct NoHook {
  __device__ void operator()(uint64_t) const {}
};

// One compaction round: appends the set bits of w[0..3] (this thread's four
// words of the tile) to list[] while there is room, clearing them from w;
// returns the number of entries (capped at kListCap).  Block-wide.
__device__ __forceinline__ int compact_round(uint32_t *w, uint32_t *list, int *list_n) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) *list_n = 0;
  __syncthreads();
  int c = __popc(w[0]) + __popc(w[1]) + __popc(w[2]) + __popc(w[3]);
  int incl = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += y;
  }
  int base = 0;
  if (lane == 31) base = atomicAdd(list_n, incl);
  base = __shfl_sync(0xffffffffu, base, 31);
  int pos = base + incl - c;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    while (w[i] && pos < kListCap) {
      int b = __ffs(w[i]) - 1;
      w[i] &= w[i] - 1;
      list[pos++] = (uint32_t)((threadIdx.x * 4 + i) * 32 + b);
    }
  }
  __syncthreads();
  return min(*list_n, kListCap);
}

// This thread's contiguous share [e0, e1) of n list entries.
// The n % blockDim.x threads that take one entry more are the lowest ones,
// so they fill whole warps: a warp runs as long as its busiest lane, and
// spreading the extra entries over every warp would make every warp run
// the longer time.
__device__ __forceinline__ void my_share(int n, int &e0, int &e1) {
  const int q = n / (int)blockDim.x, r = n % (int)blockDim.x, t = threadIdx.x;
  e0 = t * q + min(t, r);
  e1 = e0 + q + (t < r ? 1 : 0);
}

// The verify's scan of one tile in two passes per compaction round: quick(idx)
// runs on every candidate and returns 0 (refuted), 1 (survives the quick
// test); the survivors are compacted into list2 and full(idx) (true:
// refuted) runs on them only.  Work per thread is then nearly uniform in the
// first pass, and the divergent full check runs on a dense list, handed out
// 32 survivors at a time to whichever warp is free (n2[0]: survivors,
// n2[1]: next survivor to hand out).
template <class Q, class F>
__device__ __forceinline__ void scan_tile_verify(uint64_t t, uint32_t *bits, uint64_t nbits,
                                                 uint32_t *list, uint32_t *list2, uint32_t *clr,
                                                 int *list_n, int *n2, Q &&quick, F &&full,
                                                 uint32_t *out, int lo = 0, int hi = kTileWords) {
  const uint64_t nwords = (nbits + 31) >> 5;
  const uint64_t w0 = t * kTileWords + threadIdx.x * 4;
  uint32_t w[4];
  if (w0 + 4 <= nwords) {
    uint4 v = *reinterpret_cast<const uint4 *>(bits + w0);
    w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = w0 + i < nwords ? bits[w0 + i] : 0u;
  }
  uint32_t raw[4] = {w[0], w[1], w[2], w[3]};
  const bool mine = threadIdx.x * 4 >= lo && threadIdx.x * 4 < hi;  // the part's words
#pragma unroll
  for (int i = 0; i < 4; i++) {
    uint64_t base = (w0 + i) * 32;
    if (base + 32 > nbits) w[i] &= base < nbits ? (1u << (nbits - base)) - 1u : 0u;
    if (!mine) w[i] = 0;
    clr[threadIdx.x * 4 + i] = 0;
  }
  const uint64_t tbase = t * (uint64_t)kTileWords * 32;
  for (;;) {
    if (threadIdx.x == 0) *n2 = 0;
    const int n = compact_round(w, list, list_n);
    int e0, e1;
    my_share(n, e0, e1);
    for (int e = e0; e < e1; e++) {
      uint32_t off = list[e];
      if (quick(tbase + off)) list2[atomicAdd(n2, 1)] = off;
      else atomicOr(&clr[off >> 5], 1u << (off & 31));
    }
    if (threadIdx.x == 0) n2[1] = 0;
    __syncthreads();
    const int m = *n2;
    // the full checks take uneven time: warps take 32 survivors at a time
    for (;;) {
      int base = 0;
      if ((threadIdx.x & 31) == 0) base = atomicAdd(&n2[1], 32);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= m) break;
      const int e = base + (threadIdx.x & 31);
      if (e < m) {
        uint32_t off = list2[e];
        if (full(tbase + off)) atomicOr(&clr[off >> 5], 1u << (off & 31));
      }
    }
    if (!__syncthreads_or((w[0] | w[1] | w[2] | w[3]) != 0)) break;
  }
  __syncthreads();
  if (!mine) {
    // another part of the tile owns these words
  } else if (out != nullptr) {
    if (w0 + 4 <= nwords) {
      uint4 v = make_uint4(raw[0] & ~clr[threadIdx.x * 4], raw[1] & ~clr[threadIdx.x * 4 + 1],
                           raw[2] & ~clr[threadIdx.x * 4 + 2], raw[3] & ~clr[threadIdx.x * 4 + 3]);
      *reinterpret_cast<uint4 *>(out + w0) = v;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (w0 + i < nwords) out[w0 + i] = raw[i] & ~clr[threadIdx.x * 4 + i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      uint32_t cm = clr[threadIdx.x * 4 + i];
      if (cm && w0 + i < nwords) bits[w0 + i] &= ~cm;
    }
  }
  __syncthreads();
}

template <bool kClear, bool kContig, class F, class B = NoHook, class E = NoHook>
__device__ __forceinline__ void scan_tile(uint64_t t, uint32_t *bits, uint64_t nbits,
                                          uint32_t *list, uint32_t *clr, int *list_n, F &&f,
                                          uint32_t *out = nullptr, B begin = B(), E end = E(),
                                          int lo = 0, int hi = kTileWords) {
  const uint64_t nwords = (nbits + 31) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = t * kTileWords + threadIdx.x * 4;
  uint32_t w[4];
  if (w0 + 4 <= nwords) {
    uint4 v = *reinterpret_cast<const uint4 *>(bits + w0);
    w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = w0 + i < nwords ? bits[w0 + i] : 0u;
  }
  uint32_t raw[4] = {w[0], w[1], w[2], w[3]};
  const bool mine = threadIdx.x * 4 >= lo && threadIdx.x * 4 < hi;  // the part's words
#pragma unroll
  for (int i = 0; i < 4; i++) {
    uint64_t base = (w0 + i) * 32;
    if (base + 32 > nbits) w[i] &= base < nbits ? (1u << (nbits - base)) - 1u : 0u;
    if (!mine) w[i] = 0;
  }
  if (kClear) {
#pragma unroll
    for (int i = 0; i < 4; i++) clr[threadIdx.x * 4 + i] = 0;
  }
  begin(t);
  for (;;) {
    if (threadIdx.x == 0) *list_n = 0;
    __syncthreads();
    int c = __popc(w[0]) + __popc(w[1]) + __popc(w[2]) + __popc(w[3]);
    int incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += y;
    }
    int base = 0;
    if (lane == 31) base = atomicAdd(list_n, incl);
    base = __shfl_sync(0xffffffffu, base, 31);
    int pos = base + incl - c;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      while (w[i] && pos < kListCap) {
        int b = __ffs(w[i]) - 1;
        w[i] &= w[i] - 1;
        list[pos++] = (uint32_t)((threadIdx.x * 4 + i) * 32 + b);
      }
    }
    __syncthreads();
    const int n = min(*list_n, kListCap);
    const uint64_t tbase = t * (uint64_t)kTileWords * 32;
    int e0, e1, es;
    if (kContig) {
      my_share(n, e0, e1);
      es = 1;
    } else {
      e0 = threadIdx.x;
      e1 = n;
      es = blockDim.x;
    }
    for (int e = e0; e < e1; e += es) {
      uint32_t off = list[e];
      bool c2 = f(tbase + off);
      if (kClear && c2) atomicOr(&clr[off >> 5], 1u << (off & 31));
    }
    if (!__syncthreads_or((w[0] | w[1] | w[2] | w[3]) != 0)) break;
  }
  end(t);
  if (kClear) {
    __syncthreads();
    if (!mine) {
      // another part of the tile owns these words
    } else if (out != nullptr) {
      if (w0 + 4 <= nwords) {
        uint4 v = make_uint4(raw[0] & ~clr[threadIdx.x * 4], raw[1] & ~clr[threadIdx.x * 4 + 1],
                             raw[2] & ~clr[threadIdx.x * 4 + 2], raw[3] & ~clr[threadIdx.x * 4 + 3]);
        *reinterpret_cast<uint4 *>(out + w0) = v;
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++)
          if (w0 + i < nwords) out[w0 + i] = raw[i] & ~clr[threadIdx.x * 4 + i];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        uint32_t cm = clr[threadIdx.x * 4 + i];
        if (cm && w0 + i < nwords) bits[w0 + i] &= ~cm;
      }
    }
    __syncthreads();
  }
}

__device__ __forceinline__ uint64_t tiles_of(uint64_t nbits) {
  return (((nbits + 31) >> 5) + kTileWords - 1) / kTileWords;
}

// ------------------------------------------------------- incremental deindex
// Positions of one row (all digits but the last set's equal) share the
// sets 0..L-1 (L = numsets - 1); a thread walking increasing indices keeps
// them and re-unranks only the last set while the row does not change.
struct RowCache {
  uint64_t row = ~0ull;
  uint64_t row_base = 0;   // index of the row's first position
  bb occ_head = 0;         // kings + sets 0..L-1
};

template <int NS>
__device__ __forceinline__ bb unrank_cached(const DIdx &X, const uint32_t *bin, uint64_t idx,
                                           int k0, int k1, bb *set, RowCache &rc) {
  constexpr int L = NS - 1;
  uint64_t row = 0, F = X.size;
  if (L > 0) {
    F = X.factor[L > 0 ? L - 1 : 0];
    row = idx < (1ull << 32) ? fast_div32((uint32_t)idx, X.fdiv[L > 0 ? L - 1 : 0]) : idx / F;
  }
  if (row != rc.row) {
    bb occ = unrank_sets<NS>(X, bin, idx, k0, k1, set);
    bb last = 0;
#pragma unroll
    for (int k = 0; k < NS; k++)
      if (k == L) last = set[k];
    rc.row = row;
    rc.row_base = row * F;
    rc.occ_head = occ & ~last;
    return occ;
  }
  // same row: only the last set changes
  uint32_t d = (uint32_t)(idx - rc.row_base);
  bb freeb = ~rc.occ_head, sb = 0;
  int m = X.mult[L];
  for (int i = m - 1; i > 0; i--) {
    const uint32_t *rowb = bin + (i + 1) * 64;
    int lo = i, hi = 63;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (rowb[mid] <= d) lo = mid;
      else hi = mid;
    }
    d -= rowb[lo];
    sb |= bit(nth_set(freeb, lo));
  }
  if (m > 0) sb |= bit(nth_set(freeb, (int)d));
#pragma unroll
  for (int k = 0; k < NS; k++)
    if (k == L) set[k] = sb;
  return rc.occ_head | sb;
}

// ----------------------------------------------------------- W step
// mark_king_unmoves (tb8gen.c:246-262) for a position with an optional
// uncaptured piece (set kb, square xb) on the king's old square.
template <int NS>
__device__ __forceinline__ void mark_king_unmoves(const SliceJob &J, const KingDest *kd,
                                                  const DMat &M, const uint32_t *bin,
                                                  const bb *set, bb occ, int kb, bb xb,
                                                  DevStatus *st,
                                                  const RankCtx<NS> *c = nullptr) {
  int opp = J.stm ? J.k0 : J.k1;
  const int me = J.stm ? J.k1 : J.k0;
  bb dest = ~(occ | king_attacks(opp));
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = kd[d];
    if (!(dest & bit(D.to))) continue;
    uint64_t i;
    if (c != nullptr && kb < 0 && D.mirror == 0 && D.flip == 0)
      i = rank_king_move<NS>(*c, M.ii, bin, set, D.k0, D.k1, me, D.to);
    else
      i = rank_mod<NS>(M.ii, bin, D.k0, D.k1, set, -1, 0, kb, xb, D.mirror, D.flip);
    mark(D.bits, i, M.ii.size, st);
    if (D.dbl) {
      // mirror_diagonal (tb8gen.c:240-244) of the normalised position: the
      // kings are on the diagonal, so the transpose acts on the sets only.
      int m2 = D.mirror;
      uint64_t i2 = rank_mod<NS>(M.ii, bin, D.k0, D.k1, set, -1, 0, kb, xb, m2, D.flip ^ 1);
      mark(D.bits, i2, M.ii.size, st);
    }
  }
}

// The king destinations, copied from the kernel parameters into shared
// memory once per block (indexed at run time below).
__device__ __forceinline__ void load_dests(const SliceJob &J, KingDest *kd) {
#pragma unroll
  for (int d = 0; d < 8; d++)
    if (threadIdx.x == d) kd[d] = J.kd[d];
}

// mark_unmoves (tb8gen.c:264-276) for every non-king piece of the side to
// move, optionally with an uncaptured piece (set kb, square taken from the
// moving piece's origin).
template <int NS>
__device__ __forceinline__ void mark_piece_unmoves(const SliceJob &J, const DMat &M,
                                                   const uint32_t *bin, const bb *set,
                                                   bb occ, int kb, DevStatus *st,
                                                   const RankCtx<NS> *c = nullptr) {
#pragma unroll
  for (int k = 0; k < NS; k++) {
    if (M.set_color[k] == J.stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb mv = piece_attacks(M.set_type[k], x, occ) & ~occ;
        while (mv) {
          int to = pop_lsb(mv);
          uint64_t i;
          if (kb < 0 && c != nullptr)
            i = rank_move<NS>(*c, M.ii, bin, set, k, x, to);
          else if (kb < 0)
            i = rank_mod<NS>(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), -1, 0, 0, 0);
          else
            i = rank_mod<NS>(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), kb, bit(x), 0, 0);
          mark(J.self, i, M.ii.size, st);
        }
      }
    }
  }
}

// ------------------------------------------------ incremental index updates
// A move changes few terms of the index (sq_to_idx_helper, tb8gen.c:129-149:
// per set, the sum over its squares in increasing order of C(r, i + 1), r
// the square's rank among the squares not taken by the kings and earlier
// sets).  The scatter updates the source's index by those terms instead of
// ranking the target position afresh.

// Rank of square q among the squares not in occ.
__device__ __forceinline__ int free_rank(int q, bb occ) {
  return q - __popcll(occ & (bit(q) - 1));
}

// Index change, over the sets j >= j0, when a king or a piece of a set
// below j0 moves from a to b: a square q of set j strictly between a and b
// has one occupied square more or fewer below it, so its rank r moves by
// one and its term C(r, i + 1) by C(r, i) (upward move) or by -C(r - 1, i)
// (downward), Pascal's rule, i being q's place in its set; no other term
// changes.  `kings`: the king squares before the move.
template <int NS>
__device__ __forceinline__ uint64_t seg_delta(const DIdx &X, const uint32_t *bin, const bb *set,
                                              bb kings, int j0, bb betw, bool up);

template <int NS>
__device__ __forceinline__ uint64_t cross_delta(const DIdx &X, const uint32_t *bin,
                                                const bb *set, bb kings, int j0, int a, int b) {
  return seg_delta<NS>(X, bin, set, kings, j0, between(a, b), a < b);
}

// The same sum over the squares of `betw` only (the move's squares lie on
// one side: up, or down): a slider's index along a ray adds the terms of the
// squares between one target and the next.
template <int NS>
__device__ __forceinline__ uint64_t seg_delta(const DIdx &X, const uint32_t *bin, const bb *set,
                                              bb kings, int j0, bb betw, bool up) {
  bb occ = kings;
  uint64_t d = 0;
#pragma unroll
  for (int j = 0; j < NS; j++) {
    if (j >= j0) {
      bb c = set[j] & betw;
      while (c) {
        const int q = pop_lsb(c);
        const bb below = bit(q) - 1;
        const int r = q - __popcll(occ & below);
        const int i = __popcll(set[j] & below);
        const uint64_t v = (uint64_t)(up ? bin[i * 64 + r] : bin[i * 64 + r - 1]) * X.factor[j];
        d = up ? d + v : d - v;
      }
    }
    occ |= set[j];
  }
  return d;
}

// One piece of a set of at most 4 about to move: its set's rank after the
// move to a square of rank rto with `pos` of the set's other pieces below
// it is C(rto, pos + 1) + g[pos], where, with the others' ranks o_0 < o_1
// < ..., g[pos] = sum_{i < pos} C(o_i, i + 1) + sum_{i >= pos} C(o_i, i + 2)
// (the others below the destination keep their places, those above move
// up one).
struct Mover {
  bb others;
  uint32_t g[4];
};

__device__ __forceinline__ void mover_init(Mover &mv, const uint32_t *bin, bb setk, int x,
                                           bb occk) {
  mv.others = setk & ~bit(x);
  uint32_t a[3], b[3];
  bb o = mv.others;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    a[i] = b[i] = 0;
    if (o) {
      const int r = free_rank(pop_lsb(o), occk);
      a[i] = bin[(i + 1) * 64 + r];
      b[i] = bin[(i + 2) * 64 + r];
    }
  }
  mv.g[0] = b[0] + b[1] + b[2];
  mv.g[1] = a[0] + b[1] + b[2];
  mv.g[2] = a[0] + a[1] + b[2];
  mv.g[3] = a[0] + a[1] + a[2];
}

__device__ __forceinline__ uint32_t mover_rank(const Mover &mv, const uint32_t *bin, int to,
                                               bb occk) {
  const bb below = bit(to) - 1;
  const int pos = __popcll(mv.others & below);
  const int rto = to - __popcll(occk & below);
  uint32_t g = mv.g[0];
#pragma unroll
  for (int p = 1; p < 4; p++)
    if (pos == p) g = mv.g[p];
  return bin[(pos + 1) * 64 + rto] + g;
}

// predecessors_worker's unmoves of one source position (mark_king_unmoves
// and mark_unmoves, tb8gen.c:246-276) with the targets' indices updated
// from the source's index idx: a king step without a normalising
// transform changes only the terms of the squares it passes over; a piece
// step changes its own set's rank (mover_rank) and the terms of the later
// sets' squares it passes over.  Sets of more than 4 pieces, and king steps
// into a transformed slice, are ranked afresh.
//
// With J.filter (the opponent's "wins" of slice s, tbg_candidates) the
// sliders' unmoves into slice s are filtered: a predecessor P whose piece
// stands on the ray from x at t_k can step to the ray's next square toward
// x (t_{k-1}), or, at t_1, away from it (t_2); both squares are empty, and
// the position reached is the one the unmove to that square gives.  If
// that position is not in the opponent's "wins", P has a quiet move out of
// them and cannot be lost (check_moves, tb8gen.c:594-602): it is not
// marked.  A ray of one square, knights and king unmoves are marked as
// before.
template <int NS>
__device__ __forceinline__ void mark_unmoves_inc(const SliceJob &J, const KingDest *kd,
                                                 const DMat &M, const uint32_t *bin,
                                                 const bb *set, bb occ, uint64_t idx,
                                                 DevStatus *st) {
  const DIdx &X = M.ii;
  const bb kings = bit(J.k0) | bit(J.k1);
  const int opp = J.stm ? J.k0 : J.k1;
  const int me = J.stm ? J.k1 : J.k0;
  const bb dest = ~(occ | king_attacks(opp));
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = kd[d];
    if (!(dest & bit(D.to))) continue;
    const uint64_t i =
        (D.mirror == 0 && D.flip == 0)
            ? idx + cross_delta<NS>(X, bin, set, kings, 0, me, D.to)
            : rank_mod_cold<NS>(X, bin, D.k0, D.k1, sets_v<NS>(set), -1, 0, -1, 0, D.mirror,
                                D.flip);
    mark(D.bits, i, X.size, st);
    if (D.dbl) {
      // mirror_diagonal (tb8gen.c:240-244) of the normalised position
      const uint64_t i2 = rank_mod_cold<NS>(X, bin, D.k0, D.k1, sets_v<NS>(set), -1, 0, -1, 0,
                                            D.mirror, D.flip ^ 1);
      mark(D.bits, i2, X.size, st);
    }
  }
  bb occk = kings;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const bb setk = set[k];
    if (M.set_color[k] == J.stm) {
      const bool inc = X.mult[k] <= 4;
      const uint64_t base = idx - (uint64_t)rank_one(setk, occk, bin) * X.factor[k];
      const int type = M.set_type[k];
      bb pcs = setk;
      while (pcs) {
        const int x = pop_lsb(pcs);
        Mover mv;
        if (inc) mover_init(mv, bin, setk, x, occk);
        auto index_of = [&](int to) -> uint64_t {
          return inc ? base + (uint64_t)mover_rank(mv, bin, to, occk) * X.factor[k] +
                           cross_delta<NS>(X, bin, set, kings, k + 1, x, to)
                     : rank_mod_cold<NS>(X, bin, J.k0, J.k1, sets_v<NS>(set), k,
                                         bit(x) | bit(to), -1, 0, 0, 0);
        };
        if (inc && type >= 3 && type <= 5) {
          // A slider's targets along each ray, each index updated from the
          // previous square's: the occupied squares below the target (for
          // its rank among the free squares) and the other pieces of its set
          // below it change by the squares passed in square order, and so
          // does the later sets' term sum (seg_delta).  Same indices as
          // mover_rank + cross_delta.
          const bb others = setk & ~bit(x);
          const int cnt0 = __popcll(occk & (bit(x) - 1)), pos0 = __popcll(others & (bit(x) - 1));
          const int d0 = type == 3 ? 4 : 0, d1 = type == 4 ? 4 : 8;
          for (int d = d0; d < d1; d++) {
            // directions: 0 E, 1 W, 2 N, 3 S, 4 NE, 5 NW, 6 SE, 7 SW
            const int df = (d == 0 || d == 4 || d == 6) ? 1 : (d == 1 || d == 5 || d == 7) ? -1 : 0;
            const int dr = (d == 2 || d == 4 || d == 5) ? 1 : (d == 3 || d == 6 || d == 7) ? -1 : 0;
            const bool up = dr > 0 || (dr == 0 && df > 0);
            int f = x & 7, r = x >> 3, n = 0, cur = x, cnt = cnt0, pos = pos0;
            uint64_t dx = 0, i_prev = 0, i_first = 0;
            for (;;) {
              f += df;
              r += dr;
              if ((unsigned)f > 7u || (unsigned)r > 7u) break;
              const int to = r * 8 + f;
              if ((occ >> to) & 1) break;
              const bb seg = between(cur, to);
              const int sc = __popcll(occk & seg), so = __popcll(others & seg);
              cnt += up ? sc : -sc;
              pos += up ? so : -so;
              if (seg) dx += seg_delta<NS>(X, bin, set, kings, k + 1, seg, up);
              cur = to;
              uint32_t g = mv.g[0];
#pragma unroll
              for (int p = 1; p < 4; p++)
                if (pos == p) g = mv.g[p];
              const uint64_t i =
                  base + (uint64_t)(bin[(pos + 1) * 64 + (to - cnt)] + g) * X.factor[k] + dx;
              if (J.filter == nullptr) {
                mark(J.self, i, X.size, st);
              } else if (n == 0) {
                i_first = i;
              } else {
                if (n == 1 && test(J.filter, i, X.size, st)) mark(J.self, i_first, X.size, st);
                if (test(J.filter, i_prev, X.size, st)) mark(J.self, i, X.size, st);
              }
              i_prev = i;
              n++;
            }
            if (J.filter != nullptr && n == 1) mark(J.self, i_first, X.size, st);
          }
        } else if (J.filter != nullptr && type >= 3 && type <= 5) {
          const int d0 = type == 3 ? 4 : 0, d1 = type == 4 ? 4 : 8;
          for (int d = d0; d < d1; d++) {
            // directions: 0 E, 1 W, 2 N, 3 S, 4 NE, 5 NW, 6 SE, 7 SW
            const int df = (d == 0 || d == 4 || d == 6) ? 1 : (d == 1 || d == 5 || d == 7) ? -1 : 0;
            const int dr = (d == 2 || d == 4 || d == 5) ? 1 : (d == 3 || d == 6 || d == 7) ? -1 : 0;
            int f = x & 7, r = x >> 3, n = 0;
            uint64_t i_prev = 0, i_first = 0;
            for (;;) {
              f += df;
              r += dr;
              if ((unsigned)f > 7u || (unsigned)r > 7u) break;
              const int to = r * 8 + f;
              if ((occ >> to) & 1) break;
              const uint64_t i = index_of(to);
              if (n == 0) {
                i_first = i;
              } else {
                if (n == 1 && test(J.filter, i, X.size, st)) mark(J.self, i_first, X.size, st);
                if (test(J.filter, i_prev, X.size, st)) mark(J.self, i, X.size, st);
              }
              i_prev = i;
              n++;
            }
            if (n == 1) mark(J.self, i_first, X.size, st);
          }
        } else {
          bb to_set = piece_attacks(type, x, occ) & ~occ;
          while (to_set) mark(J.self, index_of(pop_lsb(to_set)), X.size, st);
        }
      }
    }
    occk |= setk;
  }
}

// ------------------------------------------------------ bulk tile staging
// A scatter tile's words come into shared memory by the copy engine
// (cp.async.bulk, completing on an mbarrier), the next tile of an item
// while the block processes the current one.  The phase bits of the two
// buffers' barriers (bit b: the parity buffer b's next copy completes) are
// kept by the kernel in a register, the same in every thread.  The source is this GPU's own
// memory and nothing is multicast.  Every wait is bounded: a copy that has
// not landed after kBulkPolls polls is reported (status 5) and the block
// reads its tiles with plain loads from then on.
#ifndef TBG_BULK
#define TBG_BULK 1
#endif
constexpr long kBulkPolls = 1L << 22;

struct BulkStage {
  uint4 buf[2][kThreads];       // two tiles of kTileWords words
  unsigned long long bar[2];    // their mbarriers
  int off;                      // a wait ran out: plain loads only
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bulk_init(BulkStage &B) {
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; b++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&B.bar[b])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    B.off = 0;
  }
}

// Thread 0: tile t of a bitmap of `words` 32-bit words (a multiple of 16:
// bitmaps are 64-byte rounded) into buffer b.  The block's earlier reads of
// that buffer are done (a barrier lies between them and this call).
__device__ __forceinline__ void bulk_issue(BulkStage &B, int b, const uint32_t *bits,
                                           uint64_t words, uint64_t t) {
  const uint64_t w0 = t * kTileWords;
  const uint32_t bytes = (uint32_t)(min((uint64_t)kTileWords, words - w0) * 4);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&B.bar[b])),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(&B.buf[b][0])),
      "l"(bits + w0), "r"(bytes), "r"(smem_addr(&B.bar[b]))
      : "memory");
}

// Every thread: waits (bounded) for buffer b's copy; false if it ran out.
__device__ __forceinline__ bool bulk_wait(BulkStage &B, int b, uint32_t ph, DevStatus *st) {
  const uint32_t parity = (ph >> b) & 1u;
  for (long n = 0; n < kBulkPolls; n++) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_addr(&B.bar[b])), "r"(parity)
        : "memory");
    if (done) return true;
  }
  report(st, 5, (unsigned)b, 0);
  return false;
}

// The sources of tiles [t0, t0 + ntile) of bits[] (within each tile only
// its words [lo, hi)), gathered into one shared list until it holds
// kFlush entries (or a tile's sources do not fit), then handed to f(idx)
// in contiguous shares: every thread of the block gets the same number of
// sources, give or take one, and neighbouring indices.  An entry is the
// tile's place in the group (bits 15 and up) and the position's offset in
// its tile.
//
// The list's entry count alternates between two counters, gcnt[gp] and
// gcnt[gp ^ 1] (gp: the block's current one, kept by the caller across
// calls; both counters start at zero with the kernel): a flush zeroes the
// other counter, whose last readers read it before the previous flush's
// closing barrier, so a flushed round costs two barriers (the count's and
// the flush's), not a reset with barriers of its own.
constexpr int kFlush = kThreads * 4;

template <class F>
__device__ __forceinline__ void scan_group(uint64_t t0, int ntile, const uint32_t *bits,
                                           uint64_t nbits, uint32_t *list, int *gcnt, int &gp,
                                           BulkStage &B, uint32_t &ph, DevStatus *st, F &&f,
                                           int lo = 0, int hi = kTileWords) {
  const uint64_t nwords = (nbits + 31) >> 5;
  const uint64_t words64 = ((nbits + 511) >> 9) << 4;  // the 64-byte rounded bitmap
  const int lane = threadIdx.x & 31;
  const bool mine = threadIdx.x * 4 >= lo && threadIdx.x * 4 < hi;
  const bool bulk = TBG_BULK && !B.off;
  if (bulk && threadIdx.x == 0) bulk_issue(B, 0, bits, words64, t0);
  for (int g = 0; g < ntile; g++) {
    const uint64_t t = t0 + g;
    const uint64_t w0 = t * kTileWords + threadIdx.x * 4;
    const int b = g & 1;
    // the next tile's copy, into the buffer every thread finished reading
    // before the last tile's first barrier
    if (bulk && g + 1 < ntile && threadIdx.x == 0) bulk_issue(B, b ^ 1, bits, words64, t + 1);
    bool staged = false;
    if (bulk) {
      staged = bulk_wait(B, b, ph, st);
      ph ^= 1u << b;
      if (!staged && threadIdx.x == 0) B.off = 1;
    }
    uint32_t w[4];
    if (staged) {
      const uint4 v = w0 + 4 <= words64 ? B.buf[b][threadIdx.x] : make_uint4(0, 0, 0, 0);
      w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else if (w0 + 4 <= nwords) {
      const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(bits + w0));
      w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) w[i] = w0 + i < nwords ? bits[w0 + i] : 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint64_t base = (w0 + i) * 32;
      if (base + 32 > nbits) w[i] &= base < nbits ? (1u << (nbits - base)) - 1u : 0u;
      if (!mine) w[i] = 0;
    }
    for (;;) {
      const int c = __popc(w[0]) + __popc(w[1]) + __popc(w[2]) + __popc(w[3]);
      int incl = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
      }
      int *cnt = gcnt + gp;
      int base = 0;
      if (lane == 31 && incl) base = atomicAdd(cnt, incl);
      base = __shfl_sync(0xffffffffu, base, 31);
      int pos = base + incl - c;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        while (w[i] && pos < kListCap) {
          const int b = __ffs(w[i]) - 1;
          w[i] &= w[i] - 1;
          list[pos++] = ((uint32_t)g << 15) | (uint32_t)((threadIdx.x * 4 + i) * 32 + b);
        }
      }
      const int more = __syncthreads_or((w[0] | w[1] | w[2] | w[3]) != 0);
      const int n = min(*cnt, kListCap);
      if (more || n >= kFlush || g == ntile - 1) {
        if (threadIdx.x == 0) gcnt[gp ^ 1] = 0;
        int e0, e1;
        my_share(n, e0, e1);
        for (int e = e0; e < e1; e++) {
          const uint32_t v = list[e];
          f((t0 + (v >> 15)) * (uint64_t)(kTileWords * 32) + (v & 32767u));
        }
        // every entry is read (and the count by everyone) before the next
        // round appends, on the other counter
        __syncthreads();
        gp ^= 1;
      } else {
        // every thread has read the count before the next tile appends
        __syncthreads();
      }
      if (!more) break;
    }
  }
}

// Shared memory of the sparse kernels (one tile at a time).
struct SparseSmem {
  uint32_t bin[7 * 64];
  KingDest kd[8];
  uint32_t list[kListCap];
  uint32_t clr[kTileWords];     // verify: cleared candidates of the tile
  uint32_t list2[kListCap];     // verify: survivors of the quick test
  int list_n;
  int n2[2];
  int gcnt[2];                  // scatter: the list's two alternating counts
  __align__(128) BulkStage B;   // scatter: staged source tiles
};

// The scatter's alternating counts start at zero (before the kernel's
// first barrier); gp selects the current one.
__device__ __forceinline__ void init_gcnt(SparseSmem &S) {
  if (threadIdx.x == 0) {
    S.gcnt[0] = 0;
    S.gcnt[1] = 0;
  }
}

// Tiles [t0, t0 + ntile) of predecessors_worker (tb8gen.c:484-516): every
// source's unmoves marked (within each tile only the words [lo, hi)).
template <int NS>
__device__ __forceinline__ void tile_predecessors(const SliceJob &J, SparseSmem &S, int &gp,
                                                  uint32_t &ph, uint64_t t0, int ntile,
                                                  DevStatus *st, int lo = 0,
                                                  int hi = kTileWords) {
  const DMat &M = c_mats[J.mat];
  bb set[NS];
  RowCache rc;
  scan_group(
      t0, ntile, J.src, J.nbits, S.list, S.gcnt, gp, S.B, ph, st,
      [&](uint64_t idx) {
        const bb occ = unrank_cached<NS>(M.ii, S.bin, idx, J.k0, J.k1, set, rc);
        mark_unmoves_inc<NS>(J, S.kd, M, S.bin, set, occ, idx, st);
      },
      lo, hi);
}

// predecessors_sub_worker (tb8gen.c:346-394): the source is the sub bitmap
// of captured set J.set (colour stm^1); each position is uncaptured by the
// king and by every non-king piece of stm.
template <int NS>
__device__ __forceinline__ void tile_predecessors_sub(const SliceJob &J, SparseSmem &S,
                                                      uint64_t t, DevStatus *st, int lo = 0,
                                                      int hi = kTileWords) {
  const DMat &M = c_mats[J.mat];
  const int kc = J.set;
  const DIdx &X = M.capt[kc];
  bb set[NS];
  RowCache rc;
  scan_tile<false, true>(t, const_cast<uint32_t *>(J.src), J.nbits, S.list, nullptr, &S.list_n,
                         [&](uint64_t idx) {
                           bb occ = unrank_cached<NS>(X, S.bin, idx, J.k0, J.k1, set, rc);
                           int me = J.stm ? J.k1 : J.k0;
                           if (J.legality &&
                               attacked_by<NS>(M, set, J.k0, J.k1, occ, me, J.stm ^ 1))
                             return false;
                           mark_king_unmoves<NS>(J, S.kd, M, S.bin, set, occ, kc, bit(me), st);
                           mark_piece_unmoves<NS>(J, M, S.bin, set, occ, kc, st);
                           return false;
                         },
                         nullptr, NoHook(), NoHook(), lo, hi);
}

// ----------------------------------------------------------- L step
// check_successors_worker (tb8gen.c:607-650) with check_moves (571-605) and
// check_king_moves (537-569).  True iff the candidate is to be cleared.
//
// A candidate survives iff it is legal and every successor is won for the
// opponent: a conjunction, so the tests may run in any order as long as the
// king captures, whose capture index the reference computes in its own way
// (see below), are reached exactly when the reference reaches them -- after
// legality and every non-king piece passed.  The quiet moves of the side's
// sets run first, the last set first: they are the cheapest (only the sets
// from the moving one on are re-ranked) and, at the densities of a ply, the
// most likely to refute.
template <int NS>
__device__ __forceinline__ bool refute(const SliceJob &J, const KingDest *kd, const DMat &M,
                                       const uint32_t *bin, const bb *set, bb occ,
                                       const RowCache &rc, DevStatus *st) {
  const int stm = J.stm;
  const int opp = stm ? J.k0 : J.k1;
  const int me = stm ? J.k1 : J.k0;
  // each set's share of the index, for the moves below
  RankCtx<NS> c;
  rank_ctx<NS>(c, M.ii, bin, J.k0, J.k1, set);
  bb own = 0;
#pragma unroll
  for (int k = 0; k < NS; k++)
    if (M.set_color[k] == stm) own |= set[k];
  // 1. quiet moves of the non-king pieces into "wins"
#pragma unroll
  for (int k = NS - 1; k >= 0; k--) {
    if (M.set_color[k] == stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb quiet = piece_attacks(M.set_type[k], x, occ) & ~occ;
        while (quiet) {
          int to = pop_lsb(quiet);
          uint64_t i = rank_move<NS>(c, M.ii, bin, set, k, x, to);
          if (!test(J.self, i, M.ii.size, st)) return true;
        }
      }
    }
  }
  // 2. legality: the side to move must not attack the other king
  if (attacked_by<NS>(M, set, J.k0, J.k1, occ, opp, stm)) return true;
  // 3. captures by the non-king pieces into sub/win
#pragma unroll
  for (int k = 0; k < NS; k++) {
    if (M.set_color[k] == stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb caps = piece_attacks(M.set_type[k], x, occ) & occ & ~own & ~bit(opp);
        while (caps) {
          int to = pop_lsb(caps);
          // one rank site for every captured set (keeps the code small)
          const int l = set_of<NS>(set, to);
          if (l < 0) continue;
          uint64_t i = rank_mod<NS>(M.capt[l], bin, J.k0, J.k1, set, k, bit(x) | bit(to), l,
                                    bit(to), 0, 0);
          if (!test_sub(J.self_sub, J.self_sub_len, M.sub_offset[l], i, st)) return true;
        }
      }
    }
  }
  // 4. King captures leave the captured piece in its slot and drop the set's
  // last slot (its highest square) from the capture index, as the reference
  // computes it (tb8gen.c:543-555).
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = kd[d];
    if (!(occ & bit(D.to))) continue;
    if (own & bit(D.to)) continue;
    const int l = set_of<NS>(set, D.to);
    if (l < 0) continue;
    uint64_t i = rank_mod<NS>(M.capt[l], bin, D.k0, D.k1, set, -1, 0, l,
                              bit(msb64(set_at<NS>(set, l))), D.mirror, D.flip);
    if (!test_sub(D.sub, D.sub_len, M.sub_offset[l], i, st)) return true;
  }
  // 5. quiet king moves into the neighbouring slices' "wins"
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = kd[d];
    if (occ & bit(D.to)) continue;
    const uint64_t i =
        (D.mirror == 0 && D.flip == 0)
            ? rank_king_move<NS>(c, M.ii, bin, set, D.k0, D.k1, me, D.to)
            : rank_mod<NS>(M.ii, bin, D.k0, D.k1, set, -1, 0, -1, 0, D.mirror, D.flip);
    if (!test(D.bits, i, M.ii.size, st)) return true;
  }
  return false;
}

// refute for the candidates that pass the quick test (out of line, TBG_COLD).
template <int NS>
__device__ TBG_COLD_FN bool refute_cold(const SliceJob &J, const KingDest *kd, const DMat &M,
                                        const uint32_t *bin, SetsV<NS> v, bb occ,
                                        DevStatus *st) {
  RowCache rc;
  return refute<NS>(J, kd, M, bin, v.s, occ, rc, st);
}

// The quick test of the verify: the first quiet move of the side's pieces,
// last set first, must lead into "wins".  Returns false when that refutes the
// candidate, true when the candidate needs the full check.
template <int NS>
__device__ __forceinline__ bool survives_quick(const SliceJob &J, const DMat &M,
                                               const uint32_t *bin, const bb *set, bb occ,
                                               const RowCache &rc, DevStatus *st) {
#pragma unroll
  for (int k = NS - 1; k >= 0; k--) {
    if (M.set_color[k] == J.stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb quiet = piece_attacks(M.set_type[k], x, occ) & ~occ;
        if (quiet) {
          int to = ctz64(quiet);
          bb po = k == 0 ? (bit(J.k0) | bit(J.k1)) : (k == NS - 1 ? rc.occ_head : 0);
          uint64_t pi = k == NS - 1 ? rc.row_base : 0;
          uint64_t i = (k == 0 || k == NS - 1)
                           ? rank_mod<NS>(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), -1, 0,
                                          0, 0, k, po, pi)
                           : rank_mod<NS>(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), -1, 0,
                                          0, 0);
          return test(J.self, i, M.ii.size, st);
        }
      }
    }
  }
  return true;
}

// Candidates are read from J.cand; survivors are written back in place, or
// to `out` (every word up to out_words; words past the scanned range copied
// by the block that owns tile 0).
template <int NS>
__device__ __forceinline__ void tile_check(const SliceJob &J, SparseSmem &S, uint64_t t,
                                           DevStatus *st, uint32_t *out, uint64_t out_words,
                                           int lo = 0, int hi = kTileWords) {
  const DMat &M = c_mats[J.mat];
  bb set[NS];
  RowCache rc;
  scan_tile_verify(
      t, J.cand, J.nbits, S.list, S.list2, S.clr, &S.list_n, S.n2,
      [&](uint64_t idx) {
        bb occ = unrank_cached<NS>(M.ii, S.bin, idx, J.k0, J.k1, set, rc);
        return survives_quick<NS>(J, M, S.bin, set, occ, rc, st);
      },
      [&](uint64_t idx) {
        bb occ = unrank_cached<NS>(M.ii, S.bin, idx, J.k0, J.k1, set, rc);
        return refute_cold<NS>(J, S.kd, M, S.bin, sets_v<NS>(set), occ, st);
      },
      out, lo, hi);
  if (out != nullptr && t == 0 && lo == 0) {
    for (uint64_t w = ((J.nbits + 31) >> 5) + threadIdx.x; w < out_words; w += blockDim.x)
      out[w] = J.cand[w];
  }
}

// ------------------------------------------------ dense per-position kernels
// Seeded 7-piece WDL stub standing in for probe_wdl (probe.c:1677):
// VALS[mix64(seed ^ key7) % modulus] with key7 the XOR over the pieces of
// mix64(((type << 6) | sq) * GAMMA + GAMMA), ^ STM_KEY with black to move;
// bare kings are a draw, as probe_table has it.
constexpr uint64_t kGamma = 0x9e3779b97f4a7c15ull;
constexpr uint64_t kStmKey = 0xd1b54a32d192ed03ull;

__device__ __forceinline__ uint64_t piece_key(int type, int sq) {
  return mix64(((uint64_t)((type << 6) | sq)) * kGamma + kGamma);
}

template <int NS>
__device__ __forceinline__ int stub_wdl(const DMat &M, const bb *set, int k0, int k1, int stm) {
  // A capture that leaves the two kings alone is a draw (KvK, probe.c:1525).
  if (M.num == 3) return 0;
  uint64_t key = stm ? kStmKey : 0;
  key ^= piece_key(M.king_type[0], k0) ^ piece_key(M.king_type[1], k1);
#pragma unroll
  for (int k = 0; k < NS; k++) {
    {
      bb b = set[k];
      int t = M.set_type[k] | (M.set_color[k] << 3);
      while (b) key ^= piece_key(t, pop_lsb(b));
    }
  }
  uint64_t h = mix64(c_stub_seed ^ key);
  if (c_stub_mod == 5) return (int)(h % 5) - 2;
  return (int)(h % 3) * 2 - 2;
}

// Write one 32-bit word of a region whose meaningful bits end at nbits: the
// bytes that hold bits below nbits are replaced, later bytes are kept.
__device__ __forceinline__ void store_partial(uint32_t *p, uint64_t w, uint64_t nbits,
                                              uint32_t v) {
  uint64_t base = w * 32;
  if (base + 32 <= nbits) {
    p[w] = v;
    return;
  }
  uint64_t nbytes = (nbits - base + 7) >> 3;  // 1..4
  uint32_t keep = nbytes >= 4 ? 0u : ~0u << (8 * nbytes);
  p[w] = (p[w] & keep) | (v & ~keep);
}

// calc_sub_worker (tb8gen.c:280-314) for captured set J.set of colour stm:
// cls[0..4] = loss, bloss, draw, cwin, win; illegal positions -> cwin+win.
template <int NS>
__global__ void __launch_bounds__(kThreads) k_calc_sub(SliceJob J, uint32_t *c0, uint32_t *c1,
                                                       uint32_t *c2, uint32_t *c3, uint32_t *c4) {
  __shared__ uint32_t bin[7 * 64];
  load_binomials(bin);
  __syncthreads();
  const DMat &M = c_mats[J.mat];
  const DIdx &X = M.capt[J.set];
  const uint64_t n = X.size, nwords = (n + 31) >> 5;
  const int stm = J.stm, opp = stm ? J.k0 : J.k1;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t o[5] = {0, 0, 0, 0, 0};
    bb set[NS], occ = 0;
    uint64_t left = 0;
    for (int b = 0; b < 32; b++) {
      uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      occ = walk_sets<NS>(X, bin, idx, J.k0, J.k1, set, occ, left);
      uint32_t m = 1u << b;
      if (attacked_by<NS>(M, set, J.k0, J.k1, occ, opp, stm)) {
        o[3] |= m;
        o[4] |= m;
      } else {
        int v = stub_wdl<NS>(M, set, J.k0, J.k1, stm);
        o[v + 2] |= m;
        if (v == 2) o[3] |= m;
      }
    }
    store_partial(c0, w, n, o[0]);
    store_partial(c1, w, n, o[1]);
    store_partial(c2, w, n, o[2]);
    store_partial(c3, w, n, o[3]);
    store_partial(c4, w, n, o[4]);
  }
}

// calc_illegal_worker (tb8gen.c:664-684) in gather form: a position is
// illegal for colour c to move iff a piece of colour c attacks the other
// king.  Every word of both outputs is written (padding words zero), as
// after the kslice_clear_addr of tb8gen.c:738-739.
template <int NS>
__global__ void __launch_bounds__(kThreads) k_calc_illegal(SliceJob J, uint32_t *ill_w,
                                                           uint32_t *ill_b, uint64_t nwords) {
  __shared__ uint32_t bin[7 * 64];
  load_binomials(bin);
  __syncthreads();
  const DMat &M = c_mats[J.mat];
  const uint64_t n = M.ii.size;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t ow = 0, ob = 0;
    bb set[NS], occ = 0;
    uint64_t left = 0;
    for (int b = 0; b < 32; b++) {
      uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      occ = walk_sets<NS>(M.ii, bin, idx, J.k0, J.k1, set, occ, left);
      if (attacked_by<NS>(M, set, J.k0, J.k1, occ, J.k1, 0)) ow |= 1u << b;
      if (attacked_by<NS>(M, set, J.k0, J.k1, occ, J.k0, 1)) ob |= 1u << b;
    }
    ill_w[w] = ow;
    ill_b[w] = ob;
  }
}

// has_legal_moves || has_legal_caps (movegen.c:75-111) for side stm.
template <int NS>
__device__ __forceinline__ bool has_legal(const DMat &M, const bb *set0, int k0, int k1, bb occ,
                                          int stm) {
  bb set[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) set[k] = set0[k];
  const int me = stm ? k1 : k0;
  bb own = bit(me), theirs = bit(stm ? k0 : k1);
#pragma unroll
  for (int k = 0; k < NS; k++)
    {
      if (M.set_color[k] == stm) own |= set[k];
      else theirs |= set[k];
    }
  // King steps and captures.
  bb kb = king_attacks(me) & ~own;
  while (kb) {
    int to = pop_lsb(kb);
    bb tb = bit(to);
    int nk0 = stm ? k0 : to, nk1 = stm ? to : k1;
    bb sv[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) sv[k] = set[k] & ~tb;
    bb occ2 = (occ & ~bit(me)) | tb;
    if (!attacked_by<NS>(M, sv, nk0, nk1, occ2, to, stm ^ 1)) return true;
  }
  // Other pieces.
#pragma unroll
  for (int k = 0; k < NS; k++) {
    if (M.set_color[k] == stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb mv = piece_attacks(M.set_type[k], x, occ) & ~own;
        while (mv) {
          int to = pop_lsb(mv);
          bb tb = bit(to);
          bb sv[NS];
#pragma unroll
          for (int q = 0; q < NS; q++) sv[q] = set[q] & ~tb;
          sv[k] = (set[k] ^ bit(x)) | tb;
          bb occ2 = (occ & ~bit(x)) | tb;
          if (!attacked_by<NS>(M, sv, k0, k1, occ2, me, stm ^ 1)) return true;
        }
      }
    }
  }
  (void)theirs;
  return false;
}

// calc_mate_worker (tb8gen.c:686-727): positions legal for exactly one side
// to move, where that side has no legal move or capture.
template <int NS>
__global__ void __launch_bounds__(kThreads) k_calc_mate(SliceJob J, const uint32_t *ill_w,
                                                        const uint32_t *ill_b, uint32_t *mate_w,
                                                        uint32_t *mate_b, uint64_t nwords) {
  __shared__ uint32_t bin[7 * 64];
  load_binomials(bin);
  __syncthreads();
  const DMat &M = c_mats[J.mat];
  const uint64_t n = M.ii.size;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t iw = ill_w[w], ib = ill_b[w];
    uint32_t cand = iw ^ ib, ow = 0, ob = 0;
    while (cand) {
      int b = __ffs(cand) - 1;
      cand &= cand - 1;
      uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      bb set[NS];
      bb occ = unrank_sets<NS>(M.ii, bin, idx, J.k0, J.k1, set);
      int stm = (ib >> b) & 1 ? 0 : 1;
      if (!has_legal<NS>(M, set, J.k0, J.k1, occ, stm)) {
        if (stm == 0) ow |= 1u << b;
        else ob |= 1u << b;
      }
    }
    mate_w[w] = ow;
    mate_b[w] = ob;
  }
}

// ------------------------------------------------------- bitmap algebra
__device__ __forceinline__ uint32_t popc4(uint4 v) {
  return __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
}

// The plain (non-template) kernels below are defined in tbg_api.cu only; the
// persistent-kernel units include this header for its device functions.
#ifndef TBG_PERSIST_UNIT
// Fused W-step epilogue (tb8gen.c:1072-1077): T &= ~wins; cnt += popcount(T)
// below nbits; wins |= T.  One pass, 16-B loads and stores; 4 * N/8 bytes.
// wins_in may equal wins_out (the reference's in-place form).
__global__ void __launch_bounds__(kThreads) k_epilogue_W(uint4 *T, const uint4 *wins_in,
                                                         uint4 *wins_out, uint64_t n16,
                                                         uint64_t nbits,
                                                         unsigned long long *cnt) {
  uint64_t c = 0;
  const uint64_t full16 = nbits >> 7;  // vectors wholly below nbits
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 t = T[i], w = wins_in[i];
    t.x &= ~w.x; t.y &= ~w.y; t.z &= ~w.z; t.w &= ~w.w;
    w.x |= t.x; w.y |= t.y; w.z |= t.z; w.w |= t.w;
    T[i] = t;
    wins_out[i] = w;
    if (i < full16) {
      c += popc4(t);
    } else if (i == full16) {
      uint32_t v[4] = {t.x, t.y, t.z, t.w};
      uint64_t base = i * 128;
      for (int j = 0; j < 4; j++) {
        uint64_t b0 = base + 32 * j;
        if (b0 >= nbits) break;
        uint32_t m = b0 + 32 <= nbits ? ~0u : (1u << (nbits - b0)) - 1u;
        c += __popc(v[j] & m);
      }
    }
  }
  for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
  __shared__ unsigned long long part[kThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int i = 0; i < kThreads / 32; i++) s += part[i];
    if (s) atomicAdd(cnt, s);
  }
}

// kslice_count_addr (kslice.c:500-522): ones below nbits, blocks blk of nblk
// striding over the bitmap; one atomic add per block.
__device__ __forceinline__ void count_bits(const uint4 *p, uint64_t n16, uint64_t nbits,
                                           unsigned long long *cnt, uint64_t blk, uint64_t nblk) {
  uint64_t c = 0;
  const uint64_t full16 = nbits >> 7;
  for (uint64_t i = blk * blockDim.x + threadIdx.x; i < n16 && i <= full16;
       i += nblk * blockDim.x) {
    uint4 t = p[i];
    if (i < full16) {
      c += popc4(t);
    } else {
      uint32_t v[4] = {t.x, t.y, t.z, t.w};
      uint64_t base = i * 128;
      for (int j = 0; j < 4; j++) {
        uint64_t b0 = base + 32 * j;
        if (b0 >= nbits) break;
        uint32_t m = b0 + 32 <= nbits ? ~0u : (1u << (nbits - b0)) - 1u;
        c += __popc(v[j] & m);
      }
    }
  }
  for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
  __shared__ unsigned long long part[kThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int i = 0; i < kThreads / 32; i++) s += part[i];
    if (s) atomicAdd(cnt, s);
  }
}

__global__ void __launch_bounds__(kThreads) k_count(const uint4 *p, uint64_t n16, uint64_t nbits,
                                                    unsigned long long *cnt) {
  count_bits(p, n16, nbits, cnt, blockIdx.x, gridDim.x);
}

// The count over the slices of a plane: bitmap blockIdx.y at base + y * stride.
__global__ void __launch_bounds__(kThreads) k_count_strided(const uint8_t *base, uint64_t stride,
                                                            uint64_t n16, uint64_t nbits,
                                                            unsigned long long *cnt) {
  const uint4 *p = reinterpret_cast<const uint4 *>(base + (uint64_t)blockIdx.y * stride);
  count_bits(p, n16, nbits, cnt, blockIdx.x, gridDim.x);
}

// p &= ~q over n16 vectors (kslice_sub_and_not, kslice.c:481-487).
__global__ void __launch_bounds__(kThreads) k_and_not(uint4 *p, const uint4 *q, uint64_t n16) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 a = p[i], b = q[i];
    a.x &= ~b.x; a.y &= ~b.y; a.z &= ~b.z; a.w &= ~b.w;
    p[i] = a;
  }
}

// Seeded Bernoulli bitmap (synthetic inputs): bit i < nbits set iff the
// (i+1)-th output of the splitmix64 stream keyed by (seed, tag) is < thr.
__global__ void __launch_bounds__(kThreads) k_gen_bernoulli(uint32_t *p, uint64_t nwords,
                                                            uint64_t nbits, uint64_t key,
                                                            uint64_t thr) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = 0;
    for (int b = 0; b < 32; b++) {
      uint64_t i = w * 32 + b;
      if (i >= nbits) break;
      if (mix64(key + (i + 1) * kGamma) < thr) v |= 1u << b;
    }
    p[w] = v;
  }
}

#endif  // TBG_PERSIST_UNIT

}  // namespace tbg
