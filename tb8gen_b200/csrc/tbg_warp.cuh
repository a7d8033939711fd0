// Batched ply with warp-granular work items (tbg_batch_run mode 2).
//
// The same recorded queue as k_batch (tbg_batch.cuh), with every block item
// cut into one sub-item per warp of a block: a warp takes the next sub-item
// with its own atomicAdd, waits (bounded) for the op's predecessors, and
// runs it alone.  No block barrier is left on the ply path: in k_batch a
// block hands a tile's sources out in shares and meets at a barrier after
// every round, so the warps with two sources per lane hold up those with
// one; here each warp feeds its own ring of source positions and processes
// them 32 at a time, one per lane, carrying the remainder (< 32) to its next
// sub-item of the same op.
//
// A sub-item is 128 words (4,096 positions) of a scatter's, an uncapture's
// or a verify's bitmap (gt x 128 words for a scatter op of gt tiles per
// item), or an eighth of a streaming op's 1 MiB chunk.  An op's sub-items
// are counted done (done[op] reaches ntiles x warps per block) when the
// warp's ring holds none of their sources: a warp flushes its ring before
// it waits for another op's predecessors, so, as in k_batch, the earliest
// unfinished sub-item can always proceed.
//
// The same runners drive the one-launch-per-call kernel k_op_w (the plain
// path and the per-call entry points): one op, sub-items of 32 words (one
// per lane: a small bitmap still spreads over many warps) dealt to the
// warps of the grid in turn.
#pragma once

#include "tbg_batch.cuh"

namespace tbg {

constexpr int kWarps = kThreads / 32;           // sub-items per block item
constexpr int kSubWords = kTileWords / kWarps;  // 128: four words per lane
static_assert(kSubWords == 128, "a sub-item is four words per lane");
constexpr int kRing = 256;                      // a warp's source ring
constexpr int kRing2 = 128;                     // verify: survivors of the quick test
constexpr unsigned kFull = 0xffffffffu;
constexpr int kRun = 4;                         // k_op_w: sub-items per run of a warp

struct WarpSmem {
  Op op;                       // the op the warp runs: descriptor and king destinations
  uint64_t ring[kRing];        // source positions waiting for a lane
  uint64_t ring2[kRing2];      // verify: candidates that passed the quick test
};

// A warp's ring: head and tail count entries (warp-uniform registers).
struct Ring {
  uint32_t head = 0, tail = 0;
};

__device__ __forceinline__ unsigned long long warp_fetch(unsigned long long *next) {
  unsigned long long it = 0;
  if ((threadIdx.x & 31) == 0) it = atomicAdd(next, 1ull);
  return __shfl_sync(kFull, it, 0);
}

// This lane's WPL words (4 or 1; the others zero) of the 32 x WPL-word
// chunk at word c0 of a bitmap of nbits positions: raw[] as stored, w[]
// with the positions >= nbits masked off.  Returns the word index of w[0].
template <int WPL>
__device__ __forceinline__ uint64_t load_chunk(const uint32_t *bits, uint64_t nbits, uint64_t c0,
                                               uint32_t w[4], uint32_t raw[4]) {
  const uint64_t nwords = (nbits + 31) >> 5;
  const uint64_t w0 = c0 + (uint64_t)(threadIdx.x & 31) * WPL;
  if (WPL == 1) {
    raw[0] = w0 < nwords ? __ldcs(bits + w0) : 0u;
    raw[1] = raw[2] = raw[3] = 0u;
  } else if (w0 + 4 <= nwords) {
    const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(bits + w0));
    raw[0] = v.x; raw[1] = v.y; raw[2] = v.z; raw[3] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) raw[i] = w0 + i < nwords ? bits[w0 + i] : 0u;
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint64_t base = (w0 + i) * 32;
    w[i] = raw[i];
    if (base + 32 > nbits) w[i] &= base < nbits ? (1u << (nbits - base)) - 1u : 0u;
  }
  return w0;
}

// Appends the set bits of this lane's words w[] (word index w0) to the
// warp's ring and hands every full batch of 32 to f(idx), one entry per
// lane (consecutive positions in consecutive lanes); fewer than 32 stay in
// the ring.  Warp-wide.
template <class F>
__device__ __forceinline__ void ring_feed(uint32_t w[4], uint64_t w0, uint64_t *ring, Ring &r,
                                          F &&f) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    const int c = __popc(w[0]) + __popc(w[1]) + __popc(w[2]) + __popc(w[3]);
    int incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += y;
    }
    const int tot = __shfl_sync(kFull, incl, 31);
    if (tot == 0) return;
    const int room = kRing - (int)(r.tail - r.head);
    int pos = incl - c;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      while (w[i] && pos < room) {
        const int b = __ffs(w[i]) - 1;
        w[i] &= w[i] - 1;
        ring[(r.tail + pos) & (kRing - 1)] = (w0 + i) * 32 + b;
        pos++;
      }
    }
    r.tail += min(tot, room);
    __syncwarp();
    while (r.tail - r.head >= 32) {
      const uint64_t e = ring[(r.head + lane) & (kRing - 1)];
      r.head += 32;
      f(e);
      __syncwarp();
    }
    if (tot <= room) return;
  }
}

// The last entries of the ring (fewer than 32), one per lane.
template <class F>
__device__ __forceinline__ void ring_flush(uint64_t *ring, Ring &r, F &&f) {
  const int n = (int)(r.tail - r.head);
  if (n <= 0) return;
  const int lane = threadIdx.x & 31;
  if (lane < n) f(ring[(r.head + lane) & (kRing - 1)]);
  r.head = r.tail;
  __syncwarp();
}

// First word of sub-item u of an op whose block items are gt tiles each
// (WPL 4: gt chunks of 128 words per sub-item), or of sub-item u of 32
// words (WPL 1: one chunk).
template <int WPL>
__device__ __forceinline__ uint64_t sub_word0(uint64_t u, int gt) {
  if (WPL == 1) return u * 32;
  const uint64_t b = u / kWarps, s = u % kWarps;
  return b * (uint64_t)gt * kTileWords + s * (uint64_t)gt * kSubWords;
}

// The chunk's cleared candidates into dst (out of place: every word; in
// place: only words that held candidates).
template <int WPL>
__device__ __forceinline__ void store_cleared(uint32_t *dst, bool always, uint64_t w0,
                                              uint64_t nwords, const uint32_t w[4],
                                              const uint32_t raw[4]) {
  if (WPL == 1) {
    if (w0 < nwords && (always || w[0])) dst[w0] = raw[0] & ~w[0];
    return;
  }
  if (w0 + 4 <= nwords) {
    if (always || (w[0] | w[1] | w[2] | w[3]))
      *reinterpret_cast<uint4 *>(dst + w0) =
          make_uint4(raw[0] & ~w[0], raw[1] & ~w[1], raw[2] & ~w[2], raw[3] & ~w[3]);
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (w0 + i < nwords) dst[w0 + i] = raw[i] & ~w[i];
  }
}

// The sparse runners are compiled out of line (TBG_RUNNER): each gets its own
// register allocation, as a kernel of one op kind would, instead of sharing
// one across every kind the persistent kernel dispatches to.
#ifndef TBG_RUNNER
#define TBG_RUNNER __noinline__
#endif

// The sparse runners below process sub-items it, fetch(it), ... of one op
// (those below hi: sub-items are handed out in increasing order) and return
// the first sub-item at or past hi.  o: the op (in shared memory); ring,
// ring2: the warp's rings; cnt: sub-items run.

// ---- scatter (predecessors_worker, tb8gen.c:484-516) and candidates
template <int NS, int WPL, class Fetch>
__device__ TBG_RUNNER unsigned long long run_scatter(const Op &o, const uint32_t *bin,
                                                          uint64_t *ring, uint64_t *,
                                                          unsigned long long it, uint64_t lo,
                                                          uint64_t hi, Fetch &&fetch,
                                                          DevStatus *st, unsigned &cnt) {
  const SliceJob &J = o.J;
  const DMat &M = c_mats[J.mat];
  const uint64_t nwords = (J.nbits + 31) >> 5;
  const int nch = WPL == 1 ? 1 : o.gt;
  bb set[NS];
  RowCache rc;
  Ring r;
  auto f = [&](uint64_t idx) {
    const bb occ = unrank_cached<NS>(M.ii, bin, idx, J.k0, J.k1, set, rc);
    mark_unmoves_inc<NS>(J, J.kd, M, bin, set, occ, idx, st);
  };
  for (;;) {
    const uint64_t c0 = sub_word0<WPL>(it - lo, o.gt);
    for (int g = 0; g < nch && c0 + (uint64_t)g * 32 * WPL < nwords; g++) {
      uint32_t w[4], raw[4];
      const uint64_t w0 = load_chunk<WPL>(J.src, J.nbits, c0 + (uint64_t)g * 32 * WPL, w, raw);
      ring_feed(w, w0, ring, r, f);
    }
    cnt++;
    it = fetch(it);
    if (it >= hi) break;
  }
  ring_flush(ring, r, f);
  return it;
}

// ---- uncaptures (predecessors_sub_worker, tb8gen.c:346-394)
template <int NS, int WPL, class Fetch>
__device__ TBG_RUNNER unsigned long long run_scatter_sub(const Op &o, const uint32_t *bin,
                                                              uint64_t *ring, uint64_t *,
                                                              unsigned long long it, uint64_t lo,
                                                              uint64_t hi, Fetch &&fetch,
                                                              DevStatus *st, unsigned &cnt) {
  const SliceJob &J = o.J;
  const DMat &M = c_mats[J.mat];
  const int kc = J.set;
  const DIdx &X = M.capt[kc];
  const uint64_t nwords = (J.nbits + 31) >> 5;
  bb set[NS];
  RowCache rc;
  Ring r;
  auto f = [&](uint64_t idx) {
    const bb occ = unrank_cached<NS>(X, bin, idx, J.k0, J.k1, set, rc);
    const int me = J.stm ? J.k1 : J.k0;
    if (J.legality && attacked_by<NS>(M, set, J.k0, J.k1, occ, me, J.stm ^ 1)) return;
    mark_king_unmoves<NS>(J, J.kd, M, bin, set, occ, kc, bit(me), st);
    mark_piece_unmoves<NS>(J, M, bin, set, occ, kc, st);
  };
  for (;;) {
    const uint64_t c0 = sub_word0<WPL>(it - lo, 1);
    if (c0 < nwords) {
      uint32_t w[4], raw[4];
      const uint64_t w0 = load_chunk<WPL>(J.src, J.nbits, c0, w, raw);
      ring_feed(w, w0, ring, r, f);
    }
    cnt++;
    it = fetch(it);
    if (it >= hi) break;
  }
  ring_flush(ring, r, f);
  return it;
}

// ---- verify (check_successors_worker, tb8gen.c:607-650)
// A chunk's candidate bits are cleared in the output as the chunk is read
// (out, or the candidate bitmap in place; bits past nbits and every other
// bit kept), and a candidate that survives both tests is set again; only
// this warp touches the chunk's words.
template <int NS, int WPL, class Fetch>
__device__ TBG_RUNNER unsigned long long run_verify(const Op &o, const uint32_t *bin,
                                                         uint64_t *ring, uint64_t *ring2,
                                                         unsigned long long it, uint64_t lo,
                                                         uint64_t hi, Fetch &&fetch,
                                                         DevStatus *st, unsigned &cnt) {
  const SliceJob &J = o.J;
  const DMat &M = c_mats[J.mat];
  const uint64_t nwords = (J.nbits + 31) >> 5;
  uint32_t *dst = o.out != nullptr ? o.out : J.cand;
  const int lane = threadIdx.x & 31;
  bb set[NS];
  RowCache rc;
  Ring r, r2;
  // full check of 32 (or, at the end, fewer) survivors of the quick test
  auto full = [&](uint64_t idx) {
    const bb occ = unrank_cached<NS>(M.ii, bin, idx, J.k0, J.k1, set, rc);
    if (!refute_cold<NS>(J, J.kd, M, bin, sets_v<NS>(set), occ, st))
      asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(
                       __cvta_generic_to_global(dst + (idx >> 5))),
                   "r"(1u << (idx & 31))
                   : "memory");
  };
  // quick test of one candidate per lane; survivors go to ring2
  auto quick_batch = [&](uint64_t idx, bool active) {
    bool keep = false;
    if (active) {
      const bb occ = unrank_cached<NS>(M.ii, bin, idx, J.k0, J.k1, set, rc);
      keep = survives_quick<NS>(J, M, bin, set, occ, rc, st);
    }
    const unsigned m = __ballot_sync(kFull, keep);
    if (keep) ring2[(r2.tail + __popc(m & ((1u << lane) - 1u))) & (kRing2 - 1)] = idx;
    r2.tail += __popc(m);
    __syncwarp();
    if (r2.tail - r2.head >= 32) {
      const uint64_t e = ring2[(r2.head + lane) & (kRing2 - 1)];
      r2.head += 32;
      full(e);
      __syncwarp();
    }
  };
  for (;;) {
    const uint64_t c0 = sub_word0<WPL>(it - lo, 1);
    if (c0 < nwords) {
      uint32_t w[4], raw[4];
      const uint64_t w0 = load_chunk<WPL>(J.cand, J.nbits, c0, w, raw);
      store_cleared<WPL>(dst, o.out != nullptr, w0, nwords, w, raw);
      __syncwarp();
      ring_feed(w, w0, ring, r, [&](uint64_t e) { quick_batch(e, true); });
    }
    // words past the scanned range, copied once (out of place only)
    if (o.out != nullptr && it == lo) {
      for (uint64_t x = nwords + lane; x < o.out_words; x += 32) o.out[x] = J.cand[x];
    }
    cnt++;
    it = fetch(it);
    if (it >= hi) break;
  }
  {
    const int n = (int)(r.tail - r.head);
    if (n > 0) {
      const uint64_t e = ring[(r.head + lane) & (kRing - 1)];
      r.head = r.tail;
      quick_batch(e, lane < n);
    }
  }
  {
    const int n = (int)(r2.tail - r2.head);
    if (n > 0) {
      if (lane < n) full(ring2[(r2.head + lane) & (kRing2 - 1)]);
      r2.head = r2.tail;
      __syncwarp();
    }
  }
  return it;
}

// ---- streaming ops: the fused W epilogue, a clear, a count
template <class Fetch>
__device__ __forceinline__ unsigned long long run_stream(const Op &o, unsigned long long it,
                                                         uint64_t lo, uint64_t hi, Fetch &&fetch,
                                                         unsigned &cnt) {
  const int lane = threadIdx.x & 31;
  constexpr uint64_t kPart = kChunk16 / kWarps;
  const uint64_t full16 = o.nbits >> 7;
  unsigned long long c = 0;
  for (;;) {
    const uint64_t i0 = (it - lo) * kPart;
    const uint64_t i1 = i0 + kPart < o.n16 ? i0 + kPart : o.n16;
    if (o.kind == OP_CLEAR) {
      const uint4 z = make_uint4(0, 0, 0, 0);
      for (uint64_t i = i0 + lane; i < i1; i += 32) o.T[i] = z;
    } else {
      const bool count_only = o.kind == OP_COUNT;
      for (uint64_t i = i0 + lane; i < i1; i += 32) {
        uint4 t4 = o.T[i];
        if (!count_only) {
          uint4 w = o.win[i];
          t4.x &= ~w.x; t4.y &= ~w.y; t4.z &= ~w.z; t4.w &= ~w.w;
          w.x |= t4.x; w.y |= t4.y; w.z |= t4.z; w.w |= t4.w;
          o.T[i] = t4;
          o.wout[i] = w;
        }
        if (i < full16) {
          c += popc4(t4);
        } else if (i == full16) {
          const uint32_t v[4] = {t4.x, t4.y, t4.z, t4.w};
          for (int j = 0; j < 4; j++) {
            const uint64_t b0 = i * 128 + 32 * j;
            if (b0 >= o.nbits) break;
            const uint32_t m = b0 + 32 <= o.nbits ? ~0u : (1u << (o.nbits - b0)) - 1u;
            c += __popc(v[j] & m);
          }
        }
      }
    }
    cnt++;
    it = fetch(it);
    if (it >= hi) break;
  }
  if (o.cnt != nullptr && o.kind != OP_CLEAR) {
    for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(kFull, c, d);
    if (lane == 0 && c) atomicAdd(o.cnt, c);
  }
  return it;
}

template <int NS, class Fetch>
__device__ __forceinline__ unsigned long long run_sparse(const Op &o, const uint32_t *bin,
                                                         uint64_t *ring, uint64_t *ring2,
                                                         unsigned long long it, uint64_t lo,
                                                         uint64_t hi, Fetch &&fetch,
                                                         DevStatus *st, unsigned &cnt) {
  switch (o.kind) {
  case OP_SCATTER: return run_scatter<NS, 4>(o, bin, ring, ring2, it, lo, hi, fetch, st, cnt);
  case OP_SCATTER_SUB:
    return run_scatter_sub<NS, 4>(o, bin, ring, ring2, it, lo, hi, fetch, st, cnt);
  default: return run_verify<NS, 4>(o, bin, ring, ring2, it, lo, hi, fetch, st, cnt);
  }
}

template <int NSMAX>
__global__ void __launch_bounds__(kThreads, TBG_MINB_BATCH)
k_batch_w(const Op *__restrict__ ops, int nops, const int *__restrict__ preds, uint64_t total,
          unsigned long long *next, unsigned int *done, DevStatus *st, long long spin_limit) {
  __shared__ uint32_t bin[7 * 64];
  __shared__ __align__(16) WarpSmem W[kWarps];
  load_binomials(bin);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  WarpSmem &S = W[threadIdx.x >> 5];
  const uint64_t total_w = total * kWarps;
  int cur_op = -1;  // the op whose descriptor is in S.op
  unsigned long long it = warp_fetch(next);
  while (it < total_w) {
    // the op of sub-item it (sub-items come in increasing order: the next
    // op is found by stepping forward, or, far ahead, by a binary search),
    // and its predecessors (lane 0 waits, bounded)
    const uint64_t b = it / kWarps;
    int op = cur_op < 0 ? 0 : cur_op;
    for (int n = 0; n < 4 && op + 1 < nops && ops[op + 1].first <= b; n++) op++;
    if (op + 1 < nops && ops[op + 1].first <= b) {
      int lo = op, hi = nops - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ops[mid].first <= b) lo = mid;
        else hi = mid - 1;
      }
      op = lo;
    }
    int abort = 0;
    if (lane == 0) {
      const int np = ops[op].npred, po = ops[op].pred_off;
      for (int p = 0; p < np && !abort; p++) {
        const int q = preds[po + p];
        const unsigned int need = ops[q].ntiles * (unsigned)kWarps;
        long long n = 0;
        while (load_acquire(&done[q]) < need) {
          if (++n > spin_limit) {
            report(st, 3, (unsigned)q, it);
            abort = 1;
            break;
          }
          __nanosleep(64);
        }
      }
    }
    abort = __shfl_sync(kFull, abort, 0);
    if (abort) break;
    __syncwarp();
    __threadfence();
    // the op's descriptor (with its king destinations) into this warp's slot
    {
      const int4 *src = reinterpret_cast<const int4 *>(&ops[op]);
      int4 *dst = reinterpret_cast<int4 *>(&S.op);
      for (int i = lane; i < (int)(sizeof(Op) / 16); i += 32) dst[i] = src[i];
    }
    cur_op = op;
    __syncwarp();
    const uint64_t first_w = S.op.first * kWarps;
    const uint64_t end_w = first_w + (uint64_t)S.op.ntiles * kWarps;
    unsigned cnt = 0;
    const unsigned long long cur = it;
    auto fetch = [next](unsigned long long) { return warp_fetch(next); };
#define TBG_RUN(N) run_sparse<N>(S.op, bin, S.ring, S.ring2, it, first_w, end_w, fetch, st, cnt)
    if (op_streams(S.op.kind)) {
      it = run_stream(S.op, it, first_w, end_w, fetch, cnt);
    } else {
      switch (S.op.ns) {
      case 1: it = TBG_RUN(1); break;
      case 2: if (NSMAX >= 2) it = TBG_RUN(NSMAX >= 2 ? 2 : 1); break;
      case 3: if (NSMAX >= 3) it = TBG_RUN(NSMAX >= 3 ? 3 : 1); break;
      case 4: if (NSMAX >= 4) it = TBG_RUN(NSMAX >= 4 ? 4 : 1); break;
      case 5: if (NSMAX >= 5) it = TBG_RUN(NSMAX >= 5 ? 5 : 1); break;
      default: if (NSMAX >= 6) it = TBG_RUN(NSMAX >= 6 ? 6 : 1); break;
      }
    }
#undef TBG_RUN
    if (it == cur) {
      // no instance for this many piece sets (the host launches one that has)
      report(st, 6, (unsigned)S.op.ns, cur);
      break;
    }
    // every source of the op's sub-items this warp took is processed
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      atomicAdd(&done[op], cnt);
    }
  }
}

// ---- one launch per call (the plain path and the per-call entry points)
// One sparse op: its sub-items of 32 words taken in runs of kRun
// consecutive ones, the runs dealt to the grid's warps in turn, each warp
// feeding its own ring.  Within a run a lane batch holds neighbouring
// positions (shared leading index digits, marks into one target row);
// across the grid the warps work on one window of the bitmap at a time
// (warps x kRun x 1,024 positions), whose marks and reads stay in L2.
// The op is copied into shared memory once per block.
template <int NS, int KIND>
__global__ void __launch_bounds__(kThreads, TBG_MINB_BATCH)
k_op_w(const __grid_constant__ Op o, DevStatus *st, uint64_t nsub) {
  __shared__ uint32_t bin[7 * 64];
  __shared__ __align__(16) Op so;
  __shared__ uint64_t ring[kWarps][kRing];
  __shared__ uint64_t ring2[KIND == OP_VERIFY ? kWarps : 1][kRing2];
  load_binomials(bin);
  {
    const int4 *src = reinterpret_cast<const int4 *>(&o);
    int4 *dst = reinterpret_cast<int4 *>(&so);
    for (int i = threadIdx.x; i < (int)(sizeof(Op) / 16); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int wid = threadIdx.x >> 5;
  const uint64_t skip = ((uint64_t)gridDim.x * kWarps - 1) * kRun;  // the other warps' runs
  const unsigned long long it = ((uint64_t)blockIdx.x * kWarps + wid) * kRun;
  if (it >= nsub) return;
  auto fetch = [skip](unsigned long long cur) {
    return (cur + 1) % kRun ? cur + 1 : cur + 1 + skip;
  };
  unsigned cnt = 0;
  // sub-item numbers are op-relative (lo = 0)
  if (KIND == OP_SCATTER)
    run_scatter<NS, 1>(so, bin, ring[wid], nullptr, it, 0, nsub, fetch, st, cnt);
  else if (KIND == OP_SCATTER_SUB)
    run_scatter_sub<NS, 1>(so, bin, ring[wid], nullptr, it, 0, nsub, fetch, st, cnt);
  else
    run_verify<NS, 1>(so, bin, ring[wid], ring2[KIND == OP_VERIFY ? wid : 0], it, 0, nsub, fetch,
                      st, cnt);
}

}  // namespace tbg
