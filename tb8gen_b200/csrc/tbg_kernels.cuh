// The ply-step kernels (sm_100a).  All arithmetic is integer and bitwise.
//
//  k_predecessors        predecessors_worker      tb8gen.c:484-527   (W step / L candidates)
//  k_predecessors_sub    predecessors_sub_worker  tb8gen.c:346-414   (uncaptures)
//  k_check_successors    check_successors_worker  tb8gen.c:607-661   (L-step verify)
//  k_calc_sub            calc_sub_worker          tb8gen.c:280-342   (capture classes, seeded stub)
//  k_calc_illegal        calc_illegal_worker      tb8gen.c:664-684
//  k_calc_mate           calc_mate_worker         tb8gen.c:686-727
//  k_epilogue_W          kslice_and_not + kslice_count + kslice_or  (tb8gen.c:1072-1077)
//
// Sparse kernels (the first three) walk the source bitmap in tiles of
// TILE_WORDS 32-bit words: each thread loads 16 B (coalesced), the block
// compacts the set bits of the tile into a shared-memory list, and the
// threads then take list entries round-robin.  The list is drained in rounds,
// so any density is handled; at the densities of a ply (1-5 %) one round
// holds the whole tile and every thread gets one or two positions.
#pragma once

#include "tbg_device.cuh"

namespace tbg {

constexpr int kThreads = 256;
constexpr int kTileWords = kThreads * 4;      // 1024 words = 32768 positions
constexpr int kListCap = 4096;

// Materials and stub parameters, uniform across a launch: constant memory.
// (This header is compiled into exactly one translation unit, tbg_api.cu.)
__constant__ DMat c_mats[TBG_MAX_MATS];
__constant__ uint64_t c_stub_seed;
__constant__ int c_stub_mod;

// ------------------------------------------------------------------ ranks
// Rank of a position given as kings + sets, with up to two per-set bit
// toggles applied first (a move is a toggle of two bits; a capture removes
// one; an uncapture adds one), then the normalisation transform.  Sets
// below kfrom keep the contribution idx0 and the occupancy occ0.
__device__ __forceinline__ uint64_t rank_mod(const DIdx &X, const uint32_t *bin, int k0,
                                            int k1, const bb *set, int ka, bb xa, int kb,
                                            bb xb, int mirror, int flip, int kfrom = 0,
                                            bb occ0 = 0, uint64_t idx0 = 0) {
  bb occ = kfrom == 0 ? (bit(k0) | bit(k1)) : occ0;
  uint64_t idx = kfrom == 0 ? 0 : idx0;
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++) {
    if (k >= kfrom && k < X.numsets) {
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
  atomicOr(bits + (idx >> 5), 1u << (idx & 31));
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
// Calls f(idx) for every set bit idx < nbits of bits[].  If clr is given,
// f returns true to clear the bit and the tile is written back in place.
// With kClear and out != nullptr the surviving bits go to out (every word
// of the scanned range, out = in & ~cleared) and bits[] is left untouched.
template <bool kClear, class F>
__device__ __forceinline__ void scan_tiles(uint32_t *bits, uint64_t nbits, uint32_t *list,
                                           uint32_t *clr, int *list_n, F &&f,
                                           uint32_t *out = nullptr) {
  const uint64_t nwords = (nbits + 31) >> 5;
  const uint64_t ntiles = (nwords + kTileWords - 1) / kTileWords;
  const int lane = threadIdx.x & 31;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
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
#pragma unroll
    for (int i = 0; i < 4; i++) {
      uint64_t base = (w0 + i) * 32;
      if (base + 32 > nbits) w[i] &= base < nbits ? (1u << (nbits - base)) - 1u : 0u;
    }
    if (kClear) {
#pragma unroll
      for (int i = 0; i < 4; i++) clr[threadIdx.x * 4 + i] = 0;
    }
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
      int n = min(*list_n, kListCap);
      const uint64_t tbase = t * (uint64_t)kTileWords * 32;
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        uint32_t off = list[e];
        bool c2 = f(tbase + off);
        if (kClear && c2) atomicOr(&clr[off >> 5], 1u << (off & 31));
      }
      if (!__syncthreads_or((w[0] | w[1] | w[2] | w[3]) != 0)) break;
    }
    if (kClear) {
      __syncthreads();
      if (out != nullptr) {
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
}

// ----------------------------------------------------------- W step
// mark_king_unmoves (tb8gen.c:246-262) for a position with an optional
// uncaptured piece (set kb, square xb) on the king's old square.
__device__ __forceinline__ void mark_king_unmoves(const SliceJob &J, const DMat &M,
                                                  const uint32_t *bin, const bb *set, bb occ,
                                                  int kb, bb xb, DevStatus *st) {
  int opp = J.stm ? J.k0 : J.k1;
  bb dest = ~(occ | king_attacks(opp));
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = J.kd[d];
    if (!(dest & bit(D.to))) continue;
    uint64_t i = rank_mod(M.ii, bin, D.k0, D.k1, set, -1, 0, kb, xb, D.mirror, D.flip);
    mark(D.bits, i, M.ii.size, st);
    if (D.dbl) {
      // mirror_diagonal (tb8gen.c:240-244) of the normalised position: the
      // kings are on the diagonal, so the transpose acts on the sets only.
      int m2 = D.mirror;
      uint64_t i2 = rank_mod(M.ii, bin, D.k0, D.k1, set, -1, 0, kb, xb, m2, D.flip ^ 1);
      mark(D.bits, i2, M.ii.size, st);
    }
  }
}

// mark_unmoves (tb8gen.c:264-276) for every non-king piece of the side to
// move, optionally with an uncaptured piece (set kb, square taken from the
// moving piece's origin).
__device__ __forceinline__ void mark_piece_unmoves(const SliceJob &J, const DMat &M,
                                                   const uint32_t *bin, const bb *set,
                                                   bb occ, int kb, DevStatus *st) {
  bb occk = bit(J.k0) | bit(J.k1);
  uint64_t idxk = 0;
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++) {
    if (k < M.ii.numsets && M.set_color[k] == J.stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb mv = piece_attacks(M.set_type[k], x, occ) & ~occ;
        while (mv) {
          int to = pop_lsb(mv);
          uint64_t i;
          if (kb < 0)
            i = rank_mod(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), -1, 0, 0, 0, k,
                         occk, idxk);
          else
            i = rank_mod(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), kb, bit(x), 0, 0);
          mark(J.self, i, M.ii.size, st);
        }
      }
    }
    // Sets below the next moving set keep their rank contribution.
    if (k < M.ii.numsets) {
      bb b = set[k];
      bb occ2 = occk | b;
      uint32_t s = 0;
      int j = 1;
      while (b) {
        int x = pop_lsb(b);
        s += bin[j * 64 + x - __popcll(occk & (bit(x) - 1))];
        j++;
      }
      idxk += (uint64_t)s * M.ii.factor[k];
      occk = occ2;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_predecessors(SliceJob J, DevStatus *st) {
  __shared__ uint32_t bin[7 * 64];
  __shared__ uint32_t list[kListCap];
  __shared__ int list_n;
  load_binomials(bin);
  __syncthreads();
  const DMat &M = c_mats[J.mat];
  scan_tiles<false>(const_cast<uint32_t *>(J.src), J.nbits, list, nullptr, &list_n,
                    [&](uint64_t idx) {
                      bb set[TBG_MAX_SETS];
                      bb occ = unrank_sets(M.ii, bin, idx, J.k0, J.k1, set);
                      mark_king_unmoves(J, M, bin, set, occ, -1, 0, st);
                      mark_piece_unmoves(J, M, bin, set, occ, -1, st);
                      return false;
                    });
}

// predecessors_sub_worker (tb8gen.c:346-394): the source is the sub bitmap
// of captured set J.set (colour stm^1); each position is uncaptured by the
// king and by every non-king piece of stm.
__global__ void __launch_bounds__(kThreads) k_predecessors_sub(SliceJob J, DevStatus *st) {
  __shared__ uint32_t bin[7 * 64];
  __shared__ uint32_t list[kListCap];
  __shared__ int list_n;
  load_binomials(bin);
  __syncthreads();
  const DMat &M = c_mats[J.mat];
  const int kc = J.set;
  const DIdx &X = M.capt[kc];
  scan_tiles<false>(const_cast<uint32_t *>(J.src), J.nbits, list, nullptr, &list_n,
                    [&](uint64_t idx) {
                      bb set[TBG_MAX_SETS];
                      bb occ = unrank_sets(X, bin, idx, J.k0, J.k1, set);
                      int me = J.stm ? J.k1 : J.k0;
                      if (J.legality &&
                          attacked_by(M, set, J.k0, J.k1, occ, me, J.stm ^ 1))
                        return false;
                      mark_king_unmoves(J, M, bin, set, occ, kc, bit(me), st);
                      mark_piece_unmoves(J, M, bin, set, occ, kc, st);
                      return false;
                    });
}

// ----------------------------------------------------------- L step
// check_successors_worker (tb8gen.c:607-650) with check_moves (571-605) and
// check_king_moves (537-569).  True iff the candidate is to be cleared.
__device__ __forceinline__ bool refute(const SliceJob &J, const DMat &M, const uint32_t *bin,
                                       uint64_t idx, DevStatus *st) {
  bb set[TBG_MAX_SETS];
  bb occ = unrank_sets(M.ii, bin, idx, J.k0, J.k1, set);
  const int stm = J.stm;
  const int me = stm ? J.k1 : J.k0, opp = stm ? J.k0 : J.k1;
  if (attacked_by(M, set, J.k0, J.k1, occ, opp, stm)) return true;
  bb own = 0;
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++)
    if (k < M.ii.numsets && M.set_color[k] == stm) own |= set[k];
  // Non-king pieces: captures must lead into sub/win, quiet moves into wins.
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++) {
    if (k < M.ii.numsets && M.set_color[k] == stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb att = piece_attacks(M.set_type[k], x, occ);
        bb caps = att & occ & ~own & ~bit(opp);
        while (caps) {
          int to = pop_lsb(caps);
#pragma unroll
          for (int l = 0; l < TBG_MAX_SETS; l++) {
            if (l < M.ii.numsets && (set[l] & bit(to))) {
              uint64_t i = rank_mod(M.capt[l], bin, J.k0, J.k1, set, k, bit(x) | bit(to), l,
                                    bit(to), 0, 0);
              if (!test_sub(J.self_sub, J.self_sub_len, M.sub_offset[l], i, st)) return true;
            }
          }
        }
        bb quiet = att & ~occ;
        while (quiet) {
          int to = pop_lsb(quiet);
          uint64_t i = rank_mod(M.ii, bin, J.k0, J.k1, set, k, bit(x) | bit(to), -1, 0, 0, 0);
          if (!test(J.self, i, M.ii.size, st)) return true;
        }
      }
    }
  }
  // King: captures leave the captured piece in its slot and drop the set's
  // last slot (its highest square) from the capture index, as the reference
  // computes it (tb8gen.c:543-555); quiet moves go to neighbouring slices.
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = J.kd[d];
    if (!(occ & bit(D.to))) continue;
    if (own & bit(D.to)) continue;
#pragma unroll
    for (int l = 0; l < TBG_MAX_SETS; l++) {
      if (l < M.ii.numsets && (set[l] & bit(D.to))) {
        uint64_t i = rank_mod(M.capt[l], bin, D.k0, D.k1, set, -1, 0, l,
                              bit(msb64(set[l])), D.mirror, D.flip);
        if (!test_sub(D.sub, D.sub_len, M.sub_offset[l], i, st)) return true;
      }
    }
  }
  for (int d = 0; d < J.nk; d++) {
    const KingDest &D = J.kd[d];
    if (occ & bit(D.to)) continue;
    uint64_t i = rank_mod(M.ii, bin, D.k0, D.k1, set, -1, 0, -1, 0, D.mirror, D.flip);
    if (!test(D.bits, i, M.ii.size, st)) return true;
  }
  (void)me;
  return false;
}

// Candidates are read from J.cand; survivors are written back in place, or
// to `out` (every word up to out_words; words past the scanned range copied).
__global__ void __launch_bounds__(kThreads) k_check_successors(SliceJob J, DevStatus *st,
                                                               uint32_t *out, uint64_t out_words) {
  __shared__ uint32_t bin[7 * 64];
  __shared__ uint32_t list[kListCap];
  __shared__ uint32_t clr[kTileWords];
  __shared__ int list_n;
  load_binomials(bin);
  __syncthreads();
  const DMat &M = c_mats[J.mat];
  scan_tiles<true>(J.cand, J.nbits, list, clr, &list_n,
                   [&](uint64_t idx) { return refute(J, M, bin, idx, st); }, out);
  if (out != nullptr && blockIdx.x == 0) {
    for (uint64_t w = ((J.nbits + 31) >> 5) + threadIdx.x; w < out_words; w += blockDim.x)
      out[w] = J.cand[w];
  }
}

// ------------------------------------------------ dense per-position kernels
// Seeded 7-piece WDL stub standing in for probe_wdl (probe.c:1677):
// VALS[mix64(seed ^ key7) % modulus] with key7 the XOR over the pieces of
// mix64(((type << 6) | sq) * GAMMA + GAMMA), ^ STM_KEY with black to move.
constexpr uint64_t kGamma = 0x9e3779b97f4a7c15ull;
constexpr uint64_t kStmKey = 0xd1b54a32d192ed03ull;

__device__ __forceinline__ uint64_t piece_key(int type, int sq) {
  return mix64(((uint64_t)((type << 6) | sq)) * kGamma + kGamma);
}

__device__ __forceinline__ int stub_wdl(const DMat &M, const bb *set, int k0, int k1, int stm) {
  uint64_t key = stm ? kStmKey : 0;
  key ^= piece_key(M.king_type[0], k0) ^ piece_key(M.king_type[1], k1);
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++) {
    if (k < M.ii.numsets) {
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
    for (int b = 0; b < 32; b++) {
      uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      bb set[TBG_MAX_SETS];
      bb occ = unrank_sets(X, bin, idx, J.k0, J.k1, set);
      uint32_t m = 1u << b;
      if (attacked_by(M, set, J.k0, J.k1, occ, opp, stm)) {
        o[3] |= m;
        o[4] |= m;
      } else {
        int v = stub_wdl(M, set, J.k0, J.k1, stm);
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
    for (int b = 0; b < 32; b++) {
      uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      bb set[TBG_MAX_SETS];
      bb occ = unrank_sets(M.ii, bin, idx, J.k0, J.k1, set);
      if (attacked_by(M, set, J.k0, J.k1, occ, J.k1, 0)) ow |= 1u << b;
      if (attacked_by(M, set, J.k0, J.k1, occ, J.k0, 1)) ob |= 1u << b;
    }
    ill_w[w] = ow;
    ill_b[w] = ob;
  }
}

// has_legal_moves || has_legal_caps (movegen.c:75-111) for side stm.
__device__ __forceinline__ bool has_legal(const DMat &M, const bb *set0, int k0, int k1, bb occ,
                                          int stm) {
  bb set[TBG_MAX_SETS];
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++) set[k] = set0[k];
  const int me = stm ? k1 : k0;
  bb own = bit(me), theirs = bit(stm ? k0 : k1);
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++)
    if (k < M.ii.numsets) {
      if (M.set_color[k] == stm) own |= set[k];
      else theirs |= set[k];
    }
  // King steps and captures.
  bb kb = king_attacks(me) & ~own;
  while (kb) {
    int to = pop_lsb(kb);
    bb tb = bit(to);
    int nk0 = stm ? k0 : to, nk1 = stm ? to : k1;
    bb sv[TBG_MAX_SETS];
#pragma unroll
    for (int k = 0; k < TBG_MAX_SETS; k++) sv[k] = set[k] & ~tb;
    bb occ2 = (occ & ~bit(me)) | tb;
    if (!attacked_by(M, sv, nk0, nk1, occ2, to, stm ^ 1)) return true;
  }
  // Other pieces.
#pragma unroll
  for (int k = 0; k < TBG_MAX_SETS; k++) {
    if (k < M.ii.numsets && M.set_color[k] == stm) {
      bb pcs = set[k];
      while (pcs) {
        int x = pop_lsb(pcs);
        bb mv = piece_attacks(M.set_type[k], x, occ) & ~own;
        while (mv) {
          int to = pop_lsb(mv);
          bb tb = bit(to);
          bb sv[TBG_MAX_SETS];
#pragma unroll
          for (int q = 0; q < TBG_MAX_SETS; q++) sv[q] = set[q] & ~tb;
          sv[k] = (set[k] ^ bit(x)) | tb;
          bb occ2 = (occ & ~bit(x)) | tb;
          if (!attacked_by(M, sv, k0, k1, occ2, me, stm ^ 1)) return true;
        }
      }
    }
  }
  (void)theirs;
  return false;
}

// calc_mate_worker (tb8gen.c:686-727): positions legal for exactly one side
// to move, where that side has no legal move or capture.
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
      bb set[TBG_MAX_SETS];
      bb occ = unrank_sets(M.ii, bin, idx, J.k0, J.k1, set);
      int stm = (ib >> b) & 1 ? 0 : 1;
      if (!has_legal(M, set, J.k0, J.k1, occ, stm)) {
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

// kslice_count_addr (kslice.c:500-522): ones below nbits.
__global__ void __launch_bounds__(kThreads) k_count(const uint4 *p, uint64_t n16, uint64_t nbits,
                                                    unsigned long long *cnt) {
  uint64_t c = 0;
  const uint64_t full16 = nbits >> 7;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16 && i <= full16;
       i += (uint64_t)gridDim.x * blockDim.x) {
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

}  // namespace tbg
