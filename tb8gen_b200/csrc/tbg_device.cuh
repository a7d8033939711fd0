// Device-side building blocks of the ply step: bitboard attacks, the
// king-slice symmetry transforms and the combinatorial position index.
//
// A position inside a kernel is held as bitboards: the two king squares and
// one 64-bit occupancy mask per like-piece set (struct IdxInfo sets,
// tb8gen.h:4-13).  Because every set is ranked as a set (the reference sorts
// each set before ranking it, tb8gen.c:136), a mask carries all the index
// needs, and moving one piece is a two-bit update of one mask.
#pragma once

#include <cstdint>

#include "tbg_types.h"

namespace tbg {

typedef uint64_t bb;

__device__ __forceinline__ bb bit(int sq) { return 1ull << sq; }
__device__ __forceinline__ int ctz64(bb b) { return __ffsll((long long)b) - 1; }
__device__ __forceinline__ int pop_lsb(bb &b) {
  int s = ctz64(b);
  b &= b - 1;
  return s;
}
__device__ __forceinline__ int msb64(bb b) { return 63 - __clzll((long long)b); }

// ---------------------------------------------------------------- attacks
// Sliding attacks by the subtraction/bit-reversal line method ("hyperbola
// quintessence", chessprogramming wiki): for a line mask m that excludes the
// origin s, attacks = ((o - 2s) ^ rev(rev(o) - 2 rev(s))) & m with o = occ & m.
// No lookup table; the reference's magic tables (magic.h:23-38) are matched
// exhaustively in tests/test_gpu_parity.py::test_attacks_exhaustive.
__device__ __forceinline__ bb line_attacks(bb occ, int sq, bb mask) {
  bb o = occ & mask;
  bb s = bit(sq);
  bb fwd = o - (s << 1);
  bb rev = __brevll(__brevll(o) - (__brevll(s) << 1));
  return (fwd ^ rev) & mask;
}

__device__ __forceinline__ bb rook_attacks(int sq, bb occ) {
  bb s = bit(sq);
  bb file = (0x0101010101010101ull << (sq & 7)) ^ s;
  bb rank = (0xffull << (sq & 56)) ^ s;
  return line_attacks(occ, sq, file) | line_attacks(occ, sq, rank);
}

__device__ __forceinline__ bb bishop_attacks(int sq, bb occ) {
  const bb MAIN = 0x8040201008040201ull, ANTI = 0x0102040810204080ull;
  int f = sq & 7, r = sq >> 3;
  int d = f - r, c = r + f;
  bb diag = d >= 0 ? MAIN >> (8 * d) : MAIN << (-8 * d);
  bb anti = c <= 7 ? ANTI >> (8 * (7 - c)) : ANTI << (8 * (c - 7));
  bb s = bit(sq);
  return line_attacks(occ, sq, diag ^ s) | line_attacks(occ, sq, anti ^ s);
}

__device__ __forceinline__ bb knight_attacks(int sq) {
  bb b = bit(sq);
  bb l1 = (b >> 1) & 0x7f7f7f7f7f7f7f7full, l2 = (b >> 2) & 0x3f3f3f3f3f3f3f3full;
  bb r1 = (b << 1) & 0xfefefefefefefefeull, r2 = (b << 2) & 0xfcfcfcfcfcfcfcfcull;
  bb h1 = l1 | r1, h2 = l2 | r2;
  return (h1 << 16) | (h1 >> 16) | (h2 << 8) | (h2 >> 8);
}

__device__ __forceinline__ bb king_attacks(int sq) {
  bb b = bit(sq);
  bb k = b | ((b << 1) & 0xfefefefefefefefeull) | ((b >> 1) & 0x7f7f7f7f7f7f7f7full);
  k |= (k << 8) | (k >> 8);
  return k ^ b;
}

// non_king_piece_attacks, movegen.h:103-117 (piece type & 7: 2 N, 3 B, 4 R, 5 Q).
__device__ __forceinline__ bb piece_attacks(int type, int sq, bb occ) {
  switch (type) {
  case 2: return knight_attacks(sq);
  case 3: return bishop_attacks(sq, occ);
  case 4: return rook_attacks(sq, occ);
  case 5: return rook_attacks(sq, occ) | bishop_attacks(sq, occ);
  default: return king_attacks(sq);
  }
}

// ------------------------------------------------------------- transforms
// normalize (tb8gen.c:230-238) on a whole bitboard: xor of every square with
// the mirror mask (0x07 mirrors files, 0x38 ranks), then optionally the a1-h8
// transpose (FlipDiag).
__device__ __forceinline__ bb bswap64(bb x) {
  uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
  return ((bb)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

// a1-h8 transpose by three delta swaps (chessprogramming wiki,
// "Flipping Mirroring and Rotating").
__device__ __forceinline__ bb transpose(bb x) {
  bb t;
  t = 0x0f0f0f0f00000000ull & (x ^ (x << 28));
  x ^= t ^ (t >> 28);
  t = 0x3333000033330000ull & (x ^ (x << 14));
  x ^= t ^ (t >> 14);
  t = 0x5500550055005500ull & (x ^ (x << 7));
  x ^= t ^ (t >> 7);
  return x;
}

__device__ __forceinline__ bb xform(bb x, int mirror, int flip) {
  if (mirror == 0x3f) x = __brevll(x);
  else if (mirror == 0x07) x = bswap64(__brevll(x));
  else if (mirror == 0x38) x = bswap64(x);
  return flip ? transpose(x) : x;
}

// ------------------------------------------------------------------ index
// Binomials C(n, k) for k <= 6, n < 64 (Binomial, probe.c:541-546), staged in
// shared memory by every kernel that ranks or unranks: bin[k * 64 + n].
struct BinTable {
  uint32_t v[7 * 64];
};

__device__ __forceinline__ void load_binomials(uint32_t *bin) {
  for (int i = threadIdx.x; i < 7 * 64; i += blockDim.x) {
    int k = i >> 6, n = i & 63;
    // C(n, k) by the multiplicative formula; exact in 64 bits for n < 64, k <= 6.
    uint64_t c = 1;
    for (int j = 0; j < k; j++) c = c * (uint64_t)(n - j) / (uint64_t)(j + 1);
    bin[i] = n < k ? 0u : (uint32_t)c;
  }
}

// Quotient n / d for n < 2^32 by a precomputed M = ceil(2^64 / d) (Lemire,
// Kaser, Kurz, "Faster remainder by direct computation", 2019): q = hi64(M n).
// d == 1 is encoded as M == 0.
__device__ __forceinline__ uint32_t fast_div32(uint32_t n, uint64_t M) {
  return M ? (uint32_t)__umul64hi(M, (uint64_t)n) : n;
}

// Combinatorial rank of the sets of a position (sq_to_idx_helper,
// tb8gen.c:129-149): each set's squares, in increasing order, ranked among
// the squares not taken by the kings and earlier sets.
template <int NS>
__device__ __forceinline__ uint64_t rank_sets(const DIdx &X, const uint32_t *bin,
                                             int k0, int k1, const bb *set) {
  bb occ = bit(k0) | bit(k1);
  uint64_t idx = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    {
      bb b = set[k];
      uint32_t s = 0;
      int j = 1;
      while (b) {
        int x = pop_lsb(b);
        int r = x - __popcll(occ & (bit(x) - 1));
        s += bin[j * 64 + r];
        j++;
      }
      idx += (uint64_t)s * X.factor[k];
      occ |= set[k];
    }
  }
  return idx;
}

// The r-th (0-based) set bit of b.
__device__ __forceinline__ int nth_set(bb b, int r) {
  uint32_t lo = (uint32_t)b;
  int c = __popc(lo);
  if (r < c) return __fns(lo, 0, r + 1);
  return 32 + __fns((uint32_t)(b >> 32), 0, r - c + 1);
}

// Inverse of rank_sets (idx_to_sq_init + unrank_binomial, tb8gen.c:105-126,
// 169-175): fills set[] and returns the occupancy, kings included.
template <int NS>
__device__ __forceinline__ bb unrank_sets(const DIdx &X, const uint32_t *bin,
                                         uint64_t idx, int k0, int k1, bb *set) {
  bb occ = bit(k0) | bit(k1);
  uint32_t rem32 = (uint32_t)idx;
  bool small = idx < (1ull << 32);
#pragma unroll
  for (int k = 0; k < NS; k++) {
    set[k] = 0;
    {
      uint32_t d;
      if (small) {
        d = fast_div32(rem32, X.fdiv[k]);
        rem32 -= d * (uint32_t)X.factor[k];
      } else {
        uint64_t q = idx / X.factor[k];
        idx -= q * X.factor[k];
        d = (uint32_t)q;
        if (idx < (1ull << 32)) {
          small = true;
          rem32 = (uint32_t)idx;
        }
      }
      bb freeb = ~occ, sb = 0;
      int m = X.mult[k];
      for (int i = m - 1; i > 0; i--) {
        const uint32_t *row = bin + (i + 1) * 64;
        int lo = i, hi = 63;
        while (hi - lo > 1) {
          int mid = (lo + hi) >> 1;
          if (row[mid] <= d) lo = mid;
          else hi = mid;
        }
        d -= row[lo];
        sb |= bit(nth_set(freeb, lo));
      }
      if (m > 0) sb |= bit(nth_set(freeb, (int)d));
      set[k] = sb;
      occ |= sb;
    }
  }
  return occ;
}

// The next m-subset of the free squares in colex order, which is the order
// of the rank of a set (the combinatorial number system of unrank_sets): the
// lowest square that can move up to the next free square without reaching
// the set's next square moves there, and the squares below it drop to the
// lowest free squares.  s holds m >= 1 squares of freeb and is not the last
// subset.
__device__ __forceinline__ bb next_colex(bb s, bb freeb) {
  int passed = 0;
  for (;;) {
    const int x = __ffsll((long long)s) - 1;
    const bb rest = s & (s - 1);
    const bb up = x == 63 ? 0 : freeb & ~((bit(x) << 1) - 1);
    if (rest == 0 || (up & (rest & (~rest + 1)) - 1) != 0) {
      bb low = 0, f = freeb;
      for (int i = 0; i < passed; i++) {
        const bb lb = f & (~f + 1);
        low |= lb;
        f ^= lb;
      }
      return rest | (up & (~up + 1)) | low;
    }
    s = rest;
    passed++;
  }
}

// The sets of position idx for a caller that visits consecutive indices:
// a full unrank where a row starts (the last set's combinations under one
// placement of the others, or the whole index with a single set), else the
// next combination of the last set.  `left` (0 at the first call) counts
// the positions left in the current row; `occ` is the previous call's
// result.
template <int NS>
__device__ __forceinline__ bb walk_sets(const DIdx &X, const uint32_t *bin, uint64_t idx, int k0,
                                       int k1, bb *set, bb occ, uint64_t &left) {
  constexpr int L = NS - 1;
  if (left == 0) {
    occ = unrank_sets<NS>(X, bin, idx, k0, k1, set);
    uint64_t off = idx;
    if (L > 0) {
      const uint64_t F = X.factor[L > 0 ? L - 1 : 0];
      const uint64_t row = idx < (1ull << 32)
                               ? fast_div32((uint32_t)idx, X.fdiv[L > 0 ? L - 1 : 0])
                               : idx / F;
      off = idx - row * F;
      left = F - off;
    } else {
      left = X.size - off;
    }
  } else {
    bb last = 0;
#pragma unroll
    for (int k = 0; k < NS; k++)
      if (k == L) last = set[k];
    const bb nl = next_colex(last, ~(occ & ~last));
#pragma unroll
    for (int k = 0; k < NS; k++)
      if (k == L) set[k] = nl;
    occ = (occ & ~last) | nl;
  }
  left--;
  return occ;
}

// Whether a piece of colour `color` attacks square `target` (is_attacked_by,
// movegen.h:180-188), given each set's type/colour, the king squares and
// the occupancy.
template <int NS>
__device__ __forceinline__ bool attacked_by(const DMat &M, const bb *set, int k0, int k1,
                                            bb occ, int target, int color) {
  bb rq = 0, bq = 0, n = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    if (M.set_color[k] == color) {
      int t = M.set_type[k];
      if (t == 4 || t == 5) rq |= set[k];
      if (t == 3 || t == 5) bq |= set[k];
      if (t == 2) n |= set[k];
    }
  }
  int ksq = color ? k1 : k0;
  return ((rook_attacks(target, occ) & rq) | (bishop_attacks(target, occ) & bq) |
          (knight_attacks(target) & n) | (king_attacks(target) & bit(ksq))) != 0;
}

// Splitmix64 output function (Steele, Lea, Flood, OOPSLA 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace tbg
