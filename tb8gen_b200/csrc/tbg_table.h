// The 7-piece WDL table format the engine probes: the reference's .rtbw
// layout for pawnless tables with rANS-compressed blocks (probe.c:603-1044,
// 1049-1390; rans.h; rans.c), and the synthetic table the engine builds in
// that format.  Everything here is plain C++ usable on the host and (where
// marked TBG_HD) on the device.
//
// Formats and tables have to be alike for the reference's reader to read
// what the engine writes and vice versa; the code is this project's own.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#ifdef __CUDACC__
#define TBG_HD __host__ __device__ __forceinline__
#else
#define TBG_HD inline
#endif

namespace tbg {

// ---------------------------------------------------------------- tables
// The square tables of probe.c:299-571, generated from their rules.
struct EncTables {
  int8_t offdiag[64];      // +1 above the a1-h8 diagonal (rank > file), -1 below
  uint8_t triangle[64];    // a1-d1-d4 triangle index, off-diagonal 0..5 first
  uint8_t lower[64];       // file > rank squares 0..27 (row-major), diagonal 28..35
  uint8_t diag[64];        // a1-h8 diagonal 0..7, h1-a8 diagonal 8..15
  uint8_t flipdiag[64];
  uint8_t inv_triangle[10];
  uint8_t inv_diag[16];
  uint8_t inv_lower[36];
  int16_t kkidx[10][64];
  uint8_t kksq[462][2];
  uint32_t binom[8][64];   // C(n, k)
};

void build_enc_tables(EncTables &t);

// EncInfo (probe.h:71-76) of one side of a pawnless table.
struct EncInfoP {
  int num;                 // pieces
  int kk;                  // kk_enc: only the two kings are unique (probe.c:183-187)
  uint8_t pieces[8];       // piece codes, in table order
  uint8_t norm[8];         // group size at the group's first piece
  uint64_t factor[8];      // mixed-radix factor at the group's first piece
  uint64_t size;           // positions of the table side
};

// set_enc_info (probe.c:725-771), PIECE_ENC.
uint64_t set_enc_info(EncInfoP &ei, const uint8_t *tb, int shift, int num, int kk);

TBG_HD int popcount64(uint64_t b) {
#ifdef __CUDA_ARCH__
  return __popcll(b);
#else
  return __builtin_popcountll(b);
#endif
}

TBG_HD int lsb64(uint64_t b) {
#ifdef __CUDA_ARCH__
  return __ffsll((long long)b) - 1;
#else
  return __builtin_ctzll(b);
#endif
}

// The r-th (0-based) zero bit of occ.
TBG_HD int nth_free(uint64_t occ, int r) {
  uint64_t b = ~occ;
  for (int i = 0; i < r; i++) b &= b - 1;
  return lsb64(b);
}

// encode (probe.c:603-694) with enc == PIECE_ENC; p[] is modified.
TBG_HD uint64_t encode_piece(const EncTables &T, const EncInfoP &ei, uint8_t *p) {
  const int n = ei.num;
  if (p[0] & 0x04)
    for (int i = 0; i < 8; i++) p[i] ^= 0x07;
  if (p[0] & 0x20)
    for (int i = 0; i < 8; i++) p[i] ^= 0x38;
  for (int i = 0; i < n; i++)
    if (T.offdiag[p[i]]) {
      if (T.offdiag[p[i]] > 0 && i < (ei.kk ? 2 : 3))
        for (int j = 0; j < n; j++) p[j] = T.flipdiag[p[j]];
      break;
    }
  uint64_t idx;
  int k;
  if (ei.kk) {
    idx = (uint64_t)T.kkidx[T.triangle[p[0]]][p[1]];
    k = 2;
  } else {
    int s1 = p[1] > p[0];
    int s2 = (p[2] > p[0]) + (p[2] > p[1]);
    if (T.offdiag[p[0]])
      idx = (uint64_t)T.triangle[p[0]] * 63 * 62 + (p[1] - s1) * 62 + (p[2] - s2);
    else if (T.offdiag[p[1]])
      idx = 6 * 63 * 62 + T.diag[p[0]] * 28 * 62 + T.lower[p[1]] * 62 + p[2] - s2;
    else if (T.offdiag[p[2]])
      idx = 6 * 63 * 62 + 4 * 28 * 62 + T.diag[p[0]] * 7 * 28 + (T.diag[p[1]] - s1) * 28 +
            T.lower[p[2]];
    else
      idx = 6 * 63 * 62 + 4 * 28 * 62 + 4 * 7 * 28 + T.diag[p[0]] * 7 * 6 +
            (T.diag[p[1]] - s1) * 6 + (T.diag[p[2]] - s2);
    k = 3;
  }
  idx *= ei.factor[0];
  uint64_t occ = 0;
  for (int i = 0; i < k; i++) occ |= 1ull << p[i];
  while (k < n) {
    const int t = k + ei.norm[k];
    // the group's squares, in increasing order, ranked among the free ones
    uint64_t g = 0;
    for (int i = k; i < t; i++) g |= 1ull << p[i];
    uint64_t s = 0;
    int j = 1;
    for (uint64_t b = g; b; b &= b - 1, j++) {
      int sq = lsb64(b);
      int r = sq - popcount64(occ & ((1ull << sq) - 1));
      s += T.binom[j][r];
    }
    idx += s * ei.factor[k];
    occ |= g;
    k = t;
  }
  return idx;
}

// decode_piece (probe.c:978-994, decode_helper 883-976) for PIECE_ENC: the
// squares of the position at table index idx, in table order.
TBG_HD void decode_piece(const EncTables &T, const EncInfoP &ei, uint64_t idx, uint8_t *p) {
  const int n = ei.num;
  // digits, most significant group first
  int groups[8], ng = 0;
  for (int k = 0; k < n;) {
    groups[ng++] = k;
    k += k == 0 ? (ei.kk ? 2 : 3) : ei.norm[k];
  }
  int order[8];
  for (int g = 0; g < ng; g++) {
    int j = g;
    while (j > 0 && ei.factor[groups[order[j - 1]]] < ei.factor[groups[g]]) {
      order[j] = order[j - 1];
      j--;
    }
    order[j] = g;
  }
  uint64_t d[8], rem = idx;
  for (int h = 0; h < ng; h++) {
    const int g = order[h];
    const uint64_t f = ei.factor[groups[g]];
    d[g] = rem / f;
    rem -= d[g] * f;
  }
  uint64_t occ = 0;
  uint32_t q = (uint32_t)d[0];
  int i;
  if (ei.kk) {
    p[0] = T.kksq[q][0];
    p[1] = T.kksq[q][1];
    occ = (1ull << p[0]) | (1ull << p[1]);
    i = 2;
  } else {
    const uint64_t DIAG = 0x8040201008040201ull;
    uint32_t r;
    if (q < 6 * 63 * 62) {
      r = q / (63 * 62);
      q -= r * 63 * 62;
      p[0] = T.inv_triangle[r];
      occ = 1ull << p[0];
      r = q / 62;
      q -= r * 62;
      r += (r >= p[0]);
      p[1] = (uint8_t)r;
      occ |= 1ull << r;
      p[2] = (uint8_t)nth_free(occ, (int)q);
      occ |= 1ull << p[2];
    } else if (q < 6 * 63 * 62 + 4 * 28 * 62) {
      q -= 6 * 63 * 62;
      r = q / (28 * 62);
      q -= r * 28 * 62;
      p[0] = T.inv_diag[r];
      occ = 1ull << p[0];
      r = q / 62;
      q -= r * 62;
      p[1] = T.inv_lower[r];
      occ |= 1ull << p[1];
      p[2] = (uint8_t)nth_free(occ, (int)q);
      occ |= 1ull << p[2];
    } else if (q < 6 * 63 * 62 + 4 * 28 * 62 + 4 * 7 * 28) {
      q -= 6 * 63 * 62 + 4 * 28 * 62;
      r = q / (7 * 28);
      q -= r * 7 * 28;
      p[0] = T.inv_diag[r];
      occ = 1ull << p[0];
      r = q / 28;
      q -= r * 28;
      r += (T.inv_diag[r] >= p[0]);
      p[1] = T.inv_diag[r];
      occ |= 1ull << p[1];
      p[2] = T.inv_lower[q];
      occ |= 1ull << p[2];
    } else {
      q -= 6 * 63 * 62 + 4 * 28 * 62 + 4 * 7 * 28;
      r = q / (7 * 6);
      q -= r * 7 * 6;
      p[0] = T.inv_diag[r];
      occ = 1ull << p[0];
      r = q / 6;
      q -= r * 6;
      r += (T.inv_diag[r] >= p[0]);
      p[1] = T.inv_diag[r];
      occ |= 1ull << p[1];
      // q-th free square on the a1-h8 diagonal
      p[2] = (uint8_t)nth_free(occ | ~DIAG, (int)q);
      occ |= 1ull << p[2];
    }
    i = 3;
  }
  for (int g = 1; g < ng; g++) {
    const int k = groups[g], m = ei.norm[k];
    uint64_t v = d[g];
    const uint64_t freeocc = occ;
    uint64_t sb = 0;
    for (int j = m - 1; j > 0; j--) {
      int r = j;
      while (v >= T.binom[j + 1][r + 1]) r++;
      v -= T.binom[j + 1][r];
      int sq = nth_free(freeocc, r);
      p[k + j] = (uint8_t)sq;
      sb |= 1ull << sq;
    }
    int sq = nth_free(freeocc, (int)v);
    p[k] = (uint8_t)sq;
    sb |= 1ull << sq;
    occ |= sb;
    (void)i;
  }
}

// --------------------------------------------------------------- rANS
// 64-bit-state rANS with a 4096-bucket alias table (rans.h:10-140, after
// ryg_rans, F. Giesen).  Probabilities are 16-bit.
constexpr uint64_t kRansL = 1ull << 31;

struct RansEntry {
  uint16_t alias_div;   // alias symbol << 4 | divider & 15
  uint16_t start;
};

struct RansDecodeTab {
  RansEntry entry[4096];
  uint16_t freq[4096];
};

// Encoder side of a code (struct RansCode, rans.h:26-32).
struct RansCodeHost {
  RansDecodeTab d;
  uint16_t cum_freq[4096];
  uint16_t alias_remap[1 << 16];
  uint16_t map[4096];   // sorted symbol -> original symbol
  uint16_t inv[4096];   // original symbol -> sorted symbol
};

// create_code_rans (rans.c:145-152): normalise, sort by frequency, alias.
void create_code(RansCodeHost &c, const int64_t *freq, int num_syms);
// make_alias_table (rans.c:95-143).
void make_alias(RansDecodeTab &d, RansCodeHost *c);
// write_freq_table (rans.c:239-276): the coded frequency table bytes.
std::vector<uint8_t> freq_table_bytes(const RansCodeHost &c, int num_syms);
// read_freq_table (rans.c:278-314).
const uint8_t *read_freq_table(RansDecodeTab &d, int *num_syms, const uint8_t *p);

TBG_HD uint32_t rd_le32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
TBG_HD uint64_t rd_le64(const uint8_t *p) {
  return (uint64_t)rd_le32(p) | ((uint64_t)rd_le32(p + 4) << 32);
}
TBG_HD void wr_le32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}
TBG_HD void wr_le64(uint8_t *p, uint64_t v) {
  wr_le32(p, (uint32_t)v);
  wr_le32(p + 4, (uint32_t)(v >> 32));
}

// rans_enc_put (rans.h:39-58): encodes sorted symbol s, output moving down
// from *p; `end` is the lowest address renormalisation may write to.
// Returns false (state unchanged) when the block is full.
TBG_HD bool rans_put(uint64_t &x0, const uint16_t *freqs, const uint16_t *cum,
                     const uint16_t *remap, int s, uint8_t *&p, const uint8_t *end) {
  const uint32_t freq = freqs[s];
  const uint64_t x_max = (uint64_t)freq << 47;
  uint64_t x = x0;
  if (x >= x_max && (p != end || x >= 2 * x_max)) {
    if (p == end) return false;
    p -= 4;
    wr_le32(p, (uint32_t)x);
    x >>= 32;
  }
  x0 = ((x / freq) << 16) + remap[(x % freq) + cum[s]];
  return true;
}

// rans_enc_flush (rans.h:79-87).
TBG_HD void rans_flush(uint64_t x, uint8_t *&p, const uint8_t *start) {
  p -= 8;
  wr_le64(p, x);
  while (p > start) {
    p -= 4;
    wr_le32(p, 0);
  }
}

// rans_dec_init / rans_dec_get / rans_dec_renorm (rans.h:89-140).
TBG_HD void rans_dec_init(uint64_t &x, const uint8_t *&p, const uint8_t *end) {
  while (rd_le32(p) == 0 && p + 8 < end) p += 4;
  x = rd_le64(p);
  p += 8;
}

TBG_HD int rans_dec_get(uint64_t &x, const RansEntry *entry, const uint16_t *freq) {
  const uint64_t v = x;
  int s = (int)((v >> 4) & 4095);
  uint32_t rem = (uint32_t)(v & 15);
  const RansEntry e = entry[s];
  if (rem >= (uint32_t)(e.alias_div & 15)) {
    rem = (rem + e.start) & 0xffff;  // wraps by design
    s = e.alias_div >> 4;
  }
  x = (uint64_t)freq[s] * (v >> 16) + rem;
  return s;
}

TBG_HD void rans_dec_renorm(uint64_t &x, const uint8_t *&p) {
  if (x < kRansL) {
    x = (x << 32) | rd_le32(p);
    p += 4;
  }
}

// ---------------------------------------------------------- synthetic table
// Table sides are cut into blocks of exactly kBlockPositions positions (the
// size table counts positions in 16 bits, probe.c:1360-1365), coded as
// "quad" symbols of four consecutive values: sympat holds the leaves (one
// per value), the pairs of leaves and the quads (pairs of pairs), the
// Re-Pair tree the reader descends (probe.c:1049-1062, 1380-1389).
constexpr int kBlockBits = 16;                 // 64 KiB blocks (block_size)
constexpr uint32_t kBlockPositions = 65536;    // positions per block
constexpr int kQuadsPerBlock = kBlockPositions / 4;
constexpr int kIdxBits = 16;                   // one index entry per block

// Per-position value of the synthetic table: VALS[mix64(seed ^ idx ^
// bside << 63) % modulus], VALS = {-2, 0, 2} or {-2, -1, 0, 1, 2}; stored +2.
TBG_HD uint64_t tbl_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

TBG_HD int table_value(uint64_t seed, int modulus, uint64_t idx, int bside) {
  uint64_t h = tbl_mix64(seed ^ idx ^ ((uint64_t)bside << 63));
  if (modulus == 5) return (int)(h % 5);      // stored value wdl + 2
  return (int)(h % 3) * 2;
}

// Symbol numbering before frequency sorting: leaves 0..M-1, pairs
// M + a*M + b, quads M + M*M + (a*M + b)*M*M + (c*M + d).
TBG_HD int quad_symbol(int M, int a, int b, int c, int d) {
  return M + M * M + (a * M + b) * M * M + (c * M + d);
}

// Positions in block b of a side of `size` positions.
TBG_HD uint32_t block_positions(uint64_t size, uint64_t b) {
  const uint64_t start = b * kBlockPositions;
  const uint64_t n = size - start;
  return n < kBlockPositions ? (uint32_t)n : kBlockPositions;
}

// Quads in block b.  A block whose position count is not a multiple of 4
// (only the last block of a side can be one) gets front padding: its first
// quad starts `pad` positions before the block, so that every quad ends on
// a position the reader counts back to from the block's end
// (decompress_rans decodes the last symbol first, probe.c:1362-1372).
TBG_HD uint32_t block_quads(uint64_t size, uint64_t b) { return (block_positions(size, b) + 3) / 4; }
TBG_HD uint32_t block_pad(uint32_t npos) { return (4 - (npos & 3)) & 3; }

TBG_HD uint64_t side_blocks(uint64_t size) { return (size + kBlockPositions - 1) / kBlockPositions; }
TBG_HD uint64_t side_quads(uint64_t size) {
  const uint64_t nb = side_blocks(size);
  return nb ? (nb - 1) * kQuadsPerBlock + block_quads(size, nb - 1) : 0;
}

// The four values (0..M-1, most significant first) of quad q of a side as
// one base-M number; padding positions hold 0.
TBG_HD int quad_values(uint64_t seed, int M, int bside, uint64_t size, uint64_t q) {
  const uint64_t b = q / kQuadsPerBlock, j = q % kQuadsPerBlock;
  const uint64_t start = b * kBlockPositions;
  const uint32_t pad = block_pad(block_positions(size, b));
  int code = 0;
  for (int t = 0; t < 4; t++) {
    const uint64_t rel = 4 * j + t;
    int v = 0;
    if (rel >= pad) v = table_value(seed, M, start + rel - pad, bside) / (M == 5 ? 1 : 2);
    code = code * M + v;
  }
  return code;
}

}  // namespace tbg
