// WDL probes into rANS-compressed 7-piece tables (probe_table, decompress_rans,
// probe.c:1346-1390, 1522-1597) and the builder of the synthetic table.
//
// A probe batch runs in passes instead of one independent decode per
// position: (1) every position is encoded (encode_piece) and located in its
// block through the index and size tables, counting the positions per block
// and the lowest position asked for; (2) a scan numbers the touched blocks;
// (3) every touched block is decoded once, by one thread, from its end down
// to the lowest position asked for, into a scratch array of symbol ids;
// (4) each position reads its symbol and descends the Re-Pair tree to its
// value.  A 64 KiB block holds up to 65,536 positions, so per-position
// decoding costs up to 16,384 rANS steps per probe; grouped, the cost is
// one decode per touched block.
#pragma once

#include "tbg_device.cuh"
#include "tbg_table.h"

namespace tbg {

struct ProbeSide {
  EncInfoP ei;
  const uint8_t *index;     // 6 B per 2^idx_bits positions
  const uint8_t *sizes;     // u16 per block: positions in the block - 1
  const uint8_t *data;      // blocks of 2^block_size bytes
  const uint16_t *start;    // per block: word offset of its stream (k_block_starts), or null
  const RansEntry *entry;   // decode table (device copy)
  const uint16_t *freq;
  const uint8_t *sympat;    // 3 B per symbol (inside the table)
  const uint8_t *symlen;    // per symbol (device copy)
  uint64_t nblocks;
  uint32_t key0;            // first block key of this side
  int idx_bits, block_size;
  int sym_positions;        // positions per top-level symbol if all equal, else 0
  int nsym_emit;            // symbols with nonzero frequency: ids 0 .. nsym_emit-1
};

struct ProbeTable {
  int num;
  int symmetric;
  uint8_t pt[8];            // piece types of the queries' squares (material order)
  const EncTables *T;
  ProbeSide side[2];
};

// A query: squares in material order and the side to move (16 bytes).
struct Query {
  uint8_t sq[8];
  uint8_t stm;
  uint8_t pad[7];
};

// Output of a query that is not a placement of the material: a square
// outside the board or used twice, stm not 0/1, or (kk-encoded tables,
// where KKIdx has no entry for them) kings on adjacent squares.  The
// reference has no such check: its callers only pass legal positions.
constexpr int8_t kWdlInvalid = -128;

// Byte i of eight squares packed into a 64-bit register.
__device__ __forceinline__ int pk_get(uint64_t p, int i) { return (int)(p >> (8 * i)) & 0xff; }

// encode_piece (probe.c:603-694, PIECE_ENC) with the squares packed one per
// byte of a register (byte i: table piece i) and the square tables in
// shared memory: the steps of the host function in tbg_table.h, without a
// square array indexed at run time (which would live in local memory).
__device__ __forceinline__ uint64_t encode_packed(const EncTables &T, const EncInfoP &ei,
                                                  uint64_t p) {
  const int n = ei.num;
  if (p & 0x04) p ^= 0x0707070707070707ull;
  if (p & 0x20) p ^= 0x3838383838383838ull;
  const int lim = ei.kk ? 2 : 3;
  for (int i = 0; i < n; i++) {
    const int o = T.offdiag[pk_get(p, i)];
    if (o) {
      if (o > 0 && i < lim) {
        uint64_t q = p;
        for (int j = 0; j < n; j++) {
          const int sh = 8 * j;
          q = (q & ~(0xffull << sh)) | ((uint64_t)T.flipdiag[pk_get(p, j)] << sh);
        }
        p = q;
      }
      break;
    }
  }
  const int p0 = pk_get(p, 0), p1 = pk_get(p, 1), p2 = pk_get(p, 2);
  uint64_t idx;
  int k;
  uint64_t occ = (1ull << p0) | (1ull << p1);
  if (ei.kk) {
    idx = (uint64_t)T.kkidx[T.triangle[p0]][p1];
    k = 2;
  } else {
    const int s1 = p1 > p0;
    const int s2 = (p2 > p0) + (p2 > p1);
    if (T.offdiag[p0])
      idx = (uint64_t)T.triangle[p0] * 63 * 62 + (p1 - s1) * 62 + (p2 - s2);
    else if (T.offdiag[p1])
      idx = 6 * 63 * 62 + T.diag[p0] * 28 * 62 + T.lower[p1] * 62 + p2 - s2;
    else if (T.offdiag[p2])
      idx = 6 * 63 * 62 + 4 * 28 * 62 + T.diag[p0] * 7 * 28 + (T.diag[p1] - s1) * 28 +
            T.lower[p2];
    else
      idx = 6 * 63 * 62 + 4 * 28 * 62 + 4 * 7 * 28 + T.diag[p0] * 7 * 6 +
            (T.diag[p1] - s1) * 6 + (T.diag[p2] - s2);
    occ |= 1ull << p2;
    k = 3;
  }
  idx *= ei.factor[0];
  while (k < n) {
    const int t = k + ei.norm[k];
    uint64_t g = 0;
    for (int i = k; i < t; i++) g |= 1ull << pk_get(p, i);
    uint64_t sum = 0;
    int j = 1;
    for (uint64_t b = g; b; b &= b - 1, j++) {
      const int sq = __ffsll((long long)b) - 1;
      sum += T.binom[j][sq - __popcll(occ & ((1ull << sq) - 1))];
    }
    idx += sum * ei.factor[k];
    occ |= g;
    k = t;
  }
  return idx;
}

// The square tables of a ProbeTable copied into a block's shared memory.
__device__ __forceinline__ void load_enc_tables(const EncTables *g, EncTables &s) {
  const uint32_t *src = reinterpret_cast<const uint32_t *>(g);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(EncTables) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// A query loaded as one vector: squares packed, side to move.  A 16-byte
// query is tbg_query; an 8-byte one (materials of at most 7 pieces) holds
// the squares in bytes 0-6 and the side to move in byte 7.
__device__ __forceinline__ void load_query(const Query *q, uint64_t i, int qbytes, uint64_t &sqs,
                                           int &stm) {
  if (qbytes == 8) {
    const uint2 v = reinterpret_cast<const uint2 *>(q)[i];
    sqs = (uint64_t)v.x | ((uint64_t)(v.y & 0x00ffffffu) << 32);
    stm = (int)(v.y >> 24);
    return;
  }
  const uint4 v = reinterpret_cast<const uint4 *>(q)[i];
  sqs = (uint64_t)v.x | ((uint64_t)v.y << 32);
  stm = (int)(v.z & 0xff);
}

// list_squares (probe.c:1511-1520) then encode_piece: table index and side.
// Returns false for a query that is not a placement (see kWdlInvalid).
__device__ __forceinline__ bool query_index(const ProbeTable &P, const EncTables &T, uint64_t sqs,
                                            int stm, int &bside, uint64_t &idx) {
  uint64_t occ = 0;
  int wk = 0, bk = 0;
  for (int j = 0; j < P.num; j++) {
    const int sq = pk_get(sqs, j);
    if (sq >= 64 || ((occ >> sq) & 1)) return false;
    occ |= 1ull << sq;
    if (P.pt[j] == 6) wk = sq;
    if (P.pt[j] == 14) bk = sq;
  }
  if (stm > 1) return false;
  int flip;
  if (!P.symmetric) {
    flip = 0;
    bside = stm == 1;
  } else {
    flip = stm != 0;
    bside = 0;
  }
  const ProbeSide &S = P.side[bside];
  if (S.ei.kk) {
    const int df = (wk & 7) - (bk & 7), dr = (wk >> 3) - (bk >> 3);
    if (df >= -1 && df <= 1 && dr >= -1 && dr <= 1) return false;
  }
  const int fx = flip ? 0x38 : 0x00;
  uint64_t p = 0;
  for (int i = 0; i < P.num;) {
    const int t = S.ei.pieces[i] ^ (flip << 3);
    for (int j = 0; j < P.num; j++)
      if (P.pt[j] == t) {
        p |= (uint64_t)(pk_get(sqs, j) ^ fx) << (8 * i);
        i++;
      }
  }
  idx = encode_packed(T, S.ei, p);
  return idx < S.ei.size;
}

// The block of idx and its position there, counted from the block's start
// (the walk of decompress_rans, probe.c:1348-1360).
__device__ __forceinline__ void locate(const ProbeSide &S, uint64_t idx, uint32_t &block,
                                       int &lit) {
  uint32_t main_idx = (uint32_t)(idx >> S.idx_bits);
  lit = (int)((uint32_t)idx & ((1u << S.idx_bits) - 1)) - (int)(1u << (S.idx_bits - 1));
  const uint8_t *e = S.index + 6ull * main_idx;
  block = rd_le32(e);
  lit += (int)((uint32_t)e[4] | ((uint32_t)e[5] << 8));
  auto sz = [&](uint32_t b) { return (int)((uint32_t)S.sizes[2 * b] | ((uint32_t)S.sizes[2 * b + 1] << 8)); };
  if (lit < 0)
    while (lit < 0) lit += sz(--block) + 1;
  else
    while (lit > sz(block)) lit -= sz(block++) + 1;
}

__device__ __forceinline__ int block_npos(const ProbeSide &S, uint32_t block) {
  return (int)((uint32_t)S.sizes[2 * block] | ((uint32_t)S.sizes[2 * block + 1] << 8)) + 1;
}

// The Re-Pair descent of decompress_rans (probe.c:1380-1389): the value
// byte of position `lit` inside symbol `sym`.
__device__ __forceinline__ uint8_t descend(const ProbeSide &S, int sym, int lit) {
  while (S.symlen[sym] != 0) {
    const uint8_t *w = S.sympat + 3 * sym;
    int s1 = ((w[1] & 0xf) << 8) | w[0];
    if (lit < (int)S.symlen[s1] + 1) {
      sym = s1;
    } else {
      lit -= (int)S.symlen[s1] + 1;
      sym = (w[2] << 4) | (w[1] >> 4);
    }
  }
  return S.sympat[3 * sym];
}

// rans_dec_init / rans_dec_renorm (rans.h:89-95, 129-140) for a block in
// device memory, whose start is 64-byte aligned so that every word the
// reader visits is 4-byte aligned: zero words are skipped 64 bytes at a
// time while the reference's loop would skip all of them, then one at a
// time under the reference's own condition.
__device__ __forceinline__ void dev_dec_init(uint64_t &x, const uint8_t *&p, const uint8_t *end) {
  while (p + 68 < end) {
    const uint4 *c = reinterpret_cast<const uint4 *>(p);
    const uint4 a = c[0], b = c[1], d = c[2], e = c[3];
    if ((a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w | d.x | d.y | d.z | d.w | e.x | e.y | e.z |
         e.w) != 0)
      break;
    p += 64;
  }
  while (*reinterpret_cast<const uint32_t *>(p) == 0 && p + 8 < end) p += 4;
  const uint32_t *w = reinterpret_cast<const uint32_t *>(p);
  x = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
  p += 8;
}

// dev_dec_init from the block's start offset found at open (k_block_starts):
// the same first word, without reading the block's zero padding again.
__device__ __forceinline__ void dev_dec_start(const ProbeSide &S, uint32_t block, uint64_t &x,
                                              const uint8_t *&p, const uint8_t *end) {
  if (S.start == nullptr) {
    dev_dec_init(x, p, end);
    return;
  }
  p += 4 * (uint32_t)S.start[block];
  const uint32_t *w = reinterpret_cast<const uint32_t *>(p);
  x = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
  p += 8;
}

// dev_dec_init's scan for every block of one side, once per opened table:
// the word where the block's stream begins, i.e. its first nonzero 32-bit
// word, or the word 8 bytes before the block's end if that comes first
// (where the scan stops).  One warp per block, 512 bytes per step.
__global__ void __launch_bounds__(256) k_block_starts(ProbeSide S, uint16_t *start) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t nwords = 1u << (S.block_size - 2);
  const uint32_t limit = nwords - 2;
  for (uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; b < S.nblocks;
       b += nwarps) {
    const uint4 *c = reinterpret_cast<const uint4 *>(S.data + (b << S.block_size));
    uint32_t found = limit;
    for (uint32_t w0 = 0; w0 < limit; w0 += 128) {
      const uint32_t w = w0 + 4 * lane;
      const uint4 v = w < nwords ? c[w >> 2] : make_uint4(0, 0, 0, 0);
      const int first = v.x ? 0 : v.y ? 1 : v.z ? 2 : v.w ? 3 : 4;
      const unsigned m = __ballot_sync(0xffffffffu, first < 4);
      if (m) {
        const int l = __ffs(m) - 1;
        const int f = __shfl_sync(0xffffffffu, first, l);
        found = min(w0 + 4u * l + (uint32_t)f, limit);
        break;
      }
    }
    if (lane == 0) start[b] = (uint16_t)found;
  }
}

__device__ __forceinline__ void dev_dec_renorm(uint64_t &x, const uint8_t *&p) {
  if (x < kRansL) {
    x = (x << 32) | *reinterpret_cast<const uint32_t *>(p);
    p += 4;
  }
}

// The whole of decompress_rans for one index (reference path, any table).
__device__ __forceinline__ int probe_one(const ProbeSide &S, uint64_t idx) {
  uint32_t block;
  int lit;
  locate(S, idx, block, lit);
  int sz = (int)((uint32_t)S.sizes[2 * block] | ((uint32_t)S.sizes[2 * block + 1] << 8));
  lit -= sz + 1;
  const uint8_t *p = S.data + ((size_t)block << S.block_size);
  const uint8_t *end = p + ((size_t)1 << S.block_size);
  uint64_t x;
  dev_dec_start(S, block, x, p, end);
  int sym = 0;
  for (; lit < 0 && p < end; lit += S.symlen[sym] + 1) {
    sym = rans_dec_get(x, S.entry, S.freq);
    dev_dec_renorm(x, p);
  }
  for (; lit < 0; lit += S.symlen[sym] + 1) sym = rans_dec_get(x, S.entry, S.freq);
  return (int)descend(S, sym, lit) - 2;
}

// ------------------------------------------------------------ probe passes
constexpr uint32_t kNoKey = 0xffffffffu;
constexpr uint32_t kNoLit = 0xffffffffu;  // minlit of an untouched block

// Pass 1 of a grouped probe (tables whose symbols all cover L positions):
// block key and symbol-relative position of every query, and per block the
// lowest position asked for (which also marks the block touched).
__global__ void k_probe_locate(ProbeTable P, const Query *q, int qbytes, uint64_t n,
                               uint32_t *key, uint32_t *lit, uint32_t *minlit, int8_t *out) {
  __shared__ EncTables T;
  load_enc_tables(P.T, T);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int bside, stm;
    uint64_t idx, sqs;
    load_query(q, i, qbytes, sqs, stm);
    if (!query_index(P, T, sqs, stm, bside, idx)) {
      key[i] = kNoKey;
      out[i] = kWdlInvalid;
      continue;
    }
    const ProbeSide &S = P.side[bside];
    uint32_t block;
    int l;
    locate(S, idx, block, l);
    // counted from the block's first symbol: past the front padding of a
    // short last block (at most 65535 for any block)
    const int L = S.sym_positions, npos = block_npos(S, block);
    l += ((npos + L - 1) / L) * L - npos;
    const uint32_t k = S.key0 + block;
    key[i] = k;
    lit[i] = (uint32_t)l;
    atomicMin(&minlit[k], (uint32_t)l);  // also marks the block touched
  }
}

// Exclusive scan of the touched flags (minlit[k] != kNoLit) of the blocks: tpos[k]
// is block k's place among the touched blocks, list[tpos[k]] = k for the
// touched ones.  Three passes over tiles of 4096 keys: tile totals, a scan
// of the totals, then each tile's scan plus its offset.
constexpr int kScanTile = 4096;

struct Pair32 {
  uint32_t a, b;
};

// Inclusive scan of (a, b) pairs over the 1024 threads of a block.
__device__ __forceinline__ Pair32 block_scan(Pair32 v, Pair32 *warp_tot) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t ya = __shfl_up_sync(0xffffffffu, v.a, d), yb = __shfl_up_sync(0xffffffffu, v.b, d);
    if (lane >= d) {
      v.a += ya;
      v.b += yb;
    }
  }
  if (lane == 31) warp_tot[wid] = v;
  __syncthreads();
  if (wid == 0) {
    Pair32 w = warp_tot[lane];
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t ya = __shfl_up_sync(0xffffffffu, w.a, d), yb = __shfl_up_sync(0xffffffffu, w.b, d);
      if (lane >= d) {
        w.a += ya;
        w.b += yb;
      }
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  if (wid > 0) {
    v.a += warp_tot[wid - 1].a;
    v.b += warp_tot[wid - 1].b;
  }
  return v;
}

__global__ void __launch_bounds__(1024) k_scan_tiles(const uint32_t *minlit, uint64_t nkeys,
                                                      uint32_t *tile_cnt, uint32_t *tile_flag) {
  __shared__ Pair32 wt[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + 4 * threadIdx.x;
  Pair32 v = {0, 0};
  for (int e = 0; e < 4; e++)
    if (base + e < nkeys) {
      const uint32_t c = minlit[base + e] != kNoLit;
      v.a += c;
      v.b += c;
    }
  v = block_scan(v, wt);
  if (threadIdx.x == 1023) {
    tile_cnt[blockIdx.x] = v.a;
    tile_flag[blockIdx.x] = v.b;
  }
}

// Exclusive scan of the tile totals in place (one block; any number of tiles).
__global__ void __launch_bounds__(1024) k_scan_totals(uint32_t *tile_cnt, uint32_t *tile_flag,
                                                       uint32_t ntiles) {
  __shared__ Pair32 wt[32];
  __shared__ Pair32 carry;
  if (threadIdx.x == 0) carry = {0, 0};
  __syncthreads();
  for (uint32_t t0 = 0; t0 < ntiles; t0 += 1024) {
    const uint32_t t = t0 + threadIdx.x;
    Pair32 v = {0, 0};
    if (t < ntiles) v = {tile_cnt[t], tile_flag[t]};
    const Pair32 own = v;
    v = block_scan(v, wt);
    const Pair32 c = carry;
    if (t < ntiles) {
      tile_cnt[t] = c.a + v.a - own.a;
      tile_flag[t] = c.b + v.b - own.b;
    }
    __syncthreads();
    if (threadIdx.x == 1023) carry = {c.a + v.a, c.b + v.b};
    __syncthreads();
  }
}

__global__ void __launch_bounds__(1024) k_scan_finish(const uint32_t *minlit, uint64_t nkeys,
                                                       const uint32_t *tile_flag, uint32_t *tpos,
                                                       uint32_t *list) {
  __shared__ Pair32 wt[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + 4 * threadIdx.x;
  uint32_t c[4];
  Pair32 v = {0, 0};
  for (int e = 0; e < 4; e++) {
    c[e] = base + e < nkeys ? (uint32_t)(minlit[base + e] != kNoLit) : 0u;
    v.a += c[e];
    v.b += c[e] != 0;
  }
  const Pair32 own = v;
  v = block_scan(v, wt);
  uint32_t rb = tile_flag[blockIdx.x] + v.b - own.b;
  for (int e = 0; e < 4; e++) {
    const uint64_t k = base + e;
    if (k >= nkeys) break;
    tpos[k] = rb;
    if (c[e]) list[rb++] = (uint32_t)k;
  }
}

__device__ __forceinline__ const ProbeSide &side_of_key(const ProbeTable &P, uint32_t k) {
  return (P.side[1].nblocks && k >= P.side[1].key0) ? P.side[1] : P.side[0];
}

// The decode table of one side packed for shared memory, one 64-bit word
// per bucket b of rans_dec_get (rans.h:111-136): freq of b's own symbol
// (bits 0-15), freq of its alias (16-31), the alias slot start (32-47), the
// divider (48-51) and the alias symbol (52-63).
__device__ __forceinline__ uint64_t pack_bucket(const ProbeSide &S, int b) {
  const RansEntry e = S.entry[b];
  const uint32_t a = e.alias_div >> 4;
  return (uint64_t)S.freq[b] | ((uint64_t)S.freq[a] << 16) | ((uint64_t)e.start << 32) |
         ((uint64_t)e.alias_div << 48);
}

// rans_dec_get on a packed bucket table.
__device__ __forceinline__ int dec_get_packed(uint64_t &x, const uint64_t *tab) {
  const uint64_t v = x;
  const int b = (int)((v >> 4) & 4095);
  uint32_t rem = (uint32_t)(v & 15);
  const uint64_t e = tab[b];
  uint32_t f;
  int sym;
  if (rem >= (uint32_t)((e >> 48) & 15)) {
    rem = (rem + (uint32_t)(e >> 32)) & 0xffff;  // wraps by design
    f = (uint32_t)(e >> 16) & 0xffff;
    sym = (int)(e >> 52);
  } else {
    f = (uint32_t)e & 0xffff;
    sym = b;
  }
  x = (uint64_t)f * (v >> 16) + rem;
  return sym;
}

// One thread per touched block of one side: decode from the block's end
// down to the lowest symbol asked for.  Symbol j of the wave's u-th block
// goes to scratch[j * W + u] (W blocks in the wave), so that the threads of
// a warp, which step through j together, store side by side.  TS is uint8_t
// when every symbol the code emits has an id below 256, else uint16_t.
//
// The steps are those of decompress_rans (probe.c:1362-1372): get, then
// renormalise while the read pointer is inside the block.  Two things are
// arranged differently: the words renormalisations read come through two
// 16-byte chunks held in registers, the next one loaded a chunk ahead (its
// latency hides behind the steps in between), and the pointer test runs
// once per run of steps that cannot reach the block's end (one step reads
// at most one word).
template <typename TS>
__global__ void __launch_bounds__(256) k_probe_decode(ProbeSide S, const uint32_t *list,
                                                      uint32_t t0, uint32_t t1,
                                                      const uint32_t *bounds, int bside,
                                                      uint32_t wbase, uint32_t W,
                                                      const uint32_t *minlit, TS *scratch) {
  __shared__ uint64_t tab[4096];
  if (bounds) {  // touched range of this side, from k_probe_bounds
    t0 = bside ? bounds[1] : 0u;
    t1 = bside ? bounds[0] : bounds[1];
    if (t0 >= t1) return;
  }
  for (int b = threadIdx.x; b < 4096; b += blockDim.x) tab[b] = pack_bucket(S, b);
  __syncthreads();
  for (uint32_t t = t0 + blockIdx.x * blockDim.x + threadIdx.x; t < t1;
       t += gridDim.x * blockDim.x) {
    const uint32_t k = list[t];
    const uint32_t block = k - S.key0;
    const int L = S.sym_positions;
    const int nsym = (block_npos(S, block) + L - 1) / L;
    const int lo = (int)minlit[k] / L;  // positions count from the first symbol
    const uint8_t *p = S.data + ((size_t)block << S.block_size);
    const uint8_t *end = p + ((size_t)1 << S.block_size);
    uint64_t x;
    dev_dec_start(S, block, x, p, end);
    // cur: the chunk of the next word (word ci of it); nxt: the chunk after
    const uint32_t *wp = reinterpret_cast<const uint32_t *>(p);
    const uint32_t *wend = reinterpret_cast<const uint32_t *>(end);
    const uint4 *cp = reinterpret_cast<const uint4 *>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(15));
    const uint4 *cend = reinterpret_cast<const uint4 *>(end);
    const uint4 zero = make_uint4(0, 0, 0, 0);
    uint4 cur = cp < cend ? cp[0] : zero;
    uint4 nxt = cp + 1 < cend ? cp[1] : zero;
    int ci = (int)((reinterpret_cast<uintptr_t>(p) >> 2) & 3);
    TS *out = scratch + (size_t)(nsym - 1) * W + (t - wbase);
    int j = nsym - 1;
    while (j >= lo) {
      const int nsafe = (int)(wend - wp);  // renormalisations left inside the block
      if (nsafe == 0) {
        for (; j >= lo; j--, out -= W) *out = (TS)dec_get_packed(x, tab);
        break;
      }
      int jstop = j - nsafe;
      if (jstop < lo - 1) jstop = lo - 1;
#pragma unroll 2
      for (; j > jstop; j--, out -= W) {
        *out = (TS)dec_get_packed(x, tab);
        if (x < kRansL) {
          const uint32_t w = ci == 0 ? cur.x : ci == 1 ? cur.y : ci == 2 ? cur.z : cur.w;
          x = (x << 32) | w;
          ++wp;
          if (++ci == 4) {
            ci = 0;
            cur = nxt;
            ++cp;
            nxt = cp + 1 < cend ? cp[1] : zero;
          }
        }
      }
    }
  }
}

// Device-side extent of a batch's touched blocks: bounds[0] = touched
// blocks, bounds[1] = touched blocks of side 0 (tpos at side 1's first key;
// key1 == nkeys for a one-sided table).
__global__ void k_probe_bounds(const uint32_t *minlit, const uint32_t *tpos, uint64_t nkeys,
                               uint64_t key1, uint32_t *bounds) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t total = tpos[nkeys - 1] + (minlit[nkeys - 1] != kNoLit ? 1u : 0u);
    bounds[0] = total;
    bounds[1] = key1 < nkeys ? tpos[key1] : total;
  }
}

// One thread per query: the queries whose block is in the wave (touched
// blocks w0 .. w0+W-1) read their symbol from the scratch and descend to
// their value; the others wait for their wave.
template <typename TS>
__global__ void k_probe_answer(ProbeTable P, const uint32_t *key, const uint32_t *lit,
                               const uint32_t *tpos, uint64_t n, uint32_t w0, uint32_t W,
                               const TS *scratch, int8_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = key[i];
    if (k == kNoKey) continue;
    const uint32_t u = tpos[k] - w0;
    if (u >= W) continue;
    const ProbeSide &S = side_of_key(P, k);
    const int L = S.sym_positions;
    const int l = (int)lit[i];
    const int sym = scratch[(size_t)(l / L) * W + u];
    out[i] = (int8_t)((int)descend(S, sym, l % L) - 2);
  }
}

// Reference path: every position decoded on its own (any table layout).
__global__ void k_probe_direct(ProbeTable P, const Query *q, int qbytes, uint64_t n,
                               int8_t *out) {
  __shared__ EncTables T;
  load_enc_tables(P.T, T);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int bside, stm;
    uint64_t idx, sqs;
    load_query(q, i, qbytes, sqs, stm);
    out[i] = query_index(P, T, sqs, stm, bside, idx) ? (int8_t)probe_one(P.side[bside], idx)
                                                     : kWdlInvalid;
  }
}

__global__ void k_encode_batch(ProbeTable P, const Query *q, uint64_t n, uint64_t *idx_out,
                               uint8_t *side_out) {
  __shared__ EncTables T;
  load_enc_tables(P.T, T);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int bside = 0, stm;
    uint64_t idx, sqs;
    load_query(q, i, 16, sqs, stm);
    const bool ok = query_index(P, T, sqs, stm, bside, idx);
    idx_out[i] = ok ? idx : ~0ull;
    if (side_out) side_out[i] = (uint8_t)bside;
  }
}

__global__ void k_decode_batch(ProbeTable P, int bside, const uint64_t *idx, uint64_t n,
                               uint8_t *sq_out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    // an index outside the side decodes to 0xff squares
    uint8_t p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (idx[i] < P.side[bside].ei.size)
      decode_piece(*P.T, P.side[bside].ei, idx[i], p);
    else
      for (int j = 0; j < 8; j++) p[j] = 0xff;
    for (int j = 0; j < 8; j++) sq_out[8 * i + j] = p[j];
  }
}

// ---------------------------------------------------- random legal positions
// Squares drawn from a splitmix64 stream keyed by (seed, query, attempt),
// distinct, with the side to move drawn too; a position is kept when the
// side not to move is not in check (kings apart included).
__global__ void k_gen_positions(int num, const uint8_t *pt_list, uint64_t seed, uint64_t n,
                                Query *out, uint32_t *failed) {
  uint8_t pt[8];
  for (int j = 0; j < 8; j++) pt[j] = j < num ? pt_list[j] : 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    Query q;
    bool okq = false;
    for (int a = 0; a < 64 && !okq; a++) {
      uint64_t h = tbl_mix64(seed * 0x9e3779b97f4a7c15ull + i * 64 + a + 1);
      uint64_t occ = 0;
      for (int j = 0; j < num; j++) {
        int sq;
        do {
          h = tbl_mix64(h + 0x9e3779b97f4a7c15ull);
          sq = (int)(h & 63);
        } while (occ >> sq & 1);
        occ |= 1ull << sq;
        q.sq[j] = (uint8_t)sq;
      }
      q.stm = (uint8_t)(tbl_mix64(h) & 1);
      // the side not to move (q.stm ^ 1) must not be attacked
      int them = q.stm ^ 1;
      int ksq = -1;
      for (int j = 0; j < num; j++)
        if (pt[j] == (uint8_t)((them << 3) | 6)) ksq = q.sq[j];
      bool attacked = false;
      for (int j = 0; j < num && !attacked; j++)
        if ((pt[j] >> 3) == q.stm)
          attacked = (piece_attacks(pt[j] & 7, q.sq[j], occ) >> ksq) & 1;
      okq = !attacked;
    }
    for (int j = num; j < 8; j++) q.sq[j] = 0;
    for (int j = 0; j < 7; j++) q.pad[j] = 0;
    if (!okq) atomicAdd(failed, 1u);
    out[i] = q;
  }
}

// ------------------------------------------------------------ table build
// Histogram of the quad symbols of one table side (value codes 0..M^4-1).
__global__ void k_tbl_hist(uint64_t size, uint64_t seed, int bside, int M,
                           unsigned long long *hist) {
  __shared__ unsigned int h[625];
  const int nq = M * M * M * M;
  for (int i = threadIdx.x; i < nq; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const uint64_t nquads = side_quads(size);
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nquads;
       q += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(&h[quad_values(seed, M, bside, size, q)], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < nq; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

// One thread per block: the block's quads encoded in order (the reader
// decodes them last to first), renormalisation words growing down from the
// block's end, the final state in front of them, zeros before that.
__global__ void k_tbl_encode(uint64_t size, uint64_t seed, int bside, int M,
                             const uint16_t *freq, const uint16_t *cum, const uint16_t *remap,
                             const uint16_t *quad_code, uint8_t *data, uint64_t nblocks,
                             uint32_t *overflow) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblocks;
       b += (uint64_t)gridDim.x * blockDim.x) {
    uint8_t *start = data + (b << kBlockBits);
    uint8_t *p = start + (1ull << kBlockBits);
    const uint8_t *lim = start + 8;
    uint64_t x = kRansL;
    const uint64_t q0 = b * kQuadsPerBlock, q1 = q0 + block_quads(size, b);
    for (uint64_t q = q0; q < q1; q++) {
      const int s = quad_code[quad_values(seed, M, bside, size, q)];
      if (!rans_put(x, freq, cum, remap, s, p, lim)) {
        atomicAdd(overflow, 1u);
        break;
      }
    }
    rans_flush(x, p, start);
  }
}

}  // namespace tbg
