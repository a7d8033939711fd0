// WDL probes into rANS-compressed 7-piece tables (probe_table, decompress_rans,
// probe.c:1346-1390, 1522-1597) and the builder of the synthetic table.
//
// A probe batch runs in four passes instead of one independent decode per
// position: (1) every position is encoded (encode_piece) and located in its
// block through the index and size tables; (2) positions are grouped by block
// (counting sort); (3) every block some position falls in is decoded once, by
// one thread, from its end down to the lowest position asked for, into a
// scratch array of symbols; (4) each position reads its symbol and descends
// the Re-Pair tree to its value.  A 64 KiB block holds up to 65,536 positions,
// so per-position decoding would cost up to 16,384 rANS steps per probe;
// grouped, the cost is one decode per touched block.
#pragma once

#include "tbg_device.cuh"
#include "tbg_table.h"

namespace tbg {

struct ProbeSide {
  EncInfoP ei;
  const uint8_t *index;     // 6 B per 2^idx_bits positions
  const uint8_t *sizes;     // u16 per block: positions in the block - 1
  const uint8_t *data;      // blocks of 2^block_size bytes
  const RansEntry *entry;   // decode table (device copy)
  const uint16_t *freq;
  const uint8_t *sympat;    // 3 B per symbol (inside the table)
  const uint8_t *symlen;    // per symbol (device copy)
  uint64_t nblocks;
  uint32_t key0;            // first block key of this side
  int idx_bits, block_size;
  int sym_positions;        // positions per top-level symbol if all equal, else 0
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

// list_squares (probe.c:1511-1520) then encode_piece: table index and side.
// Returns false for a query that is not a placement (see kWdlInvalid).
__device__ __forceinline__ bool query_index(const ProbeTable &P, const Query &q, int &bside,
                                            uint64_t &idx) {
  uint64_t occ = 0;
  int wk = 0, bk = 0;
  for (int j = 0; j < P.num; j++) {
    const int sq = q.sq[j];
    if (sq >= 64 || ((occ >> sq) & 1)) return false;
    occ |= 1ull << sq;
    if (P.pt[j] == 6) wk = sq;
    if (P.pt[j] == 14) bk = sq;
  }
  if (q.stm > 1) return false;
  int flip;
  if (!P.symmetric) {
    flip = 0;
    bside = q.stm == 1;
  } else {
    flip = q.stm != 0;
    bside = 0;
  }
  const ProbeSide &S = P.side[bside];
  if (S.ei.kk) {
    const int df = (wk & 7) - (bk & 7), dr = (wk >> 3) - (bk >> 3);
    if (df >= -1 && df <= 1 && dr >= -1 && dr <= 1) return false;
  }
  uint8_t p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < P.num;) {
    int t = S.ei.pieces[i] ^ (flip << 3);
    for (int j = 0; j < P.num; j++)
      if (P.pt[j] == t) p[i++] = q.sq[j] ^ (flip ? 0x38 : 0x00);
  }
  idx = encode_piece(*P.T, S.ei, p);
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
  rans_dec_init(x, p, end);
  int sym = 0;
  for (; lit < 0 && p < end; lit += S.symlen[sym] + 1) {
    sym = rans_dec_get(x, S.entry, S.freq);
    rans_dec_renorm(x, p);
  }
  for (; lit < 0; lit += S.symlen[sym] + 1) sym = rans_dec_get(x, S.entry, S.freq);
  return (int)descend(S, sym, lit) - 2;
}

// ------------------------------------------------------------ probe passes
constexpr uint32_t kNoKey = 0xffffffffu;

__global__ void k_probe_locate(ProbeTable P, const Query *q, uint64_t n, uint32_t *key,
                               uint32_t *lit, uint32_t *count, uint32_t *minlit, int8_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int bside;
    uint64_t idx;
    if (!query_index(P, q[i], bside, idx)) {
      key[i] = kNoKey;
      out[i] = kWdlInvalid;
      continue;
    }
    const ProbeSide &S = P.side[bside];
    uint32_t block;
    int l;
    locate(S, idx, block, l);
    uint32_t k = S.key0 + block;
    key[i] = k;
    lit[i] = (uint32_t)l;
    atomicAdd(&count[k], 1u);
    atomicMin(&minlit[k], (uint32_t)l);
  }
}

// Exclusive scan of n counts in one block of 1024 threads (n is at most a
// few million: the number of blocks of the tables).
// With kFlag the values scanned are (in[i] != 0).
template <bool kFlag>
__global__ void __launch_bounds__(1024) k_scan_exclusive(const uint32_t *in, uint32_t *out,
                                                         uint64_t n) {
  __shared__ uint32_t part[1024];
  const uint64_t per = (n + 1023) / 1024;
  const uint64_t b0 = threadIdx.x * per, b1 = b0 + per < n ? b0 + per : n;
  uint32_t s = 0;
  for (uint64_t i = b0; i < b1; i++) s += kFlag ? (in[i] != 0) : in[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    uint32_t v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - s;
  for (uint64_t i = b0; i < b1; i++) {
    uint32_t v = kFlag ? (in[i] != 0) : in[i];
    out[i] = run;
    run += v;
  }
}

__global__ void k_probe_scatter(const uint32_t *key, uint64_t n, uint32_t *cursor,
                                uint32_t *order) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (key[i] != kNoKey) order[atomicAdd(&cursor[key[i]], 1u)] = (uint32_t)i;
}

// Touched blocks, in key order: list[tpos[k]] = k for every k with
// count > 0, and tq[tpos[k]] = offs[k], the first of k's queries in order[].
__global__ void k_probe_touched(const uint32_t *count, const uint32_t *tpos, const uint32_t *offs,
                                uint64_t nkeys, uint32_t *list, uint32_t *tq) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nkeys;
       k += (uint64_t)gridDim.x * blockDim.x)
    if (count[k]) {
      list[tpos[k]] = (uint32_t)k;
      tq[tpos[k]] = offs[k];
    }
}

__device__ __forceinline__ const ProbeSide &side_of_key(const ProbeTable &P, uint32_t k) {
  return (P.side[1].nblocks && k >= P.side[1].key0) ? P.side[1] : P.side[0];
}

// One thread per touched block of the wave: decode from the block's end
// down to the lowest symbol asked for, writing symbol ids in block order.
__global__ void k_probe_decode(ProbeTable P, const uint32_t *list, uint32_t w0, uint32_t w1,
                               const uint32_t *minlit, uint16_t *scratch, uint32_t stride) {
  for (uint32_t t = w0 + blockIdx.x * blockDim.x + threadIdx.x; t < w1;
       t += gridDim.x * blockDim.x) {
    const uint32_t k = list[t];
    const ProbeSide &S = side_of_key(P, k);
    const uint32_t block = k - S.key0;
    const int L = S.sym_positions;
    const int npos = block_npos(S, block);
    const int nsym = (npos + L - 1) / L;
    const int pad = nsym * L - npos;  // front padding of a short last block
    const int lo = ((int)minlit[k] + pad) / L;
    const uint8_t *p = S.data + ((size_t)block << S.block_size);
    const uint8_t *end = p + ((size_t)1 << S.block_size);
    uint64_t x;
    rans_dec_init(x, p, end);
    uint16_t *out = scratch + (size_t)(t - w0) * stride;
    for (int j = nsym - 1; j >= lo; j--) {
      out[j] = (uint16_t)rans_dec_get(x, S.entry, S.freq);
      if (p < end) rans_dec_renorm(x, p);
    }
  }
}

// One thread per query of the wave's blocks: queries order[tq[w0] ..
// tq[w1]) (the last wave ends at nvalid, the number of valid queries).
__global__ void k_probe_answer(ProbeTable P, const uint32_t *order, const uint32_t *tq,
                               uint32_t w0, uint32_t w1, uint32_t ntouched, uint32_t nvalid,
                               const uint32_t *key, const uint32_t *lit, const uint32_t *tpos,
                               const uint16_t *scratch, uint32_t stride, int8_t *out) {
  const uint32_t q0 = tq[w0], q1 = w1 < ntouched ? tq[w1] : nvalid;
  for (uint32_t t = q0 + blockIdx.x * blockDim.x + threadIdx.x; t < q1;
       t += gridDim.x * blockDim.x) {
    const uint32_t i = order[t];
    const uint32_t k = key[i];
    const ProbeSide &S = side_of_key(P, k);
    const int L = S.sym_positions;
    const int npos = block_npos(S, k - S.key0);
    const int l = (int)lit[i] + ((npos + L - 1) / L) * L - npos;
    const int sym = scratch[(size_t)(tpos[k] - w0) * stride + l / L];
    out[i] = (int8_t)((int)descend(S, sym, l % L) - 2);
  }
}

// Reference path: every position decoded on its own (any table layout).
__global__ void k_probe_direct(ProbeTable P, const Query *q, uint64_t n, int8_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int bside;
    uint64_t idx;
    out[i] = query_index(P, q[i], bside, idx) ? (int8_t)probe_one(P.side[bside], idx)
                                              : kWdlInvalid;
  }
}

__global__ void k_encode_batch(ProbeTable P, const Query *q, uint64_t n, uint64_t *idx_out,
                               uint8_t *side_out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int bside = 0;
    uint64_t idx;
    const bool ok = query_index(P, q[i], bside, idx);
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
