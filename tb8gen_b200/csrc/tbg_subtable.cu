// Capture classification through 7-piece tables (calc_sub_worker,
// tb8gen.c:280-314, with probe_wdl answered by the table of the material left
// after the capture instead of the seeded stub).
//
// For captured set k of colour stm, every position of the capture space is
// the position after the capture with stm to move; its value comes from the
// table of that material (the original material minus one piece of set k),
// in one of two ways:
//   mode 0  the table itself: the positions become probe queries and one
//           grouped probe batch decodes the table's rANS blocks on the GPU;
//   mode 1  the table's defining formula, VALS[splitmix64(seed ^ idx ^
//           bside << 63) mod m], at the index the table encodes the position
//           to (encode_piece, probe.c:603-694) -- what the table stores.
// Both must give the same class bitmaps; illegal positions (the side not to
// move in check) go to cwin and win, as in the reference.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/tbgpu.h"
#include "tbg_device.cuh"
#include "tbg_host.h"
#include "tbg_table.h"

namespace tbg {

int cuda_fail(cudaError_t e, const char *what);
// from tbg_probe_api.cu
int sub_layout(const char *material, EncInfoP *ei, int *symmetric, uint8_t qpt[8],
               uint8_t tpt[8], int *num);
const EncTables *enc_tables_dev();

// Where each piece of the table's (or the query's) order comes from in the
// capture position: -1 white king, -2 black king, else the set index.
struct SubMap {
  EncInfoP ei;
  int symmetric, num;
  int8_t tsrc[2][8];   // table order, [flip]
  int8_t qsrc[8];      // query order (no flip: the probe flips itself)
};

struct SubQuery {      // the probe's query layout (tbgpu.h tbg_query)
  uint8_t sq[8];
  uint8_t stm;
  uint8_t pad[7];
};

template <int NS>
__device__ __forceinline__ int take_square(bb *rem, int src, int k0, int k1) {
  if (src == -1) return k0;
  if (src == -2) return k1;
  int sq = 0;
#pragma unroll
  for (int q = 0; q < NS; q++)
    if (q == src) {
      sq = __ffsll((long long)rem[q]) - 1;
      rem[q] &= rem[q] - 1;
    }
  return sq;
}

// The table's value (wdl, -2..2) of the capture position by its formula.
template <int NS>
__device__ __forceinline__ int formula_wdl(const SubMap &S, const EncTables &T, const bb *set,
                                           int k0, int k1, int stm, uint64_t seed, int modulus) {
  if (S.num == 2) return 0;  // bare kings (probe.c:1525)
  const int flip = S.symmetric ? (stm != 0) : 0;
  const int bside = S.symmetric ? 0 : (stm == 1);
  bb rem[NS];
#pragma unroll
  for (int q = 0; q < NS; q++) rem[q] = set[q];
  uint8_t p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < S.num; i++) {
    const int sq = take_square<NS>(rem, S.tsrc[flip][i], k0, k1);
    p[i] = (uint8_t)(sq ^ (flip ? 0x38 : 0));
  }
  const uint64_t idx = encode_piece(T, S.ei, p);
  return table_value(seed, modulus, idx, bside) - 2;
}

__device__ __forceinline__ void sub_store(uint32_t *p, uint64_t w, uint64_t nbits, uint32_t v) {
  const uint64_t base = w * 32;
  if (base + 32 <= nbits) {
    p[w] = v;
    return;
  }
  const uint64_t nbytes = (nbits - base + 7) >> 3;  // bytes holding positions
  const uint32_t keep = nbytes >= 4 ? 0u : ~0u << (8 * nbytes);
  p[w] = (p[w] & keep) | (v & ~keep);
}

__device__ __forceinline__ void classify(uint32_t *o, int v, uint32_t m) {
  o[v + 2] |= m;
  if (v == 2) o[3] |= m;
}

// mode 1: classes from the formula, one thread per 32 positions.
template <int NS>
__global__ void __launch_bounds__(256) k_sub_formula(DMat M, SubMap S, const EncTables *T, int set,
                                                     int k0, int k1, int stm, uint64_t seed,
                                                     int modulus, uint32_t *c0, uint32_t *c1,
                                                     uint32_t *c2, uint32_t *c3, uint32_t *c4) {
  __shared__ uint32_t bin[7 * 64];
  load_binomials(bin);
  __syncthreads();
  const DIdx &X = M.capt[set];
  const uint64_t n = X.size, nwords = (n + 31) >> 5;
  const int opp = stm ? k0 : k1;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t o[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < 32; b++) {
      const uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      bb sets[NS];
      const bb occ = unrank_sets<NS>(X, bin, idx, k0, k1, sets);
      const uint32_t m = 1u << b;
      if (attacked_by<NS>(M, sets, k0, k1, occ, opp, stm)) {
        o[3] |= m;
        o[4] |= m;
      } else {
        classify(o, formula_wdl<NS>(S, *T, sets, k0, k1, stm, seed, modulus), m);
      }
    }
    sub_store(c0, w, n, o[0]);
    sub_store(c1, w, n, o[1]);
    sub_store(c2, w, n, o[2]);
    sub_store(c3, w, n, o[3]);
    sub_store(c4, w, n, o[4]);
  }
}

// mode 0, step 1: the capture positions as probe queries; an illegal one
// gets side to move 2, which the probe answers with -128.
template <int NS>
__global__ void __launch_bounds__(256) k_sub_queries(DMat M, SubMap S, int set, int k0, int k1,
                                                     int stm, SubQuery *q) {
  __shared__ uint32_t bin[7 * 64];
  load_binomials(bin);
  __syncthreads();
  const DIdx &X = M.capt[set];
  const int opp = stm ? k0 : k1;
  for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < X.size;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    bb sets[NS];
    const bb occ = unrank_sets<NS>(X, bin, idx, k0, k1, sets);
    SubQuery r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.sq[j] = 0;
#pragma unroll
    for (int j = 0; j < 7; j++) r.pad[j] = 0;
    r.stm = attacked_by<NS>(M, sets, k0, k1, occ, opp, stm) ? 2 : (uint8_t)stm;
    bb rem[NS];
#pragma unroll
    for (int q2 = 0; q2 < NS; q2++) rem[q2] = sets[q2];
    for (int j = 0; j < S.num; j++) r.sq[j] = (uint8_t)take_square<NS>(rem, S.qsrc[j], k0, k1);
    q[idx] = r;
  }
}

// mode 0, step 2: classes from the probed values.
__global__ void __launch_bounds__(256) k_sub_classify(const int8_t *wdl, uint64_t n, uint32_t *c0,
                                                      uint32_t *c1, uint32_t *c2, uint32_t *c3,
                                                      uint32_t *c4) {
  const uint64_t nwords = (n + 31) >> 5;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t o[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < 32; b++) {
      const uint64_t idx = w * 32 + b;
      if (idx >= n) break;
      const int v = wdl[idx];
      const uint32_t m = 1u << b;
      if (v < -2 || v > 2) {  // -128: illegal (the side not to move in check)
        o[3] |= m;
        o[4] |= m;
      } else {
        classify(o, v, m);
      }
    }
    sub_store(c0, w, n, o[0]);
    sub_store(c1, w, n, o[1]);
    sub_store(c2, w, n, o[2]);
    sub_store(c3, w, n, o[3]);
    sub_store(c4, w, n, o[4]);
  }
}

// The material left when one piece of set k is captured, and the source map.
static int make_submap(const Material &m, int k, SubMap &S, std::string &name) {
  static const char *letters = "PNBRQK";
  const int t = m.d.set_type[k] | (m.d.set_color[k] << 3);
  std::string w = "K", b = "K";
  bool dropped = false;
  for (int i = 2; i < m.num; i++) {
    if (m.pt[i] == t && !dropped) {
      dropped = true;
      continue;
    }
    (m.pt[i] & 8 ? b : w) += letters[(m.pt[i] & 7) - 1];
  }
  name = w + "v" + b;
  uint8_t qpt[8], tpt[8];
  memset(&S, 0, sizeof S);
  if (m.num == 3) {  // the kings alone: a draw, no table (probe.c:1525)
    S.num = 2;
    return TBG_OK;
  }
  int rc = sub_layout(name.c_str(), &S.ei, &S.symmetric, qpt, tpt, &S.num);
  if (rc) return rc;
  auto src_of = [&](int code) -> int {
    if (code == 6) return -1;
    if (code == 14) return -2;
    for (int q = 0; q < m.d.ii.numsets; q++)
      if ((m.d.set_type[q] | (m.d.set_color[q] << 3)) == code) return q;
    return -3;
  };
  for (int i = 0; i < S.num; i++) {
    S.tsrc[0][i] = (int8_t)src_of(tpt[i]);
    S.tsrc[1][i] = (int8_t)src_of(tpt[i] ^ 8);  // colours swapped
    S.qsrc[i] = (int8_t)src_of(qpt[i]);
    if (S.tsrc[0][i] < -2 || S.qsrc[i] < -2 || (S.symmetric && S.tsrc[1][i] < -2))
      return fail(TBG_ERR_ARG, "capture material %s does not match", name.c_str());
  }
  return TBG_OK;
}

static SubQuery *g_q = nullptr;
static int8_t *g_wdl = nullptr;
static uint64_t g_cap = 0;

#define SUB_NS_SWITCH(ns, ...)                                           \
  switch (ns) {                                                          \
    case 1: { constexpr int NS = 1; __VA_ARGS__; } break;                \
    case 2: { constexpr int NS = 2; __VA_ARGS__; } break;                \
    case 3: { constexpr int NS = 3; __VA_ARGS__; } break;                \
    case 4: { constexpr int NS = 4; __VA_ARGS__; } break;                \
    case 5: { constexpr int NS = 5; __VA_ARGS__; } break;                \
    case 6: { constexpr int NS = 6; __VA_ARGS__; } break;                \
    default: return fail(TBG_ERR_RANGE, "%d piece sets", (int)(ns));    \
  }

}  // namespace tbg

using namespace tbg;

extern "C" int tbg_calc_sub_table(int stm, int s, void *const dev_cls[5], const int handles[6],
                                  int mode, uint64_t seed, int modulus) {
  if (!g_tab.ready || !g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  if (g_eng.cur < 0) return fail(TBG_ERR_STATE, "no material selected");
  if ((stm & ~1) || s < 0 || s >= TBG_NSLICES || !dev_cls || (mode != 0 && mode != 1))
    return fail(TBG_ERR_ARG, "bad args");
  if (mode == 0 && !handles) return fail(TBG_ERR_ARG, "mode 0 needs the table handles");
  if (mode == 1 && modulus != 3 && modulus != 5) return fail(TBG_ERR_ARG, "modulus 3 or 5");
  for (int i = 0; i < 5; i++)
    if (!dev_cls[i] || (reinterpret_cast<uintptr_t>(dev_cls[i]) & 15))
      return fail(TBG_ERR_ARG, "class buffer %d", i);
  const Material &m = g_eng.mats[g_eng.cur];
  const int k0 = g_tab.kksq[s][0], k1 = g_tab.kksq[s][1];
  const cudaStream_t st = g_eng.stream;
  const EncTables *T = enc_tables_dev();
  if (!T) return fail(TBG_ERR_STATE, "encoding tables not on the device");
  for (int k = 0; k < m.d.ii.numsets; k++) {
    if (m.d.set_color[k] != stm) continue;
    SubMap S;
    std::string name;
    int rc = make_submap(m, k, S, name);
    if (rc) return rc;
    const uint64_t off = m.d.sub_offset[k];
    const uint64_t n = m.d.capt[k].size;
    uint32_t *c[5];
    for (int i = 0; i < 5; i++)
      c[i] = reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(dev_cls[i]) + off);
    const uint64_t nwords = (n + 31) / 32;
    const int gw = g_eng.grid_for((nwords + 255) / 256, 16);
    if (mode == 1 || S.num == 2) {
      SUB_NS_SWITCH(m.d.ii.numsets,
                    k_sub_formula<NS><<<gw, 256, 0, st>>>(m.d, S, T, k, k0, k1, stm, seed, modulus,
                                                          c[0], c[1], c[2], c[3], c[4]));
      rc = g_eng.check_launch("k_sub_formula");
      if (rc) return rc;
      continue;
    }
    if (n > g_cap) {
      cudaStreamSynchronize(st);
      if (g_q) cudaFree(g_q);
      if (g_wdl) cudaFree(g_wdl);
      g_q = nullptr;
      g_wdl = nullptr;
      g_cap = 0;
      cudaError_t e = cudaMalloc(&g_q, n * sizeof(SubQuery));
      if (e == cudaSuccess) e = cudaMalloc(&g_wdl, n);
      if (e != cudaSuccess) return fail(TBG_ERR_NOMEM, "capture queries: %s", cudaGetErrorString(e));
      g_cap = n;
    }
    const int gq = g_eng.grid_for((n + 255) / 256, 16);
    SUB_NS_SWITCH(m.d.ii.numsets,
                  k_sub_queries<NS><<<gq, 256, 0, st>>>(m.d, S, k, k0, k1, stm, g_q));
    rc = g_eng.check_launch("k_sub_queries");
    if (rc) return rc;
    if (handles[k] < 0) return fail(TBG_ERR_ARG, "no table for the capture of set %d (%s)", k,
                                    name.c_str());
    rc = tbg_probe_wdl_batch(handles[k], g_q, n, g_wdl, 0);
    if (rc) return rc;
    k_sub_classify<<<gw, 256, 0, st>>>(g_wdl, n, c[0], c[1], c[2], c[3], c[4]);
    rc = g_eng.check_launch("k_sub_classify");
    if (rc) return rc;
  }
  return TBG_OK;
}

extern "C" int tbg_capture_material(int set, char *name, int len) {
  if (!g_tab.ready || g_eng.cur < 0) return fail(TBG_ERR_STATE, "no material selected");
  const Material &m = g_eng.mats[g_eng.cur];
  if (set < 0 || set >= m.d.ii.numsets || !name || len < 2) return fail(TBG_ERR_ARG, "bad args");
  SubMap S;
  std::string s;
  int rc = make_submap(m, set, S, s);
  if (rc) return rc;
  if ((int)s.size() + 1 > len) return fail(TBG_ERR_RANGE, "name buffer too small");
  memcpy(name, s.c_str(), s.size() + 1);
  return TBG_OK;
}
