// C ABI of the ply-step engine (include/tbgpu.h) and its host-side state:
// king-slice tables, registered materials, the slot map and the launches.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "../../include/tbgpu.h"
#include "tbg_host.h"
#include "tbg_kernels.cuh"
#include "tbg_persist.h"

namespace tbg {

HostTables g_tab;
Engine g_eng;

static char g_errbuf[512];

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_errbuf, sizeof g_errbuf, fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(TBG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

// Kernels are compiled for each number of piece sets (1..6); NS_SWITCH picks
// the instance of the current material.
#define NS_CASE(n, ...) \
  case n: {             \
    constexpr int NS = n; \
    __VA_ARGS__;        \
  } break;
#define NS_SWITCH(ns, ...)                                                   \
  switch (ns) {                                                              \
    NS_CASE(1, __VA_ARGS__)                                                  \
    NS_CASE(2, __VA_ARGS__)                                                  \
    NS_CASE(3, __VA_ARGS__)                                                  \
    NS_CASE(4, __VA_ARGS__)                                                  \
    NS_CASE(5, __VA_ARGS__)                                                  \
    NS_CASE(6, __VA_ARGS__)                                                  \
    default: return fail(TBG_ERR_RANGE, "%d piece sets", (int)(ns));         \
  }

// ------------------------------------------------------------ host tables
// The king-pair tables of probe.c:441-539 and tb8gen.c:69-89, generated from
// their defining rules.
static const int kTriSq[10] = {1, 2, 3, 10, 11, 19, 0, 9, 18, 27};

static bool touching(int a, int b) {
  int df = (a & 7) - (b & 7), dr = (a >> 3) - (b >> 3);
  return df >= -1 && df <= 1 && dr >= -1 && dr <= 1;
}

void HostTables::build() {
  if (ready) return;
  for (int sq = 0; sq < 64; sq++) {
    uint64_t k = 0;
    for (int df = -1; df <= 1; df++)
      for (int dr = -1; dr <= 1; dr++) {
        int f = (sq & 7) + df, r = (sq >> 3) + dr;
        if ((df || dr) && f >= 0 && f < 8 && r >= 0 && r < 8) k |= 1ull << (r * 8 + f);
      }
    king[sq] = k;
    flipdiag[sq] = ((sq & 7) << 3) | (sq >> 3);
    mirror[sq] = ((sq & 7) >= 4 ? 0x07 : 0) | ((sq >> 3) >= 4 ? 0x38 : 0);
    int f = sq & 7, r = sq >> 3;
    if (f > 3) f = 7 - f;
    if (r > 3) r = 7 - r;
    if (r > f) std::swap(r, f);
    for (int t = 0; t < 10; t++)
      if (kTriSq[t] == r * 8 + f) triangle[sq] = t;
  }
  int next = 0, next_diag = 441;
  for (int t = 0; t < 10; t++)
    for (int sq = 0; sq < 64; sq++) {
      int wk = kTriSq[t];
      kkidx[t][sq] = -1;
      if (touching(wk, sq)) continue;
      if (t >= 6) {
        if ((sq & 7) < (sq >> 3)) continue;
        if ((sq & 7) == (sq >> 3)) {
          kkidx[t][sq] = next_diag++;
          continue;
        }
      }
      kkidx[t][sq] = next++;
    }
  for (int t = 0; t < 10; t++)
    for (int sq = 0; sq < 64; sq++)
      if (kkidx[t][sq] >= 0) {
        kksq[kkidx[t][sq]][0] = kTriSq[t];
        kksq[kkidx[t][sq]][1] = sq;
      }
  for (int i = 0; i < 64; i++)
    for (int j = 0; j < 64; j++) {
      int s1 = i ^ mirror[i], s2 = j ^ mirror[i];
      bool tri = (s1 & 7) <= 3 && (s1 >> 3) <= (s1 & 7);
      bool diag = tri && (s1 & 7) == (s1 >> 3);
      bool lower = (s2 & 7) >= (s2 >> 3);
      fliptest[i][j] = !tri || (diag && !lower);
      if (fliptest[i][j]) {
        s1 = flipdiag[s1];
        s2 = flipdiag[s2];
      }
      kkmap[i][j] = kkidx[triangle[s1]][s2];
    }
  ready = next == 441 && next_diag == 462;
}

// ---------------------------------------------------------------- materials
static uint64_t placements(uint64_t k, uint64_t n) {
  uint64_t f = 1;
  for (uint64_t i = 0; i < k; i++) f = f * (n - i) / (i + 1);
  return f;
}

static uint64_t rounded_bytes(uint64_t bits) { return (((bits + 7) >> 3) + 63) & ~63ull; }

static uint64_t div_magic(uint64_t d) {
  if (d <= 1) return 0;
  unsigned __int128 one = (unsigned __int128)1 << 64;
  return (uint64_t)(one / d + (one % d != 0));
}

// calc_factors (tb8gen.c:209-228) into device form.
static void fill_idx(DIdx &x, int numsets, const int *mult) {
  memset(&x, 0, sizeof x);
  x.numsets = numsets;
  uint64_t sub[TBG_MAX_SETS];
  for (int i = 0, n = 62; i < numsets; i++) {
    x.mult[i] = mult[i];
    sub[i] = placements(mult[i], n);
    n -= mult[i];
  }
  uint64_t f = 1;
  for (int i = numsets - 1; i >= 0; i--) {
    x.factor[i] = f;
    x.fdiv[i] = div_magic(f);
    f *= sub[i];
  }
  x.size = f;
}

int Engine::add_material(const int *pt, int num) {
  if (!g_tab.ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  // A material registered again gets its existing handle (slot map kept).
  for (int h = 0; h < nmats; h++) {
    bool same = mats[h].num == num;
    for (int i = 0; same && i < num; i++) same = mats[h].pt[i] == pt[i];
    if (same) {
      cur = h;
      return h;
    }
  }
  if (nmats >= TBG_MAX_MATS) return fail(TBG_ERR_RANGE, "at most %d materials", TBG_MAX_MATS);
  Material &m = mats[nmats];
  memset(&m.d, 0, sizeof m.d);
  for (int i = 0; i < 463; i++) {
    m.slot[i] = nullptr;
    m.slot_bytes[i] = 0;
    m.sub[i] = nullptr;
    m.sub_len[i] = 0;
  }
  DMat &d = m.d;
  d.num = num;
  d.king_type[0] = 6;
  d.king_type[1] = 14;
  int mult[TBG_MAX_SETS] = {0}, nsets = 0;
  for (int i = 2; i < num;) {
    int j = i;
    while (i < num && pt[i] == pt[j]) i++;
    if (nsets >= TBG_MAX_SETS) return fail(TBG_ERR_RANGE, "too many piece sets");
    d.set_type[nsets] = pt[j] & 7;
    d.set_color[nsets] = pt[j] >> 3;
    d.set_first[nsets] = j;
    mult[nsets] = i - j;
    nsets++;
  }
  fill_idx(d.ii, nsets, mult);
  d.bytes = rounded_bytes(d.ii.size);
  uint64_t sub_size[2] = {0, 0};
  for (int k = 0; k < nsets; k++) {
    int cm[TBG_MAX_SETS];
    memcpy(cm, mult, sizeof cm);
    cm[k]--;
    fill_idx(d.capt[k], nsets, cm);
    d.sub_offset[k] = sub_size[d.set_color[k]];
    sub_size[d.set_color[k]] += rounded_bytes(d.capt[k].size);
  }
  d.sub_size[0] = sub_size[0];
  d.sub_size[1] = sub_size[1];
  d.sub_bytes = std::max(sub_size[0], sub_size[1]);
  for (int i = 0; i < num; i++) m.pt[i] = pt[i];
  m.num = num;
  cudaError_t e = cudaMemcpyToSymbol(c_mats, &d, sizeof d, nmats * sizeof(DMat));
  if (e == cudaSuccess) e = persist_block_set_mat(d, nmats);
  if (e == cudaSuccess) e = persist_warp_set_mat(d, nmats);
  if (e != cudaSuccess) return cuda_fail(e, "upload material");
  // a legacy-stream upload: complete before a non-blocking stream reads it
  CK(cudaStreamSynchronize(0));
  cur = nmats;
  return nmats++;
}

// Piece order of main(): kings first, then N < B < R < Q, white before black
// within a type (piece_order, tb8gen.c:1331-1339).
static const int kOrder[16] = {0, 0, 3, 5, 7, 9, 1, 0, 0, 0, 4, 6, 8, 10, 2, 0};

// -------------------------------------------------------------- launches
bool Engine::alloc_refused() {
  alloc_calls++;
  return fail_alloc_at > 0 && alloc_calls == fail_alloc_at;
}

int Engine::ensure_device() {
  if (dev_ready) return TBG_OK;
  if (const char *v = getenv("TBG_FAIL_ALLOC_AT")) fail_alloc_at = strtol(v, nullptr, 10);
  CK(cudaGetDevice(&device));
  CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  CK(cudaMalloc(&d_status, sizeof(DevStatus)));
  CK(cudaMemset(d_status, 0, sizeof(DevStatus)));
  CK(cudaMalloc(&d_cnt, 64 * sizeof(unsigned long long)));
  CK(cudaMallocHost(&h_cnt, 64 * sizeof(unsigned long long)));
  uint64_t seed = 1;
  int mod = 3;
  CK(cudaMemcpyToSymbol(c_stub_seed, &seed, sizeof seed));
  CK(cudaMemcpyToSymbol(c_stub_mod, &mod, sizeof mod));
  CK(persist_block_set_stub(seed, mod, nullptr));
  CK(persist_warp_set_stub(seed, mod, nullptr));
  // legacy-stream set-up, complete before any stream of the caller's
  // (blocking or not) launches
  CK(cudaDeviceSynchronize());
  dev_ready = true;
  return TBG_OK;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// Fills the king destinations of (stm, s): every square the king of stm can
// step to (king_attacks(me) & ~king_attacks(opp)), with its target slice,
// the normalisation of the new king pair and the bound buffers there.
int Engine::fill_job(SliceJob &J, int stm, int s, bool need_sub) {
  Material &m = mats[cur];
  J.mat = cur;
  J.stm = stm;
  J.s = s;
  J.set = -1;
  J.k0 = g_tab.kksq[s][0];
  J.k1 = g_tab.kksq[s][1];
  J.legality = 0;
  J.self = reinterpret_cast<uint32_t *>(m.slot[s + 1]);
  J.self_sub = m.sub[s + 1];
  J.self_sub_len = m.sub_len[s + 1];
  int me = stm ? J.k1 : J.k0, opp = stm ? J.k0 : J.k1;
  uint64_t dests = g_tab.king[me] & ~g_tab.king[opp] & ~(1ull << opp);
  J.nk = 0;
  for (int to = 0; to < 64; to++) {
    if (!(dests >> to & 1)) continue;
    KingDest &D = J.kd[J.nk++];
    int w = stm ? J.k0 : to, b = stm ? to : J.k1;
    D.to = to;
    D.mirror = g_tab.mirror[w];
    D.flip = g_tab.fliptest[w][b];
    int nw = w ^ D.mirror, nb = b ^ D.mirror;
    if (D.flip) {
      nw = g_tab.flipdiag[nw];
      nb = g_tab.flipdiag[nb];
    }
    D.k0 = nw;
    D.k1 = nb;
    D.s2 = g_tab.kkmap[w][b];
    if (D.s2 < 0) return fail(TBG_ERR_ARG, "king move to an illegal pair");
    D.dbl = s < 441 && D.s2 >= 441;
    D.pad = 0;
    D.bits = reinterpret_cast<uint32_t *>(m.slot[D.s2 + 1]);
    D.sub = m.sub[D.s2 + 1];
    D.sub_len = m.sub_len[D.s2 + 1];
    if (!D.bits) return fail(TBG_ERR_UNBOUND, "slice %d (king move of slice %d) not bound", D.s2, s);
    if (need_sub && !D.sub) return fail(TBG_ERR_UNBOUND, "sub of slice %d not bound", D.s2);
  }
  if (!J.self) return fail(TBG_ERR_UNBOUND, "slice %d not bound", s);
  if (need_sub && !J.self_sub) return fail(TBG_ERR_UNBOUND, "sub of slice %d not bound", s);
  return TBG_OK;
}

int Engine::grid_for(uint64_t units, int per_sm) {
  uint64_t cap = (uint64_t)num_sms * per_sm;
  uint64_t g = units < cap ? units : cap;
  return g < 1 ? 1 : (int)g;
}

int Engine::check_launch(const char *what) {
  launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  return TBG_OK;
}

int Engine::wait(int timeout_ms) {
  auto t0 = std::chrono::steady_clock::now();
  long limit = timeout_ms > 0 ? timeout_ms : 600000;
  for (;;) {
    cudaError_t e = cudaStreamQuery(stream);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_fail(e, "stream");
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                  std::chrono::steady_clock::now() - t0).count();
    if (ms > limit) return fail(TBG_ERR_TIMEOUT, "stream did not finish within %ld ms", limit);
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  DevStatus st;
  CK(cudaMemcpy(&st, d_status, sizeof st, cudaMemcpyDeviceToHost));
  if (st.err) {
    CK(cudaMemsetAsync(d_status, 0, sizeof st, stream));
    return fail(TBG_ERR_DEVICE, "kernel status %u at site %u (byte %llu)", st.err, st.where,
                (unsigned long long)st.info);
  }
  return TBG_OK;
}

int Engine::tickets_ready() {
  if (!tick_ev.empty()) return TBG_OK;
  CK(cudaStreamCreateWithFlags(&s_in, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&s_out, cudaStreamNonBlocking));
  std::vector<cudaEvent_t> ev(kTickets);
  for (auto &e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  tick_ev.swap(ev);
  return TBG_OK;
}

int Engine::ticket_event(uint64_t t, cudaEvent_t *e) {
  if (t == 0 || t >= next_ticket || t + kTickets < next_ticket)
    return fail(TBG_ERR_ARG, "ticket %llu is not live (next %llu)", (unsigned long long)t,
                (unsigned long long)next_ticket);
  *e = tick_ev[t % kTickets];
  return TBG_OK;
}

int Engine::issue_ticket(cudaStream_t st, uint64_t *t) {
  const uint64_t k = next_ticket;
  CK(cudaEventRecord(tick_ev[k % kTickets], st));
  next_ticket++;
  *t = k;
  return TBG_OK;
}

}  // namespace tbg

using namespace tbg;

// ------------------------------------------------------------------- C ABI
#define NEED_MAT()                                                      \
  do {                                                                  \
    if (!g_tab.ready || !g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called"); \
    if (g_eng.cur < 0) return fail(TBG_ERR_STATE, "no material selected"); \
  } while (0)

extern "C" int tbg_init(void) {
  g_tab.build();
  if (!g_tab.ready) return fail(TBG_ERR_STATE, "king tables inconsistent");
  return g_eng.ensure_device();
}

extern "C" int tbg_material_from_name(const char *name) {
  if (!name) return fail(TBG_ERR_ARG, "null material");
  int pt[8], n = 0, black = 0, kings[2] = {0, 0};
  static const char *letters = "PNBRQK";
  for (const char *p = name; *p; p++) {
    if (*p == 'v' && !black) {
      black = 8;
      continue;
    }
    const char *q = strchr(letters, *p);
    if (!q) continue;
    int t = (int)(q - letters) + 1;
    if (t == 1) return fail(TBG_ERR_ARG, "pawns are not supported (tb8gen.c:1314-1317)");
    if (n >= 8) return fail(TBG_ERR_RANGE, "more than 8 pieces");
    if (t == 6) kings[black ? 1 : 0]++;
    pt[n++] = t | black;
  }
  if (!black || n < 3 || kings[0] != 1 || kings[1] != 1)
    return fail(TBG_ERR_ARG, "material %s: need one king each and >= 3 pieces", name);
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (kOrder[pt[i]] > kOrder[pt[j]]) std::swap(pt[i], pt[j]);
  return g_eng.add_material(pt, n);
}

extern "C" int tbg_material_init(const tbg_idx_info *ii, const tbg_idx_info *capt_ii,
                                 const tbg_position *pos, const int *pc_to_set) {
  if (!ii || !capt_ii || !pos || !pc_to_set) return fail(TBG_ERR_ARG, "null argument");
  if (pos->num < 3 || pos->num > 8) return fail(TBG_ERR_ARG, "bad piece count");
  int pt[8];
  for (int i = 0; i < pos->num; i++) pt[i] = pos->pt[i];
  int before = g_eng.nmats;
  int h = g_eng.add_material(pt, pos->num);
  if (h < 0) return h;
  const DMat &d = g_eng.mats[h].d;
  // The caller's IdxInfo must describe the same index (tb8gen.c:1356-1378).
  bool ok = ii->numsets == d.ii.numsets && ii->size == d.ii.size;
  for (int k = 0; ok && k < d.ii.numsets; k++) {
    ok = ii->factor[k] == d.ii.factor[k] && ii->mult[k] == d.ii.mult[k] &&
         ii->first[k] == d.set_first[k] && capt_ii[k].size == d.capt[k].size;
    for (int i = ii->first[k]; ok && i <= ii->last[k]; i++) ok = pc_to_set[i] == k;
  }
  if (!ok) {
    if (g_eng.nmats > before) g_eng.nmats--;
    g_eng.cur = g_eng.nmats - 1;
    return fail(TBG_ERR_ARG, "IdxInfo does not match the piece list");
  }
  return h;
}

extern "C" int tbg_material_select(int mat) {
  if (mat < 0 || mat >= g_eng.nmats) return fail(TBG_ERR_ARG, "no material %d", mat);
  g_eng.cur = mat;
  return TBG_OK;
}

extern "C" int tbg_geometry(uint64_t *size, uint64_t *bytes, uint64_t *sub_bytes,
                            uint64_t sub_offset[6], uint64_t capt_size[6]) {
  NEED_MAT();
  const DMat &d = g_eng.mats[g_eng.cur].d;
  if (size) *size = d.ii.size;
  if (bytes) *bytes = d.bytes;
  if (sub_bytes) *sub_bytes = d.sub_bytes;
  for (int k = 0; k < 6; k++) {
    if (sub_offset) sub_offset[k] = k < d.ii.numsets ? d.sub_offset[k] : 0;
    if (capt_size) capt_size[k] = k < d.ii.numsets ? d.capt[k].size : 0;
  }
  return TBG_OK;
}

extern "C" int tbg_set_stream(void *stream) {
  g_eng.stream = reinterpret_cast<cudaStream_t>(stream);
  return TBG_OK;
}

extern "C" int tbg_set_stub(uint64_t seed, int modulus) {
  if (modulus != 3 && modulus != 5) return fail(TBG_ERR_ARG, "stub modulus must be 3 or 5");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  CK(cudaMemcpyToSymbolAsync(c_stub_seed, &seed, sizeof seed, 0, cudaMemcpyHostToDevice,
                             g_eng.stream));
  CK(cudaMemcpyToSymbolAsync(c_stub_mod, &modulus, sizeof modulus, 0, cudaMemcpyHostToDevice,
                             g_eng.stream));
  CK(persist_block_set_stub(seed, modulus, g_eng.stream));
  CK(persist_warp_set_stub(seed, modulus, g_eng.stream));
  CK(cudaStreamSynchronize(g_eng.stream));
  return TBG_OK;
}

extern "C" int tbg_slot_bind(int s, void *dev_bitmap, size_t bytes) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "slice %d out of range", s);
  Material &m = g_eng.mats[g_eng.cur];
  if (dev_bitmap && (!aligned16(dev_bitmap) || bytes < m.d.bytes))
    return fail(TBG_ERR_ARG, "bitmap for slice %d: need %llu bytes, 16-B aligned", s,
                (unsigned long long)m.d.bytes);
  m.slot[s + 1] = static_cast<uint8_t *>(dev_bitmap);
  m.slot_bytes[s + 1] = dev_bitmap ? bytes : 0;
  return TBG_OK;
}

extern "C" int tbg_sub_bind(int s, void *dev_sub, size_t bytes) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "slice %d out of range", s);
  Material &m = g_eng.mats[g_eng.cur];
  if (dev_sub && (!aligned16(dev_sub) || bytes < m.d.sub_bytes))
    return fail(TBG_ERR_ARG, "sub buffer for slice %d: need %llu bytes, 16-B aligned", s,
                (unsigned long long)m.d.sub_bytes);
  m.sub[s + 1] = static_cast<uint8_t *>(dev_sub);
  m.sub_len[s + 1] = dev_sub ? bytes : 0;
  return TBG_OK;
}

extern "C" int tbg_unbind_all(void) {
  NEED_MAT();
  Material &m = g_eng.mats[g_eng.cur];
  for (int i = 0; i < 463; i++) {
    m.slot[i] = nullptr;
    m.sub[i] = nullptr;
    m.slot_bytes[i] = m.sub_len[i] = 0;
  }
  return TBG_OK;
}

// ---------------------------------------------------------------- ops
// Every call of the ply step becomes an Op; outside a recording it is
// launched at once, inside one it is appended to the batch.
// Work items of an op: 1 MiB chunks of a streaming op, tiles of a verify
// or an uncapture, groups of gt tiles of a scatter (tbg_batch_shape; by
// default one tile for predecessors, four for candidates): a scatter's
// block gathers the sparse sources of an item's tiles before handing them
// out.
static uint32_t op_tiles(Op &o) {
  o.gt = 1;
  if (op_streams(o.kind)) return (uint32_t)((o.n16 + kChunk16 - 1) / kChunk16);
  const uint64_t tiles = (o.J.nbits + kTileWords * 32ull - 1) / (kTileWords * 32ull);
  if (o.kind == OP_SCATTER) {
    // candidates (tbg_candidates) mark only near their source's row and read
    // the opponent's wins there: larger items pay; a plain scatter's marks
    // spread over the slice, and the fewer tiles in flight the better its
    // targets stay in L2
    const int want = o.J.filter ? g_eng.candidate_tiles : g_eng.scatter_tiles;
    const uint64_t g = want > 0 ? (uint64_t)want : (o.J.filter ? 4 : 1);
    o.gt = (int)std::min<uint64_t>(std::max<uint64_t>(g, 1), std::max<uint64_t>(tiles, 1));
  }
  return (uint32_t)((tiles + o.gt - 1) / o.gt);
}

static int launch_op(const Op &o) {
  cudaStream_t st = g_eng.stream;
  switch (o.kind) {
  case OP_SCATTER:
  case OP_SCATTER_SUB:
  case OP_VERIFY:
    // warp-wide sub-items of 32 words (k_op_w, tbg_persist_warp.cu)
    persist_warp_launch_op(o, g_eng.num_sms * TBG_MINB_SCATTER, st, g_eng.d_status);
    return g_eng.check_launch("k_op_w");
  case OP_EPILOGUE: {
    uint64_t n16 = o.n16;
    k_epilogue_W<<<g_eng.grid_for((n16 + kThreads - 1) / kThreads, 8), kThreads, 0, st>>>(
        o.T, o.win, o.wout, n16, o.nbits, o.cnt);
    return g_eng.check_launch("k_epilogue_W");
  }
  case OP_CLEAR:
    CK(cudaMemsetAsync(o.T, 0, o.n16 * 16, st));
    return TBG_OK;
  case OP_COUNT:
    k_count<<<g_eng.grid_for((o.n16 + kThreads - 1) / kThreads, 8), kThreads, 0, st>>>(
        o.T, o.n16, o.nbits, o.cnt);
    return g_eng.check_launch("k_count");
  }
  return fail(TBG_ERR_ARG, "unknown op");
}

static int submit(Op &o) {
  o.ntiles = op_tiles(o);
  if (g_eng.batch().recording) return g_eng.batch().add(o);
  return launch_op(o);
}

static Op new_op(int kind) {
  Op o;
  memset(&o, 0, sizeof o);
  o.kind = kind;
  o.cnt_slot = -1;
  o.ns = g_eng.mats[g_eng.cur].d.ii.numsets;
  return o;
}

extern "C" int tbg_predecessors(int stm, int s) {
  NEED_MAT();
  if ((stm & ~1) || s < 0 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "bad stm/slice");
  Material &m = g_eng.mats[g_eng.cur];
  Op o = new_op(OP_SCATTER);
  int rc = g_eng.fill_job(o.J, stm, s, false);
  if (rc) return rc;
  if (!m.slot[0]) return fail(TBG_ERR_UNBOUND, "scratch slot not bound");
  o.J.src = reinterpret_cast<const uint32_t *>(m.slot[0]);
  o.J.cand = nullptr;
  o.J.nbits = m.d.ii.size;
  return submit(o);
}

extern "C" int tbg_candidates(int stm, int s, const void *opp_wins, size_t bytes) {
  NEED_MAT();
  if ((stm & ~1) || s < 0 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "bad stm/slice");
  Material &m = g_eng.mats[g_eng.cur];
  if (!opp_wins || !aligned16(opp_wins) || bytes < m.d.bytes)
    return fail(TBG_ERR_ARG, "opponent wins of slice %d: need %llu bytes, 16-B aligned", s,
                (unsigned long long)m.d.bytes);
  Op o = new_op(OP_SCATTER);
  int rc = g_eng.fill_job(o.J, stm, s, false);
  if (rc) return rc;
  if (!m.slot[0]) return fail(TBG_ERR_UNBOUND, "scratch slot not bound");
  o.J.src = reinterpret_cast<const uint32_t *>(m.slot[0]);
  o.J.cand = nullptr;
  o.J.nbits = m.d.ii.size;
  o.J.filter = static_cast<const uint32_t *>(opp_wins);
  return submit(o);
}

extern "C" int tbg_predecessors_sub(int stm, int s, int legality) {
  NEED_MAT();
  if ((stm & ~1) || s < 0 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "bad stm/slice");
  Material &m = g_eng.mats[g_eng.cur];
  Op o = new_op(OP_SCATTER_SUB);
  int rc = g_eng.fill_job(o.J, stm, s, false);
  if (rc) return rc;
  if (!o.J.self_sub) return fail(TBG_ERR_UNBOUND, "sub of slice %d not bound", s);
  o.J.legality = legality != 0;
  o.J.cand = nullptr;
  for (int k = 0; k < m.d.ii.numsets; k++) {
    if (m.d.set_color[k] == stm) continue;
    o.J.set = k;
    o.J.src = reinterpret_cast<const uint32_t *>(o.J.self_sub + m.d.sub_offset[k]);
    o.J.nbits = m.d.capt[k].size;
    rc = submit(o);
    if (rc) return rc;
  }
  return TBG_OK;
}

static int check_successors(int stm, int s, uint32_t *out) {
  NEED_MAT();
  if ((stm & ~1) || s < 0 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "bad stm/slice");
  Material &m = g_eng.mats[g_eng.cur];
  Op o = new_op(OP_VERIFY);
  int rc = g_eng.fill_job(o.J, stm, s, true);
  if (rc) return rc;
  if (!m.slot[0]) return fail(TBG_ERR_UNBOUND, "scratch slot not bound");
  o.J.cand = reinterpret_cast<uint32_t *>(m.slot[0]);
  o.J.src = o.J.cand;
  o.J.nbits = m.d.ii.size;
  o.out = out;
  o.out_words = out ? m.d.bytes / 4 : 0;
  return submit(o);
}

extern "C" int tbg_check_successors(int stm, int s) { return check_successors(stm, s, nullptr); }

extern "C" int tbg_check_successors_to(int stm, int s, void *dev_out) {
  if (!dev_out || !aligned16(dev_out)) return fail(TBG_ERR_ARG, "bad output");
  return check_successors(stm, s, static_cast<uint32_t *>(dev_out));
}

extern "C" int tbg_calc_sub(int stm, int s, void *const dev_cls[5]) {
  NEED_MAT();
  if ((stm & ~1) || s < 0 || s >= TBG_NSLICES || !dev_cls) return fail(TBG_ERR_ARG, "bad args");
  for (int i = 0; i < 5; i++)
    if (!dev_cls[i] || !aligned16(dev_cls[i])) return fail(TBG_ERR_ARG, "class buffer %d", i);
  Material &m = g_eng.mats[g_eng.cur];
  SliceJob J;
  memset(&J, 0, sizeof J);
  J.mat = g_eng.cur;
  J.stm = stm;
  J.s = s;
  J.k0 = g_tab.kksq[s][0];
  J.k1 = g_tab.kksq[s][1];
  for (int k = 0; k < m.d.ii.numsets; k++) {
    if (m.d.set_color[k] != stm) continue;
    J.set = k;
    uint64_t off = m.d.sub_offset[k];
    uint64_t nwords = (m.d.capt[k].size + 31) / 32;
    uint32_t *c[5];
    for (int i = 0; i < 5; i++) c[i] = reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(dev_cls[i]) + off);
    NS_SWITCH(m.d.ii.numsets, k_calc_sub<NS><<<g_eng.grid_for((nwords + kThreads - 1) / kThreads, 16), kThreads, 0,
                 g_eng.stream>>>(J, c[0], c[1], c[2], c[3], c[4]));
    int rc = g_eng.check_launch("k_calc_sub");
    if (rc) return rc;
  }
  return TBG_OK;
}

extern "C" int tbg_calc_illegal(int s, void *dev_ill_w, void *dev_ill_b) {
  NEED_MAT();
  if (s < 0 || s >= TBG_NSLICES || !dev_ill_w || !dev_ill_b ||
      !aligned16(dev_ill_w) || !aligned16(dev_ill_b))
    return fail(TBG_ERR_ARG, "bad args");
  Material &m = g_eng.mats[g_eng.cur];
  SliceJob J;
  memset(&J, 0, sizeof J);
  J.mat = g_eng.cur;
  J.s = s;
  J.k0 = g_tab.kksq[s][0];
  J.k1 = g_tab.kksq[s][1];
  uint64_t nwords = m.d.bytes / 4;
  NS_SWITCH(m.d.ii.numsets, k_calc_illegal<NS><<<g_eng.grid_for((nwords + kThreads - 1) / kThreads, 16), kThreads, 0,
                   g_eng.stream>>>(J, static_cast<uint32_t *>(dev_ill_w),
                                   static_cast<uint32_t *>(dev_ill_b), nwords));
  return g_eng.check_launch("k_calc_illegal");
}

extern "C" int tbg_calc_mate(int s, const void *dev_ill_w, const void *dev_ill_b,
                             void *dev_mate_w, void *dev_mate_b) {
  NEED_MAT();
  if (s < 0 || s >= TBG_NSLICES || !dev_ill_w || !dev_ill_b || !dev_mate_w || !dev_mate_b)
    return fail(TBG_ERR_ARG, "bad args");
  Material &m = g_eng.mats[g_eng.cur];
  SliceJob J;
  memset(&J, 0, sizeof J);
  J.mat = g_eng.cur;
  J.s = s;
  J.k0 = g_tab.kksq[s][0];
  J.k1 = g_tab.kksq[s][1];
  uint64_t nwords = m.d.bytes / 4;
  NS_SWITCH(m.d.ii.numsets, k_calc_mate<NS><<<g_eng.grid_for((nwords + kThreads - 1) / kThreads, 16), kThreads, 0,
                g_eng.stream>>>(J, static_cast<const uint32_t *>(dev_ill_w),
                                static_cast<const uint32_t *>(dev_ill_b),
                                static_cast<uint32_t *>(dev_mate_w),
                                static_cast<uint32_t *>(dev_mate_b), nwords));
  return g_eng.check_launch("k_calc_mate");
}

static int epilogue(uint8_t *T, const uint8_t *Win, uint8_t *Wout, uint64_t *cnt) {
  Material &m = g_eng.mats[g_eng.cur];
  Op o = new_op(OP_EPILOGUE);
  o.T = reinterpret_cast<uint4 *>(T);
  o.win = reinterpret_cast<const uint4 *>(Win);
  o.wout = reinterpret_cast<uint4 *>(Wout);
  o.n16 = m.d.bytes / 16;
  o.nbits = m.d.ii.size;
  if (g_eng.batch().recording) {
    if (cnt) return fail(TBG_ERR_STATE, "counts of a recorded epilogue come from tbg_batch_counts");
    o.cnt_slot = g_eng.batch().ncounts++;
    o.cnt = nullptr;
    return submit(o);
  }
  CK(cudaMemsetAsync(g_eng.d_cnt, 0, sizeof(unsigned long long), g_eng.stream));
  o.cnt = g_eng.d_cnt;
  int rc = submit(o);
  if (rc || !cnt) return rc;
  CK(cudaMemcpyAsync(g_eng.h_cnt, g_eng.d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     g_eng.stream));
  rc = g_eng.wait(0);
  if (rc) return rc;
  *cnt = g_eng.h_cnt[0];
  return TBG_OK;
}

extern "C" int tbg_epilogue_W(int s, int s_wins, uint64_t *cnt) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES || s_wins < -1 || s_wins >= TBG_NSLICES)
    return fail(TBG_ERR_ARG, "bad slice");
  Material &m = g_eng.mats[g_eng.cur];
  uint8_t *T = m.slot[s + 1], *W = m.slot[s_wins + 1];
  if (!T || !W) return fail(TBG_ERR_UNBOUND, "epilogue slices not bound");
  return epilogue(T, W, W, cnt);
}

extern "C" int tbg_epilogue_W_to(int s, const void *dev_wins_in, void *dev_wins_out,
                                 uint64_t *cnt) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES || !dev_wins_in || !dev_wins_out ||
      !aligned16(dev_wins_in) || !aligned16(dev_wins_out))
    return fail(TBG_ERR_ARG, "bad args");
  Material &m = g_eng.mats[g_eng.cur];
  uint8_t *T = m.slot[s + 1];
  if (!T) return fail(TBG_ERR_UNBOUND, "slice %d not bound", s);
  return epilogue(T, static_cast<const uint8_t *>(dev_wins_in), static_cast<uint8_t *>(dev_wins_out),
                  cnt);
}

extern "C" int tbg_count(int s, uint64_t *cnt) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES || !cnt) return fail(TBG_ERR_ARG, "bad args");
  Material &m = g_eng.mats[g_eng.cur];
  uint8_t *P = m.slot[s + 1];
  if (!P) return fail(TBG_ERR_UNBOUND, "slice %d not bound", s);
  CK(cudaMemsetAsync(g_eng.d_cnt, 0, sizeof(unsigned long long), g_eng.stream));
  uint64_t n16 = m.d.bytes / 16;
  k_count<<<g_eng.grid_for((n16 + kThreads - 1) / kThreads, 8), kThreads, 0, g_eng.stream>>>(
      reinterpret_cast<const uint4 *>(P), n16, m.d.ii.size, g_eng.d_cnt);
  int rc = g_eng.check_launch("k_count");
  if (rc) return rc;
  CK(cudaMemcpyAsync(g_eng.h_cnt, g_eng.d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     g_eng.stream));
  rc = g_eng.wait(0);
  if (rc) return rc;
  *cnt = g_eng.h_cnt[0];
  return TBG_OK;
}

extern "C" int tbg_count_strided(const void *dev_base, uint64_t stride_bytes, int n,
                                 uint64_t *cnt) {
  NEED_MAT();
  Material &m = g_eng.mats[g_eng.cur];
  if (!dev_base || !cnt || n < 1 || n > 65535 || !aligned16(dev_base) || stride_bytes % 16 ||
      (n > 1 && stride_bytes < m.d.bytes))
    return fail(TBG_ERR_ARG, "bad strided count");
  CK(cudaMemsetAsync(g_eng.d_cnt, 0, sizeof(unsigned long long), g_eng.stream));
  const uint64_t n16 = m.d.bytes / 16;
  const uint64_t per = (n16 + kThreads - 1) / kThreads;
  const uint64_t want = std::max<uint64_t>(1, (uint64_t)g_eng.num_sms * 8 / (uint64_t)n);
  dim3 grid((unsigned)std::min(per, want), (unsigned)n);
  k_count_strided<<<grid, kThreads, 0, g_eng.stream>>>(static_cast<const uint8_t *>(dev_base),
                                                       stride_bytes, n16, m.d.ii.size, g_eng.d_cnt);
  int rc = g_eng.check_launch("k_count_strided");
  if (rc) return rc;
  CK(cudaMemcpyAsync(g_eng.h_cnt, g_eng.d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                     g_eng.stream));
  rc = g_eng.wait(0);
  if (rc) return rc;
  *cnt = g_eng.h_cnt[0];
  return TBG_OK;
}

extern "C" int tbg_clear(int s) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "bad slice");
  Material &m = g_eng.mats[g_eng.cur];
  if (!m.slot[s + 1]) return fail(TBG_ERR_UNBOUND, "slice %d not bound", s);
  Op o = new_op(OP_CLEAR);
  o.T = reinterpret_cast<uint4 *>(m.slot[s + 1]);
  o.n16 = m.d.bytes / 16;
  return submit(o);
}

extern "C" int tbg_batch_count(int s) {
  NEED_MAT();
  if (s < -1 || s >= TBG_NSLICES) return fail(TBG_ERR_ARG, "bad slice");
  if (!g_eng.batch().recording) return fail(TBG_ERR_STATE, "tbg_batch_count records into a batch");
  Material &m = g_eng.mats[g_eng.cur];
  if (!m.slot[s + 1]) return fail(TBG_ERR_UNBOUND, "slice %d not bound", s);
  Op o = new_op(OP_COUNT);
  o.T = reinterpret_cast<uint4 *>(m.slot[s + 1]);
  o.n16 = m.d.bytes / 16;
  o.nbits = m.d.ii.size;
  o.cnt_slot = g_eng.batch().ncounts++;
  return submit(o);
}

extern "C" int tbg_sub_and_not(int s1, int s2, int stm) {
  NEED_MAT();
  if (s1 < -1 || s1 >= TBG_NSLICES || s2 < -1 || s2 >= TBG_NSLICES || (stm & ~1))
    return fail(TBG_ERR_ARG, "bad args");
  Material &m = g_eng.mats[g_eng.cur];
  // kslice_sub_get_base(-1) is the scratch bitmap buffer (kslice.h:63-68).
  uint8_t *p = s1 == -1 ? m.slot[0] : m.sub[s1 + 1];
  uint8_t *q = s2 == -1 ? m.slot[0] : m.sub[s2 + 1];
  if (!p || !q) return fail(TBG_ERR_UNBOUND, "sub buffers not bound");
  if ((s1 == -1 || s2 == -1) && m.d.sub_size[stm] > m.d.bytes)
    return fail(TBG_ERR_RANGE, "sub bitmaps larger than the scratch slot");
  uint64_t n16 = m.d.sub_size[stm] / 16;
  k_and_not<<<g_eng.grid_for((n16 + kThreads - 1) / kThreads, 8), kThreads, 0, g_eng.stream>>>(
      reinterpret_cast<uint4 *>(p), reinterpret_cast<const uint4 *>(q), n16);
  return g_eng.check_launch("k_and_not");
}

extern "C" int tbg_sync(int timeout_ms) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  return g_eng.wait(timeout_ms);
}

extern "C" const char *tbg_last_error(void) { return g_errbuf; }

extern "C" int tbg_gen_bernoulli(void *dev, uint64_t nbits, uint64_t bytes, uint64_t seed,
                                 uint64_t tag, uint64_t thr) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  if (!dev || !aligned16(dev) || (bytes & 3) || nbits > bytes * 8) return fail(TBG_ERR_ARG, "bad buffer");
  uint64_t key = tbg_host_mix64(tbg_host_mix64(seed + 0x9e3779b97f4a7c15ull) ^ tag);
  uint64_t nwords = bytes / 4;
  k_gen_bernoulli<<<g_eng.grid_for((nwords + kThreads - 1) / kThreads, 16), kThreads, 0,
                    g_eng.stream>>>(static_cast<uint32_t *>(dev), nwords, nbits, key, thr);
  return g_eng.check_launch("k_gen_bernoulli");
}

namespace tbg {
__global__ void k_attacks(int type, const uint8_t *sq, const uint64_t *occ, uint64_t *out,
                          uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = piece_attacks(type, sq[i], occ[i]);
}
}  // namespace tbg

extern "C" int tbg_attacks(int type, const uint8_t *dev_sq, const uint64_t *dev_occ,
                           uint64_t *dev_out, uint64_t n) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  if (type < 2 || type > 6 || !dev_sq || !dev_occ || !dev_out) return fail(TBG_ERR_ARG, "bad args");
  k_attacks<<<g_eng.grid_for((n + kThreads - 1) / kThreads, 8), kThreads, 0, g_eng.stream>>>(type, dev_sq, dev_occ,
                                                                        dev_out, n);
  return g_eng.check_launch("k_attacks");
}

extern "C" int tbg_launches(uint64_t *n) {
  if (!n) return fail(TBG_ERR_ARG, "null");
  *n = g_eng.launches;
  return TBG_OK;
}

// ------------------------------------------------------------- batches
namespace tbg {

void Batch::clear() {
  ops.clear();
  bufs.clear();
  preds.clear();
  ncounts = 0;
  nsmax = 1;
  total = 0;
  ready = false;
}

static void access_of(const Op &o, Batch::Access &a) {
  const SliceJob &J = o.J;
  switch (o.kind) {
  case OP_SCATTER:
    a.rd.push_back(J.src);
    if (J.filter) a.rd.push_back(J.filter);
    a.wacc.push_back(J.self);
    for (int d = 0; d < J.nk; d++) a.wacc.push_back(J.kd[d].bits);
    break;
  case OP_SCATTER_SUB:
    a.rd.push_back(J.self_sub);
    a.wacc.push_back(J.self);
    for (int d = 0; d < J.nk; d++) a.wacc.push_back(J.kd[d].bits);
    break;
  case OP_VERIFY:
    a.rd.push_back(J.cand);
    a.rd.push_back(J.self);
    a.rd.push_back(J.self_sub);
    for (int d = 0; d < J.nk; d++) {
      a.rd.push_back(J.kd[d].bits);
      a.rd.push_back(J.kd[d].sub);
    }
    a.wplain.push_back(o.out ? static_cast<const void *>(o.out) : J.cand);
    break;
  case OP_EPILOGUE:
    a.rd.push_back(o.T);
    a.rd.push_back(o.win);
    a.wplain.push_back(o.T);
    a.wplain.push_back(o.wout);
    break;
  case OP_CLEAR:
    a.wplain.push_back(o.T);
    break;
  case OP_COUNT:
    a.rd.push_back(o.T);
    break;
  }
}

static bool contains(const std::vector<const void *> &v, const void *p) {
  return p != nullptr && std::find(v.begin(), v.end(), p) != v.end();
}

// Op b (recorded after a) must wait for a when a write of one meets a read or
// write of the other; two accumulating scatters commute.  Per buffer this
// means: a read waits for the last outright write and the accumulations
// since; an accumulation for the last write and the reads since; an outright
// write for all three.  Earlier accesses are covered through those ops' own
// waits.
int Batch::add(Op &o) {
  Access a;
  access_of(o, a);
  std::vector<int> dep;
  auto need = [&](const void *x, bool rd, bool accs) {
    if (!x) return;
    auto it = bufs.find(x);
    if (it == bufs.end()) return;
    const BufState &b = it->second;
    if (b.writer >= 0) dep.push_back(b.writer);
    if (rd) dep.insert(dep.end(), b.readers.begin(), b.readers.end());
    if (accs) dep.insert(dep.end(), b.accs.begin(), b.accs.end());
  };
  for (const void *x : a.rd) need(x, false, true);
  for (const void *x : a.wacc) need(x, true, false);
  for (const void *x : a.wplain) need(x, true, true);
  std::sort(dep.begin(), dep.end());
  dep.erase(std::unique(dep.begin(), dep.end()), dep.end());
  o.pred_off = (int)preds.size();
  o.npred = (int)dep.size();
  preds.insert(preds.end(), dep.begin(), dep.end());
  const int me = (int)ops.size();
  for (const void *x : a.wplain) {
    if (!x) continue;
    BufState &b = bufs[x];
    b.writer = me;
    b.readers.clear();
    b.accs.clear();
  }
  auto note = [&](const void *x, bool rd) {
    if (!x || contains(a.wplain, x)) return;
    std::vector<int> &v = rd ? bufs[x].readers : bufs[x].accs;
    if (v.empty() || v.back() != me) v.push_back(me);
  };
  for (const void *x : a.rd) note(x, true);
  for (const void *x : a.wacc) note(x, false);
  if (!op_streams(o.kind)) nsmax = std::max(nsmax, o.ns);
  o.first = total;
  total += o.ntiles;
  ops.push_back(o);
  return TBG_OK;
}

template <class T>
static int grow(T **p, size_t *cap, size_t n) {
  if (n <= *cap) return TBG_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  size_t c = std::max(n, (size_t)64);
  cudaError_t e = cudaMalloc(p, c * sizeof(T));
  if (e != cudaSuccess) return fail(TBG_ERR_NOMEM, "batch queue: %s", cudaGetErrorString(e));
  *cap = c;
  return TBG_OK;
}

int Batch::finish() {
  int rc;
  if ((rc = grow(&d_ops, &cap_ops, ops.size()))) return rc;
  if ((rc = grow(&d_preds, &cap_preds, std::max<size_t>(preds.size(), 1)))) return rc;
  if ((rc = grow(&d_done, &cap_done, ops.size()))) return rc;
  if ((rc = grow(&d_counts, &cap_counts, std::max(ncounts, 1)))) return rc;
  if (!d_next) {
    cudaError_t e = cudaMalloc(&d_next, sizeof(unsigned long long));
    if (e != cudaSuccess) return fail(TBG_ERR_NOMEM, "batch queue: %s", cudaGetErrorString(e));
  }
  for (Op &o : ops) o.cnt = o.cnt_slot >= 0 ? d_counts + o.cnt_slot : nullptr;
  // Stream-ordered after a run of the previous batch that may still read the
  // queue; from pageable memory the call returns once the bytes are staged.
  CK(cudaMemcpyAsync(d_ops, ops.data(), ops.size() * sizeof(Op), cudaMemcpyHostToDevice,
                     g_eng.stream));
  if (!preds.empty())
    CK(cudaMemcpyAsync(d_preds, preds.data(), preds.size() * sizeof(int), cudaMemcpyHostToDevice,
                       g_eng.stream));
  ready = true;
  return TBG_OK;
}

}  // namespace tbg

extern "C" int tbg_batch_begin(void) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  if (g_eng.batch().recording) return fail(TBG_ERR_STATE, "already recording");
  g_eng.batch().clear();
  g_eng.batch().recording = true;
  return TBG_OK;
}

extern "C" int tbg_batch_end(int *nops, uint64_t *nitems) {
  Batch &b = g_eng.batch();
  if (!b.recording) return fail(TBG_ERR_STATE, "not recording");
  b.recording = false;
  if (b.ops.empty()) return fail(TBG_ERR_ARG, "empty batch");
  int rc = b.finish();
  if (rc) return rc;
  if (nops) *nops = (int)b.ops.size();
  if (nitems) *nitems = b.total;
  return TBG_OK;
}

extern "C" int tbg_batch_select(int slot) {
  if (slot < 0 || slot >= Engine::kBatchSlots) return fail(TBG_ERR_ARG, "batch slot 0..%d", Engine::kBatchSlots - 1);
  for (const Batch &b : g_eng.batches)
    if (b.recording) return fail(TBG_ERR_STATE, "a batch is being recorded");
  g_eng.bslot = slot;
  return TBG_OK;
}

extern "C" int tbg_batch_shape(int scatter_tiles, int candidate_tiles, uint64_t *nitems) {
  if (scatter_tiles < 0 || scatter_tiles > 64 || candidate_tiles < 0 || candidate_tiles > 64)
    return fail(TBG_ERR_ARG, "tiles per item 0..64");
  for (const Batch &b : g_eng.batches)
    if (b.recording) return fail(TBG_ERR_STATE, "a batch is being recorded");
  g_eng.scatter_tiles = scatter_tiles;
  g_eng.candidate_tiles = candidate_tiles;
  Batch &b = g_eng.batch();
  if (nitems) *nitems = 0;
  if (!b.ready) return TBG_OK;
  // re-cut the selected batch's work items and upload its queue again
  b.total = 0;
  for (Op &o : b.ops) {
    o.ntiles = op_tiles(o);
    o.first = b.total;
    b.total += o.ntiles;
  }
  if (nitems) *nitems = b.total;
  return b.finish();
}

extern "C" int tbg_batch_tune(int ctas_per_sm, long long spin_limit) {
  if (ctas_per_sm < 1 || ctas_per_sm > 32) return fail(TBG_ERR_ARG, "ctas_per_sm 1..32");
  for (Batch &b : g_eng.batches) {
    b.ctas_per_sm = ctas_per_sm;
    if (spin_limit > 0) b.spin_limit = spin_limit;
  }
  return TBG_OK;
}

extern "C" int tbg_batch_run(int mode) {
  Batch &b = g_eng.batch();
  if (!b.ready) return fail(TBG_ERR_STATE, "no recorded batch");
  cudaStream_t st = g_eng.stream;
  CK(cudaMemsetAsync(b.d_counts, 0, std::max(b.ncounts, 1) * sizeof(unsigned long long), st));
  if (mode == 0) {
    for (const Op &o : b.ops) {
      int rc = launch_op(o);
      if (rc) return rc;
    }
    return TBG_OK;
  }
  if (mode != 1 && mode != 2)
    return fail(TBG_ERR_ARG, "mode 0 (one launch per call), 1 or 2 (persistent)");
  CK(cudaMemsetAsync(b.d_done, 0, b.ops.size() * sizeof(unsigned int), st));
  CK(cudaMemsetAsync(b.d_next, 0, sizeof(unsigned long long), st));
  int grid = g_eng.num_sms * b.ctas_per_sm;
  const PersistArgs pa{b.d_ops, (int)b.ops.size(), b.d_preds, b.total,
                       b.d_next, b.d_done, g_eng.d_status, b.spin_limit};
  if (mode == 2) {
    persist_warp_launch(b.nsmax, grid, st, pa);
    return g_eng.check_launch("k_batch_w");
  }
  persist_block_launch(b.nsmax, grid, st, pa);
  return g_eng.check_launch("k_batch");
}

extern "C" int tbg_batch_counts(uint64_t *out, int n) {
  Batch &b = g_eng.batch();
  if (!b.ready || !out || n < 0 || n > b.ncounts) return fail(TBG_ERR_ARG, "bad count request");
  if (n == 0) return TBG_OK;
  int rc = g_eng.wait(0);
  if (rc) return rc;
  CK(cudaMemcpy(out, b.d_counts, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return TBG_OK;
}

extern "C" int tbg_batch_counts_async(uint64_t *host_out, int n) {
  Batch &b = g_eng.batch();
  if (!b.ready || !host_out || n < 0 || n > b.ncounts) return fail(TBG_ERR_ARG, "bad count request");
  if (n == 0) return TBG_OK;
  CK(cudaMemcpyAsync(host_out, b.d_counts, n * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                     g_eng.stream));
  return TBG_OK;
}

extern "C" int tbg_alloc(size_t bytes, void **dev) {
  if (!dev || bytes == 0) return fail(TBG_ERR_ARG, "bad allocation request");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  *dev = nullptr;
  if (g_eng.alloc_refused())
    return fail(TBG_ERR_NOMEM, "cudaMalloc(%zu): allocation %ld refused (TBG_FAIL_ALLOC_AT)",
                bytes, g_eng.alloc_calls);
  cudaError_t e = cudaMalloc(dev, bytes);
  if (e != cudaSuccess) return fail(TBG_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  // Zeroed on a stream of its own and waited for: a plain cudaMemset would
  // queue on the legacy default stream, unordered with the caller's
  // non-blocking streams, and could land after the caller's first copy.
  if (!g_eng.s_zero) CK(cudaStreamCreateWithFlags(&g_eng.s_zero, cudaStreamNonBlocking));
  CK(cudaMemsetAsync(*dev, 0, bytes, g_eng.s_zero));
  CK(cudaStreamSynchronize(g_eng.s_zero));
  return TBG_OK;
}

extern "C" int tbg_free(void *dev) {
  if (!dev) return TBG_OK;
  CK(cudaFree(dev));
  return TBG_OK;
}

extern "C" int tbg_copy_to_device(void *dev, const void *host, size_t bytes) {
  if (!dev || !host) return fail(TBG_ERR_ARG, "null pointer");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, g_eng.stream));
  CK(cudaStreamSynchronize(g_eng.stream));
  return TBG_OK;
}

extern "C" int tbg_copy_to_device_async(void *dev, const void *host, size_t bytes) {
  if (!dev || !host) return fail(TBG_ERR_ARG, "null pointer");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, g_eng.stream));
  return TBG_OK;
}

extern "C" int tbg_copy_to_host_async(void *host, const void *dev, size_t bytes) {
  if (!dev || !host) return fail(TBG_ERR_ARG, "null pointer");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, g_eng.stream));
  return TBG_OK;
}

// ---------------------------------------------------------- copy streams
extern "C" int tbg_mark(uint64_t *ticket) {
  if (!ticket) return fail(TBG_ERR_ARG, "null ticket");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  int rc = g_eng.tickets_ready();
  if (rc) return rc;
  return g_eng.issue_ticket(g_eng.stream, ticket);
}

static int side_copy(cudaStream_t st, void *dst, const void *src, size_t n, cudaMemcpyKind kind,
                     uint64_t after, uint64_t *ticket) {
  if (after) {
    cudaEvent_t e;
    int rc = g_eng.ticket_event(after, &e);
    if (rc) return rc;
    CK(cudaStreamWaitEvent(st, e, 0));
  }
  if (n) CK(cudaMemcpyAsync(dst, src, n, kind, st));
  if (ticket) return g_eng.issue_ticket(st, ticket);
  return TBG_OK;
}

static int side_ready(size_t n, const void *a, const void *b) {
  if (n && (!a || !b)) return fail(TBG_ERR_ARG, "null pointer");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  return g_eng.tickets_ready();
}

extern "C" int tbg_copy_in(void *dev, const void *host, size_t bytes, uint64_t after,
                           uint64_t *ticket) {
  int rc = side_ready(bytes, dev, host);
  if (rc) return rc;
  return side_copy(g_eng.s_in, dev, host, bytes, cudaMemcpyHostToDevice, after, ticket);
}

extern "C" int tbg_copy_out(void *host, const void *dev, size_t bytes, uint64_t after,
                            uint64_t *ticket) {
  int rc = side_ready(bytes, dev, host);
  if (rc) return rc;
  return side_copy(g_eng.s_out, host, dev, bytes, cudaMemcpyDeviceToHost, after, ticket);
}

extern "C" int tbg_join(uint64_t ticket) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  cudaEvent_t e;
  int rc = g_eng.ticket_event(ticket, &e);
  if (rc) return rc;
  CK(cudaStreamWaitEvent(g_eng.stream, e, 0));
  return TBG_OK;
}

extern "C" int tbg_wait_ticket(uint64_t ticket, int timeout_ms) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  cudaEvent_t e;
  int rc = g_eng.ticket_event(ticket, &e);
  if (rc) return rc;
  auto t0 = std::chrono::steady_clock::now();
  const long limit = timeout_ms > 0 ? timeout_ms : 600000;
  for (;;) {
    cudaError_t q = cudaEventQuery(e);
    if (q == cudaSuccess) return TBG_OK;
    if (q != cudaErrorNotReady) return cuda_fail(q, "ticket");
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                  std::chrono::steady_clock::now() - t0).count();
    if (ms > limit) return fail(TBG_ERR_TIMEOUT, "ticket not reached within %ld ms", limit);
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

extern "C" int tbg_host_alloc(size_t bytes, void **host) {
  if (!host || bytes == 0) return fail(TBG_ERR_ARG, "bad allocation request");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  *host = nullptr;
  if (g_eng.alloc_refused())
    return fail(TBG_ERR_NOMEM, "cudaHostAlloc(%zu): allocation %ld refused (TBG_FAIL_ALLOC_AT)",
                bytes, g_eng.alloc_calls);
  cudaError_t e = cudaHostAlloc(host, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(TBG_ERR_NOMEM, "cudaHostAlloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return TBG_OK;
}

extern "C" int tbg_host_free(void *host) {
  if (!host) return TBG_OK;
  CK(cudaFreeHost(host));
  return TBG_OK;
}

extern "C" int tbg_copy_to_host(void *host, const void *dev, size_t bytes) {
  if (!dev || !host) return fail(TBG_ERR_ARG, "null pointer");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, g_eng.stream));
  CK(cudaStreamSynchronize(g_eng.stream));
  return TBG_OK;
}

namespace tbg {
__global__ void __launch_bounds__(kThreads) k_and_not3(uint4 *d, const uint4 *a, const uint4 *b,
                                                       uint64_t n16) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 x = a[i], y = b[i];
    d[i] = make_uint4(x.x & ~y.x, x.y & ~y.y, x.z & ~y.z, x.w & ~y.w);
  }
}
}  // namespace tbg

extern "C" int tbg_bitmap_and_not(void *dst, const void *a, const void *b, size_t bytes) {
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  if (!dst || !a || !b || !aligned16(dst) || !aligned16(a) || !aligned16(b) || (bytes & 15))
    return fail(TBG_ERR_ARG, "bad buffers");
  uint64_t n16 = bytes / 16;
  k_and_not3<<<g_eng.grid_for((n16 + kThreads - 1) / kThreads, 8), kThreads, 0, g_eng.stream>>>(
      static_cast<uint4 *>(dst), static_cast<const uint4 *>(a), static_cast<const uint4 *>(b), n16);
  return g_eng.check_launch("k_and_not3");
}
