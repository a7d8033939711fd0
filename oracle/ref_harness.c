/*
 * Oracle test infrastructure -- NOT product code.
 *
 * Drives the reference generator's own per-king-slice workers, compiled in
 * place from the reference sources (tb8gen.c and kslice.c are #included so
 * that their `static` workers and schedule tables are reachable), over
 * caller-provided host buffers.  Only tests, the smoke check and the CPU
 * baseline leg of bench.py load the resulting oracle/_ref/libtbref.so, and
 * only as the checker / the timed reference arm.
 *
 * Build: oracle/Makefile (the reference's Makefile is not used: it asks for
 * -std=c23, which gcc 13 rejects, and links a non-existent bitmap.o).
 *
 * Substitutions, all outside the reference's algorithm:
 *  - probe_wdl (probe.c:1677) is renamed at compile time to
 *    harness_probe_wdl, the seeded 7-piece WDL stub defined below.  It stands
 *    in for the 7-piece tables, which do not exist here.
 *  - The zstd entry points the disk tier (util.c:218-255) links against are
 *    defined as aborting stubs: the harness never reads or writes files.
 *  - main() (tb8gen.c:1245) is renamed tb8gen_main and never called;
 *    harness_setup() below restates its material set-up (tb8gen.c:1284-1385)
 *    without the disk-side steps (directory creation, table scan).
 */
#include <stdlib.h>

#include "tb8gen.c"
#include "kslice.c"
#include <zstd.h>

/* ---- zstd stubs: the disk tier is out of reach of every harness entry ---- */
size_t ZSTD_compressBound(size_t n) { (void)n; abort(); }
ZSTD_CCtx *ZSTD_createCCtx(void) { abort(); }
ZSTD_DCtx *ZSTD_createDCtx(void) { abort(); }
size_t ZSTD_compressCCtx(ZSTD_CCtx *c, void *d, size_t dc, const void *s,
                         size_t sn, int l)
{ (void)c; (void)d; (void)dc; (void)s; (void)sn; (void)l; abort(); }
size_t ZSTD_decompressDCtx(ZSTD_DCtx *c, void *d, size_t dc, const void *s,
                           size_t sn)
{ (void)c; (void)d; (void)dc; (void)s; (void)sn; abort(); }

/* ---- seeded 7-piece WDL stub -------------------------------------------
 * v = VALS[mix64(seed ^ key7(pos)) % modulus], with
 *   key7(pos) = XOR over pieces of mix64(((pt << 6) | sq) * GAMMA + GAMMA)
 *               ^ (stm ? STM_KEY : 0)
 * VALS = {-2, 0, 2} for modulus 3, {-2, -1, 0, 1, 2} for modulus 5.
 * mix64 is the splitmix64 output function (Steele, Lea, Flood 2014). */
static uint64_t h_seed = 1;
static int h_mod = 3;

static uint64_t h_mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static constexpr uint64_t H_GAMMA = 0x9e3779b97f4a7c15ULL;
static constexpr uint64_t H_STM_KEY = 0xd1b54a32d192ed03ULL;

/* ---- table-formula stub ----------------------------------------------
 * The value a synthetic table of the engine stores for the position:
 * VALS[mix64(seed ^ idx ^ bside << 63) % modulus], idx = the reference's own
 * encode_piece (probe.c:603-699) of the position under the table's piece
 * layout (the kings; unless only the kings are unique, the first other
 * unique piece in piece order; then the rest in piece order), bside/flip as
 * probe_table chooses them for a table of the position's own material
 * (probe.c:1554-1580).  Used to pin capture classification through tables. */
size_t set_enc_info(struct EncInfo *ei, struct BaseEntry *be, const uint8_t *tb, int shift,
                    int fr, const int enc);
static int h_table_mode = 0;

static int table_formula_wdl(Position *pos)
{
  static const int order[16] = { 0, 0, 3, 5, 7, 9, 1, 0, 0, 0, 4, 6, 8, 10, 2, 0 };
  int n = pos->num, cnt[16] = { 0 };
  uint8_t pt[8];
  for (int i = 0; i < n; i++) {
    pt[i] = pos->pt[i];
    cnt[pos->pt[i]]++;
  }
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (order[pt[i]] > order[pt[j]]) {
        uint8_t t = pt[i];
        pt[i] = pt[j];
        pt[j] = t;
      }
  int uniq = 0;
  for (int i = 0; i < 16; i++) uniq += cnt[i] == 1;
  bool symmetric = true;
  for (int t = 1; t <= 6; t++) symmetric = symmetric && cnt[t] == cnt[t + 8];
  uint8_t table[8], used[8] = { 0 };
  int k = 0;
  table[k++] = 6;
  table[k++] = 14;
  used[0] = used[1] = 1;
  if (uniq != 2)
    for (int i = 2; i < n; i++)
      if (cnt[pt[i]] == 1) {
        table[k++] = pt[i];
        used[i] = 1;
        break;
      }
  for (int i = 2; i < n; i++)
    if (!used[i]) table[k++] = pt[i];
  uint8_t hdr[9] = { 0 };
  for (int i = 0; i < n; i++) hdr[1 + i] = table[i] | (table[i] << 4);
  struct BaseEntry be;
  memset(&be, 0, sizeof be);
  be.num = n;
  be.kk_enc = uniq == 2;
  be.symmetric = symmetric;
  struct EncInfo ei;
  memset(&ei, 0, sizeof ei);
  set_enc_info(&ei, &be, hdr, 0, 0, PIECE_ENC);
  bool flip = symmetric ? pos->stm != WHITE : false;
  int bside = symmetric ? 0 : pos->stm == BLACK;
  uint8_t p[8] = { 0 };
  for (int i = 0; i < n;) {
    int t = ei.pieces[i] ^ (flip << 3);
    for (int j = 0; j < n; j++)
      if (pos->pt[j] == t) p[i++] = pos->sq[j] ^ (flip ? 0x38 : 0x00);
  }
  uint64_t idx = encode_piece(p, &ei, &be);
  uint64_t h = h_mix64(h_seed ^ idx ^ ((uint64_t)bside << 63));
  if (h_mod == 5) return (int)(h % 5) - 2;
  return (int)(h % 3) * 2 - 2;
}

void ref_set_stub_table(uint64_t seed, int modulus)
{
  h_seed = seed;
  h_mod = modulus == 5 ? 5 : 3;
  h_table_mode = 1;
}

int harness_probe_wdl(Position *pos, int alpha, int beta)
{
  (void)alpha;
  (void)beta;
  if (pos->num == 2) return 0;  /* KvK, as probe_table (probe.c:1525) */
  if (h_table_mode) return table_formula_wdl(pos);
  uint64_t key = pos->stm ? H_STM_KEY : 0;
  for (int i = 0; i < pos->num; i++)
    key ^= h_mix64((((uint64_t)pos->pt[i] << 6) | pos->sq[i]) * H_GAMMA
                   + H_GAMMA);
  uint64_t h = h_mix64(h_seed ^ key);
  if (h_mod == 5)
    return (int)(h % 5) - 2;
  static const int v3[3] = { -2, 0, 2 };
  return v3[h % 3];
}

void ref_set_stub(uint64_t seed, int modulus)
{
  h_seed = seed;
  h_mod = modulus == 5 ? 5 : 3;
  h_table_mode = 0;
}

/* ---- set-up ------------------------------------------------------------ */
static bool h_global_init = false;

/* Restates tb8gen.c:1280-1385 for one material; returns 0 or -1. */
int ref_setup(const char *material, int nthreads)
{
  if (!h_global_init) {
    init_indices();
    init_movegen();
    init_tables();
    g_num_threads = nthreads < 1 ? 1 : nthreads;
    init_threads();
    h_global_init = true;
  }
  g_total_work = g_num_threads > 1 ? g_num_threads : 1;

  uint8_t cnt[16] = { 0 }, pt[8];
  int color = 0, k = 0;
  for (const char *c = material; *c; c++) {
    if (*c == 'v' && !color) {
      color = 8;
      continue;
    }
    for (int i = PAWN; i <= KING; i++)
      if (*c == PieceChar[i]) {
        if (k >= 8) return -1;
        cnt[i | color]++;
        pt[k++] = i | color;
        break;
      }
  }
  if (!color || k < 3 || cnt[WKING] != 1 || cnt[BKING] != 1
      || cnt[WPAWN] || cnt[BPAWN])
    return -1;

  static const int order[16] = { 0, 0, 3, 5, 7, 9, 1, 0,
                                 0, 0, 4, 6, 8, 10, 2, 0 };
  for (int i = 0; i < k; i++)
    for (int j = i + 1; j < k; j++)
      if (order[pt[i]] > order[pt[j]]) {
        uint8_t t = pt[i]; pt[i] = pt[j]; pt[j] = t;
      }

  memset(&g_pos, 0, sizeof g_pos);
  g_pos.num = k;
  for (int i = 0; i < k; i++)
    g_pos.pt[i] = pt[i];
  int w = 0, b = 0;
  for (int i = 0; i < k; i++) {
    if (pt[i] & 8) g_pos.pcs[BLACK][b++] = i;
    else g_pos.pcs[WHITE][w++] = i;
  }
  g_pos.pcs[WHITE][w] = -1;
  g_pos.pcs[BLACK][b] = -1;

  memset(&ii, 0, sizeof ii);
  int nsets = 0;
  for (int i = 2; i < k;) {
    int j = i;
    while (i < k && pt[i] == pt[j]) pc_to_set[i++] = nsets;
    ii.first[nsets] = j;
    ii.mult[nsets] = i - j;
    ii.last[nsets] = i - 1;
    nsets++;
  }
  ii.numsets = nsets;
  calc_factors(&ii);
  kslice_size = ii.size;
  for (int s = 0; s < nsets; s++) {
    capt_ii[s] = ii;
    capt_ii[s].mult[s]--;
    calc_factors(&capt_ii[s]);
    kslice_sub_size[s] = capt_ii[s].size;
  }

  free(work_g);
  work_g = create_work(g_total_work, kslice_size, 0x1ff);
  for (int s = 0; s < MAX_SETS; s++) {
    free(work_capt[s]);
    work_capt[s] = s < nsets
        ? create_work(g_total_work, capt_ii[s].size, 0x1ff) : nullptr;
  }

  /* kslice_setup (kslice.c:98-127) without the buffer allocations. */
  init_kslice_manager();
  kslice_cache_lines = bits_to_aligned(kslice_size) >> 6;
  free(work_cl);
  free(work_clc);
  work_cl = create_work(g_total_work, kslice_cache_lines, 0);
  work_clc = create_work(g_total_work, kslice_cache_lines - 1, 0);
  sub_size[0] = sub_size[1] = 0;
  for (int s = 0; s < nsets; s++) {
    int c = g_pos.pt[ii.first[s]] >> 3;
    sub_offset[s] = sub_size[c];
    sub_size[c] += bits_to_aligned(kslice_sub_size[s]);
  }
  for (int c = 0; c < 2; c++) {
    free(work_sub_cl[c]);
    work_sub_cl[c] = create_work(g_total_work, sub_size[c] >> 6, 0);
  }
  for (int i = 0; i < 20; i++) kslice_buf[i] = nullptr;
  for (int i = 0; i < 19; i++) {
    kslice_sub_buf[i] = nullptr;
    kslice_in_use[i] = false;
  }
  kslice_slot[0] = 19;
  for (int s = 0; s < 462; s++) kslice_slot[s + 1] = -1;
  return 0;
}

/* ---- slot binding (mirrors kslice_reserve/kslice_release) --------------- */
void ref_unbind_all(void)
{
  for (int s = 0; s < 462; s++)
    if (kslice_slot[s + 1] >= 0) kslice_release(s);
  kslice_buf[19] = nullptr;
}

/* Bind caller memory to slice s (-1 = the scratch slot, buffer 19). */
int ref_bind(int s, void *bitmap, void *sub)
{
  if (s == -1) {
    kslice_buf[19] = bitmap;
    return 0;
  }
  if (s < 0 || s >= 462 || kslice_slot[s + 1] >= 0) return -1;
  for (int i = 0; i < 19; i++)
    if (!kslice_in_use[i]) {
      kslice_reserve(s);
      int slot = kslice_slot[s + 1];
      kslice_buf[slot] = bitmap;
      kslice_sub_buf[slot] = sub;
      return 0;
    }
  return -1;
}

/* ---- the workers -------------------------------------------------------- */
void ref_predecessors(int stm, int s) { predecessors(stm, s); }

void ref_predecessors_sub(int stm, int s, int legality)
{
  predecessors_sub(stm, s, legality != 0);
}

void ref_check_successors(int stm, int s) { check_successors(stm, s); }

/* calc_sub_kslices (tb8gen.c:317-342) for one slice, into caller buffers
 * cls[0..4] = loss, bloss, draw, cwin, win (each sub_size[stm] bytes). */
void ref_calc_sub(int stm, int s, void *const cls[5])
{
  uint8_t *saved[5];
  for (int i = 0; i < 5; i++) {
    saved[i] = kslice_sub_buf[i];
    kslice_sub_buf[i] = cls[i];
  }
  g_pos.stm = stm;
  g_pos.sq[0] = KKSquare[s][0];
  g_pos.sq[1] = KKSquare[s][1];
  for (int k = 0; k < ii.numsets; k++) {
    if ((g_pos.pt[ii.first[k]] >> 3) != stm) continue;
    work_set = k;
    run_threaded(calc_sub_worker, work_capt[k], 0);
  }
  for (int i = 0; i < 5; i++) kslice_sub_buf[i] = saved[i];
}

/* Illegal-position masks of calc_illegal_and_mate (tb8gen.c:734-745). */
void ref_calc_illegal(int s, void *illegal_w, void *illegal_b)
{
  uint8_t *saved0 = kslice_buf[0], *saved1 = kslice_buf[1];
  kslice_buf[0] = illegal_w;
  kslice_buf[1] = illegal_b;
  g_pos.sq[0] = KKSquare[s][0];
  g_pos.sq[1] = KKSquare[s][1];
  kslice_clear_addr(kslice_buf[0]);
  kslice_clear_addr(kslice_buf[1]);
  for (int k = 0; k < ii.numsets; k++) {
    work_set = k;
    run_threaded(calc_illegal_worker, work_capt[k], 0);
  }
  kslice_buf[0] = saved0;
  kslice_buf[1] = saved1;
}

/* Mate (L0) step of calc_illegal_and_mate (tb8gen.c:752-758). */
void ref_calc_mate(int s, void *illegal_w, void *illegal_b, void *mate_w,
                   void *mate_b)
{
  uint8_t *saved[4];
  void *bufs[4] = { illegal_w, illegal_b, mate_w, mate_b };
  for (int i = 0; i < 4; i++) {
    saved[i] = kslice_buf[i];
    kslice_buf[i] = bufs[i];
  }
  g_pos.sq[0] = KKSquare[s][0];
  g_pos.sq[1] = KKSquare[s][1];
  kslice_clear_addr(kslice_buf[2]);
  kslice_clear_addr(kslice_buf[3]);
  run_threaded(calc_mate_worker, work_g, 0);
  for (int i = 0; i < 4; i++) kslice_buf[i] = saved[i];
}

/* W-step epilogue of calc_W_n (tb8gen.c:1072-1077):
 * T &= ~wins; cnt = count(T); wins |= T. */
uint64_t ref_epilogue_W(void *T, void *wins)
{
  work_p = T;
  work_q = wins;
  run_threaded(and_not_worker, work_cl, 0);
  uint64_t cnt = kslice_count_addr(T);
  work_p = wins;
  work_q = T;
  run_threaded(or_worker, work_cl, 0);
  return cnt;
}

uint64_t ref_count(void *p) { return kslice_count_addr(p); }

/* kslice_sub_and_not (kslice.c:481-487) on explicit buffers. */
void ref_sub_and_not(int stm, void *p, void *q)
{
  work_p = p;
  work_q = q;
  run_threaded(and_not_worker, work_sub_cl[stm], 0);
}

/* ---- read-only views of the reference's tables, for pinning ------------ */
uint64_t ref_kslice_size(void) { return kslice_size; }
uint64_t ref_kslice_bytes(void) { return kslice_cache_lines << 6; }
uint64_t ref_sub_size(int stm) { return sub_size[stm]; }
uint64_t ref_sub_offset(int k) { return sub_offset[k]; }
uint64_t ref_capt_size(int k) { return capt_ii[k].size; }
int ref_numsets(void) { return ii.numsets; }
int ref_num_threads(void) { return g_num_threads; }
int ref_kksquare(int s, int i) { return KKSquare[s][i]; }
int ref_kkmap(int a, int b) { return KKMap[a][b]; }
int ref_kkidx(int t, int sq) { return KKIdx[t][sq]; }
int ref_fliptest(int a, int b) { return FlipTest[a][b]; }
int ref_mirrormask(int sq) { return MirrorMask[sq]; }
int ref_pc_to_set(int i) { return pc_to_set[i]; }
int ref_piece_type(int i) { return g_pos.pt[i]; }
uint64_t ref_binomial(int k, int n) { return Binomial[k][n]; }
uint64_t ref_rook_attacks(int sq, uint64_t occ) { return rook_attacks(sq, occ); }
uint64_t ref_bishop_attacks(int sq, uint64_t occ)
{
  return bishop_attacks(sq, occ);
}
uint64_t ref_knight_attacks(int sq) { return knight_attacks(sq); }
uint64_t ref_king_attacks(int sq) { return king_attacks(sq); }

/* Index views: sq_to_idx_helper (tb8gen.c:129-149) and its inverse
 * (tb8gen.c:161-180) on the main IdxInfo or capture IdxInfo k (k >= 0). */
uint64_t ref_sq_to_idx(const uint8_t *sq8, int k)
{
  uint8_t tmp[8];
  memcpy(tmp, sq8, 8);
  return k < 0 ? sq_to_idx(tmp) : capt_sq_to_idx(tmp, k);
}

uint64_t ref_idx_to_sq(uint64_t idx, int s, int k, uint8_t *sq8)
{
  uint32_t sub[MAX_SETS];
  struct IdxInfo *info = k < 0 ? &ii : &capt_ii[k];
  memset(sq8, 0xff, 8);
  sq8[0] = KKSquare[s][0];
  sq8[1] = KKSquare[s][1];
  idx_to_sq_init(idx, sub, info);
  return idx_to_sq_unpack(sub, sq8, info);
}

/* Manager schedule (kslice.c:41-84): writes in[] and out[] (-1 ended). */
int ref_manager(int stm, int i, int16_t *in, int16_t *out)
{
  struct KSliceManager *m = kslice_get_manager(stm, i);
  memcpy(in, m->in, sizeof m->in);
  memcpy(out, m->out, sizeof m->out);
  return m->kslice;
}
