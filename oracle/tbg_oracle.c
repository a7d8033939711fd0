/*
 * Oracle test infrastructure -- NOT product code.  See tbg_oracle.h.
 *
 * Single-threaded restatement of the reference's ply-step workers.  Attack
 * sets are computed by walking rays (the reference uses fixed-shift magic
 * tables, magic.h:23-38); the KKIdx table is generated from its defining
 * rule rather than transcribed.  Both are pinned exhaustively against the
 * reference in tests/test_oracle_pin.py.
 */
#include "tbg_oracle.h"

#include <stdbool.h>
#include <string.h>

typedef uint64_t bb_t;

static inline bb_t bit(int sq) { return 1ULL << sq; }
static inline int lsb(bb_t b) { return __builtin_ctzll(b); }
static inline int popcnt(bb_t b) { return __builtin_popcountll(b); }
static inline int pop_lsb(bb_t *b)
{
  int s = lsb(*b);
  *b &= *b - 1;
  return s;
}

/* ---------------------------------------------------------------- tables */

static uint64_t Bin[8][64];          /* Bin[k][n] = C(n,k), probe.c:541-546 */
static int16_t KKIdx_[10][64];       /* probe.c:441-522 */
static uint8_t KKSq[462][2];         /* probe.c:534-539 */
static uint8_t TriIdx[64];           /* Triangle, probe.c:310-319 */
static uint8_t Flip[64];             /* FlipDiag, probe.c:331-340 */
static uint8_t Mirror[64];           /* MirrorMask, tb8gen.c:75-76 */
static bool FlipT[64][64];           /* FlipTest, tb8gen.c:78-88 */
static int16_t KKMap_[64][64];       /* KKMap, tb8gen.c:78-88 */
static bb_t KingAtt[64], KnightAtt[64];
static int16_t Mgr[2][462][23];      /* kslice_get_manager: kslice, in[11], out[11] */
static bool tables_ready = false;

/* Canonical squares of the a1-d1-d4 triangle: off-diagonal ones first, then
 * the diagonal, each in square order (InvTriangle, probe.c:327-329). */
static const uint8_t TriSq[10] = { 1, 2, 3, 10, 11, 19, 0, 9, 18, 27 };

static int file_of(int sq) { return sq & 7; }
static int rank_of(int sq) { return sq >> 3; }

static bool adjacent_or_same(int a, int b)
{
  int df = file_of(a) - file_of(b), dr = rank_of(a) - rank_of(b);
  return df >= -1 && df <= 1 && dr >= -1 && dr <= 1;
}

static bb_t step_attacks(int sq, const int (*d)[2], int n)
{
  bb_t b = 0;
  for (int i = 0; i < n; i++) {
    int f = file_of(sq) + d[i][0], r = rank_of(sq) + d[i][1];
    if (f >= 0 && f < 8 && r >= 0 && r < 8) b |= bit(r * 8 + f);
  }
  return b;
}

static bb_t ray_attacks(int sq, bb_t occ, const int (*d)[2])
{
  bb_t b = 0;
  for (int i = 0; i < 4; i++) {
    int f = file_of(sq), r = rank_of(sq);
    for (;;) {
      f += d[i][0];
      r += d[i][1];
      if (f < 0 || f > 7 || r < 0 || r > 7) break;
      b |= bit(r * 8 + f);
      if (occ & bit(r * 8 + f)) break;
    }
  }
  return b;
}

static const int RookDir[4][2] = { { 1, 0 }, { -1, 0 }, { 0, 1 }, { 0, -1 } };
static const int BishopDir[4][2] = { { 1, 1 }, { -1, 1 }, { 1, -1 }, { -1, -1 } };

uint64_t orc_rook_attacks(int sq, uint64_t occ)
{
  return ray_attacks(sq, occ, RookDir);
}

uint64_t orc_bishop_attacks(int sq, uint64_t occ)
{
  return ray_attacks(sq, occ, BishopDir);
}

/* non_king_piece_attacks / piece_attacks, movegen.h:79-117 (types 2..6). */
static bb_t piece_attacks(int pt, int sq, bb_t occ)
{
  switch (pt & 7) {
  case 2: return KnightAtt[sq];
  case 3: return orc_bishop_attacks(sq, occ);
  case 4: return orc_rook_attacks(sq, occ);
  case 5: return orc_rook_attacks(sq, occ) | orc_bishop_attacks(sq, occ);
  default: return KingAtt[sq];
  }
}

int orc_init(void)
{
  if (tables_ready) return 0;
  static const int kd[8][2] = { { 1, 0 }, { -1, 0 }, { 0, 1 }, { 0, -1 },
                                { 1, 1 }, { -1, 1 }, { 1, -1 }, { -1, -1 } };
  static const int nd[8][2] = { { 1, 2 }, { 2, 1 }, { -1, 2 }, { -2, 1 },
                                { 1, -2 }, { 2, -1 }, { -1, -2 }, { -2, -1 } };
  for (int sq = 0; sq < 64; sq++) {
    KingAtt[sq] = step_attacks(sq, kd, 8);
    KnightAtt[sq] = step_attacks(sq, nd, 8);
    Flip[sq] = (uint8_t)((file_of(sq) << 3) | rank_of(sq));
    Mirror[sq] = (uint8_t)((file_of(sq) >= 4 ? 0x07 : 0) | (rank_of(sq) >= 4 ? 0x38 : 0));
    /* Triangle: fold the square into a1-d1-d4 by the board symmetries. */
    int f = file_of(sq), r = rank_of(sq);
    if (f > 3) f = 7 - f;
    if (r > 3) r = 7 - r;
    if (r > f) { int t = r; r = f; f = t; }
    for (int t = 0; t < 10; t++)
      if (TriSq[t] == r * 8 + f) TriIdx[sq] = (uint8_t)t;
  }

  for (int k = 0; k < 8; k++)
    for (int n = 0; n < 64; n++) {
      if (k == 0) Bin[k][n] = 1;
      else if (n == 0) Bin[k][n] = 0;
      else Bin[k][n] = Bin[k - 1][n - 1] + Bin[k][n - 1];
    }

  /* KKIdx: legal (non-touching) king pairs, white king on the triangle.
   * With the white king on the a1-d4 diagonal only black-king squares on or
   * below that diagonal (file >= rank) are kept; the pairs with both kings on
   * the diagonal are numbered last, from 441, in the same scan order. */
  int next = 0, next_diag = 441;
  for (int t = 0; t < 10; t++)
    for (int sq = 0; sq < 64; sq++) {
      int wk = TriSq[t];
      KKIdx_[t][sq] = -1;
      if (adjacent_or_same(wk, sq)) continue;
      if (t >= 6) {
        if (file_of(sq) < rank_of(sq)) continue;
        if (file_of(sq) == rank_of(sq)) {
          KKIdx_[t][sq] = (int16_t)next_diag++;
          continue;
        }
      }
      KKIdx_[t][sq] = (int16_t)next++;
    }
  if (next != 441 || next_diag != 462) return -1;
  for (int t = 0; t < 10; t++)
    for (int sq = 0; sq < 64; sq++)
      if (KKIdx_[t][sq] >= 0) {
        KKSq[KKIdx_[t][sq]][0] = TriSq[t];
        KKSq[KKIdx_[t][sq]][1] = (uint8_t)sq;
      }

  /* FlipTest / KKMap (tb8gen.c:69-89). */
  for (int i = 0; i < 64; i++)
    for (int j = 0; j < 64; j++) {
      int s1 = i ^ Mirror[i], s2 = j ^ Mirror[i];
      bool in_tri = file_of(s1) <= 3 && rank_of(s1) <= file_of(s1);
      bool on_diag = in_tri && file_of(s1) == rank_of(s1);
      bool s2_lower = file_of(s2) >= rank_of(s2);
      FlipT[i][j] = !in_tri || (on_diag && !s2_lower);
      if (FlipT[i][j]) {
        s1 = Flip[s1];
        s2 = Flip[s2];
      }
      KKMap_[i][j] = KKIdx_[TriIdx[s1]][s2];
    }

  /* Manager schedule, kslice.c:41-84. */
  int s = 0;
  bb_t loaded = 0;
  for (int t = 0; t < 10; t++) {
    for (int bk = 0; bk < 64; bk++) {
      if (KKIdx_[t][bk] < 0) continue;
      int16_t *m = Mgr[1][s];
      m[0] = KKIdx_[t][bk];
      int j = 0;
      bb_t b = (bit(bk) | KingAtt[bk]) & ~loaded;
      while (b) {
        int sq = pop_lsb(&b);
        if (KKIdx_[t][sq] >= 0) {
          m[1 + j++] = KKIdx_[t][sq];
          loaded |= bit(sq);
        }
      }
      m[1 + j] = -1;
      b = bk == 63 ? loaded : bk >= 9 ? (loaded & (bit(bk - 8) - 1)) : 0;
      j = 0;
      while (b) {
        int sq = pop_lsb(&b);
        m[12 + j++] = KKIdx_[t][sq];
        loaded ^= bit(sq);
      }
      m[12 + j] = -1;
      s++;
    }
  }
  for (int i = 0; i < 462; i++) {
    for (int j = 0; j < 23; j++) {
      int16_t x = Mgr[1][i][j];
      Mgr[0][i][j] = x < 0 ? x : KKMap_[KKSq[x][1]][KKSq[x][0]];
    }
  }
  tables_ready = true;
  return 0;
}

int orc_kkidx(int t, int sq) { return KKIdx_[t][sq]; }
int orc_kkmap(int a, int b) { return KKMap_[a][b]; }
int orc_kksquare(int s, int i) { return KKSq[s][i]; }
int orc_fliptest(int a, int b) { return FlipT[a][b]; }

int orc_manager(int stm, int i, int16_t *in, int16_t *out)
{
  for (int j = 0; j < 11; j++) {
    in[j] = Mgr[stm][i][1 + j];
    out[j] = Mgr[stm][i][12 + j];
  }
  return Mgr[stm][i][0];
}

/* ------------------------------------------------------------ material */

/* subfactor, probe.c:715-723 */
static uint64_t placements(uint64_t k, uint64_t n)
{
  uint64_t f = 1;
  for (uint64_t i = 0; i < k; i++) f = f * (n - i) / (i + 1);
  return f;
}

/* calc_factors, tb8gen.c:209-228 (without the +64 guard on subfactor[0],
 * which only protects the reference's incremental carry). */
static void set_factors(orc_idx *x)
{
  for (int i = 0, n = 62; i < x->numsets; i++) {
    x->subfactor[i] = (uint32_t)placements(x->mult[i], n);
    n -= x->mult[i];
  }
  uint64_t f = 1;
  for (int i = x->numsets - 1; i >= 0; i--) {
    x->factor[i] = f;
    f *= x->subfactor[i];
  }
  x->size = f;
}

static uint64_t rounded_bytes(uint64_t bits)
{
  return (((bits + 7) >> 3) + 63) & ~(uint64_t)63;
}

/* Material set-up of main(), tb8gen.c:1284-1385. */
int orc_setup(orc_ctx *c, const char *material)
{
  if (orc_init()) return -1;
  memset(c, 0, sizeof *c);
  c->stub_seed = 1;
  c->stub_mod = 3;
  static const char *letters = "PNBRQK";
  uint8_t pt[8];
  int n = 0, black = 0, kings[2] = { 0, 0 };
  for (const char *p = material; *p; p++) {
    if (*p == 'v' && !black) { black = 8; continue; }
    const char *q = strchr(letters, *p);
    if (!q || !*p) continue;
    int t = (int)(q - letters) + 1;
    if (n >= 8 || t == 1) return -1;
    if (t == 6) kings[black ? 1 : 0]++;
    pt[n++] = (uint8_t)(t | black);
  }
  if (!black || n < 3 || kings[0] != 1 || kings[1] != 1) return -1;
  /* piece_order, tb8gen.c:1331-1339: kings, then N < B < R < Q, white
   * before black within a type. */
  static const int order[16] = { 0, 0, 3, 5, 7, 9, 1, 0, 0, 0, 4, 6, 8, 10, 2, 0 };
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (order[pt[i]] > order[pt[j]]) { uint8_t t = pt[i]; pt[i] = pt[j]; pt[j] = t; }
  c->num = n;
  memcpy(c->pt, pt, (size_t)n);
  int nw = 0, nb = 0;
  for (int i = 0; i < n; i++) {
    if (pt[i] & 8) c->pcs[1][nb++] = (int8_t)i;
    else c->pcs[0][nw++] = (int8_t)i;
  }
  c->pcs[0][nw] = -1;
  c->pcs[1][nb] = -1;
  int k = 0;
  for (int i = 2; i < n;) {
    int j = i;
    while (i < n && pt[i] == pt[j]) c->pc_to_set[i++] = k;
    c->ii.first[k] = j;
    c->ii.mult[k] = i - j;
    c->ii.last[k] = i - 1;
    k++;
  }
  c->ii.numsets = k;
  set_factors(&c->ii);
  c->bytes = rounded_bytes(c->ii.size);
  for (int s = 0; s < k; s++) {
    c->capt[s] = c->ii;
    c->capt[s].mult[s]--;
    set_factors(&c->capt[s]);
    int col = pt[c->ii.first[s]] >> 3;
    c->sub_offset[s] = c->sub_size[col];
    c->sub_size[col] += rounded_bytes(c->capt[s].size);
  }
  c->sub_bytes = c->sub_size[0] > c->sub_size[1] ? c->sub_size[0] : c->sub_size[1];
  return 0;
}

void orc_bind(orc_ctx *c, int s, void *bitmap, void *sub)
{
  c->slot[s + 1] = bitmap;
  c->sub[s + 1] = sub;
}

void orc_unbind_all(orc_ctx *c)
{
  for (int i = 0; i < 463; i++) c->slot[i] = c->sub[i] = NULL;
}

/* ------------------------------------------------------------ indexing */

/* sq_to_idx_helper, tb8gen.c:129-149: per set, the squares sorted, ranked
 * among the squares not taken by the kings and the earlier sets, combined
 * in the combinatorial number system; the last set varies fastest. */
static uint64_t rank_position(const orc_idx *x, const uint8_t *sq)
{
  uint64_t idx = 0;
  bb_t occ = bit(sq[0]) | bit(sq[1]);
  for (int k = 0; k < x->numsets; k++) {
    uint8_t v[8];
    int m = x->mult[k];
    memcpy(v, sq + x->first[k], (size_t)m);
    for (int i = 1; i < m; i++)
      for (int j = i; j > 0 && v[j - 1] > v[j]; j--) {
        uint8_t t = v[j]; v[j] = v[j - 1]; v[j - 1] = t;
      }
    uint64_t s = 0;
    bb_t occ2 = occ;
    for (int j = 0; j < m; j++) {
      int r = v[j] - popcnt(occ & (bit(v[j]) - 1));
      s += Bin[j + 1][r];
      occ2 |= bit(v[j]);
    }
    idx += s * x->factor[k];
    occ = occ2;
  }
  return idx;
}

/* idx_to_sq_init + unrank_binomial, tb8gen.c:105-126, 161-180.  Writes the
 * squares of the sets into sq (kings must already be there); returns the
 * occupancy. */
static bb_t unrank_position(const orc_idx *x, uint64_t idx, uint8_t *sq)
{
  bb_t occ = bit(sq[0]) | bit(sq[1]);
  for (int k = 0; k < x->numsets; k++) {
    uint64_t d = idx / x->factor[k];
    idx -= d * x->factor[k];
    int m = x->mult[k];
    bb_t freeb = ~occ;
    for (int i = m - 1; i >= 0; i--) {
      int r;
      if (i > 0) {
        r = i;
        while (d >= Bin[i + 1][r + 1]) r++;
        d -= Bin[i + 1][r];
      } else {
        r = (int)d;
      }
      bb_t b = freeb;
      for (int t = 0; t < r; t++) b &= b - 1;
      int s = lsb(b);
      sq[x->first[k] + i] = (uint8_t)s;
      occ |= bit(s);
    }
  }
  return occ;
}

uint64_t orc_sq_to_idx(orc_ctx *c, const uint8_t *sq8, int k)
{
  return rank_position(k < 0 ? &c->ii : &c->capt[k], sq8);
}

uint64_t orc_idx_to_sq(orc_ctx *c, uint64_t idx, int s, int k, uint8_t *sq8)
{
  memset(sq8, 0xff, 8);
  sq8[0] = KKSq[s][0];
  sq8[1] = KKSq[s][1];
  return unrank_position(k < 0 ? &c->ii : &c->capt[k], idx, sq8);
}

/* normalize, tb8gen.c:230-238 */
static void normalize(const uint8_t *sq, uint8_t *out)
{
  int m = Mirror[sq[0]];
  bool f = FlipT[sq[0]][sq[1]];
  for (int i = 0; i < 8; i++) {
    int t = sq[i] ^ m;
    out[i] = f ? Flip[t] : (uint8_t)t;
  }
}

/* is_attacked_by, movegen.h:180-188, over pieces 0..num-1 with types pt. */
static bool attacked_by(const uint8_t *pt, const uint8_t *sq, int num, bb_t occ,
                        int target, int color)
{
  for (int i = 0; i < num; i++)
    if ((pt[i] >> 3) == color && (piece_attacks(pt[i], sq[i], occ) & bit(target)))
      return true;
  return false;
}

static inline void set_bit(uint8_t *p, uint64_t idx)
{
  p[idx >> 3] |= (uint8_t)(1u << (idx & 7));
}

static inline bool test_bit(const uint8_t *p, uint64_t idx)
{
  return (p[idx >> 3] >> (idx & 7)) & 1;
}

/* ----------------------------------------------------------- W step */

/* mark_king_unmoves, tb8gen.c:246-262 */
static void mark_king_unmoves(orc_ctx *c, int stm, bb_t occ, uint8_t *sq, int s)
{
  uint8_t sq2[8];
  bb_t b = KingAtt[sq[stm]] & ~(occ | KingAtt[sq[stm ^ 1]]);
  while (b) {
    sq[stm] = (uint8_t)pop_lsb(&b);
    normalize(sq, sq2);
    int s2 = KKMap_[sq2[0]][sq2[1]];
    uint8_t *p = c->slot[s2 + 1];
    set_bit(p, rank_position(&c->ii, sq2));
    if (s < 441 && s2 >= 441) {
      for (int i = 2; i < 8; i++) sq2[i] = Flip[sq2[i]];
      set_bit(p, rank_position(&c->ii, sq2));
    }
  }
}

/* mark_unmoves, tb8gen.c:264-276 */
static void mark_unmoves(orc_ctx *c, int j, uint8_t *p, bb_t occ, uint8_t *sq)
{
  bb_t b = piece_attacks(c->pt[j], sq[j], occ) & ~occ;
  while (b) {
    sq[j] = (uint8_t)pop_lsb(&b);
    set_bit(p, rank_position(&c->ii, sq));
  }
}

/* predecessors_worker / predecessors, tb8gen.c:484-527: every set bit of
 * the scratch slot (opponent to move) is unmoved by the side stm. */
void orc_predecessors(orc_ctx *c, int stm, int s)
{
  const uint64_t *src = (const uint64_t *)c->slot[0];
  uint8_t *self = c->slot[s + 1];
  uint64_t n = c->ii.size;
  for (uint64_t w = 0; w * 64 < n; w++) {
    uint64_t word = src[w];
    while (word) {
      uint64_t idx = w * 64 + (uint64_t)pop_lsb(&word);
      if (idx >= n) break;
      uint8_t sq[8];
      memset(sq, 0, 8);
      sq[0] = KKSq[s][0];
      sq[1] = KKSq[s][1];
      bb_t occ = unrank_position(&c->ii, idx, sq);
      uint8_t keep = sq[stm];
      mark_king_unmoves(c, stm, occ, sq, s);
      sq[stm] = keep;
      for (int i = 1; c->pcs[stm][i] >= 0; i++) {
        int j = c->pcs[stm][i];
        uint8_t t = sq[j];
        mark_unmoves(c, j, self, occ, sq);
        sq[j] = t;
      }
    }
  }
}

/* predecessors_sub_worker / predecessors_sub, tb8gen.c:346-414: uncaptures
 * into stm positions from the sub bitmaps of the sets of colour stm^1. */
void orc_predecessors_sub(orc_ctx *c, int stm, int s, int legality)
{
  uint8_t *self = c->slot[s + 1];
  int n = c->num - 1;
  for (int k = 0; k < c->ii.numsets; k++) {
    int m = c->ii.last[k];
    if ((c->pt[m] >> 3) == stm) continue;
    const orc_idx *x = &c->capt[k];
    const uint64_t *src = (const uint64_t *)(c->sub[s + 1] + c->sub_offset[k]);
    uint8_t pt7[8];
    memcpy(pt7, c->pt, 8);
    pt7[m] = c->pt[n];
    for (uint64_t w = 0; w * 64 < x->size; w++) {
      uint64_t word = src[w];
      while (word) {
        uint64_t idx = w * 64 + (uint64_t)pop_lsb(&word);
        if (idx >= x->size) break;
        uint8_t sq[8];
        memset(sq, 0, 8);
        sq[0] = KKSq[s][0];
        sq[1] = KKSq[s][1];
        bb_t occ = unrank_position(x, idx, sq);
        if (legality) {
          sq[m] = sq[n];
          if (attacked_by(pt7, sq, n, occ, sq[stm], stm ^ 1)) continue;
        }
        sq[m] = sq[stm];
        uint8_t keep = sq[stm];
        mark_king_unmoves(c, stm, occ, sq, s);
        sq[stm] = keep;
        for (int i = 1; c->pcs[stm][i] >= 0; i++) {
          int j = c->pcs[stm][i];
          sq[m] = sq[j];
          mark_unmoves(c, j, self, occ, sq);
          sq[j] = sq[m];
        }
      }
    }
  }
}

/* ----------------------------------------------------------- L step */

static int piece_on(const uint8_t *sq, int to)
{
  for (int i = 0;; i++)
    if (sq[i] == to) return i;
}

static bool sub_bit(orc_ctx *c, int s, int l, uint64_t idx)
{
  uint64_t byte = c->sub_offset[l] + (idx >> 3);
  if (byte >= c->sub_bytes) {
    c->oob_reads++;
    return false;
  }
  return test_bit(c->sub[s + 1] + c->sub_offset[l], idx);
}

/* check_king_moves, tb8gen.c:537-569.  For a king capture the captured
 * piece stays in its slot (on the king's new square) and the capture index
 * drops the last slot of its set, exactly as the reference computes it. */
static bool check_king_moves(orc_ctx *c, int stm, bb_t occ, uint8_t *sq)
{
  uint8_t sq2[8];
  bb_t b = KingAtt[sq[stm]] & ~KingAtt[sq[stm ^ 1]];
  bb_t caps = b & occ;
  while (caps) {
    int to = pop_lsb(&caps);
    int j = piece_on(sq, to);
    if ((c->pt[j] >> 3) == stm) continue;
    sq[stm] = (uint8_t)to;
    normalize(sq, sq2);
    int l = c->pc_to_set[j];
    int s2 = KKMap_[sq2[0]][sq2[1]];
    if (!sub_bit(c, s2, l, rank_position(&c->capt[l], sq2))) return false;
  }
  b &= ~occ;
  while (b) {
    sq[stm] = (uint8_t)pop_lsb(&b);
    normalize(sq, sq2);
    int s2 = KKMap_[sq2[0]][sq2[1]];
    if (!test_bit(c->slot[s2 + 1], rank_position(&c->ii, sq2))) return false;
  }
  return true;
}

/* check_moves, tb8gen.c:571-605 */
static bool check_moves(orc_ctx *c, int k, int s, const uint8_t *wins, bb_t occ,
                        uint8_t *sq)
{
  uint8_t sq2[8];
  bb_t b = piece_attacks(c->pt[k], sq[k], occ);
  bb_t caps = b & occ;
  while (caps) {
    int to = pop_lsb(&caps);
    int j = piece_on(sq, to);
    if (!((c->pt[k] ^ c->pt[j]) & 8)) continue;
    memcpy(sq2, sq, 8);
    int l = c->pc_to_set[j];
    sq2[k] = (uint8_t)to;
    sq2[j] = sq2[c->ii.last[l]];
    if (!sub_bit(c, s, l, rank_position(&c->capt[l], sq2))) return false;
  }
  b &= ~occ;
  while (b) {
    sq[k] = (uint8_t)pop_lsb(&b);
    if (!test_bit(wins, rank_position(&c->ii, sq))) return false;
  }
  return true;
}

/* check_successors_worker / check_successors, tb8gen.c:607-661: a candidate
 * (scratch slot, stm to move) survives iff it is legal and every move leads
 * to a position won for stm^1 (quiet: "wins" bitmap; capture: sub bitmap). */
void orc_check_successors(orc_ctx *c, int stm, int s)
{
  uint64_t *x = (uint64_t *)c->slot[0];
  const uint8_t *wins = c->slot[s + 1];
  uint64_t n = c->ii.size;
  for (uint64_t w = 0; w * 64 < n; w++) {
    uint64_t word = x[w], keep = word;
    while (word) {
      int bt = pop_lsb(&word);
      uint64_t idx = w * 64 + (uint64_t)bt;
      if (idx >= n) break;
      uint8_t sq[8];
      memset(sq, 0, 8);
      sq[0] = KKSq[s][0];
      sq[1] = KKSq[s][1];
      bb_t occ = unrank_position(&c->ii, idx, sq);
      bool ok = !attacked_by(c->pt, sq, c->num, occ, sq[stm ^ 1], stm);
      for (int i = 1; ok && c->pcs[stm][i] >= 0; i++) {
        int j = c->pcs[stm][i];
        uint8_t t = sq[j];
        ok = check_moves(c, j, s, wins, occ, sq);
        sq[j] = t;
      }
      if (ok) {
        uint8_t t = sq[stm];
        ok = check_king_moves(c, stm, occ, sq);
        sq[stm] = t;
      }
      if (!ok) keep ^= 1ULL << bt;
    }
    x[w] = keep;
  }
}

/* ------------------------------------------------ capture classification */

uint64_t orc_mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

#define GAMMA 0x9e3779b97f4a7c15ULL
#define STM_KEY 0xd1b54a32d192ed03ULL

/* The seeded 7-piece WDL stub that stands in for probe_wdl (probe.c:1677)
 * on both sides: VALS[mix64(seed ^ key7) % modulus], key7 the XOR of
 * mix64(((pt << 6) | sq) * GAMMA + GAMMA) over the pieces, ^ STM_KEY when
 * black is to move. */
int orc_stub_value(uint64_t seed, int modulus, const uint8_t *pt,
                   const uint8_t *sq, int num, int stm)
{
  if (num == 2) return 0;  /* KvK, as probe_table (probe.c:1525) */
  uint64_t key = stm ? STM_KEY : 0;
  for (int i = 0; i < num; i++)
    key ^= orc_mix64((((uint64_t)pt[i] << 6) | sq[i]) * GAMMA + GAMMA);
  uint64_t h = orc_mix64(seed ^ key);
  if (modulus == 5) return (int)(h % 5) - 2;
  return (int)(h % 3) * 2 - 2;
}

/* calc_sub_worker / calc_sub_kslices, tb8gen.c:280-342 for one slice:
 * positions after stm^1 captured a piece of a set of colour stm, stm to
 * move, classified loss/bloss/draw/cwin/win (illegal -> cwin + win). */
void orc_calc_sub(orc_ctx *c, int stm, int s, void *const cls[5])
{
  int n = c->num - 1;
  for (int k = 0; k < c->ii.numsets; k++) {
    int m = c->ii.last[k];
    if ((c->pt[c->ii.first[k]] >> 3) != stm) continue;
    const orc_idx *x = &c->capt[k];
    uint8_t *p[5];
    for (int i = 0; i < 5; i++) {
      p[i] = (uint8_t *)cls[i] + c->sub_offset[k];
      memset(p[i], 0, (x->size + 7) >> 3);
    }
    uint8_t pt7[8];
    memcpy(pt7, c->pt, 8);
    pt7[m] = c->pt[n];
    for (uint64_t idx = 0; idx < x->size; idx++) {
      uint8_t sq[8];
      memset(sq, 0, 8);
      sq[0] = KKSq[s][0];
      sq[1] = KKSq[s][1];
      bb_t occ = unrank_position(x, idx, sq);
      sq[m] = sq[n];
      if (attacked_by(pt7, sq, n, occ, sq[stm ^ 1], stm)) {
        set_bit(p[3], idx);
        set_bit(p[4], idx);
      } else {
        int v = orc_stub_value(c->stub_seed, c->stub_mod, pt7, sq, n, stm);
        set_bit(p[v + 2], idx);
        if (v == 2) set_bit(p[3], idx);
      }
    }
  }
}

/* calc_illegal_worker, tb8gen.c:664-684 with the clears of :738-739:
 * ill[c] marks the positions, c to move, in which a piece of colour c
 * attacks the king of colour c^1. */
void orc_calc_illegal(orc_ctx *c, int s, void *ill_w, void *ill_b)
{
  uint8_t *ill[2] = { ill_w, ill_b };
  memset(ill_w, 0, c->bytes);
  memset(ill_b, 0, c->bytes);
  for (int k = 0; k < c->ii.numsets; k++) {
    int m = c->ii.last[k];
    int col = c->pt[m] >> 3;
    const orc_idx *x = &c->capt[k];
    for (uint64_t idx = 0; idx < x->size; idx++) {
      uint8_t sq[8];
      memset(sq, 0, 8);
      sq[0] = KKSq[s][0];
      sq[1] = KKSq[s][1];
      bb_t occ = unrank_position(x, idx, sq);
      int ksq = sq[col ^ 1];
      sq[m] = (uint8_t)ksq;
      mark_unmoves(c, m, ill[col], occ, sq);
    }
  }
}

/* has_legal_moves / has_legal_caps, movegen.c:75-111, for the pieces of the
 * side to move; a move is legal iff afterwards the mover's king is not
 * attacked by the other side. */
static bool has_legal_move(orc_ctx *c, int stm, const uint8_t *sq0, bb_t occ0)
{
  uint8_t sq[8], pt[8];
  memcpy(sq, sq0, 8);
  memcpy(pt, c->pt, 8);
  int num = c->num;
  for (int i = 0; i < num; i++) {
    if ((pt[i] >> 3) != stm) continue;
    int from = sq[i];
    bb_t b = piece_attacks(pt[i], from, occ0) & ~occ0;
    while (b) {
      int to = pop_lsb(&b);
      bb_t occ = occ0 ^ bit(from) ^ bit(to);
      sq[i] = (uint8_t)to;
      bool ok = !attacked_by(pt, sq, num, occ, sq[stm], stm ^ 1);
      sq[i] = (uint8_t)from;
      if (ok) return true;
    }
  }
  for (int i = 0; i < num; i++) {
    if ((pt[i] >> 3) != stm) continue;
    int from = sq[i];
    bb_t b = piece_attacks(pt[i], from, occ0) & occ0;
    while (b) {
      int to = pop_lsb(&b);
      int j = piece_on(sq, to);
      if (!((pt[i] ^ pt[j]) & 8)) continue;
      /* do_capture, movegen.h:219-234: the last piece takes slot j. */
      uint8_t sq2[8], pt2[8];
      memcpy(sq2, sq, 8);
      memcpy(pt2, pt, 8);
      bb_t occ = occ0 ^ bit(from);
      sq2[i] = (uint8_t)to;
      pt2[j] = pt2[num - 1];
      sq2[j] = sq2[num - 1];
      if (!attacked_by(pt2, sq2, num - 1, occ, sq2[stm], stm ^ 1)) return true;
    }
  }
  return false;
}

/* calc_mate_worker, tb8gen.c:686-727: legal positions (exactly one of the
 * two illegal bitmaps clear) without a legal move or capture. */
void orc_calc_mate(orc_ctx *c, int s, void *ill_w, void *ill_b, void *mate_w,
                   void *mate_b)
{
  const uint64_t *p0 = ill_w, *p1 = ill_b;
  uint64_t *q0 = mate_w, *q1 = mate_b;
  memset(mate_w, 0, c->bytes);
  memset(mate_b, 0, c->bytes);
  uint64_t n = c->ii.size;
  for (uint64_t w = 0; w * 64 < n; w++) {
    uint64_t word = p0[w] ^ p1[w], white = 0, blk = 0;
    while (word) {
      int bt = pop_lsb(&word);
      uint64_t idx = w * 64 + (uint64_t)bt;
      if (idx >= n) break;
      uint8_t sq[8];
      memset(sq, 0, 8);
      sq[0] = KKSq[s][0];
      sq[1] = KKSq[s][1];
      bb_t occ = unrank_position(&c->ii, idx, sq);
      int stm = (p1[w] >> bt) & 1 ? 0 : 1;
      if (!has_legal_move(c, stm, sq, occ)) {
        if (stm == 0) white |= 1ULL << bt;
        else blk |= 1ULL << bt;
      }
    }
    q0[w] = white;
    q1[w] = blk;
  }
}

/* ------------------------------------------------------ bitmap algebra */

/* kslice_and_not + kslice_count + kslice_or, tb8gen.c:1072-1077 */
uint64_t orc_epilogue_W(orc_ctx *c, void *T, void *wins)
{
  uint64_t *t = T, *w = wins;
  for (uint64_t i = 0; i < c->bytes / 8; i++) t[i] &= ~w[i];
  uint64_t cnt = orc_count(c, T);
  for (uint64_t i = 0; i < c->bytes / 8; i++) w[i] |= t[i];
  return cnt;
}

/* kslice_count_addr, kslice.c:389-422: ones below the slice size. */
uint64_t orc_count(orc_ctx *c, const void *p)
{
  const uint64_t *q = p;
  uint64_t n = c->ii.size, cnt = 0;
  for (uint64_t i = 0; i < n / 64; i++) cnt += (uint64_t)popcnt(q[i]);
  if (n & 63) cnt += (uint64_t)popcnt(q[n / 64] & ((1ULL << (n & 63)) - 1));
  return cnt;
}

/* Seeded Bernoulli bitmap: bit i (i < nbits) is set iff the (i+1)-th
 * output of the splitmix64 stream keyed by (seed, tag) is below thr. */
void orc_gen_bernoulli(void *p, uint64_t nbits, uint64_t bytes, uint64_t seed,
                       uint64_t tag, uint64_t thr)
{
  uint64_t key = orc_mix64(orc_mix64(seed + GAMMA) ^ tag);
  uint64_t *q = p;
  memset(p, 0, bytes);
  #pragma omp parallel for schedule(static)
  for (uint64_t w = 0; w < (nbits + 63) / 64; w++) {
    uint64_t word = 0;
    for (int b = 0; b < 64; b++) {
      uint64_t i = w * 64 + (uint64_t)b;
      if (i >= nbits) break;
      if (orc_mix64(key + (i + 1) * GAMMA) < thr) word |= 1ULL << b;
    }
    q[w] = word;
  }
}
