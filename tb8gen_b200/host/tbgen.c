/*
 * tbgen -- the retrograde generation loop of tb8gen (tb8gen.c main,
 * calc_sub_kslices, calc_illegal_and_mate, calc_L_n, calc_W_n) as a C host
 * over the tbgpu C ABI, with every king slice resident in HBM.
 *
 *   tbgen [-s seed] [-m 3|5] [-q] MATERIAL
 *
 * Prints the reference's per-ply counts ("broken_w = ...", "l<n>_<c> = ...",
 * "w<n>_<c> = ...") in the reference's order.  There is no disk tier: each
 * slice's "wins", the previous and current W/L bitmaps of both sides and the
 * capture-class bitmaps stay on the device for the whole run, so the
 * reference's KSliceManager window (kslice.c:41-84) reduces to "all slices
 * bound": the order in which slices are scattered does not change a bitmap
 * (marks are ORed), and every scatter of a half-ply finishes before its
 * epilogue or verify starts, as in the reference.  7-piece capture values
 * come from the seeded stub (tbg_set_stub); a capture that leaves the two
 * kings alone is a draw, as in the reference.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../../include/tbgpu.h"

enum { WHITE = 0, BLACK = 1, NS = 462, DRAW_RULE = 100 };
enum { C_LOSS = 0, C_BLOSS = 1, C_DRAW = 2, C_CWIN = 3, C_WIN = 4 };

static void ok(int rc, const char *what)
{
  if (rc < 0) {
    fprintf(stderr, "tbgen: %s: %s\n", what, tbg_last_error());
    exit(EXIT_FAILURE);
  }
}

static uint64_t g_bytes, g_sub;
/* per side: wins, previous W and L (sources of this ply), current W and L */
static uint8_t *wins[2][NS], *Wp[2][NS], *Lp[2][NS], *Wc[2][NS], *Lc[2][NS];
/* capture classes per side (the side to move after the capture) */
static uint8_t *sub[2][5][NS], *subtmp[NS];
static int quiet;

static void bind_all(uint8_t *bm[NS], uint8_t *sb[NS])
{
  for (int s = 0; s < NS; s++) {
    ok(tbg_slot_bind(s, bm ? bm[s] : NULL, g_bytes), "bind");
    ok(tbg_sub_bind(s, sb ? sb[s] : NULL, g_sub), "bind sub");
  }
}

static void swap_planes(uint8_t *a[NS], uint8_t *b[NS])
{
  for (int s = 0; s < NS; s++) {
    uint8_t *t = a[s];
    a[s] = b[s];
    b[s] = t;
  }
}

/* calc_sub_kslices, tb8gen.c:317-342, for both sides. */
static void calc_subs(void)
{
  for (int stm = 0; stm < 2; stm++)
    for (int s = 0; s < NS; s++) {
      void *cls[5] = { sub[stm][0][s], sub[stm][1][s], sub[stm][2][s], sub[stm][3][s],
                       sub[stm][4][s] };
      ok(tbg_calc_sub(stm, s, cls), "calc_sub");
    }
}

/* calc_illegal_and_mate, tb8gen.c:730-768: wins = illegal, L0 = mates. */
static void illegal_and_mate(void)
{
  uint64_t bw = 0, bb = 0, lw = 0, lb = 0, c;
  for (int s = 0; s < NS; s++) {
    ok(tbg_calc_illegal(s, wins[WHITE][s], wins[BLACK][s]), "illegal");
    ok(tbg_calc_mate(s, wins[WHITE][s], wins[BLACK][s], Lp[WHITE][s], Lp[BLACK][s]), "mate");
  }
  for (int s = 0; s < NS; s++) {
    ok(tbg_slot_bind(0, wins[WHITE][s], g_bytes), "bind");
    ok(tbg_count(0, &c), "count");
    bw += c;
    ok(tbg_slot_bind(0, wins[BLACK][s], g_bytes), "bind");
    ok(tbg_count(0, &c), "count");
    bb += c;
    ok(tbg_slot_bind(0, Lp[WHITE][s], g_bytes), "bind");
    ok(tbg_count(0, &c), "count");
    lw += c;
    ok(tbg_slot_bind(0, Lp[BLACK][s], g_bytes), "bind");
    ok(tbg_count(0, &c), "count");
    lb += c;
  }
  printf("broken_w = %llu\nbroken_b = %llu\nl0_w = %llu\nl0_b = %llu\n",
         (unsigned long long)bw, (unsigned long long)bb, (unsigned long long)lw,
         (unsigned long long)lb);
}

/* calc_L_n, tb8gen.c:943-1026: stm losses in n, into Lc[stm]. */
static int calc_L_n(int stm, int n, int more_l)
{
  uint64_t cnt = 0, c;
  /* candidates: predecessors of stm^1's W(n-1) and of its winning captures */
  bind_all(Lc[stm], NULL);
  for (int s = 0; s < NS; s++) ok(tbg_clear(s), "clear");
  for (int s = 0; s < NS; s++) {
    if (n == 1) {
      ok(tbg_sub_bind(s, sub[stm ^ 1][C_WIN][s], g_sub), "bind sub");
      ok(tbg_predecessors_sub(stm, s, 1), "predecessors_sub");
    } else if (n == DRAW_RULE + 1) {
      /* cwin \ win (tb8gen.c:964-970) */
      ok(tbg_bitmap_and_not(subtmp[s], sub[stm ^ 1][C_CWIN][s], sub[stm ^ 1][C_WIN][s], g_sub),
         "and_not");
      ok(tbg_sub_bind(s, subtmp[s], g_sub), "bind sub");
      ok(tbg_predecessors_sub(stm, s, 0), "predecessors_sub");
    }
    if (more_l && n > 1) {
      ok(tbg_slot_bind(-1, Wp[stm ^ 1][s], g_bytes), "bind");
      ok(tbg_predecessors(stm, s), "predecessors");
    }
  }
  /* verify against stm^1's wins and winning captures */
  int cls = n <= DRAW_RULE ? C_WIN : C_CWIN;
  bind_all(wins[stm ^ 1], sub[stm ^ 1][cls]);
  for (int s = 0; s < NS; s++) {
    ok(tbg_slot_bind(-1, Lc[stm][s], g_bytes), "bind");
    ok(tbg_check_successors(stm, s), "check_successors");
  }
  for (int s = 0; s < NS; s++) {
    ok(tbg_slot_bind(-1, Lc[stm][s], g_bytes), "bind");
    ok(tbg_count(-1, &c), "count");
    cnt += c;
  }
  printf("l%d_%c = %llu\n", n, "wb"[stm], (unsigned long long)cnt);
  return cnt != 0;
}

/* calc_W_n, tb8gen.c:1028-1084: stm wins in n, into Wc[stm]. */
static int calc_W_n(int stm, int n, int more_w)
{
  uint64_t cnt = 0, c;
  bind_all(Wc[stm], NULL);
  for (int s = 0; s < NS; s++) ok(tbg_clear(s), "clear");
  for (int s = 0; s < NS; s++) {
    if (n == 1 || n == DRAW_RULE + 1) {
      ok(tbg_sub_bind(s, sub[stm ^ 1][n == 1 ? C_LOSS : C_BLOSS][s], g_sub), "bind sub");
      ok(tbg_predecessors_sub(stm, s, 0), "predecessors_sub");
    }
    if (more_w) {
      ok(tbg_slot_bind(-1, Lp[stm ^ 1][s], g_bytes), "bind");
      ok(tbg_predecessors(stm, s), "predecessors");
    }
  }
  for (int s = 0; s < NS; s++) {
    ok(tbg_epilogue_W_to(s, wins[stm][s], wins[stm][s], &c), "epilogue");
    cnt += c;
  }
  printf("w%d_%c = %llu\n", n, "wb"[stm], (unsigned long long)cnt);
  return cnt != 0;
}

int main(int argc, char **argv)
{
  uint64_t seed = 1;
  int mod = 3, opt;
  while ((opt = getopt(argc, argv, "s:m:q")) != -1) {
    if (opt == 's') seed = strtoull(optarg, NULL, 10);
    else if (opt == 'm') mod = atoi(optarg);
    else if (opt == 'q') quiet = 1;
  }
  if (optind >= argc) {
    fprintf(stderr, "usage: tbgen [-s seed] [-m 3|5] MATERIAL\n");
    return EXIT_FAILURE;
  }
  ok(tbg_init(), "init");
  ok(tbg_material_from_name(argv[optind]), "material");
  ok(tbg_set_stub(seed, mod), "stub");
  uint64_t size, offs[6], capt[6];
  ok(tbg_geometry(&size, &g_bytes, &g_sub, offs, capt), "geometry");

  /* one allocation for everything: 10 bitmap planes, 10 sub planes + temp */
  size_t per = (size_t)g_bytes, persub = (size_t)g_sub;
  size_t total = per * NS * 10 + persub * NS * 11;
  uint8_t *base;
  ok(tbg_alloc(total, (void **)&base), "alloc");
  uint8_t *p = base;
  for (int c = 0; c < 2; c++)
    for (int s = 0; s < NS; s++) {
      wins[c][s] = p; p += per;
      Wp[c][s] = p; p += per;
      Lp[c][s] = p; p += per;
      Wc[c][s] = p; p += per;
      Lc[c][s] = p; p += per;
    }
  for (int c = 0; c < 2; c++)
    for (int k = 0; k < 5; k++)
      for (int s = 0; s < NS; s++) {
        sub[c][k][s] = p;
        p += persub;
      }
  for (int s = 0; s < NS; s++) {
    subtmp[s] = p;
    p += persub;
  }

  calc_subs();
  illegal_and_mate();  /* L0 into Lp */

  int more_ww = 1, more_wb = 1, more_lw = 1, more_lb = 1, more_wb_next, more_ww_next;
  int n;
  /* tb8gen.c:1414-1444; after each ply the current W/L become the sources */
  for (n = 1; ; n++) {
    int special = n == DRAW_RULE + 1;
    if (n > DRAW_RULE + 1 && !(more_ww || more_wb || more_lw || more_lb)) break;
    if (special) {
      more_wb_next = calc_L_n(WHITE, n, more_lw);
      more_ww_next = calc_L_n(BLACK, n, more_lb);
      more_lb = calc_W_n(WHITE, n, more_ww);
      more_lw = calc_W_n(BLACK, n, more_wb);
    } else {
      more_wb_next = more_lw && calc_L_n(WHITE, n, more_lw);
      more_ww_next = more_lb && calc_L_n(BLACK, n, more_lb);
      more_lb = more_ww && calc_W_n(WHITE, n, more_ww);
      more_lw = more_wb && calc_W_n(BLACK, n, more_wb);
    }
    more_wb = more_wb_next;
    more_ww = more_ww_next;
    for (int c = 0; c < 2; c++) {
      swap_planes(Wp[c], Wc[c]);
      swap_planes(Lp[c], Lc[c]);
    }
  }
  ok(tbg_sync(0), "sync");
  ok(tbg_free(base), "free");
  return 0;
}
