/*
 * tbgen -- the retrograde generation loop of tb8gen (tb8gen.c main,
 * calc_sub_kslices, calc_illegal_and_mate, calc_L_n, calc_W_n) as a C host
 * over the tbgpu C ABI, with every king slice resident in HBM.
 *
 *   tbgen [-s seed] [-m 3|5] [-b device_MB] [-S [-H]] [-g steps] [-P] [-p] [-n max_ply]
 *         [-o dir] [-c slices] MATERIAL
 *
 * Prints the reference's per-ply counts ("broken_w = ...", "l<n>_<c> = ...",
 * "w<n>_<c> = ...") in the reference's order.
 *
 * Resident mode (default when everything fits the device budget -b): each
 * slice's "wins", the previous and current W/L bitmaps of both sides and the
 * capture-class bitmaps stay on the device for the whole run, so the
 * reference's KSliceManager window (kslice.c:41-84) reduces to "all slices
 * bound": the order in which slices are scattered does not change a bitmap
 * (marks are ORed), and every scatter of a half-ply finishes before its
 * epilogue or verify starts, as in the reference.
 *
 * Streamed mode (-S, or when the planes exceed -b): the planes live in host
 * memory, the tier that replaces the reference's slice files
 * (kslice_read/kslice_write, kslice.c:317-379), and the device holds a
 * window of slices that follows the schedule's slice order, as the
 * reference's manager does: a slice is brought in before the first step
 * that unmoves into it (or reads it) and written out after the last one.
 * The "wins" planes stay in HBM (-H: in the host tier as well).  The steps
 * run in segments of -g steps (default 32 for slices up to 16 MB,
 * else 8), pipelined: a
 * segment's reads from the host tier and the previous segment's writes
 * overlap the kernels of the segment between them.
 *
 * In resident mode each half-ply is recorded as one batch and run by the
 * persistent kernel (tbg_batch_run mode 1, block-wide work items: a
 * half-ply's ~1,400 ops of small slices switch ops at every item, which a
 * block pays once for its warps; -k 2 for warp-wide items); -P launches
 * every call on its own instead, in the reference's call order.
 *
 * -o dir writes the reference's per-ply files under dir (n/W/<c>/<wk><bk>,
 * n/L/..., 0/L and, at the end, 0/wins; write_data's zstd frames), so that
 * the output can be compared with the reference program's file by file.
 *
 * -c K prints after each half-ply a digest of K seeded slices of its output
 * ("sum <w|l><n>_<c> = <hex>"), to compare runs slice-exactly.
 *
 * -p prints a timing line per half-ply ("time <kind><n>_<c> ms=...").
 * 7-piece capture values come from the seeded stub (tbg_set_stub); a capture
 * that leaves the two kings alone is a draw, as in the reference.
 */
#define _POSIX_C_SOURCE 200809L
#include <dlfcn.h>
#include <errno.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
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

/* The reference's per-ply files (-o DIR): defined with the king tables. */
static const char *g_outdir;
static void out_plane_dev(int n, const char *name, int stm, uint8_t *const pl[]);
static void out_plane_host(int n, const char *name, int stm, const uint8_t *plane,
                           const uint8_t *empty);

/* -c K: a digest of K seeded slices of every half-ply's output (defined
 * with the king tables). */
static int g_nsum;
static uint64_t g_sum_seed = 1;
static void sum_plane_dev(const char *kind, int n, int stm, uint8_t *const pl[]);
static void sum_plane_host(const char *kind, int n, int stm, const uint8_t *plane,
                           const uint8_t *empty);

/* A half-ply's output for -o and -c, written after its timing line: the
 * slices as device buffers (dev) or as a host-tier plane with its empty
 * flags. */
static struct {
  int pending, n, stm;
  const char *kind, *name;
  uint8_t *const *dev;
  const uint8_t *host, *empty;
} g_last;

static void note_output(const char *kind, const char *name, int n, int stm, uint8_t *const *dev,
                        const uint8_t *host, const uint8_t *empty)
{
  g_last.pending = g_outdir || g_nsum;
  g_last.kind = kind;
  g_last.name = name;
  g_last.n = n;
  g_last.stm = stm;
  g_last.dev = dev;
  g_last.host = host;
  g_last.empty = empty;
}

static void emit_output(void)
{
  if (!g_last.pending) return;
  g_last.pending = 0;
  if (g_last.dev) {
    if (g_outdir) out_plane_dev(g_last.n, g_last.name, g_last.stm, g_last.dev);
    if (g_nsum) sum_plane_dev(g_last.kind, g_last.n, g_last.stm, g_last.dev);
  } else {
    if (g_outdir) out_plane_host(g_last.n, g_last.name, g_last.stm, g_last.host, g_last.empty);
    if (g_nsum) sum_plane_host(g_last.kind, g_last.n, g_last.stm, g_last.host, g_last.empty);
  }
}

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
  if (g_outdir)
    for (int c = 0; c < 2; c++) out_plane_dev(0, "L", c, Lp[c]);
}

/* Half-plies of the resident mode run as one recorded batch (a persistent
 * kernel whose work queue follows the calls' buffer dependencies) unless -P
 * asks for one launch per call. */
static int g_plain;
static int g_kmode = 1;   /* persistent kernel: tbg_batch_run mode (-k) */

static void batch_begin(void)
{
  if (!g_plain) ok(tbg_batch_begin(), "batch begin");
}

static void batch_run(void)
{
  if (g_plain) return;
  int nops;
  uint64_t items;
  ok(tbg_batch_end(&nops, &items), "batch end");
  ok(tbg_batch_run(g_kmode), "batch run");
}

/* Ones in the slices of a plane: one strided count when the slices lie at
 * a fixed stride (the resident layout), else slice by slice. */
static uint64_t plane_total(uint8_t *pl[NS])
{
  uint64_t cnt = 0, c;
  const ptrdiff_t stride = pl[1] - pl[0];
  int uniform = stride > 0;
  for (int s = 1; s < NS && uniform; s++) uniform = pl[s] - pl[0] == stride * s;
  if (uniform) {
    ok(tbg_count_strided(pl[0], (uint64_t)stride, NS, &cnt), "count");
    return cnt;
  }
  for (int s = 0; s < NS; s++) {
    ok(tbg_slot_bind(-1, pl[s], g_bytes), "bind");
    ok(tbg_count(-1, &c), "count");
    cnt += c;
  }
  return cnt;
}

/* calc_L_n, tb8gen.c:943-1026: stm losses in n, into Lc[stm]. */
static int calc_L_n(int stm, int n, int more_l)
{
  uint64_t cnt;
  if (n == DRAW_RULE + 1)  /* cwin \ win (tb8gen.c:964-970) */
    for (int s = 0; s < NS; s++)
      ok(tbg_bitmap_and_not(subtmp[s], sub[stm ^ 1][C_CWIN][s], sub[stm ^ 1][C_WIN][s], g_sub),
         "and_not");
  /* candidates: predecessors of stm^1's W(n-1) and of its winning captures */
  bind_all(Lc[stm], NULL);
  batch_begin();
  for (int s = 0; s < NS; s++) ok(tbg_clear(s), "clear");
  for (int s = 0; s < NS; s++) {
    if (n == 1) {
      ok(tbg_sub_bind(s, sub[stm ^ 1][C_WIN][s], g_sub), "bind sub");
      ok(tbg_predecessors_sub(stm, s, 1), "predecessors_sub");
    } else if (n == DRAW_RULE + 1) {
      ok(tbg_sub_bind(s, subtmp[s], g_sub), "bind sub");
      ok(tbg_predecessors_sub(stm, s, 0), "predecessors_sub");
    }
    if (more_l && n > 1) {
      /* predecessors() less those a slider step takes out of stm^1's wins,
       * which the verify below would clear (tbg_candidates) */
      ok(tbg_slot_bind(-1, Wp[stm ^ 1][s], g_bytes), "bind");
      ok(tbg_candidates(stm, s, wins[stm ^ 1][s], g_bytes), "candidates");
    }
  }
  /* verify against stm^1's wins and winning captures */
  int cls = n <= DRAW_RULE ? C_WIN : C_CWIN;
  bind_all(wins[stm ^ 1], sub[stm ^ 1][cls]);
  for (int s = 0; s < NS; s++) {
    ok(tbg_slot_bind(-1, Lc[stm][s], g_bytes), "bind");
    ok(tbg_check_successors(stm, s), "check_successors");
  }
  batch_run();
  cnt = plane_total(Lc[stm]);
  printf("l%d_%c = %llu\n", n, "wb"[stm], (unsigned long long)cnt);
  note_output("l", "L", n, stm, Lc[stm], NULL, NULL);
  return cnt != 0;
}

/* calc_W_n, tb8gen.c:1028-1084: stm wins in n, into Wc[stm]. */
static int calc_W_n(int stm, int n, int more_w)
{
  uint64_t cnt = 0, c[NS];
  bind_all(Wc[stm], NULL);
  batch_begin();
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
  for (int s = 0; s < NS; s++)
    ok(tbg_epilogue_W_to(s, wins[stm][s], wins[stm][s], g_plain ? &c[s] : NULL), "epilogue");
  if (!g_plain) {
    batch_run();
    ok(tbg_batch_counts(c, NS), "counts");
  }
  for (int s = 0; s < NS; s++) cnt += c[s];
  printf("w%d_%c = %llu\n", n, "wb"[stm], (unsigned long long)cnt);
  note_output("w", "W", n, stm, Wc[stm], NULL, NULL);
  return cnt != 0;
}

/* ------------------------------------------------------------ streamed mode */
static uint64_t g_size;        /* positions per slice */
static int g_timing;

static double now_ms(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

/* The host tier's reads and writes (kslice_read / kslice_write,
 * kslice.c:317-379), through the library's stream. */
static uint64_t g_h2d_bytes, g_d2h_bytes;

/* Set-up copies are queued on the library's stream, in order with the
 * kernels. */
static void d2h(void *host, const void *dev, size_t n)
{
  ok(tbg_copy_to_host_async(host, dev, n), "copy to host");
  g_d2h_bytes += n;
}

/* King-pair tables, generated from their rules (probe.c:441-539,
 * tb8gen.c:69-89): KKIdx over the a1-d1-d4 triangle, KKSquare, KKMap. */
static int KKIdx[10][64], KKSq[NS][2], KKMap[64][64];

static uint64_t katt(int sq)
{
  uint64_t b = 0;
  for (int df = -1; df <= 1; df++)
    for (int dr = -1; dr <= 1; dr++) {
      int f = (sq & 7) + df, r = (sq >> 3) + dr;
      if ((df || dr) && f >= 0 && f < 8 && r >= 0 && r < 8) b |= 1ULL << (r * 8 + f);
    }
  return b;
}

static void init_king_tables(void)
{
  static const int tri[10] = { 1, 2, 3, 10, 11, 19, 0, 9, 18, 27 };
  int next = 0, nd = 441;
  for (int t = 0; t < 10; t++)
    for (int sq = 0; sq < 64; sq++) {
      KKIdx[t][sq] = -1;
      if (sq == tri[t] || (katt(tri[t]) >> sq & 1)) continue;
      if (t >= 6) {
        if ((sq & 7) < (sq >> 3)) continue;
        if ((sq & 7) == (sq >> 3)) {
          KKIdx[t][sq] = nd++;
          continue;
        }
      }
      KKIdx[t][sq] = next++;
    }
  for (int t = 0; t < 10; t++)
    for (int sq = 0; sq < 64; sq++)
      if (KKIdx[t][sq] >= 0) {
        KKSq[KKIdx[t][sq]][0] = tri[t];
        KKSq[KKIdx[t][sq]][1] = sq;
      }
  int triangle[64];
  for (int sq = 0; sq < 64; sq++) {
    int f = sq & 7, r = sq >> 3;
    if (f > 3) f = 7 - f;
    if (r > 3) r = 7 - r;
    if (r > f) { int x = f; f = r; r = x; }
    for (int t = 0; t < 10; t++)
      if (tri[t] == r * 8 + f) triangle[sq] = t;
  }
  for (int i = 0; i < 64; i++)
    for (int j = 0; j < 64; j++) {
      int m = ((i & 7) >= 4 ? 0x07 : 0) | ((i >> 3) >= 4 ? 0x38 : 0);
      int s1 = i ^ m, s2 = j ^ m;
      int tri_ok = (s1 & 7) <= 3 && (s1 >> 3) <= (s1 & 7);
      int diag = tri_ok && (s1 & 7) == (s1 >> 3);
      int lower = (s2 & 7) >= (s2 >> 3);
      if (!tri_ok || (diag && !lower)) {
        s1 = ((s1 & 7) << 3) | (s1 >> 3);
        s2 = ((s2 & 7) << 3) | (s2 >> 3);
      }
      KKMap[i][j] = (i == j || (katt(i) >> j & 1)) ? -1 : KKIdx[triangle[s1]][s2];
    }
}

/* ---- the reference's per-ply files (-o DIR) ----
 * write_data (util.c:272-343) into the paths of create_name
 * (kslice.c:306-315): DIR/<n>/<name>/<w|b>/<wk><bk>, each file the slice's
 * bitmap in chunks of 50 KiB, every chunk one frame: {compressed size, chunk
 * size, offset} as three size_t, then the chunk compressed by zstd at level
 * 6, as the reference's Makefile sets it.  libzstd is opened on first use. */
enum { OUT_CHUNK = 50 * 1024, OUT_LEVEL = 6 };
static size_t (*z_bound)(size_t);
static size_t (*z_compress)(void *, size_t, const void *, size_t, int);
static unsigned (*z_iserror)(size_t);
static uint8_t *out_frame, *out_host, *out_zero;

static void out_init(void)
{
  if (z_compress) return;
  void *h = dlopen("libzstd.so.1", RTLD_NOW);
  if (!h) {
    fprintf(stderr, "tbgen: -o needs libzstd.so.1: %s\n", dlerror());
    exit(EXIT_FAILURE);
  }
  *(void **)&z_bound = dlsym(h, "ZSTD_compressBound");
  *(void **)&z_compress = dlsym(h, "ZSTD_compress");
  *(void **)&z_iserror = dlsym(h, "ZSTD_isError");
  if (!z_bound || !z_compress || !z_iserror) {
    fprintf(stderr, "tbgen: libzstd.so.1 lacks the compression entry points\n");
    exit(EXIT_FAILURE);
  }
  out_frame = malloc(3 * sizeof(size_t) + z_bound(OUT_CHUNK));
  out_host = malloc(g_bytes);
  out_zero = calloc(1, g_bytes);
  if (!out_frame || !out_host || !out_zero) {
    fprintf(stderr, "tbgen: out of host memory\n");
    exit(EXIT_FAILURE);
  }
}

static void out_mkdirs(char *path)
{
  for (char *p = path + 1; *p; p++)
    if (*p == '/') {
      *p = 0;
      if (mkdir(path, 0777) != 0 && errno != EEXIST) {
        fprintf(stderr, "tbgen: cannot create %s\n", path);
        exit(EXIT_FAILURE);
      }
      *p = '/';
    }
}

static void out_slice(int n, const char *name, int stm, int s, const uint8_t *p)
{
  char path[512];
  const int wk = KKSq[s][0], bk = KKSq[s][1];
  snprintf(path, sizeof path, "%s/%d/%s/%c/%c%c%c%c", g_outdir, n, name, "wb"[stm],
           'a' + (wk & 7), '1' + (wk >> 3), 'a' + (bk & 7), '1' + (bk >> 3));
  out_mkdirs(path);
  FILE *F = fopen(path, "wb");
  if (!F) {
    fprintf(stderr, "tbgen: cannot write %s\n", path);
    exit(EXIT_FAILURE);
  }
  const size_t head = 3 * sizeof(size_t), cap = z_bound(OUT_CHUNK);
  for (size_t idx = 0; idx < g_bytes; idx += OUT_CHUNK) {
    const size_t chunk = g_bytes - idx < OUT_CHUNK ? g_bytes - idx : OUT_CHUNK;
    const size_t c = z_compress(out_frame + head, cap, p + idx, chunk, OUT_LEVEL);
    if (z_iserror(c)) {
      fprintf(stderr, "tbgen: zstd failed on %s\n", path);
      exit(EXIT_FAILURE);
    }
    const size_t h3[3] = { c, chunk, idx };
    memcpy(out_frame, h3, head);
    if (fwrite(out_frame, 1, head + c, F) != head + c) {
      fprintf(stderr, "tbgen: cannot write %s\n", path);
      exit(EXIT_FAILURE);
    }
  }
  fclose(F);
}

/* A plane whose slices are device buffers (pl[s]). */
static void out_plane_dev(int n, const char *name, int stm, uint8_t *const pl[])
{
  out_init();
  for (int s = 0; s < NS; s++) {
    ok(tbg_copy_to_host(out_host, pl[s], g_bytes), "copy to host");
    out_slice(n, name, stm, s, out_host);
  }
}

/* A plane of the host tier; slices flagged empty are zero. */
static void out_plane_host(int n, const char *name, int stm, const uint8_t *plane,
                           const uint8_t *empty)
{
  out_init();
  for (int s = 0; s < NS; s++)
    out_slice(n, name, stm, s, empty && empty[s] ? out_zero : plane + (size_t)s * g_bytes);
}

/* ---- digests of seeded slices (-c K) ----
 * After each half-ply: "sum <w|l><n>_<c> = <hex>", a 64-bit FNV-1a digest
 * (over 64-bit little-endian words) of the output bitmaps of K slices drawn with splitmix64 from the seed, so
 * that two runs (resident and streamed) can be compared slice-exactly at
 * every ply without writing the planes out. */
static uint64_t sum_mix(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

static int sum_slice(int i) { return (int)(sum_mix(g_sum_seed * 1000003u + (uint64_t)i) % NS); }

static uint64_t sum_bytes(uint64_t h, const uint8_t *p, size_t n)
{
  for (size_t i = 0; i + 8 <= n; i += 8) {  /* n is a multiple of 64 */
    uint64_t w;
    memcpy(&w, p + i, 8);
    h = (h ^ w) * 0x100000001b3ull;
  }
  return h;
}

static void sum_print(const char *kind, int n, int stm, uint64_t h)
{
  printf("sum %s%d_%c = %016llx\n", kind, n, "wb"[stm], (unsigned long long)h);
}

static void sum_plane_dev(const char *kind, int n, int stm, uint8_t *const pl[])
{
  static uint8_t *buf;
  if (!buf && !(buf = malloc(g_bytes))) {
    fprintf(stderr, "tbgen: out of host memory\n");
    exit(EXIT_FAILURE);
  }
  uint64_t h = 0xcbf29ce484222325ull;
  for (int i = 0; i < g_nsum; i++) {
    ok(tbg_copy_to_host(buf, pl[sum_slice(i)], g_bytes), "copy to host");
    h = sum_bytes(h, buf, g_bytes);
  }
  sum_print(kind, n, stm, h);
}

static void sum_plane_host(const char *kind, int n, int stm, const uint8_t *plane,
                           const uint8_t *empty)
{
  static uint8_t *zero;
  if (!zero && !(zero = calloc(1, g_bytes))) {
    fprintf(stderr, "tbgen: out of host memory\n");
    exit(EXIT_FAILURE);
  }
  uint64_t h = 0xcbf29ce484222325ull;
  for (int i = 0; i < g_nsum; i++) {
    const int s = sum_slice(i);
    h = sum_bytes(h, empty && empty[s] ? zero : plane + (size_t)s * g_bytes, g_bytes);
  }
  sum_print(kind, n, stm, h);
}

/* The slices a step on slice s of side stm touches: s and the slices its
 * king moves reach (the targets of predecessors, the wins that
 * check_successors reads). */
static int step_slices(int stm, int s, int *out)
{
  int n = 0, me = KKSq[s][stm], opp = KKSq[s][stm ^ 1];
  out[n++] = s;
  uint64_t b = katt(me) & ~katt(opp) & ~(1ULL << opp);
  while (b) {
    int to = __builtin_ctzll(b);
    b &= b - 1;
    int k[2] = { KKSq[s][0], KKSq[s][1] };
    k[stm] = to;
    int t = KKMap[k[0]][k[1]];
    int seen = t < 0;
    for (int j = 0; j < n && !seen; j++) seen = out[j] == t;
    if (!seen) out[n++] = t;
  }
  return n;
}

/* Step order per side to move: for black, the rows of KKIdx (black-king
 * moves keep the normalised white king, so they stay within a row); for
 * white, the same steps through the colour flip, as the reference's
 * manager (kslice.c:41-84) orders them. */
static int order[2][NS];
static int touch[2][NS][12], ntouch[2][NS];
static int last_use[2][NS];
static int window_max;

static void init_schedule(void)
{
  int k = 0;
  for (int i = 0; i < 10; i++)
    for (int bk = 0; bk < 64; bk++)
      if (KKIdx[i][bk] >= 0) order[BLACK][k++] = KKIdx[i][bk];
  for (k = 0; k < NS; k++) {
    int s = order[BLACK][k];
    order[WHITE][k] = KKMap[KKSq[s][1]][KKSq[s][0]];
  }
  for (int stm = 0; stm < 2; stm++) {
    int live = 0, resident[NS] = { 0 };
    for (k = 0; k < NS; k++) {
      ntouch[stm][k] = step_slices(stm, order[stm][k], touch[stm][k]);
      for (int j = 0; j < ntouch[stm][k]; j++) last_use[stm][touch[stm][k][j]] = k;
    }
    for (k = 0; k < NS; k++) {
      for (int j = 0; j < ntouch[stm][k]; j++)
        if (!resident[touch[stm][k][j]]) {
          resident[touch[stm][k][j]] = 1;
          live++;
        }
      if (live > window_max) window_max = live;
      for (int j = 0; j < ntouch[stm][k]; j++) {
        int t = touch[stm][k][j];
        if (last_use[stm][t] == k && resident[t]) {
          resident[t] = 0;
          live--;
        }
      }
    }
  }
}

/* host tier: per side the planes of all slices */
enum { P_WINS, P_WP, P_LP, P_WC, P_LC, P_X, NPLANE };
static uint8_t *HP[2][NPLANE], *HS[2][5];
#define HSL(plane, c, s) (HP[c][plane] + (size_t)(s) * g_bytes)
#define HSUB(c, k, s) (HS[c][k] + (size_t)(s) * g_sub)

/* Slices of a host-tier plane known to hold no position (from the counts of
 * the step that wrote them): their bytes are not kept and never read.  An
 * empty source is neither copied nor scattered; a slice that no scatter
 * reaches stays empty, so it is neither cleared, nor finished by an
 * epilogue, nor written back; a verify step with no candidates is skipped. */
static uint8_t hempty[2][NPLANE][NS];

/* The "wins" planes of both sides stay in HBM unless -H: every half-ply
 * reads a whole wins plane (the W step also rewrites its own), so they are
 * the largest stream of the host tier, and both fit a B200 even for a
 * 7-piece material (2 x 71 GB for KRRRvKRRR). */
static int g_host_wins;
static uint8_t *g_dwins[2];
#define DWIN(c, s) (g_dwins[c] + (size_t)(s) * g_bytes)

/* device buffers of the set-up steps (calc_sub, illegal and mate) */
static uint8_t *setup_bm[4], *setup_sub[5], *setup_base;

static void st_calc_subs(void)
{
  for (int stm = 0; stm < 2; stm++)
    for (int s = 0; s < NS; s++) {
      void *cls[5] = { setup_sub[0], setup_sub[1], setup_sub[2], setup_sub[3], setup_sub[4] };
      ok(tbg_calc_sub(stm, s, cls), "calc_sub");
      for (int k = 0; k < 5; k++) d2h(HSUB(stm, k, s), setup_sub[k], g_sub);
    }
}

static void st_illegal_and_mate(void)
{
  uint64_t cnt[4] = { 0, 0, 0, 0 }, c;
  uint8_t *b[4] = { setup_bm[0], setup_bm[1], setup_bm[2], setup_bm[3] };
  for (int s = 0; s < NS; s++) {
    if (g_dwins[0]) {
      b[0] = DWIN(WHITE, s);
      b[1] = DWIN(BLACK, s);
    }
    ok(tbg_calc_illegal(s, b[0], b[1]), "illegal");
    ok(tbg_calc_mate(s, b[0], b[1], b[2], b[3]), "mate");
    for (int j = 0; j < 4; j++) {
      ok(tbg_slot_bind(0, b[j], g_bytes), "bind");
      ok(tbg_count(0, &c), "count");
      cnt[j] += c;
      if (j >= 2) hempty[j - 2][P_LP][s] = c == 0;
    }
    ok(tbg_slot_bind(0, NULL, 0), "unbind");
    if (!g_dwins[0]) {
      d2h(HSL(P_WINS, WHITE, s), b[0], g_bytes);
      d2h(HSL(P_WINS, BLACK, s), b[1], g_bytes);
    }
    d2h(HSL(P_LP, WHITE, s), b[2], g_bytes);
    d2h(HSL(P_LP, BLACK, s), b[3], g_bytes);
  }
  printf("broken_w = %llu\nbroken_b = %llu\nl0_w = %llu\nl0_b = %llu\n",
         (unsigned long long)cnt[0], (unsigned long long)cnt[1], (unsigned long long)cnt[2],
         (unsigned long long)cnt[3]);
}

/* ---- the pipeline of the streamed half-plies ----
 * A part of a half-ply (the scatter of calc_W_n, the candidates of
 * calc_L_n, or its verify) runs the schedule's steps in segments of g_seg
 * steps, numbered across parts.  For segment q:
 *   reads   the host-tier planes it needs go to the device on the inbound
 *           copy stream, queued before segment q-1's kernels so that they
 *           run meanwhile; they wait only for segment q-3's writes, the last
 *           users of the staging set (q mod 3) and of the window buffers
 *           released three segments back;
 *   kernels its calls are recorded as one batch and run by the persistent
 *           kernel on the library stream, after its reads;
 *   writes  the slices that step their last in q go back to the host tier
 *           on the outbound copy stream after the kernels; their window
 *           buffers are taken again two segments later at the earliest.
 * Slices enter the window (the reference's KSliceManager, kslice.c:41-84)
 * before the first step that touches them and leave after the last. */
enum { NPAR = 3, TK_RING = 8, MAX_SEG = 64 };
static int g_seg;                              /* 0: chosen from the slice size */
static int g_lw;                               /* most last uses in a segment */
static int64_t g_seq;                          /* segments issued so far */
static uint64_t in_tk[TK_RING], out_tk[TK_RING];
static uint8_t *st_src[NPAR][MAX_SEG], *st_sub[NPAR][MAX_SEG], *st_subt[NPAR][MAX_SEG];
static uint8_t **st_win[NPAR];
static uint64_t *hcnt;                         /* counts of a half-ply (page-locked) */
static int ncnt;

typedef struct {
  uint8_t *bm, *sub;
  int64_t rel;  /* segment whose kernels used it last */
  int used;
} WinBuf;
static WinBuf *win;
static int nwin, capwin, where_[NS];

/* A window buffer released at segment <= max_rel, else a new one. */
static int take(int64_t max_rel)
{
  for (int b = 0; b < nwin; b++)
    if (!win[b].used && win[b].rel <= max_rel) {
      win[b].used = 1;
      return b;
    }
  if (nwin == capwin) {
    capwin = capwin ? 2 * capwin : 64;
    win = realloc(win, capwin * sizeof *win);
    if (!win) {
      fprintf(stderr, "tbgen: out of host memory\n");
      exit(EXIT_FAILURE);
    }
  }
  uint8_t *p;
  ok(tbg_alloc(g_bytes + g_sub, (void **)&p), "window buffer");
  win[nwin] = (WinBuf){ p, p + g_bytes, INT64_MIN, 1 };
  return nwin++;
}

/* After a wait that covers every earlier use: all free buffers may be taken. */
static void reset_window(void)
{
  for (int b = 0; b < nwin; b++)
    if (!win[b].used) win[b].rel = INT64_MIN;
}

static void release(int t, int64_t q)
{
  ok(tbg_slot_bind(t, NULL, 0), "unbind");
  ok(tbg_sub_bind(t, NULL, 0), "unbind sub");
  win[where_[t]].used = 0;
  win[where_[t]].rel = q;
  where_[t] = -1;
}

static void cin(void *dev, const void *host, size_t n)
{
  ok(tbg_copy_in(dev, host, n, 0, NULL), "copy in");
  g_h2d_bytes += n;
}

static void cout_(void *host, const void *dev, size_t n)
{
  ok(tbg_copy_out(host, dev, n, 0, NULL), "copy out");
  g_d2h_bytes += n;
}

enum { PART_W, PART_CAND, PART_VERIFY };
typedef struct {
  int kind, stm, n, more, cls;
  uint64_t after;  /* inbound copies of the part wait for this point (0: none) */
} Part;

static int seg_lo(int h) { return h * g_seg; }
static int seg_hi(int h) { return (h + 1) * g_seg < NS ? (h + 1) * g_seg : NS; }

static uint8_t act[NS];      /* schedule step k of the current part has work */
static uint8_t hit[NS];      /* slice t is marked (scatters) or read (verify) */
static int cnt_slice[NS];    /* slice of each count queued in the half-ply */

static int has_sub(const Part *P)
{
  return P->kind != PART_VERIFY && (P->n == 1 || P->n == DRAW_RULE + 1);
}

static int has_src(const Part *P, int s)
{
  if (P->kind == PART_W) return P->more && !hempty[P->stm ^ 1][P_LP][s];
  if (P->kind == PART_CAND) return P->more && P->n > 1 && !hempty[P->stm ^ 1][P_WP][s];
  return 0;
}

static void plan_part(const Part *P)
{
  const int stm = P->stm;
  memset(hit, 0, sizeof hit);
  for (int k = 0; k < NS; k++) {
    const int s = order[stm][k];
    act[k] = P->kind == PART_VERIFY ? !hempty[stm][P_X][s] : has_sub(P) || has_src(P, s);
    if (act[k])
      for (int x = 0; x < ntouch[stm][k]; x++) hit[touch[stm][k][x]] = 1;
  }
}

/* Reads of segment h (number q) of part P, into staging set q mod 3. */
static void prep(const Part *P, int h, int64_t q)
{
  const int p = (int)(q % NPAR), stm = P->stm, n = P->n;
  if (h == 0 && P->after) ok(tbg_copy_in(NULL, NULL, 0, P->after, NULL), "wait");
  if (q >= 3) ok(tbg_copy_in(NULL, NULL, 0, out_tk[(q - 3) % TK_RING], NULL), "wait");
  int i = 0;
  for (int k = seg_lo(h); k < seg_hi(h); k++) {
    const int j = k - seg_lo(h), s = order[stm][k];
    if (P->kind == PART_VERIFY) {
      if (!act[k]) continue;
      for (int x = 0; x < ntouch[stm][k]; x++) {
        const int t = touch[stm][k][x];
        if (where_[t] >= 0) continue;
        const int b = take(q - 3);
        where_[t] = b;
        if (!g_dwins[stm ^ 1]) cin(win[b].bm, HSL(P_WINS, stm ^ 1, t), g_bytes);
        cin(win[b].sub, HSUB(stm ^ 1, P->cls, t), g_sub);
      }
      cin(st_src[p][j], HSL(P_X, stm, s), g_bytes);
      continue;
    }
    if (has_sub(P)) {
      if (P->kind == PART_W) {
        cin(st_sub[p][j], HSUB(stm ^ 1, n == 1 ? C_LOSS : C_BLOSS, s), g_sub);
      } else if (n == 1) {
        cin(st_sub[p][j], HSUB(stm ^ 1, C_WIN, s), g_sub);
      } else {
        cin(st_sub[p][j], HSUB(stm ^ 1, C_CWIN, s), g_sub);
        cin(st_subt[p][j], HSUB(stm ^ 1, C_WIN, s), g_sub);
      }
    }
    if (has_src(P, s))
      cin(st_src[p][j], HSL(P->kind == PART_W ? P_LP : P_WP, stm ^ 1, s), g_bytes);
    if (P->kind == PART_W)
      for (int x = 0; x < ntouch[stm][k]; x++) {
        const int t = touch[stm][k][x];
        if (last_use[stm][t] == k && hit[t] && !g_dwins[stm])
          cin(st_win[p][i++], HSL(P_WINS, stm, t), g_bytes);
      }
  }
  ok(tbg_copy_in(NULL, NULL, 0, 0, &in_tk[q % TK_RING]), "fence");
}

static int g_recording;

static void rec(void)
{
  if (!g_recording) ok(tbg_batch_begin(), "batch begin");
  g_recording = 1;
}

/* Kernels and writes of segment h (number q) of part P. */
static void compute(const Part *P, int h, int64_t q)
{
  const int p = (int)(q % NPAR), stm = P->stm, n = P->n;
  ok(tbg_join(in_tk[q % TK_RING]), "join");
  if (q >= 2) ok(tbg_join(out_tk[(q - 2) % TK_RING]), "join");
  if (P->kind == PART_CAND && n == DRAW_RULE + 1) /* cwin \ win (tb8gen.c:964-970) */
    for (int k = seg_lo(h); k < seg_hi(h); k++) {
      const int j = k - seg_lo(h);
      ok(tbg_bitmap_and_not(st_sub[p][j], st_sub[p][j], st_subt[p][j], g_sub), "and_not");
    }
  int i = 0, nc = 0;
  for (int k = seg_lo(h); k < seg_hi(h); k++) {
    const int j = k - seg_lo(h), s = order[stm][k];
    if (P->kind == PART_VERIFY) {
      if (!act[k]) continue;
      rec();
      for (int x = 0; x < ntouch[stm][k]; x++) {
        const int t = touch[stm][k][x];
        ok(tbg_slot_bind(t, g_dwins[stm ^ 1] ? DWIN(stm ^ 1, t) : win[where_[t]].bm, g_bytes),
           "bind");
        ok(tbg_sub_bind(t, win[where_[t]].sub, g_sub), "bind sub");
      }
      ok(tbg_slot_bind(-1, st_src[p][j], g_bytes), "bind");
      ok(tbg_check_successors(stm, s), "check_successors");
      ok(tbg_batch_count(-1), "count");
      cnt_slice[ncnt + nc++] = s;
      continue;
    }
    if (act[k]) {
      rec();
      for (int x = 0; x < ntouch[stm][k]; x++) {
        const int t = touch[stm][k][x];
        if (where_[t] >= 0) continue;
        const int b = take(q - 2);
        where_[t] = b;
        ok(tbg_slot_bind(t, win[b].bm, g_bytes), "bind");
        ok(tbg_clear(t), "clear");
      }
      if (has_sub(P)) {
        ok(tbg_sub_bind(s, st_sub[p][j], g_sub), "bind sub");
        ok(tbg_predecessors_sub(stm, s, P->kind == PART_CAND && n == 1), "predecessors_sub");
        ok(tbg_sub_bind(s, NULL, 0), "unbind sub");
      }
      if (has_src(P, s)) {
        ok(tbg_slot_bind(-1, st_src[p][j], g_bytes), "bind");
        if (P->kind == PART_CAND && g_dwins[stm ^ 1])
          ok(tbg_candidates(stm, s, DWIN(stm ^ 1, s), g_bytes), "candidates");
        else
          ok(tbg_predecessors(stm, s), "predecessors");
      }
    }
    if (P->kind == PART_W)
      for (int x = 0; x < ntouch[stm][k]; x++) {
        const int t = touch[stm][k][x];
        if (last_use[stm][t] != k || !hit[t]) continue;
        rec();
        uint8_t *wb = g_dwins[stm] ? DWIN(stm, t) : st_win[p][i++];
        ok(tbg_epilogue_W_to(t, wb, wb, NULL), "epilogue");
        cnt_slice[ncnt + nc++] = t;
      }
  }
  if (g_recording) {
    int nops;
    uint64_t items;
    ok(tbg_batch_end(&nops, &items), "batch end");
    ok(tbg_batch_run(g_kmode), "batch run");
    if (nc) ok(tbg_batch_counts_async(hcnt + ncnt, nc), "counts");
    g_recording = 0;
  }
  ncnt += nc;
  uint64_t mk;
  ok(tbg_mark(&mk), "mark");
  ok(tbg_copy_out(NULL, NULL, 0, mk, NULL), "wait");
  i = 0;
  for (int k = seg_lo(h); k < seg_hi(h); k++) {
    const int j = k - seg_lo(h), s = order[stm][k];
    if (P->kind == PART_VERIFY) {
      if (act[k]) cout_(HSL(P_LC, stm, s), st_src[p][j], g_bytes);
      else hempty[stm][P_LC][s] = 1;
      continue;
    }
    for (int x = 0; x < ntouch[stm][k]; x++) {
      const int t = touch[stm][k][x];
      if (last_use[stm][t] != k) continue;
      if (P->kind == PART_W) {
        if (hit[t]) {
          cout_(HSL(P_WC, stm, t), win[where_[t]].bm, g_bytes);
          if (!g_dwins[stm]) cout_(HSL(P_WINS, stm, t), st_win[p][i++], g_bytes);
        } else {
          hempty[stm][P_WC][t] = 1;
        }
      } else {
        if (hit[t]) cout_(HSL(P_X, stm, t), win[where_[t]].bm, g_bytes);
        hempty[stm][P_X][t] = !hit[t];
      }
    }
  }
  ok(tbg_copy_out(NULL, NULL, 0, 0, &out_tk[q % TK_RING]), "fence");
  for (int k = seg_lo(h); k < seg_hi(h); k++)
    for (int x = 0; x < ntouch[stm][k]; x++) {
      const int t = touch[stm][k][x];
      if (last_use[stm][t] == k && where_[t] >= 0) release(t, q);
    }
}

/* Runs a part; returns the outbound point after its last writes. */
static uint64_t run_part(const Part *P)
{
  const int nseg = (NS + g_seg - 1) / g_seg;
  const int64_t base = g_seq;
  g_seq += nseg;
  plan_part(P);
  if (P->after) reset_window();  /* its reads wait for every earlier write */
  prep(P, 0, base);
  for (int h = 0; h < nseg; h++) {
    if (h + 1 < nseg) prep(P, h + 1, base + h + 1);
    compute(P, h, base + h);
  }
  return out_tk[(base + nseg - 1) % TK_RING];
}

/* Sum of the counts the half-ply queued, once its last writes are done;
 * a slice whose count is 0 is flagged empty in `plane`. */
static uint64_t half_ply_count(uint64_t last, int stm, int plane)
{
  ok(tbg_wait_ticket(last, 0), "wait");
  ok(tbg_sync(0), "sync");
  reset_window();
  uint64_t cnt = 0;
  for (int k = 0; k < ncnt; k++) {
    cnt += hcnt[k];
    hempty[stm][plane][cnt_slice[k]] = hcnt[k] == 0;
  }
  ncnt = 0;
  return cnt;
}

/* calc_W_n streamed (tb8gen.c:1028-1084). */
static int st_calc_W_n(int stm, int n, int more_w)
{
  Part P = { PART_W, stm, n, more_w, 0, 0 };
  uint64_t cnt = half_ply_count(run_part(&P), stm, P_WC);
  printf("w%d_%c = %llu\n", n, "wb"[stm], (unsigned long long)cnt);
  note_output("w", "W", n, stm, NULL, HP[stm][P_WC], hempty[stm][P_WC]);
  return cnt != 0;
}

/* calc_L_n streamed (tb8gen.c:943-1026): candidates, written to the X
 * plane, then the verify. */
static int st_calc_L_n(int stm, int n, int more_l)
{
  Part P = { PART_CAND, stm, n, more_l, 0, 0 };
  uint64_t done = run_part(&P);
  Part V = { PART_VERIFY, stm, n, more_l, n <= DRAW_RULE ? C_WIN : C_CWIN, done };
  uint64_t cnt = half_ply_count(run_part(&V), stm, P_LC);
  printf("l%d_%c = %llu\n", n, "wb"[stm], (unsigned long long)cnt);
  note_output("l", "L", n, stm, NULL, HP[stm][P_LC], hempty[stm][P_LC]);
  return cnt != 0;
}

/* Host-tier planes: page-locked while the host allows, else ordinary. */
static void *host_alloc(size_t n)
{
  void *p = NULL;
  if (tbg_host_alloc(n, &p) == TBG_OK) return p;
  p = malloc(n);
  if (!p) {
    fprintf(stderr, "tbgen: out of host memory (%zu bytes)\n", n);
    exit(EXIT_FAILURE);
  }
  return p;
}

/* Sets up the streamed mode: host planes, the set-up buffers and the
 * staging sets of the pipeline (the window grows as it needs). */
static void st_setup(void)
{
  if (g_seg == 0) g_seg = g_bytes <= (16u << 20) ? 32 : 8;
  init_schedule();
  if (!g_host_wins && tbg_alloc((size_t)2 * NS * g_bytes, (void **)&g_dwins[0]) == TBG_OK)
    g_dwins[1] = g_dwins[0] + (size_t)NS * g_bytes;
  for (int c = 0; c < 2; c++) {
    for (int p = 0; p < NPLANE; p++)
      if (p != P_WINS || !g_dwins[0]) HP[c][p] = host_alloc((size_t)g_bytes * NS);
    for (int k = 0; k < 5; k++) HS[c][k] = host_alloc((size_t)g_sub * NS);
  }
  hcnt = host_alloc(NS * sizeof *hcnt);
  for (int stm = 0; stm < 2; stm++)
    for (int h = 0; h * g_seg < NS; h++) {
      int lw = 0;
      for (int k = seg_lo(h); k < seg_hi(h); k++)
        for (int x = 0; x < ntouch[stm][k]; x++) lw += last_use[stm][touch[stm][k][x]] == k;
      if (lw > g_lw) g_lw = lw;
    }
  ok(tbg_alloc(4 * g_bytes + 5 * g_sub, (void **)&setup_base), "alloc");
  for (int j = 0; j < 4; j++) setup_bm[j] = setup_base + j * g_bytes;
  for (int k = 0; k < 5; k++) setup_sub[k] = setup_base + 4 * g_bytes + k * g_sub;
  const int nwin_stage = g_dwins[0] ? 0 : g_lw;
  const size_t per_set = (size_t)g_seg * (g_bytes + 2 * g_sub) + (size_t)nwin_stage * g_bytes;
  for (int p = 0; p < NPAR; p++) {
    uint8_t *base;
    ok(tbg_alloc(per_set, (void **)&base), "alloc");
    for (int j = 0; j < g_seg; j++) {
      st_src[p][j] = base;
      base += g_bytes;
      st_sub[p][j] = base;
      base += g_sub;
      st_subt[p][j] = base;
      base += g_sub;
    }
    st_win[p] = calloc(g_lw, sizeof *st_win[p]);
    for (int i = 0; i < nwin_stage; i++) {
      st_win[p][i] = base;
      base += g_bytes;
    }
  }
  for (int s = 0; s < NS; s++) where_[s] = -1;
  if (!quiet)
    fprintf(stderr,
            "tbgen: streamed, segments of %d steps, schedule window %d slices, host tier %.1f GB, "
            "wins planes %s\n",
            g_seg, window_max,
            (double)((NPLANE - (g_dwins[0] ? 1 : 0)) * g_bytes + 5 * g_sub) * NS * 2 / 1e9,
            g_dwins[0] ? "in HBM" : "in the host tier");
}

/* After the set-up steps (copies on the library stream): the host tier is
 * complete before the pipeline's streams read it. */
static void st_setup_done(void)
{
  ok(tbg_sync(0), "sync");
  ok(tbg_free(setup_base), "free");
}

static void swap_host_planes(void)
{
  for (int c = 0; c < 2; c++) {
    for (int s = 0; s < NS; s++) {
      uint8_t e = hempty[c][P_WP][s];
      hempty[c][P_WP][s] = hempty[c][P_WC][s];
      hempty[c][P_WC][s] = e;
      e = hempty[c][P_LP][s];
      hempty[c][P_LP][s] = hempty[c][P_LC][s];
      hempty[c][P_LC][s] = e;
    }
    uint8_t *t = HP[c][P_WP];
    HP[c][P_WP] = HP[c][P_WC];
    HP[c][P_WC] = t;
    t = HP[c][P_LP];
    HP[c][P_LP] = HP[c][P_LC];
    HP[c][P_LC] = t;
  }
}

typedef int (*step_fn)(int stm, int n, int more);

/* One half-ply call with its timing line (-p). */
static int timed(step_fn f, const char *kind, int stm, int n, int more)
{
  double t0 = now_ms();
  int r = f(stm, n, more);
  if (g_timing) {
    ok(tbg_sync(0), "sync");
    double ms = now_ms() - t0;
    fprintf(stderr, "time %s%d_%c ms=%.3f positions=%llu\n", kind, n, "wb"[stm], ms,
            (unsigned long long)(g_size * NS));
  }
  emit_output();  /* -o files and -c digests, outside the timed half-ply */
  return r;
}

int main(int argc, char **argv)
{
  uint64_t seed = 1;
  int mod = 3, opt, force_stream = 0, max_ply = 1 << 30;
  double budget_mb = 0;
  while ((opt = getopt(argc, argv, "s:m:qb:SHPpn:g:o:c:k:")) != -1) {
    if (opt == 's') seed = strtoull(optarg, NULL, 10);
    else if (opt == 'm') mod = atoi(optarg);
    else if (opt == 'q') quiet = 1;
    else if (opt == 'b') budget_mb = atof(optarg);
    else if (opt == 'S') force_stream = 1;
    else if (opt == 'P') g_plain = 1;
    else if (opt == 'H') g_host_wins = 1;
    else if (opt == 'p') g_timing = 1;
    else if (opt == 'n') max_ply = atoi(optarg);
    else if (opt == 'g') g_seg = atoi(optarg);
    else if (opt == 'o') g_outdir = optarg;
    else if (opt == 'c') g_nsum = atoi(optarg);
    else if (opt == 'k') g_kmode = atoi(optarg);
  }
  if (optind >= argc) {
    fprintf(stderr,
            "usage: tbgen [-s seed] [-m 3|5] [-b device_MB] [-S [-H]] [-g steps] [-P] [-p] [-n max_ply] "
            "[-o dir] [-c slices] [-k 1|2] "
            "MATERIAL\n");
    return EXIT_FAILURE;
  }
  if (g_seg < 0 || g_seg > MAX_SEG) {
    fprintf(stderr, "tbgen: -g takes 1..%d steps per segment (0: automatic)\n", MAX_SEG);
    return EXIT_FAILURE;
  }
  if (g_kmode != 1 && g_kmode != 2) {
    fprintf(stderr, "tbgen: -k takes 1 (block-wide) or 2 (warp-wide work items)\n");
    return EXIT_FAILURE;
  }
  if (g_nsum < 0 || g_nsum > NS) {
    fprintf(stderr, "tbgen: -c takes 0..%d slices\n", NS);
    return EXIT_FAILURE;
  }
  g_sum_seed = seed;
  ok(tbg_init(), "init");
  ok(tbg_material_from_name(argv[optind]), "material");
  ok(tbg_set_stub(seed, mod), "stub");
  uint64_t offs[6], capt[6];
  ok(tbg_geometry(&g_size, &g_bytes, &g_sub, offs, capt), "geometry");
  init_king_tables();

  /* resident: 10 bitmap planes, 10 sub planes + temp */
  size_t per = (size_t)g_bytes, persub = (size_t)g_sub;
  size_t total = per * NS * 10 + persub * NS * 11;
  int streamed = force_stream || (budget_mb > 0 && total > budget_mb * 1e6);
  step_fn W = calc_W_n, L = calc_L_n;
  uint8_t *base = NULL;
  if (streamed) {
    st_setup();
    st_calc_subs();
    st_illegal_and_mate();
    st_setup_done();
    if (g_outdir)
      for (int c = 0; c < 2; c++) out_plane_host(0, "L", c, HP[c][P_LP], hempty[c][P_LP]);
    W = st_calc_W_n;
    L = st_calc_L_n;
  } else {
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
  }

  int more_ww = 1, more_wb = 1, more_lw = 1, more_lb = 1, more_wb_next, more_ww_next;
  int n;
  /* tb8gen.c:1414-1444; after each ply the current W/L become the sources */
  for (n = 1; n <= max_ply; n++) {
    int special = n == DRAW_RULE + 1;
    if (n > DRAW_RULE + 1 && !(more_ww || more_wb || more_lw || more_lb)) break;
    if (special) {
      more_wb_next = timed(L, "l", WHITE, n, more_lw);
      more_ww_next = timed(L, "l", BLACK, n, more_lb);
      more_lb = timed(W, "w", WHITE, n, more_ww);
      more_lw = timed(W, "w", BLACK, n, more_wb);
    } else {
      more_wb_next = more_lw && timed(L, "l", WHITE, n, more_lw);
      more_ww_next = more_lb && timed(L, "l", BLACK, n, more_lb);
      more_lb = more_ww && timed(W, "w", WHITE, n, more_ww);
      more_lw = more_wb && timed(W, "w", BLACK, n, more_wb);
    }
    more_wb = more_wb_next;
    more_ww = more_ww_next;
    if (streamed) {
      swap_host_planes();
    } else {
      for (int c = 0; c < 2; c++) {
        swap_planes(Wp[c], Wc[c]);
        swap_planes(Lp[c], Lc[c]);
      }
    }
  }
  ok(tbg_sync(0), "sync");
  if (g_outdir)
    for (int c = 0; c < 2; c++) {
      if (!streamed) {
        out_plane_dev(0, "wins", c, wins[c]);
      } else if (g_dwins[c]) {
        uint8_t *pl[NS];
        for (int s = 0; s < NS; s++) pl[s] = DWIN(c, s);
        out_plane_dev(0, "wins", c, pl);
      } else {
        out_plane_host(0, "wins", c, HP[c][P_WINS], NULL);
      }
    }
  if (g_timing) {
    uint64_t launches = 0;
    ok(tbg_launches(&launches), "launches");
    fprintf(stderr, "stats launches=%llu h2d_bytes=%llu d2h_bytes=%llu plies=%d\n",
            (unsigned long long)launches, (unsigned long long)g_h2d_bytes,
            (unsigned long long)g_d2h_bytes, n - 1);
  }
  if (base) ok(tbg_free(base), "free");
  return 0;
}
