/*
 * Oracle test infrastructure -- NOT product code.
 *
 * Reaches the reference's 7-piece table reader and WDL probe, compiled in
 * place from the reference sources: probe.c is #included so that its
 * `static` probe_table (probe.c:1522-1597) and table registry are reachable,
 * and the rANS code construction / frequency-table writer of rans.c is
 * called as the reference defines it.  Only tests load the resulting
 * oracle/_ref/libtbprobe.so, as the checker of the engine's table writer and
 * probe kernels.
 *
 * Substitutions, all outside the reference's algorithm:
 *  - The zstd entry points util.c links against are aborting stubs (the
 *    probe path never compresses).
 *  - refp_encode / refp_decode repeat probe_table's table lookup and
 *    side/flip choice (probe.c:1527-1583) to return encode_piece's index, and
 *    build a DecInfo with set_dec_info from the table's own header for
 *    decode_piece (probe.c:773-837, 1022).
 */
#include <stdlib.h>

#include "probe.c"
#include <zstd.h>

size_t ZSTD_compressBound(size_t n) { (void)n; abort(); }
ZSTD_CCtx *ZSTD_createCCtx(void) { abort(); }
ZSTD_DCtx *ZSTD_createDCtx(void) { abort(); }
size_t ZSTD_compressCCtx(ZSTD_CCtx *c, void *d, size_t dc, const void *s,
                         size_t sn, int l)
{ (void)c; (void)d; (void)dc; (void)s; (void)sn; (void)l; abort(); }
size_t ZSTD_decompressDCtx(ZSTD_DCtx *c, void *d, size_t dc, const void *s,
                           size_t sn)
{ (void)c; (void)d; (void)dc; (void)s; (void)sn; abort(); }

/* init_tablebases over one directory; returns the WDL tables found. */
int refp_init(const char *dir)
{
  static bool once = false;
  if (once) free_tablebases();
  num_paths = 0;
  num_wdl = num_dtm = 0;
  init_tablebases(dir);
  once = true;
  return num_wdl;
}

/* A query: sq[8], stm, 7 pad bytes (16 bytes); pt[] the material order. */
static void make_pos(Position *pos, const uint8_t *pt, int num, const uint8_t *q)
{
  memset(pos, 0, sizeof *pos);
  pos->num = num;
  pos->stm = q[8];
  for (int i = 0; i < num; i++) {
    pos->pt[i] = pt[i];
    pos->sq[i] = q[i];
    pos->occ |= 1ULL << q[i];
  }
}

/* probe_table(pos, 0, WDL) for n queries. */
void refp_probe(const uint8_t *pt, int num, const uint8_t *queries, uint64_t n, int8_t *out)
{
  Position pos;
  for (uint64_t i = 0; i < n; i++) {
    make_pos(&pos, pt, num, queries + 16 * i);
    out[i] = (int8_t)probe_table(&pos, 0, WDL);
  }
}

static struct BaseEntry *entry_of(const uint8_t *pt, int num, uint64_t *key_out)
{
  uint64_t key = 0;
  for (int i = 0; i < num; i++)
    key += MaterialPieceKey[pt[i]];
  int h = key >> (64 - TB_HASHBITS);
  while (tb_hash[h].key && tb_hash[h].key != key)
    h = (h + 1) & ((1 << TB_HASHBITS) - 1);
  *key_out = key;
  return tb_hash[h].ptr;
}

/* encode_piece as probe_table reaches it: table index and side. */
int refp_encode(const uint8_t *pt, int num, const uint8_t *queries, uint64_t n,
                uint64_t *idx, uint8_t *side)
{
  Position pos;
  if (n == 0) return 0;
  make_pos(&pos, pt, num, queries);
  (void)probe_table(&pos, 0, WDL); /* maps the table */
  uint64_t key;
  struct BaseEntry *be = entry_of(pt, num, &key);
  if (!be || be->has_pawns) return -1;
  for (uint64_t i = 0; i < n; i++) {
    make_pos(&pos, pt, num, queries + 16 * i);
    bool bside, flip;
    if (!be->symmetric) {
      flip = key != be->key;
      bside = (pos.stm == WHITE) == flip;
    } else {
      flip = pos.stm != WHITE;
      bside = false;
    }
    struct EncInfo *ei = &first_ei(be, WDL)[bside];
    uint8_t p[8] = { 0 };
    list_squares(&pos, ei->pieces, flip, p, be->num);
    idx[i] = encode_piece(p, ei, be);
    side[i] = bside;
  }
  return 0;
}

/* decode_piece for side `bside` of the (already mapped) table of pt[]:
 * squares in table order, 8 bytes per index. */
int refp_decode(const uint8_t *pt, int num, int bside, const uint64_t *idx, uint64_t n,
                uint8_t *squares)
{
  uint64_t key;
  struct BaseEntry *be = entry_of(pt, num, &key);
  if (!be || !be->ready[WDL] || be->has_pawns) return -1;
  struct EncInfo *ei = &first_ei(be, WDL)[bside];
  /* set_dec_info walks its type_perm[] index from norm[0] on, one step per
   * group of like pieces; give it the table's own group sizes there. */
  uint8_t pcs[16] = { 0 }, perm[16] = { 0 };
  int k = be->kk_enc ? 2 : 3, i = k;
  for (; k < be->num; k += ei->norm[k], i++) {
    perm[i] = (uint8_t)i;
    pcs[i] = ei->norm[k];
  }
  int order = (be->data[WDL][5] >> (bside ? 4 : 0)) & 0x0f;
  struct DecInfo di;
  set_dec_info(&di, be, pcs, perm, order, 0x0f, 0, PIECE_ENC);
  for (uint64_t j = 0; j < n; j++) {
    uint8_t p[8] = { 0 };
    decode_piece(idx[j], p, &di, be);
    memcpy(squares + 8 * j, p, 8);
  }
  return 0;
}

/* create_code_rans + write_freq_table (rans.c:145-152, 239-276) for a
 * histogram: the sorted frequencies, cumulative frequencies, alias remap,
 * symbol map and the frequency-table bytes. */
int refp_code(const int64_t *freq, int num, uint16_t *freq_out, uint16_t *cum_out,
              uint16_t *remap_out, uint16_t *map_out, uint8_t *ftab, uint64_t *ftab_len)
{
  int64_t f[4096] = { 0 };
  memcpy(f, freq, num * sizeof *f);
  struct RansCode *c = create_code_rans(f, num);
  memcpy(freq_out, c->d.freq, sizeof c->d.freq);
  memcpy(cum_out, c->cum_freq, sizeof c->cum_freq);
  memcpy(remap_out, c->alias_remap, sizeof c->alias_remap);
  memcpy(map_out, c->map, sizeof c->map);
  char *buf = NULL;
  size_t len = 0;
  FILE *F = open_memstream(&buf, &len);
  if (!F) {
    free_code_rans(c);
    return -1;
  }
  size_t nb = write_freq_table(F, c, num);
  fclose(F);
  memcpy(ftab, buf, nb);
  *ftab_len = nb;
  free(buf);
  free_code_rans(c);
  return 0;
}

/* read_freq_table + make_alias_table(d, NULL) (rans.c:278-314, 95-143). */
int refp_read_code(const uint8_t *ftab, uint16_t *freq_out, uint16_t *alias_div,
                   uint16_t *start, uint64_t *consumed)
{
  struct RansDecode *d = calloc(1, sizeof *d);
  int num;
  const uint8_t *p = read_freq_table(d, &num, ftab);
  make_alias_table(d, NULL);
  memcpy(freq_out, d->freq, sizeof d->freq);
  for (int i = 0; i < 4096; i++) {
    alias_div[i] = d->entry[i].alias_div;
    start[i] = d->entry[i].start;
  }
  *consumed = (uint64_t)(p - ftab);
  free(d);
  return num;
}
