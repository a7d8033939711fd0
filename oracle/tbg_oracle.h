/*
 * Oracle test infrastructure -- NOT product code.
 *
 * A plain-C restatement of the reference generator's per-king-slice ply step
 * (tb8gen.c, kslice.c, movegen.h, probe.c index tables), used only by the
 * tests, the smoke check and bench.py's CPU-baseline leg to check the CUDA
 * path.  Each function cites the reference lines it follows.  It is pinned
 * against the reference's own workers (oracle/_ref/libtbref.so, built from the
 * reference sources by oracle/Makefile) and against fixtures generated from
 * them (tests/golden/).
 */
#ifndef TBG_ORACLE_H
#define TBG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#define ORC_MAX_SETS 6

/* struct IdxInfo, tb8gen.h:4-13 */
typedef struct {
  int numsets;
  uint64_t size;
  uint64_t factor[ORC_MAX_SETS];
  uint32_t subfactor[ORC_MAX_SETS];
  int first[ORC_MAX_SETS], mult[ORC_MAX_SETS], last[ORC_MAX_SETS];
} orc_idx;

typedef struct {
  int num;               /* pieces, kings included */
  uint8_t pt[8];         /* piece types in index order (tb8gen.c:1331-1342) */
  int8_t pcs[2][8];      /* piece indices per colour, -1 ended */
  int pc_to_set[8];
  orc_idx ii, capt[ORC_MAX_SETS];
  uint64_t bytes;        /* slice bitmap bytes, 64-B rounded (kslice.c:191-196) */
  uint64_t sub_offset[ORC_MAX_SETS];
  uint64_t sub_size[2];
  uint64_t sub_bytes;    /* per-slice sub buffer = max(sub_size) */
  /* slot map: slice -> bitmap / sub buffer (kslice_slot / kslice_buf,
   * kslice.c:23-28); index 0 is the scratch slot -1. */
  uint8_t *slot[463];
  uint8_t *sub[463];
  uint64_t oob_reads;    /* reads past a bound sub buffer (none expected) */
  uint64_t stub_seed;
  int stub_mod;
} orc_ctx;

int orc_init(void);
int orc_setup(orc_ctx *c, const char *material);
void orc_bind(orc_ctx *c, int s, void *bitmap, void *sub);
void orc_unbind_all(orc_ctx *c);

void orc_predecessors(orc_ctx *c, int stm, int s);
void orc_predecessors_sub(orc_ctx *c, int stm, int s, int legality);
void orc_check_successors(orc_ctx *c, int stm, int s);
void orc_calc_sub(orc_ctx *c, int stm, int s, void *const cls[5]);
void orc_calc_illegal(orc_ctx *c, int s, void *ill_w, void *ill_b);
void orc_calc_mate(orc_ctx *c, int s, void *ill_w, void *ill_b, void *mate_w,
                   void *mate_b);
uint64_t orc_epilogue_W(orc_ctx *c, void *T, void *wins);
uint64_t orc_count(orc_ctx *c, const void *p);

void orc_gen_bernoulli(void *p, uint64_t nbits, uint64_t bytes, uint64_t seed,
                       uint64_t tag, uint64_t thr);

/* Tables and helpers exposed for pinning. */
int orc_kkidx(int t, int sq);
int orc_kkmap(int a, int b);
int orc_kksquare(int s, int i);
int orc_fliptest(int a, int b);
uint64_t orc_rook_attacks(int sq, uint64_t occ);
uint64_t orc_bishop_attacks(int sq, uint64_t occ);
uint64_t orc_sq_to_idx(orc_ctx *c, const uint8_t *sq8, int k);
uint64_t orc_idx_to_sq(orc_ctx *c, uint64_t idx, int s, int k, uint8_t *sq8);
int orc_manager(int stm, int i, int16_t *in, int16_t *out);
int orc_stub_value(uint64_t seed, int modulus, const uint8_t *pt,
                   const uint8_t *sq, int num, int stm);
uint64_t orc_mix64(uint64_t z);

#endif
