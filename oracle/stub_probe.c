/*
 * Oracle test infrastructure -- NOT product code.
 *
 * The seeded 7-piece WDL stub linked into the unmodified reference program
 * (oracle/_ref/tb8gen_stub, recipe in oracle/Makefile) in place of
 * probe_wdl (probe.c:1677), so that the reference generates materials whose
 * capture successors would need tables that do not exist here.  Same formula
 * as oracle/ref_harness.c; seed and modulus from TB8GEN_STUB_SEED and
 * TB8GEN_STUB_MOD (default 1 and 3).
 */
#include <stdint.h>
#include <stdlib.h>

#include "movegen.h"

static uint64_t s_mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

int harness_probe_wdl(Position *pos, int alpha, int beta)
{
  (void)alpha;
  (void)beta;
  static uint64_t seed = 0;
  static int mod = 0;
  if (!mod) {
    const char *a = getenv("TB8GEN_STUB_SEED"), *b = getenv("TB8GEN_STUB_MOD");
    seed = a ? strtoull(a, NULL, 10) : 1;
    mod = b && atoi(b) == 5 ? 5 : 3;
  }
  if (pos->num == 2) return 0;  /* KvK, as probe_table (probe.c:1525) */
  const uint64_t gamma = 0x9e3779b97f4a7c15ULL;
  uint64_t key = pos->stm ? 0xd1b54a32d192ed03ULL : 0;
  for (int i = 0; i < pos->num; i++)
    key ^= s_mix64((((uint64_t)pos->pt[i] << 6) | pos->sq[i]) * gamma + gamma);
  uint64_t h = s_mix64(seed ^ key);
  if (mod == 5)
    return (int)(h % 5) - 2;
  return (int)(h % 3) * 2 - 2;
}
