// Host side of the table format (tbg_table.h): the square tables of
// probe.c, set_enc_info, and the rANS code construction and frequency-table
// codec of rans.c, restated.
#include "tbg_table.h"

#include <algorithm>
#include <climits>

namespace tbg {

void build_enc_tables(EncTables &t) {
  memset(&t, 0, sizeof t);
  static const uint8_t tri_sq[10] = {1, 2, 3, 10, 11, 19, 0, 9, 18, 27};
  for (int i = 0; i < 10; i++) t.inv_triangle[i] = tri_sq[i];
  int nl = 0;
  for (int sq = 0; sq < 64; sq++) {
    int f = sq & 7, r = sq >> 3;
    t.offdiag[sq] = r > f ? 1 : r < f ? -1 : 0;
    t.flipdiag[sq] = (uint8_t)((f << 3) | r);
    int ff = f > 3 ? 7 - f : f, rr = r > 3 ? 7 - r : r;
    if (rr > ff) std::swap(rr, ff);
    for (int i = 0; i < 10; i++)
      if (tri_sq[i] == rr * 8 + ff) t.triangle[sq] = (uint8_t)i;
    if (f == r) t.diag[sq] = (uint8_t)f;
    else if (f + r == 7) t.diag[sq] = (uint8_t)(8 + r);
    if (f > r) {
      t.lower[sq] = (uint8_t)nl;
      t.inv_lower[nl++] = (uint8_t)sq;
    }
  }
  for (int sq = 0; sq < 64; sq++) {
    int f = sq & 7, r = sq >> 3;
    if (f < r) t.lower[sq] = t.lower[t.flipdiag[sq]];
    if (f == r) {
      t.lower[sq] = (uint8_t)(28 + f);
      t.inv_lower[28 + f] = (uint8_t)sq;
    }
  }
  for (int i = 0; i < 8; i++) {
    t.inv_diag[i] = (uint8_t)(9 * i);
    t.inv_diag[8 + i] = (uint8_t)(7 * (i + 1));
  }
  // KKIdx and KKSquare (probe.c:441-539)
  int next = 0, next_diag = 441;
  for (int k = 0; k < 10; k++)
    for (int sq = 0; sq < 64; sq++) {
      int wk = tri_sq[k];
      t.kkidx[k][sq] = -1;
      int df = (wk & 7) - (sq & 7), dr = (wk >> 3) - (sq >> 3);
      if (df >= -1 && df <= 1 && dr >= -1 && dr <= 1) continue;
      if (k >= 6) {
        if ((sq & 7) < (sq >> 3)) continue;
        if ((sq & 7) == (sq >> 3)) {
          t.kkidx[k][sq] = (int16_t)next_diag++;
          continue;
        }
      }
      t.kkidx[k][sq] = (int16_t)next++;
    }
  for (int k = 0; k < 10; k++)
    for (int sq = 0; sq < 64; sq++)
      if (t.kkidx[k][sq] >= 0) {
        t.kksq[t.kkidx[k][sq]][0] = tri_sq[k];
        t.kksq[t.kkidx[k][sq]][1] = (uint8_t)sq;
      }
  for (int k = 0; k < 8; k++)
    for (int n = 0; n < 64; n++) {
      uint64_t c = 1;
      for (int j = 0; j < k; j++) c = c * (uint64_t)(n - j) / (uint64_t)(j + 1);
      t.binom[k][n] = n < k ? 0u : (uint32_t)c;
    }
}

static uint64_t placements(uint64_t k, uint64_t n) {
  uint64_t f = 1;
  for (uint64_t i = 0; i < k; i++) f = f * (n - i) / (i + 1);
  return f;
}

uint64_t set_enc_info(EncInfoP &ei, const uint8_t *tb, int shift, int num, int kk) {
  memset(&ei, 0, sizeof ei);
  ei.num = num;
  ei.kk = kk;
  for (int i = 0; i < num; i++) ei.pieces[i] = (tb[i + 1] >> shift) & 0x0f;
  const int order = (tb[0] >> shift) & 0x0f;
  int k = ei.norm[0] = kk ? 2 : 3;
  for (int i = k; i < num; i += ei.norm[i])
    for (int j = i; j < num && ei.pieces[j] == ei.pieces[i]; j++) ei.norm[i]++;
  int n = 64 - k;
  uint64_t f = 1;
  for (int i = 0; k < num || i == order; i++) {
    if (i == order) {
      ei.factor[0] = f;
      f *= kk ? 462 : 31332;
    } else {
      ei.factor[k] = f;
      f *= placements(ei.norm[k], n);
      n -= ei.norm[k];
      k += ei.norm[k];
    }
  }
  ei.size = f;
  return f;
}

// normalize_freqs (rans.c:24-73): cumulative frequencies scaled to 2^16 in
// 16-bit arithmetic, every symbol that occurs keeping a nonzero width.
static void normalize(RansCodeHost &c, const int64_t *freq, int num) {
  uint64_t total = 0;
  for (int i = 0; i < num; i++) total += (uint64_t)freq[i];
  uint64_t sum = 0;
  c.cum_freq[0] = 0;
  for (int i = 0; i < num; i++) {
    sum += (uint64_t)freq[i];
    c.cum_freq[i + 1] = (uint16_t)(sum * (1ull << 16) / total);
  }
  for (int i = num + 1; i < 4096; i++) c.cum_freq[i] = c.cum_freq[num];
  for (int i = 0; i < num; i++)
    if (freq[i] && c.cum_freq[i + 1] == c.cum_freq[i]) {
      uint32_t best = UINT32_MAX;
      int steal = -1;
      for (int j = 0; j < 4095; j++) {
        uint32_t fr = (uint16_t)(c.cum_freq[j + 1] - c.cum_freq[j]);
        if (fr > 1 && fr < best) {
          best = fr;
          steal = j;
        }
      }
      if (steal < i)
        for (int j = steal + 1; j <= i; j++) c.cum_freq[j]--;
      else
        for (int j = i + 1; j <= steal; j++) c.cum_freq[j]++;
    }
  for (int i = 0; i < 4095; i++) c.d.freq[i] = (uint16_t)(c.cum_freq[i + 1] - c.cum_freq[i]);
  c.d.freq[4095] = 0;
}

// sort_freqs (rans.c:75-91): symbols renumbered by decreasing frequency.
static void sort_by_freq(RansCodeHost &c) {
  for (int i = 0; i < 4096; i++) c.map[i] = (uint16_t)i;
  for (int i = 0; i < 4096; i++)
    for (int j = i + 1; j < 4096; j++)
      if (c.d.freq[i] < c.d.freq[j]) {
        std::swap(c.d.freq[i], c.d.freq[j]);
        std::swap(c.map[i], c.map[j]);
      }
  for (int i = 0; i < 4096; i++) c.inv[c.map[i]] = (uint16_t)i;
  uint32_t sum = 0;
  for (int i = 0; i < 4096; i++) {
    c.cum_freq[i] = (uint16_t)sum;
    sum += c.d.freq[i];
  }
}

// make_alias_table (rans.c:95-143): 4096 buckets of 16 slots; a bucket's
// slots below its divider belong to the bucket's own symbol, the rest to
// its alias.  With an encoder code, alias_remap maps each symbol's
// cumulative slot to its bucket slot.
void make_alias(RansDecodeTab &d, RansCodeHost *c) {
  const uint16_t tgt = (uint16_t)((1u << 16) / 4096);
  static uint16_t remaining[4096], alias[4096], assigned[4096];
  static uint8_t divider[4096];
  for (int i = 0; i < 4096; i++) {
    remaining[i] = d.freq[i];
    divider[i] = (uint8_t)tgt;
    alias[i] = (uint16_t)i;
  }
  int large = 0, small = 0;
  for (;;) {
    while (large < 4096 && remaining[large] <= tgt) large++;
    if (large == 4096) break;
    while (remaining[small] >= tgt) small = (small + 1) & 4095;
    alias[small] = (uint16_t)large;
    divider[small] = (uint8_t)remaining[small];
    remaining[large] = (uint16_t)(remaining[large] - (tgt - remaining[small]));
    remaining[small] = tgt;
  }
  for (int b = 0; b < 4096; b++) {
    if (c)
      for (int i = 0; i < divider[b]; i++)
        c->alias_remap[c->cum_freq[b] + i] = (uint16_t)(b * tgt + i);
    assigned[b] = divider[b];
    d.entry[b].alias_div = (uint16_t)((alias[b] << 4) | (divider[b] & 15));
  }
  for (int b = 0; b < 4096; b++) {
    int s = alias[b];
    d.entry[b].start = (uint16_t)(s != b ? assigned[s] - divider[b] : 0);
    if (c)
      for (int i = divider[b]; i < tgt; i++)
        c->alias_remap[(uint16_t)(c->cum_freq[s] + assigned[s] + i - divider[b])] =
            (uint16_t)(b * tgt + i);
    assigned[s] = (uint16_t)(assigned[s] + tgt - divider[b]);
  }
}

void create_code(RansCodeHost &c, const int64_t *freq, int num_syms) {
  memset(&c, 0, sizeof c);
  normalize(c, freq, num_syms);
  sort_by_freq(c);
  make_alias(c.d, &c);
}

// Uniform and "top-weighted" value codes of the frequency table
// (rans_enc_val_uni / rans_enc_val_top, rans.c:155-199, and their decoders
// rans_dec_val_uni / rans_dec_val_top, rans.c:201-237).
static void enc_uni(uint64_t &r, uint32_t v, uint32_t vmin, uint32_t vmax, uint8_t *&p) {
  if (vmin == vmax) return;
  v -= vmin;
  uint32_t range = vmax - vmin + 1;
  uint32_t cum = (v << 16) / range;
  uint32_t fr = ((v + 1) << 16) / range - cum;
  uint64_t xmax = (uint64_t)fr << 47, x = r;
  if (x >= xmax) {
    p -= 4;
    wr_le32(p, (uint32_t)x);
    x >>= 32;
  }
  r = ((x / fr) << 16) + (x % fr) + cum;
}

static void enc_top(uint64_t &r, uint32_t v, uint32_t vmin, uint32_t vmax, uint32_t f,
                    uint8_t *&p) {
  if (vmin == vmax) return;
  uint32_t cum = (v - vmin) * f;
  uint32_t fr = v == vmax ? 65536 - cum : f;
  uint64_t xmax = (uint64_t)fr << 47, x = r;
  if (x >= xmax) {
    p -= 4;
    wr_le32(p, (uint32_t)x);
    x >>= 32;
  }
  r = ((x / fr) << 16) + (x % fr) + cum;
}

static uint32_t dec_uni(uint64_t &r, uint32_t vmin, uint32_t vmax) {
  if (vmin == vmax) return vmin;
  uint32_t range = vmax - vmin + 1;
  uint64_t x = r;
  uint32_t w = (uint32_t)(x & 0xffff);
  uint32_t v = (w * range + range - 1) >> 16;
  uint32_t cum = (v << 16) / range;
  uint32_t fr = ((v + 1) << 16) / range - cum;
  r = fr * (x >> 16) + (w - cum);
  return v + vmin;
}

static uint32_t dec_top(uint64_t &r, uint32_t vmin, uint32_t vmax, uint32_t f) {
  if (vmin == vmax) return vmin;
  uint64_t x = r;
  uint32_t w = (uint32_t)(x & 0xffff);
  uint32_t v = vmin + std::min(w / f, vmax - vmin);
  uint32_t cum = (v - vmin) * f;
  uint32_t fr = v == vmax ? 65536 - cum : f;
  r = fr * (x >> 16) + (w - cum);
  return v;
}

// The frequency-table codec decides between its two value codes with 32-bit
// int arithmetic (rans.c:256-263, 300-310); these reproduce that arithmetic,
// wraparound included, so that both sides take the same decisions.
static inline bool uni_wins(int vmax, int vmin, int left) {
  return (int32_t)((uint32_t)vmax * (uint32_t)(vmax - vmin + 1)) >= left;
}
static inline uint32_t top_weight(int vmax, int left) {
  return (uint32_t)((int32_t)((uint32_t)vmax << 16) / left);
}

std::vector<uint8_t> freq_table_bytes(const RansCodeHost &c, int num) {
  std::vector<uint8_t> buf(10000);
  uint8_t *end = buf.data() + buf.size(), *p = end;
  uint64_t r = kRansL;
  int bound[4097];
  bound[num] = 0;
  int R = 0;
  const uint16_t *fq = c.d.freq;
  for (int s = num - 1; s >= 0; s--) {
    int P = s > 0 ? fq[s - 1] : INT32_MAX;
    R += fq[s];
    int vmax = std::min(R, P);
    bound[s] = std::max(1, std::max(bound[s + 1], vmax - (int)fq[s]));
    if (bound[s] > bound[s + 1]) continue;
    int vmin = std::max((R + num - s - 1) / (num - s), vmax - bound[s]);
    if (uni_wins(vmax, vmin, num - s))
      enc_uni(r, fq[s], vmin, vmax, p);
    else
      enc_top(r, fq[s], vmin, vmax, top_weight(vmax, num - s), p);
  }
  for (int s = num - 1; s > 0; s--) enc_top(r, bound[s], 1, bound[s - 1], 1, p);
  enc_uni(r, bound[0], 0, (1 << 16) - ((1 << 16) + num - 1) / num, p);
  enc_uni(r, num, 2, 4095, p);
  rans_flush(r, p, p - 8);
  return std::vector<uint8_t>(p, end);
}

const uint8_t *read_freq_table(RansDecodeTab &d, int *num_syms, const uint8_t *p) {
  uint64_t r;
  rans_dec_init(r, p, p + 8);
  int num = (int)dec_uni(r, 2, 4095);
  *num_syms = num;
  memset(d.freq, 0, sizeof d.freq);
  rans_dec_renorm(r, p);
  d.freq[0] = (uint16_t)dec_uni(r, 0, (1 << 16) - ((1 << 16) + num - 1) / num);
  for (int s = 1; s < num; s++) {
    rans_dec_renorm(r, p);
    d.freq[s] = (uint16_t)dec_top(r, 1, d.freq[s - 1], 1);
  }
  int R = 1 << 16;
  for (int s = 0; s < num; s++) {
    int P = s > 0 ? d.freq[s - 1] : INT32_MAX;
    if (d.freq[s] > d.freq[s + 1] && s < num - 1) {
      d.freq[s] = (uint16_t)(std::min(R, P) - d.freq[s]);
      R -= d.freq[s];
      continue;
    }
    rans_dec_renorm(r, p);
    int vmax = std::min(R, P);
    int vmin = std::max((R + num - s - 1) / (num - s), vmax - (int)d.freq[s]);
    if (uni_wins(vmax, vmin, num - s))
      d.freq[s] = (uint16_t)dec_uni(r, vmin, vmax);
    else
      d.freq[s] = (uint16_t)dec_top(r, vmin, vmax, top_weight(vmax, num - s));
    R -= d.freq[s];
  }
  return p;
}

}  // namespace tbg
