// C ABI of the table probe (include/tbgpu.h, "7-piece table probes"): the
// synthetic table builder, the table reader (init_table, probe.c:1210-1344)
// and the probe, encode and decode batches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/tbgpu.h"
#include "tbg_host.h"
#include "tbg_probe.cuh"

namespace tbg {

int cuda_fail(cudaError_t e, const char *what);

#define PCK(call)                                           \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);     \
  } while (0)

static EncTables g_enc;
static bool g_enc_ready = false;
static EncTables *d_enc = nullptr;

static int enc_tables() {
  if (!g_enc_ready) {
    build_enc_tables(g_enc);
    g_enc_ready = true;
  }
  return TBG_OK;
}

static int enc_tables_device() {
  enc_tables();
  if (!d_enc) {
    PCK(cudaMalloc(&d_enc, sizeof(EncTables)));
    PCK(cudaMemcpy(d_enc, &g_enc, sizeof(EncTables), cudaMemcpyHostToDevice));
    PCK(cudaStreamSynchronize(0));  // legacy-stream upload, before any stream reads it
  }
  return TBG_OK;
}

static const uint32_t kTableMagic = 0x5d23e871;  // WDL tables (probe.c:33)

// A material as the probe sees it: the query squares' piece types in the
// order of main() (tb8gen.c:1331-1339), and the table's piece order: the
// kings first, then, when more than the kings are unique (no kk_enc), one
// more unique piece, then the groups of like pieces.
struct Spec {
  int num = 0, kk = 0, symmetric = 0;
  uint8_t pt[8] = {0};      // query order
  uint8_t table[8] = {0};   // table order
};

static int spec_from_name(const char *name, Spec &sp) {
  static const int order[16] = {0, 0, 3, 5, 7, 9, 1, 0, 0, 0, 4, 6, 8, 10, 2, 0};
  static const char *letters = "PNBRQK";
  int pt[8], n = 0, black = 0, cnt[16] = {0};
  for (const char *p = name; *p; p++) {
    if (*p == 'v' && !black) {
      black = 8;
      continue;
    }
    const char *q = strchr(letters, *p);
    if (!q) continue;
    int t = (int)(q - letters) + 1;
    if (t == 1 || n >= 8) return fail(TBG_ERR_ARG, "material %s not supported", name);
    pt[n++] = t | black;
    cnt[t | black]++;
  }
  if (!black || n < 3 || cnt[6] != 1 || cnt[14] != 1) return fail(TBG_ERR_ARG, "bad material %s", name);
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (order[pt[i]] > order[pt[j]]) std::swap(pt[i], pt[j]);
  sp.num = n;
  for (int i = 0; i < n && i < 8; i++) sp.pt[i] = (uint8_t)pt[i];
  int uniq = 0;
  for (int i = 0; i < 16; i++) uniq += cnt[i] == 1;
  sp.kk = uniq == 2;
  sp.symmetric = 1;
  for (int t = 1; t <= 6; t++) sp.symmetric &= cnt[t] == cnt[t + 8];
  int k = 0;
  sp.table[k++] = 6;
  sp.table[k++] = 14;
  bool used[8] = {false};
  used[0] = used[1] = true;
  if (!sp.kk)
    for (int i = 2; i < n; i++)
      if (cnt[pt[i]] == 1) {
        sp.table[k++] = (uint8_t)pt[i];
        used[i] = true;
        break;
      }
  for (int i = 2; i < n; i++)
    if (!used[i]) sp.table[k++] = (uint8_t)pt[i];
  return TBG_OK;
}

// The table layout of a material (for callers outside this file): its
// EncInfo, symmetry, the query order and the table order of its pieces.
int sub_layout(const char *material, EncInfoP *ei, int *symmetric, uint8_t qpt[8],
               uint8_t tpt[8], int *num) {
  Spec sp;
  int rc = spec_from_name(material, sp);
  if (rc) return rc;
  uint8_t hdr[9] = {0};
  for (int i = 0; i < sp.num; i++) hdr[1 + i] = (uint8_t)(sp.table[i] | (sp.table[i] << 4));
  set_enc_info(*ei, hdr, 0, sp.num, sp.kk);
  *symmetric = sp.symmetric;
  memcpy(qpt, sp.pt, 8);
  memcpy(tpt, sp.table, 8);
  *num = sp.num;
  return TBG_OK;
}

const EncTables *enc_tables_dev() { return enc_tables_device() == TBG_OK ? d_enc : nullptr; }

// ------------------------------------------------------------------ build
// Layout of one table side's pairs data (setup_pairs / setup_rans,
// probe.c:1179-1206, 1156-1177).
struct SideBuild {
  EncInfoP ei;
  uint64_t nblocks = 0;
  RansCodeHost *code = nullptr;
  int num_syms = 0;
  std::vector<uint8_t> pairs;   // flags .. freq table .. sympat (+pad)
  std::vector<uint16_t> quad_code;
  uint64_t off_index = 0, off_sizes = 0, off_data = 0;
};

static void make_pairs(SideBuild &sb, const std::vector<int64_t> &quad_hist, int M, int modulus) {
  const int nsyms = M + M * M + M * M * M * M;
  std::vector<int64_t> freq(nsyms, 0);
  for (int q = 0; q < M * M * M * M; q++) freq[M + M * M + q] = quad_hist[q];
  sb.code = new RansCodeHost;
  create_code(*sb.code, freq.data(), nsyms);
  sb.num_syms = nsyms;
  const RansCodeHost &c = *sb.code;
  sb.quad_code.resize(M * M * M * M);
  for (int q = 0; q < M * M * M * M; q++) sb.quad_code[q] = c.inv[M + M * M + q];
  std::vector<uint8_t> ft = freq_table_bytes(c, nsyms);
  sb.pairs.assign(10, 0);
  sb.pairs[0] = 0x40;                       // rANS
  sb.pairs[1] = kBlockBits;                 // block_size
  sb.pairs[2] = kIdxBits;                   // idx_bits
  sb.pairs[3] = 0;
  wr_le32(&sb.pairs[4], (uint32_t)sb.nblocks);
  sb.pairs.insert(sb.pairs.end(), ft.begin(), ft.end());
  // sympat in code order: leaves (value byte, s2 = 0xfff), pairs, quads
  std::vector<uint8_t> sym(3 * nsyms);
  for (int i = 0; i < nsyms; i++) {
    int o = c.map[i];
    uint8_t *w = &sym[3 * i];
    if (o < M) {
      w[0] = (uint8_t)(modulus == 5 ? o : 2 * o);
      w[1] = 0xf0;
      w[2] = 0xff;
      continue;
    }
    int s1, s2;
    if (o < M + M * M) {
      int ab = o - M;
      s1 = c.inv[ab / M];
      s2 = c.inv[ab % M];
    } else {
      int q = o - M - M * M;
      s1 = c.inv[M + q / (M * M)];
      s2 = c.inv[M + q % (M * M)];
    }
    w[0] = (uint8_t)(s1 & 0xff);
    w[1] = (uint8_t)(((s1 >> 8) & 0xf) | ((s2 & 0xf) << 4));
    w[2] = (uint8_t)(s2 >> 4);
  }
  sb.pairs.insert(sb.pairs.end(), sym.begin(), sym.end());
  if (nsyms & 1) sb.pairs.push_back(0);
}

static int build_table(const char *material, uint64_t seed, int modulus, bool device,
                       void **out, uint64_t *out_bytes) {
  Spec sp;
  int rc = spec_from_name(material, sp);
  if (rc) return rc;
  if (modulus != 3 && modulus != 5) return fail(TBG_ERR_ARG, "modulus 3 or 5");
  enc_tables();
  const int M = modulus;
  const int sides = sp.symmetric ? 1 : 2;
  std::vector<uint8_t> head(4);
  wr_le32(head.data(), kTableMagic);
  head.push_back((uint8_t)(sides == 2 ? 1 : 0));   // split
  head.push_back(0);                                // order nibbles (0, 0)
  for (int i = 0; i < sp.num; i++) head.push_back((uint8_t)(sp.table[i] | (sp.table[i] << 4)));
  if (head.size() & 1) head.push_back(0);
  SideBuild sb[2];
  for (int b = 0; b < sides; b++) {
    set_enc_info(sb[b].ei, &head[5], b ? 4 : 0, sp.num, sp.kk);
    sb[b].nblocks = side_blocks(sb[b].ei.size);
  }
  // histograms of the quad symbols
  const int nq = M * M * M * M;
  std::vector<int64_t> hist[2];
  unsigned long long *d_hist = nullptr;
  if (device) PCK(cudaMalloc(&d_hist, nq * sizeof(unsigned long long)));
  for (int b = 0; b < sides; b++) {
    hist[b].assign(nq, 0);
    const uint64_t size = sb[b].ei.size;
    if (device) {
      PCK(cudaMemset(d_hist, 0, nq * sizeof(unsigned long long)));
      k_tbl_hist<<<g_eng.num_sms * 8, 256>>>(size, seed, b, M, d_hist);
      PCK(cudaGetLastError());
      std::vector<unsigned long long> h(nq);
      PCK(cudaMemcpy(h.data(), d_hist, nq * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
      for (int q = 0; q < nq; q++) hist[b][q] = (int64_t)h[q];
    } else {
      const uint64_t nquads = side_quads(size);
      for (uint64_t q = 0; q < nquads; q++) hist[b][quad_values(seed, M, b, size, q)]++;
    }
    make_pairs(sb[b], hist[b], M, M);
  }
  if (d_hist) cudaFree(d_hist);
  // offsets (init_table, probe.c:1296-1331)
  uint64_t off = head.size();
  for (int b = 0; b < sides; b++) off += sb[b].pairs.size();
  for (int b = 0; b < sides; b++) {
    sb[b].off_index = off;
    off += 6 * sb[b].nblocks;
  }
  for (int b = 0; b < sides; b++) {
    sb[b].off_sizes = off;
    off += 2 * sb[b].nblocks;
  }
  for (int b = 0; b < sides; b++) {
    off = (off + 63) & ~63ull;
    sb[b].off_data = off;
    off += sb[b].nblocks << kBlockBits;
  }
  const uint64_t total = off;
  // header, pairs, index and size tables on the host
  std::vector<uint8_t> front(sb[0].off_data, 0);
  memcpy(front.data(), head.data(), head.size());
  uint64_t o = head.size();
  for (int b = 0; b < sides; b++) {
    memcpy(front.data() + o, sb[b].pairs.data(), sb[b].pairs.size());
    o += sb[b].pairs.size();
  }
  for (int b = 0; b < sides; b++) {
    const uint64_t size = sb[b].ei.size;
    for (uint64_t k = 0; k < sb[b].nblocks; k++) {
      // entry k: the middle position of its 2^16 range lies in block k
      uint8_t *e = front.data() + sb[b].off_index + 6 * k;
      wr_le32(e, (uint32_t)k);
      e[4] = 0x00;
      e[5] = 0x80;
      const uint32_t npos = block_positions(size, k);
      uint8_t *z = front.data() + sb[b].off_sizes + 2 * k;
      z[0] = (uint8_t)(npos - 1);
      z[1] = (uint8_t)((npos - 1) >> 8);
    }
  }
  uint8_t *table = nullptr;
  uint32_t overflow = 0;
  if (device) {
    PCK(cudaMalloc(&table, total));
    PCK(cudaMemset(table, 0, total));
    PCK(cudaMemcpy(table, front.data(), front.size(), cudaMemcpyHostToDevice));
    uint16_t *d_code;
    uint32_t *d_over;
    PCK(cudaMalloc(&d_code, (3 * 4096 + 65536 + nq) * sizeof(uint16_t)));
    PCK(cudaMalloc(&d_over, sizeof(uint32_t)));
    PCK(cudaMemset(d_over, 0, sizeof(uint32_t)));
    for (int b = 0; b < sides; b++) {
      const RansCodeHost &c = *sb[b].code;
      PCK(cudaMemcpy(d_code, c.d.freq, 4096 * 2, cudaMemcpyHostToDevice));
      PCK(cudaMemcpy(d_code + 4096, c.cum_freq, 4096 * 2, cudaMemcpyHostToDevice));
      PCK(cudaMemcpy(d_code + 8192, c.alias_remap, 65536 * 2, cudaMemcpyHostToDevice));
      PCK(cudaMemcpy(d_code + 8192 + 65536, sb[b].quad_code.data(), nq * 2, cudaMemcpyHostToDevice));
      const uint64_t nb = sb[b].nblocks;
      k_tbl_encode<<<(unsigned)((nb + 127) / 128), 128>>>(
          sb[b].ei.size, seed, b, M, d_code, d_code + 4096, d_code + 8192, d_code + 8192 + 65536,
          table + sb[b].off_data, nb, d_over);
      PCK(cudaGetLastError());
    }
    PCK(cudaDeviceSynchronize());
    PCK(cudaMemcpy(&overflow, d_over, sizeof overflow, cudaMemcpyDeviceToHost));
    cudaFree(d_code);
    cudaFree(d_over);
  } else {
    table = static_cast<uint8_t *>(calloc(total, 1));
    if (!table) return fail(TBG_ERR_NOMEM, "host table of %llu bytes", (unsigned long long)total);
    memcpy(table, front.data(), front.size());
    for (int b = 0; b < sides; b++) {
      const RansCodeHost &c = *sb[b].code;
      for (uint64_t k = 0; k < sb[b].nblocks; k++) {
        uint8_t *start = table + sb[b].off_data + (k << kBlockBits);
        uint8_t *p = start + (1ull << kBlockBits);
        uint64_t x = kRansL;
        const uint64_t q0 = k * kQuadsPerBlock, q1 = q0 + block_quads(sb[b].ei.size, k);
        for (uint64_t q = q0; q < q1; q++) {
          int s = sb[b].quad_code[quad_values(seed, M, b, sb[b].ei.size, q)];
          if (!rans_put(x, c.d.freq, c.cum_freq, c.alias_remap, s, p, start + 8)) {
            overflow++;
            break;
          }
        }
        rans_flush(x, p, start);
      }
    }
  }
  for (int b = 0; b < sides; b++) delete sb[b].code;
  if (overflow) return fail(TBG_ERR_DEVICE, "%u blocks overflowed", overflow);
  *out = table;
  *out_bytes = total;
  return TBG_OK;
}

// ------------------------------------------------------------------ open
struct ProbeHandle {
  bool used = false;
  ProbeTable P;
  Spec sp;
  const uint8_t *base = nullptr;  // the table image
  void *dev_alloc = nullptr;   // decode tables and symlen of both sides
  uint16_t *dev_starts = nullptr;  // stream start of every block (k_block_starts)
  uint64_t stream_bytes[2] = {0, 0};  // per side: bytes from each stream's start to its block's end
  uint64_t nkeys = 0;
  // scratch, grown on demand
  uint32_t *key = nullptr, *lit = nullptr;
  uint64_t cap_q = 0;
  uint32_t *minlit = nullptr, *tpos = nullptr, *list = nullptr, *tile = nullptr;
  uint8_t *symbuf = nullptr;   // decoded symbols (bytes)
  uint64_t cap_sym = 0;
  // events of the last grouped batch: start, first decode, after the last
  // decode, end
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool timed = false;
  uint64_t touched = 0;        // blocks decoded by the last grouped batch
  bool touched_on_device = false;  // ... still in bounds[0] (no host read yet)
  uint32_t *bounds = nullptr;  // touched blocks, touched blocks of side 0
};

static ProbeHandle g_probe[8];
// Device bytes of decoded-symbol scratch a grouped probe may hold.
static uint64_t g_probe_scratch = 16ull << 30;

static void calc_symlen(std::vector<uint8_t> &len, std::vector<char> &done, const uint8_t *sympat,
                        int s) {
  const uint8_t *w = sympat + 3 * s;
  int s2 = (w[2] << 4) | (w[1] >> 4);
  if (s2 == 0xfff) {
    len[s] = 0;
  } else {
    int s1 = ((w[1] & 0xf) << 8) | w[0];
    if (!done[s1]) calc_symlen(len, done, sympat, s1);
    if (!done[s2]) calc_symlen(len, done, sympat, s2);
    len[s] = (uint8_t)(len[s1] + len[s2] + 1);
  }
  done[s] = 1;
}

static int open_table(const uint8_t *dev_table, uint64_t bytes, const char *material, int *handle) {
  int h = -1;
  for (int i = 0; i < 8; i++)
    if (!g_probe[i].used) {
      h = i;
      break;
    }
  if (h < 0) return fail(TBG_ERR_RANGE, "at most 8 open tables");
  if (reinterpret_cast<uintptr_t>(dev_table) & 63)
    return fail(TBG_ERR_ARG, "table image must start on a 64-byte boundary");
  ProbeHandle &H = g_probe[h];
  H = ProbeHandle();
  H.base = dev_table;
  int rc = spec_from_name(material, H.sp);
  if (rc) return rc;
  rc = enc_tables_device();
  if (rc) return rc;
  // the front of the table: header, pairs data (a few KiB)
  uint64_t nfront = std::min<uint64_t>(bytes, 1 << 20);
  std::vector<uint8_t> f(nfront);
  PCK(cudaMemcpy(f.data(), dev_table, nfront, cudaMemcpyDeviceToHost));
  if (rd_le32(f.data()) != kTableMagic) return fail(TBG_ERR_ARG, "not a WDL table");
  const bool split = f[4] & 1;
  const int sides = split ? 2 : 1;
  const int num = H.sp.num;
  uint64_t o = 5;
  for (int b = 0; b < sides; b++)
    set_enc_info(H.P.side[b].ei, &f[o], b ? 4 : 0, num, H.sp.kk);
  o += num + 1;
  o += o & 1;
  struct Parsed {
    uint64_t nblocks, num_idx;
    int idx_bits, block_size, num_syms;
    RansDecodeTab dt;
    uint64_t sympat_off;
    std::vector<uint8_t> symlen;
  } ps[2];
  for (int b = 0; b < sides; b++) {
    const uint8_t *d = &f[o];
    if (d[0] & 0x80) return fail(TBG_ERR_ARG, "constant tables are not supported");
    if (!(d[0] & 0x40)) return fail(TBG_ERR_ARG, "only rANS-compressed tables are supported");
    ps[b].block_size = d[1];
    ps[b].idx_bits = d[2];
    uint64_t real = rd_le32(d + 4);
    ps[b].nblocks = real + d[3];
    const uint8_t *p = read_freq_table(ps[b].dt, &ps[b].num_syms, d + 10);
    make_alias(ps[b].dt, nullptr);
    ps[b].sympat_off = (uint64_t)(p - f.data());
    ps[b].symlen.assign(ps[b].num_syms, 0);
    std::vector<char> done(ps[b].num_syms, 0);
    for (int s = 0; s < ps[b].num_syms; s++)
      if (!done[s]) calc_symlen(ps[b].symlen, done, p, s);
    o = (uint64_t)(p - f.data()) + 3 * ps[b].num_syms + (ps[b].num_syms & 1);
    uint64_t size = H.P.side[b].ei.size;
    ps[b].num_idx = (size + (1ull << ps[b].idx_bits) - 1) >> ps[b].idx_bits;
    ps[b].nblocks = real;
  }
  uint64_t off_index[2], off_sizes[2], off_data[2];
  for (int b = 0; b < sides; b++) {
    off_index[b] = o;
    o += 6 * ps[b].num_idx;
  }
  for (int b = 0; b < sides; b++) {
    off_sizes[b] = o;
    o += 2 * (ps[b].nblocks);
  }
  for (int b = 0; b < sides; b++) {
    o = (o + 63) & ~63ull;
    off_data[b] = o;
    o += ps[b].nblocks << ps[b].block_size;
  }
  if (o > bytes) return fail(TBG_ERR_ARG, "table truncated (%llu > %llu)", (unsigned long long)o,
                             (unsigned long long)bytes);
  // device copies of the decode tables and symbol lengths
  const size_t per = sizeof(RansDecodeTab) + 4096;
  PCK(cudaMalloc(&H.dev_alloc, per * sides));
  uint32_t key0 = 0;
  for (int b = 0; b < sides; b++) {
    uint8_t *base = static_cast<uint8_t *>(H.dev_alloc) + per * b;
    PCK(cudaMemcpy(base, &ps[b].dt, sizeof(RansDecodeTab), cudaMemcpyHostToDevice));
    PCK(cudaMemcpy(base + sizeof(RansDecodeTab), ps[b].symlen.data(), ps[b].num_syms,
                   cudaMemcpyHostToDevice));
    PCK(cudaStreamSynchronize(0));  // legacy-stream uploads, before any stream reads them
    ProbeSide &S = H.P.side[b];
    S.index = dev_table + off_index[b];
    S.sizes = dev_table + off_sizes[b];
    S.data = dev_table + off_data[b];
    S.entry = reinterpret_cast<const RansEntry *>(base);
    S.freq = reinterpret_cast<const uint16_t *>(base + offsetof(RansDecodeTab, freq));
    S.sympat = dev_table + ps[b].sympat_off;
    S.symlen = base + sizeof(RansDecodeTab);
    S.nblocks = ps[b].nblocks;
    S.key0 = key0;
    key0 += (uint32_t)ps[b].nblocks;
    S.idx_bits = ps[b].idx_bits;
    S.block_size = ps[b].block_size;
    // one position count for every symbol the code can emit
    int L = -1;
    bool same = true;
    for (int s = 0; s < ps[b].num_syms; s++)
      if (ps[b].dt.freq[s]) {
        if (L < 0) L = ps[b].symlen[s];
        else same &= L == ps[b].symlen[s];
      }
    S.sym_positions = same && L >= 0 ? L + 1 : 0;
    S.nsym_emit = 0;
    for (int s = 0; s < ps[b].num_syms; s++)
      if (ps[b].dt.freq[s]) S.nsym_emit = s + 1;
  }
  if (sides == 1) H.P.side[1] = ProbeSide();
  // where every block's stream begins: the decoders' zero-padding scan, done
  // once here (block offsets in 32-bit words fit 16 bits up to 256 KiB blocks)
  if (H.P.side[0].block_size >= 4 && H.P.side[0].block_size <= 18 &&
      (sides == 1 || H.P.side[1].block_size == H.P.side[0].block_size)) {
    const uint64_t nb = H.P.side[0].nblocks + (sides == 2 ? H.P.side[1].nblocks : 0);
    PCK(cudaMalloc(&H.dev_starts, std::max<uint64_t>(nb, 1) * sizeof(uint16_t)));
    uint16_t *st = H.dev_starts;
    for (int b = 0; b < sides; b++) {
      ProbeSide &S = H.P.side[b];
      k_block_starts<<<g_eng.num_sms * 8, 256, 0, g_eng.stream>>>(S, st);
      int rc = g_eng.check_launch("k_block_starts");
      if (rc) return rc;
      S.start = st;
      st += S.nblocks;
    }
    PCK(cudaStreamSynchronize(g_eng.stream));
    std::vector<uint16_t> hs(nb);
    PCK(cudaMemcpy(hs.data(), H.dev_starts, nb * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    uint64_t i = 0;
    for (int b = 0; b < sides; b++) {
      const uint64_t bytes = 1ull << H.P.side[b].block_size;
      for (uint64_t k = 0; k < H.P.side[b].nblocks; k++, i++) H.stream_bytes[b] += bytes - 4ull * hs[i];
    }
  }
  H.P.num = num;
  H.P.symmetric = !split;
  memcpy(H.P.pt, H.sp.pt, 8);
  H.P.T = d_enc;
  H.nkeys = key0;
  H.used = true;
  *handle = h;
  return TBG_OK;
}

template <class T>
static int grow_buf(T **p, uint64_t *cap, uint64_t n) {
  if (n <= *cap) return TBG_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(p, n * sizeof(T));
  if (e != cudaSuccess) return fail(TBG_ERR_NOMEM, "probe scratch: %s", cudaGetErrorString(e));
  *cap = n;
  return TBG_OK;
}

// Decode and answer in waves of as many touched blocks as the scratch
// budget holds (TS: the scratch symbol type); usually one wave.
template <typename TS>
static int decode_waves(ProbeHandle &H, uint64_t n, int L, uint32_t ntouched, uint32_t nside0,
                        int8_t *out) {
  cudaStream_t st = g_eng.stream;
  const bool two = H.P.side[1].nblocks != 0;
  const uint64_t per_block = (uint64_t)((kBlockPositions + L - 1) / L) * sizeof(TS);
  const uint32_t wave =
      (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ntouched, g_probe_scratch / per_block));
  int rc = grow_buf(&H.symbuf, &H.cap_sym, (uint64_t)wave * per_block);
  if (rc) return rc;
  TS *scratch = reinterpret_cast<TS *>(H.symbuf);
  const int grid = g_eng.num_sms * 8;
  PCK(cudaEventRecord(H.ev[1], st));
  for (uint32_t w0 = 0; w0 < ntouched; w0 += wave) {
    const uint32_t w1 = std::min(ntouched, w0 + wave), W = w1 - w0;
    for (int b = 0; b < (two ? 2 : 1); b++) {
      const uint32_t t0 = std::max(w0, b ? nside0 : 0u), t1 = std::min(w1, b ? ntouched : nside0);
      if (t0 >= t1) continue;
      const uint32_t grid_d = std::min<uint32_t>((t1 - t0 + 255) / 256, g_eng.num_sms * 7);
      k_probe_decode<TS><<<grid_d, 256, 0, st>>>(H.P.side[b], H.list, t0, t1, nullptr, b, w0, W,
                                                 H.minlit, scratch);
    }
    if (w1 == ntouched) PCK(cudaEventRecord(H.ev[2], st));
    k_probe_answer<TS><<<grid, 256, 0, st>>>(H.P, H.key, H.lit, H.tpos, n, w0, W, scratch, out);
    rc = g_eng.check_launch("probe decode");
    if (rc) return rc;
  }
  return TBG_OK;
}

// One wave of W = min(n, blocks) columns; the touched extent stays on the
// device (k_probe_bounds), so the call does not wait for the GPU.
template <typename TS>
static int decode_async(ProbeHandle &H, uint64_t n, uint32_t W, int8_t *out) {
  cudaStream_t st = g_eng.stream;
  const bool two = H.P.side[1].nblocks != 0;
  const int L = std::min(H.P.side[0].sym_positions, two ? H.P.side[1].sym_positions : 1 << 20);
  const uint64_t per_block = (uint64_t)((kBlockPositions + L - 1) / L) * sizeof(TS);
  int rc = grow_buf(&H.symbuf, &H.cap_sym, (uint64_t)W * per_block);
  if (rc) return rc;
  TS *scratch = reinterpret_cast<TS *>(H.symbuf);
  k_probe_bounds<<<1, 32, 0, st>>>(H.minlit, H.tpos, H.nkeys, two ? H.P.side[1].key0 : H.nkeys,
                                   H.bounds);
  PCK(cudaEventRecord(H.ev[1], st));
  const uint32_t grid_d = std::min<uint32_t>((W + 255) / 256, g_eng.num_sms * 7);
  for (int b = 0; b < (two ? 2 : 1); b++)
    k_probe_decode<TS><<<grid_d, 256, 0, st>>>(H.P.side[b], H.list, 0, 0, H.bounds, b, 0, W,
                                               H.minlit, scratch);
  PCK(cudaEventRecord(H.ev[2], st));
  k_probe_answer<TS><<<g_eng.num_sms * 8, 256, 0, st>>>(H.P, H.key, H.lit, H.tpos, n, 0, W,
                                                        scratch, out);
  H.touched_on_device = true;
  return g_eng.check_launch("probe decode");
}

static int probe_batch(ProbeHandle &H, const Query *q, int qbytes, uint64_t n, int8_t *out,
                       int mode) {
  cudaStream_t st = g_eng.stream;
  const int grid = g_eng.num_sms * 8;
  bool grouped = mode == 0 && H.P.side[0].sym_positions > 0 &&
                 (!H.P.side[1].nblocks || H.P.side[1].sym_positions > 0);
  if (!grouped) {
    k_probe_direct<<<grid, 256, 0, st>>>(H.P, q, qbytes, n, out);
    return g_eng.check_launch("k_probe_direct");
  }
  if (n >= (1ull << 32)) return fail(TBG_ERR_RANGE, "batch of 2^32 positions or more");
  if (!H.ev[0])
    for (auto &e : H.ev) PCK(cudaEventCreate(&e));
  H.timed = false;
  int rc;
  uint64_t cap = H.cap_q;
  if ((rc = grow_buf(&H.key, &cap, n))) return rc;
  cap = H.cap_q;
  if ((rc = grow_buf(&H.lit, &cap, n))) return rc;
  H.cap_q = std::max(H.cap_q, n);
  const uint32_t ntiles = (uint32_t)((H.nkeys + kScanTile - 1) / kScanTile);
  if (!H.minlit) {
    PCK(cudaMalloc(&H.minlit, H.nkeys * sizeof(uint32_t)));
    PCK(cudaMalloc(&H.tpos, H.nkeys * sizeof(uint32_t)));
    PCK(cudaMalloc(&H.list, H.nkeys * sizeof(uint32_t)));
    PCK(cudaMalloc(&H.tile, 2 * ntiles * sizeof(uint32_t)));
    PCK(cudaMalloc(&H.bounds, 2 * sizeof(uint32_t)));
  }
  PCK(cudaEventRecord(H.ev[0], st));
  PCK(cudaMemsetAsync(H.minlit, 0xff, H.nkeys * 4, st));
  k_probe_locate<<<grid, 256, 0, st>>>(H.P, q, qbytes, n, H.key, H.lit, H.minlit, out);
  k_scan_tiles<<<ntiles, 1024, 0, st>>>(H.minlit, H.nkeys, H.tile, H.tile + ntiles);
  k_scan_totals<<<1, 1024, 0, st>>>(H.tile, H.tile + ntiles, ntiles);
  k_scan_finish<<<ntiles, 1024, 0, st>>>(H.minlit, H.nkeys, H.tile + ntiles, H.tpos, H.list);
  rc = g_eng.check_launch("probe grouping");
  if (rc) return rc;
  const bool two = H.P.side[1].nblocks != 0;
  int L = H.P.side[0].sym_positions;
  if (two) L = std::min(L, H.P.side[1].sym_positions);
  const bool narrow = H.P.side[0].nsym_emit <= 256 && (!two || H.P.side[1].nsym_emit <= 256);
  // A batch touches at most min(n, blocks) blocks: when the scratch budget
  // holds that many, one wave sized so runs without the host reading the
  // touched count (no synchronisation inside the call).
  const uint64_t wmax = std::min<uint64_t>(n, H.nkeys);
  const uint64_t per_block = (uint64_t)((kBlockPositions + L - 1) / L) * (narrow ? 1 : 2);
  if (wmax * per_block <= g_probe_scratch) {
    rc = narrow ? decode_async<uint8_t>(H, n, (uint32_t)wmax, out)
                : decode_async<uint16_t>(H, n, (uint32_t)wmax, out);
    if (rc) return rc;
    PCK(cudaEventRecord(H.ev[3], st));
    H.timed = true;
    return TBG_OK;
  }
  // touched blocks (the last key's scan value) and the touched blocks of
  // side 0 (tpos at side 1's first key), read by the host to plan the waves
  uint32_t last[3] = {0, 0, 0};
  PCK(cudaMemcpyAsync(&last[0], H.tpos + H.nkeys - 1, 4, cudaMemcpyDeviceToHost, st));
  PCK(cudaMemcpyAsync(&last[1], H.minlit + H.nkeys - 1, 4, cudaMemcpyDeviceToHost, st));
  if (two) PCK(cudaMemcpyAsync(&last[2], H.tpos + H.P.side[1].key0, 4, cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  const uint32_t ntouched = last[0] + (last[1] != kNoLit ? 1 : 0);
  const uint32_t nside0 = two ? last[2] : ntouched;
  H.touched = ntouched;
  H.touched_on_device = false;
  if (ntouched == 0) return TBG_OK;
  rc = narrow ? decode_waves<uint8_t>(H, n, L, ntouched, nside0, out)
              : decode_waves<uint16_t>(H, n, L, ntouched, nside0, out);
  if (rc) return rc;
  PCK(cudaEventRecord(H.ev[3], st));
  H.timed = true;
  return TBG_OK;
}

}  // namespace tbg

using namespace tbg;

extern "C" int tbg_table_build(const char *material, uint64_t seed, int modulus, int on_device,
                               void **table, uint64_t *bytes) {
  if (!material || !table || !bytes) return fail(TBG_ERR_ARG, "null argument");
  if (on_device && !g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  return build_table(material, seed, modulus, on_device != 0, table, bytes);
}

extern "C" int tbg_table_free_host(void *table) {
  free(table);
  return TBG_OK;
}

extern "C" int tbg_probe_open(const void *dev_table, uint64_t bytes, const char *material,
                              int *handle) {
  if (!dev_table || !material || !handle) return fail(TBG_ERR_ARG, "null argument");
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  return open_table(static_cast<const uint8_t *>(dev_table), bytes, material, handle);
}

extern "C" int tbg_probe_close(int handle) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used) return fail(TBG_ERR_ARG, "bad handle");
  ProbeHandle &H = g_probe[handle];
  cudaStreamSynchronize(g_eng.stream);
  for (auto &e : H.ev)
    if (e) cudaEventDestroy(e);
  for (void *p : {(void *)H.dev_alloc, (void *)H.dev_starts, (void *)H.key, (void *)H.lit,
                  (void *)H.minlit, (void *)H.tpos, (void *)H.list, (void *)H.tile,
                  (void *)H.bounds, (void *)H.symbuf})
    if (p) cudaFree(p);
  H = ProbeHandle();
  return TBG_OK;
}

extern "C" int tbg_probe_wdl_batch(int handle, const void *dev_queries, uint64_t n, void *dev_out,
                                   int mode) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used) return fail(TBG_ERR_ARG, "bad handle");
  if (!dev_queries || !dev_out) return fail(TBG_ERR_ARG, "null buffers");
  if (reinterpret_cast<uintptr_t>(dev_queries) & 15)
    return fail(TBG_ERR_ARG, "queries must be 16-byte aligned");
  if (n == 0) return TBG_OK;
  return probe_batch(g_probe[handle], static_cast<const Query *>(dev_queries), 16, n,
                     static_cast<int8_t *>(dev_out), mode);
}

extern "C" int tbg_probe_wdl_batch8(int handle, const void *dev_queries, uint64_t n,
                                    void *dev_out, int mode) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used) return fail(TBG_ERR_ARG, "bad handle");
  if (!dev_queries || !dev_out) return fail(TBG_ERR_ARG, "null buffers");
  if (reinterpret_cast<uintptr_t>(dev_queries) & 7)
    return fail(TBG_ERR_ARG, "compact queries must be 8-byte aligned");
  if (g_probe[handle].P.num > 7) return fail(TBG_ERR_ARG, "compact queries hold at most 7 pieces");
  if (n == 0) return TBG_OK;
  return probe_batch(g_probe[handle], static_cast<const Query *>(dev_queries), 8, n,
                     static_cast<int8_t *>(dev_out), mode);
}

extern "C" int tbg_encode_batch(int handle, const void *dev_queries, uint64_t n, uint64_t *dev_idx,
                                uint8_t *dev_side) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used) return fail(TBG_ERR_ARG, "bad handle");
  if (!dev_queries || (reinterpret_cast<uintptr_t>(dev_queries) & 15))
    return fail(TBG_ERR_ARG, "queries must be 16-byte aligned");
  k_encode_batch<<<g_eng.num_sms * 8, 256, 0, g_eng.stream>>>(
      g_probe[handle].P, static_cast<const Query *>(dev_queries), n, dev_idx, dev_side);
  return g_eng.check_launch("k_encode_batch");
}

extern "C" int tbg_decode_batch(int handle, int side, const uint64_t *dev_idx, uint64_t n,
                                uint8_t *dev_squares) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used || side < 0 || side > 1)
    return fail(TBG_ERR_ARG, "bad handle/side");
  k_decode_batch<<<g_eng.num_sms * 8, 256, 0, g_eng.stream>>>(g_probe[handle].P, side, dev_idx, n,
                                                              dev_squares);
  return g_eng.check_launch("k_decode_batch");
}

extern "C" int tbg_gen_positions(const char *material, uint64_t seed, uint64_t n, void *dev_queries,
                                 uint32_t *failed) {
  Spec sp;
  int rc = spec_from_name(material, sp);
  if (rc) return rc;
  if (!g_eng.dev_ready) return fail(TBG_ERR_STATE, "tbg_init not called");
  uint8_t *d_pt;
  uint32_t *d_fail;
  PCK(cudaMalloc(&d_pt, 8));
  PCK(cudaMalloc(&d_fail, 4));
  // on the launch stream: a legacy-stream copy or memset is not ordered
  // with a non-blocking caller stream
  PCK(cudaMemcpyAsync(d_pt, sp.pt, 8, cudaMemcpyHostToDevice, g_eng.stream));
  PCK(cudaMemsetAsync(d_fail, 0, 4, g_eng.stream));
  k_gen_positions<<<g_eng.num_sms * 8, 256, 0, g_eng.stream>>>(sp.num, d_pt, seed, n,
                                                               static_cast<Query *>(dev_queries), d_fail);
  rc = g_eng.check_launch("k_gen_positions");
  uint32_t f = 0;
  PCK(cudaMemcpyAsync(&f, d_fail, 4, cudaMemcpyDeviceToHost, g_eng.stream));
  PCK(cudaStreamSynchronize(g_eng.stream));
  cudaFree(d_pt);
  cudaFree(d_fail);
  if (failed) *failed = f;
  return rc;
}

extern "C" int tbg_probe_tune(uint64_t scratch_bytes) {
  if (scratch_bytes < (64u << 10)) return fail(TBG_ERR_ARG, "scratch below 64 KiB");
  g_probe_scratch = scratch_bytes;
  return TBG_OK;
}

extern "C" int tbg_probe_layout(int handle, int side, uint64_t *data_offset, uint64_t *nblocks,
                                uint64_t *positions) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used || side < 0 || side > 1)
    return fail(TBG_ERR_ARG, "bad handle/side");
  const ProbeHandle &H = g_probe[handle];
  const ProbeSide &S = H.P.side[side];
  if (side == 1 && !S.nblocks) return fail(TBG_ERR_ARG, "the table has one side");
  if (data_offset) *data_offset = (uint64_t)(S.data - H.base);
  if (nblocks) *nblocks = S.nblocks;
  if (positions) *positions = S.ei.size;
  return TBG_OK;
}

extern "C" int tbg_probe_stream_bytes(int handle, int side, uint64_t *bytes) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used || side < 0 || side > 1 || !bytes)
    return fail(TBG_ERR_ARG, "bad handle/side");
  const ProbeHandle &H = g_probe[handle];
  if (side == 1 && !H.P.side[1].nblocks) return fail(TBG_ERR_ARG, "the table has one side");
  if (!H.dev_starts) return fail(TBG_ERR_STATE, "block starts not computed for this table");
  *bytes = H.stream_bytes[side];
  return TBG_OK;
}

extern "C" int tbg_probe_phase_ms(int handle, float ms[3], uint64_t *touched_blocks) {
  if (handle < 0 || handle >= 8 || !g_probe[handle].used || !ms) return fail(TBG_ERR_ARG, "bad handle");
  ProbeHandle &H = g_probe[handle];
  if (!H.timed) return fail(TBG_ERR_STATE, "no grouped batch with touched blocks since the last call");
  PCK(cudaEventSynchronize(H.ev[3]));
  PCK(cudaEventElapsedTime(&ms[0], H.ev[0], H.ev[1]));
  PCK(cudaEventElapsedTime(&ms[1], H.ev[1], H.ev[2]));
  PCK(cudaEventElapsedTime(&ms[2], H.ev[2], H.ev[3]));
  if (H.touched_on_device) {
    uint32_t t = 0;
    PCK(cudaMemcpy(&t, H.bounds, sizeof t, cudaMemcpyDeviceToHost));
    H.touched = t;
    H.touched_on_device = false;
  }
  if (touched_blocks) *touched_blocks = H.touched;
  return TBG_OK;
}
