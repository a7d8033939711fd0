// Types shared by the host side of the library and its kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#define TBG_MAX_SETS 6
#define TBG_MAX_MATS 16
#define TBG_NSLICES 462

namespace tbg {

// One IdxInfo (tb8gen.h:4-13) in device form: mixed-radix factors, the
// per-set piece counts and the quotient multipliers of fast_div32.
struct DIdx {
  int numsets;
  int pad;
  uint64_t size;
  uint64_t factor[TBG_MAX_SETS];
  uint64_t fdiv[TBG_MAX_SETS];
  int mult[TBG_MAX_SETS];
};

// One material: the main index, the capture index of every set (capt_ii,
// tb8gen.c:1373-1378) and the piece/set tables the workers consult.
struct DMat {
  DIdx ii;
  DIdx capt[TBG_MAX_SETS];
  int num;                        // pieces, kings included
  int set_type[TBG_MAX_SETS];     // piece type (1..6) of each set
  int set_color[TBG_MAX_SETS];    // 0 white, 1 black
  int set_first[TBG_MAX_SETS];    // first piece index of each set
  int king_type[2];
  uint64_t bytes;                 // slice bitmap bytes (64-B rounded)
  uint64_t sub_offset[TBG_MAX_SETS];  // byte offset of set k in a sub buffer
  uint64_t sub_size[2];           // sub bytes per colour of captured set
  uint64_t sub_bytes;             // max(sub_size): one slice's sub buffer
};

// One king destination of a per-slice job (mark_king_unmoves,
// check_king_moves, tb8gen.c:246-262, 537-569): where the king of the side
// to move can step, which slice that lands in and the normalisation
// transform that maps the new king pair onto it.
struct KingDest {
  int to;                 // destination square (un-normalised)
  int s2;                 // target slice
  int k0, k1;             // normalised king squares in s2
  int mirror, flip;       // transform
  int dbl;                // s < 441 && s2 >= 441: mark the diagonal mirror too
  int pad;
  uint32_t *bits;         // bitmap bound to s2
  const uint8_t *sub;     // sub buffer bound to s2 (may be null)
  uint64_t sub_len;       // bytes bound at sub
};

struct SliceJob {
  int mat, stm, s, set;   // set: captured set for sub-based kernels
  int k0, k1;             // king squares of slice s
  int nk, legality;
  uint64_t nbits;         // bits of the source scanned
  const uint32_t *src;    // source bitmap (or candidate bitmap, in place)
  uint32_t *cand;         // candidates to verify in place (check_successors)
  uint32_t *self;         // bitmap bound to slice s
  const uint8_t *self_sub;
  uint64_t self_sub_len;
  const uint32_t *filter; // candidates: the opponent's "wins" of slice s (or null)
  uint64_t pad;
  KingDest kd[8];
};

// Error word written by kernels when an access falls outside what was
// bound; the access is skipped, the host reports TBG_ERR_DEVICE.
struct DevStatus {
  unsigned int err;
  unsigned int where;
  unsigned long long info;
};

enum OpKind : int {
  OP_SCATTER = 1, OP_SCATTER_SUB = 2, OP_VERIFY = 3, OP_EPILOGUE = 4, OP_CLEAR = 5, OP_COUNT = 6
};

// The ops that stream whole bitmaps in 1 MiB chunks (the others work by tile).
__host__ __device__ inline bool op_streams(int kind) {
  return kind == OP_EPILOGUE || kind == OP_CLEAR || kind == OP_COUNT;
}

constexpr uint64_t kChunk16 = 1u << 16;   // streaming tile: 65,536 x 16 B = 1 MiB

struct alignas(16) Op {
  int kind;
  int ns;                  // piece sets of the material (sparse kernels)
  uint32_t ntiles;
  int npred, pred_off;
  int cnt_slot;            // epilogue count slot of a recorded batch (-1: none)
  int gt;                  // scatter: tiles per work item (1: one tile)
  int pad;
  uint64_t first;          // index of the op's first work item
  SliceJob J;              // sparse kernels
  uint32_t *out;           // verify: out-of-place output (or null)
  uint64_t out_words;
  uint4 *T;                // epilogue / clear target
  const uint4 *win;        // epilogue: wins in
  uint4 *wout;             // epilogue: wins out
  uint64_t n16;            // vectors of T
  uint64_t nbits;          // epilogue: positions counted
  unsigned long long *cnt; // epilogue: count slot (or null)
};

}  // namespace tbg
