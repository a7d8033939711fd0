// Host entry points of the two persistent-kernel translation units
// (tbg_persist_block.cu: k_batch, tbg_persist_warp.cu: k_batch_w).  Each
// unit keeps its own copy of the constant-memory materials and stub
// parameters, written by these calls whenever tbg_api.cu writes its own.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tbg_types.h"

namespace tbg {

struct PersistArgs {
  const Op *ops;
  int nops;
  const int *preds;
  uint64_t total;
  unsigned long long *next;
  unsigned int *done;
  DevStatus *st;
  long long spin_limit;
};

// Material descriptor `d` into constant slot `slot` (synchronous upload).
cudaError_t persist_block_set_mat(const DMat &d, int slot);
cudaError_t persist_warp_set_mat(const DMat &d, int slot);
// Stub seed and modulus, on `st` (synchronous when st is null).
cudaError_t persist_block_set_stub(uint64_t seed, int mod, cudaStream_t st);
cudaError_t persist_warp_set_stub(uint64_t seed, int mod, cudaStream_t st);
// One persistent launch of `grid` blocks on `st`, compiled for at most
// nsmax <= 3 or <= 6 piece sets.
cudaError_t persist_block_launch(int nsmax, int grid, cudaStream_t st, const PersistArgs &a);
cudaError_t persist_warp_launch(int nsmax, int grid, cudaStream_t st, const PersistArgs &a);
// One sparse op (scatter, uncapture or verify) as its own launch of k_op_w:
// sub-items of 32 words over at most max_blocks blocks.
cudaError_t persist_warp_launch_op(const Op &o, int max_blocks, cudaStream_t st, DevStatus *dst);

}  // namespace tbg
