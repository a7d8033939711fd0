// The persistent batched-ply kernel with block-wide work items (tbg_batch_run mode 1),
// compiled in a translation unit of its own (with its own copy of the
// constant-memory materials) so that it builds beside tbg_api.cu.
#include <cuda_runtime.h>

#define TBG_PERSIST_UNIT 1
#include "tbg_batch.cuh"
#include "tbg_persist.h"

namespace tbg {

cudaError_t persist_block_set_mat(const DMat &d, int slot) {
  return cudaMemcpyToSymbol(c_mats, &d, sizeof d, slot * sizeof(DMat));
}

cudaError_t persist_block_set_stub(uint64_t seed, int mod, cudaStream_t st) {
  cudaError_t e;
  if (st == nullptr) {
    if ((e = cudaMemcpyToSymbol(c_stub_seed, &seed, sizeof seed)) != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_stub_mod, &mod, sizeof mod);
  }
  if ((e = cudaMemcpyToSymbolAsync(c_stub_seed, &seed, sizeof seed, 0, cudaMemcpyHostToDevice,
                                   st)) != cudaSuccess)
    return e;
  return cudaMemcpyToSymbolAsync(c_stub_mod, &mod, sizeof mod, 0, cudaMemcpyHostToDevice, st);
}

cudaError_t persist_block_launch(int nsmax, int grid, cudaStream_t st, const PersistArgs &a) {
  if (nsmax <= 3)
    k_batch<3><<<grid, kThreads, 0, st>>>(a.ops, a.nops, a.preds, a.total, a.next, a.done, a.st,
                                          a.spin_limit);
  else
    k_batch<6><<<grid, kThreads, 0, st>>>(a.ops, a.nops, a.preds, a.total, a.next, a.done, a.st,
                                          a.spin_limit);
  return cudaPeekAtLastError();
}

}  // namespace tbg
