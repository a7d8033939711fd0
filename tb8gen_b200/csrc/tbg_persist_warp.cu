// The persistent batched-ply kernel with warp-wide work items (tbg_batch_run mode 2),
// compiled in a translation unit of its own (with its own copy of the
// constant-memory materials) so that it builds beside tbg_api.cu.
#include <cuda_runtime.h>

#define TBG_PERSIST_UNIT 1
#include "tbg_warp.cuh"
#include "tbg_persist.h"

namespace tbg {

cudaError_t persist_warp_set_mat(const DMat &d, int slot) {
  return cudaMemcpyToSymbol(c_mats, &d, sizeof d, slot * sizeof(DMat));
}

cudaError_t persist_warp_set_stub(uint64_t seed, int mod, cudaStream_t st) {
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

cudaError_t persist_warp_launch(int nsmax, int grid, cudaStream_t st, const PersistArgs &a) {
  if (nsmax <= 3)
    k_batch_w<3><<<grid, kThreads, 0, st>>>(a.ops, a.nops, a.preds, a.total, a.next, a.done, a.st,
                                          a.spin_limit);
  else
    k_batch_w<6><<<grid, kThreads, 0, st>>>(a.ops, a.nops, a.preds, a.total, a.next, a.done, a.st,
                                          a.spin_limit);
  return cudaPeekAtLastError();
}

template <int KIND>
static void launch_op_kind(const Op &o, int grid, cudaStream_t st, DevStatus *dst,
                           uint64_t nsub) {
  switch (o.ns) {
  case 1: k_op_w<1, KIND><<<grid, kThreads, 0, st>>>(o, dst, nsub); break;
  case 2: k_op_w<2, KIND><<<grid, kThreads, 0, st>>>(o, dst, nsub); break;
  case 3: k_op_w<3, KIND><<<grid, kThreads, 0, st>>>(o, dst, nsub); break;
  case 4: k_op_w<4, KIND><<<grid, kThreads, 0, st>>>(o, dst, nsub); break;
  case 5: k_op_w<5, KIND><<<grid, kThreads, 0, st>>>(o, dst, nsub); break;
  default: k_op_w<6, KIND><<<grid, kThreads, 0, st>>>(o, dst, nsub); break;
  }
}

cudaError_t persist_warp_launch_op(const Op &o, int max_blocks, cudaStream_t st,
                                   DevStatus *dst) {
  if (o.ns < 1 || o.ns > 6) return cudaErrorInvalidValue;
  const uint64_t nwords = (o.J.nbits + 31) >> 5;
  const uint64_t nsub = nwords > 0 ? (nwords + 31) / 32 : 1;
  const uint64_t want = (nsub + kWarps - 1) / kWarps;
  const int grid = (int)(want < (uint64_t)max_blocks ? want : (uint64_t)max_blocks);
  switch (o.kind) {
  case OP_SCATTER: launch_op_kind<OP_SCATTER>(o, grid, st, dst, nsub); break;
  case OP_SCATTER_SUB: launch_op_kind<OP_SCATTER_SUB>(o, grid, st, dst, nsub); break;
  case OP_VERIFY: launch_op_kind<OP_VERIFY>(o, grid, st, dst, nsub); break;
  default: return cudaErrorInvalidValue;
  }
  return cudaPeekAtLastError();
}

}  // namespace tbg
