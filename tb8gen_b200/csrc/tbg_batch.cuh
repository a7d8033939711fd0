// Batched ply: many per-slice calls of different slices and materials run
// by one persistent kernel fed from a device work queue.
//
// Recording (tbg_batch_begin .. tbg_batch_end) turns every per-slice call
// into an Op with its bindings resolved.  An Op is cut into tiles (32,768
// positions for the sparse kernels, 1 MiB for the streaming ones); the queue
// is the list of (op, tile) items in record order.  Each op lists the earlier
// ops it waits for, found per buffer (read-after-write, write-after-read,
// write-after-write; two scatters into one bitmap commute and do not
// conflict; the waits of the listed ops cover older accesses).  A CTA takes the next item with one atomicAdd, waits -- with an
// iteration bound -- until the item's predecessor ops have all their tiles
// done, runs the tile and counts it done (at its next fetch, after the
// block's barrier).  Consecutive items of one op reuse the op's descriptor
// in shared memory.  Items are taken in record order,
// so every predecessor of the earliest unfinished item was taken earlier and
// is finished: that item can always proceed, whatever the grid size.
#pragma once

#include "tbg_kernels.cuh"

namespace tbg {

#ifndef TBG_MINB_BATCH
#define TBG_MINB_BATCH (1024 / TBG_THREADS)
#endif

__device__ __forceinline__ unsigned int load_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// One 1 MiB chunk of the fused epilogue (k_epilogue_W), of a clear or of a
// count.
__device__ __forceinline__ void tile_stream(const Op &o, uint64_t t) {
  const uint64_t i0 = t * kChunk16;
  const uint64_t i1 = i0 + kChunk16 < o.n16 ? i0 + kChunk16 : o.n16;
  if (o.kind == OP_CLEAR) {
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) o.T[i] = z;
    return;
  }
  unsigned long long c = 0;
  const uint64_t full16 = o.nbits >> 7;
  const bool count_only = o.kind == OP_COUNT;
  for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    uint4 t4 = o.T[i];
    if (!count_only) {
      uint4 w = o.win[i];
      t4.x &= ~w.x; t4.y &= ~w.y; t4.z &= ~w.z; t4.w &= ~w.w;
      w.x |= t4.x; w.y |= t4.y; w.z |= t4.z; w.w |= t4.w;
      o.T[i] = t4;
      o.wout[i] = w;
    }
    if (i < full16) {
      c += popc4(t4);
    } else if (i == full16) {
      uint32_t v[4] = {t4.x, t4.y, t4.z, t4.w};
      for (int j = 0; j < 4; j++) {
        uint64_t b0 = i * 128 + 32 * j;
        if (b0 >= o.nbits) break;
        uint32_t m = b0 + 32 <= o.nbits ? ~0u : (1u << (o.nbits - b0)) - 1u;
        c += __popc(v[j] & m);
      }
    }
  }
  if (o.cnt == nullptr) return;
  for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(o.cnt, c);
}

template <int NS>
__device__ __forceinline__ void tile_sparse(const Op &o, SparseSmem &S, int &gp, uint32_t &ph,
                                            uint64_t t, DevStatus *st) {
  switch (o.kind) {
  case OP_SCATTER: {
    const uint64_t t0 = t * o.gt, tiles = tiles_of(o.J.nbits);
    tile_predecessors<NS>(o.J, S, gp, ph, t0, (int)min((uint64_t)o.gt, tiles - t0), st);
    break;
  }
  case OP_SCATTER_SUB: tile_predecessors_sub<NS>(o.J, S, t, st); break;
  default: tile_check<NS>(o.J, S, t, st, o.out, o.out_words); break;
  }
}

template <int NSMAX>
__global__ void __launch_bounds__(kThreads, TBG_MINB_BATCH)
k_batch(const Op *__restrict__ ops, int nops, const int *__restrict__ preds, uint64_t total,
        unsigned long long *next, unsigned int *done, DevStatus *st, long long spin_limit) {
  __shared__ SparseSmem S;
  __shared__ __align__(16) Op so;
  __shared__ unsigned long long s_item;
  __shared__ int s_op, s_abort;
  load_binomials(S.bin);
  init_gcnt(S);
  bulk_init(S.B);
  int gp = 0;        // the scatter list's current count (scan_group)
  uint32_t ph = 0;   // the staged tiles' barrier phases (scan_group)
  int cur_op = -1;   // the op whose descriptor (and king destinations) are in `so`
  int prev_op = -1;  // thread 0: the op of the item this block finished last
  for (;;) {
    // every thread has finished the previous item (and read `so` and S.kd)
    __syncthreads();
    if (threadIdx.x == 0) {
      if (prev_op >= 0) {
        __threadfence();
        atomicAdd(&done[prev_op], 1u);
      }
      unsigned long long it = atomicAdd(next, 1ull);
      s_item = it;
      s_abort = 0;
      if (it < total) {
        int lo = 0, hi = nops - 1;
        while (lo < hi) {
          int mid = (lo + hi + 1) >> 1;
          if (ops[mid].first <= it) lo = mid;
          else hi = mid - 1;
        }
        s_op = lo;
        const int np = ops[lo].npred, po = ops[lo].pred_off;
        for (int p = 0; p < np && !s_abort; p++) {
          const int q = preds[po + p];
          const unsigned int need = ops[q].ntiles;
          long long n = 0;
          while (load_acquire(&done[q]) < need) {
            if (++n > spin_limit) {
              report(st, 3, (unsigned)q, it);
              s_abort = 1;
              break;
            }
            __nanosleep(64);
          }
        }
      }
    }
    __syncthreads();
    if (s_item >= total || s_abort) break;
    __threadfence();
    const int op = s_op;
    if (op != cur_op) {
      // a new op: its descriptor (and its king destinations) into shared memory
      const int4 *src = reinterpret_cast<const int4 *>(&ops[op]);
      int4 *dst = reinterpret_cast<int4 *>(&so);
      for (int i = threadIdx.x; i < (int)(sizeof(Op) / 16); i += blockDim.x) dst[i] = src[i];
      __syncthreads();
      if (!op_streams(so.kind)) {
        load_dests(so.J, S.kd);
        __syncthreads();
      }
      cur_op = op;
    }
    const uint64_t t = s_item - so.first;
    if (op_streams(so.kind)) {
      tile_stream(so, t);
    } else {
      switch (so.ns) {
      case 1: tile_sparse<1>(so, S, gp, ph, t, st); break;
      case 2: if (NSMAX >= 2) tile_sparse<(NSMAX >= 2 ? 2 : 1)>(so, S, gp, ph, t, st); break;
      case 3: if (NSMAX >= 3) tile_sparse<(NSMAX >= 3 ? 3 : 1)>(so, S, gp, ph, t, st); break;
      case 4: if (NSMAX >= 4) tile_sparse<(NSMAX >= 4 ? 4 : 1)>(so, S, gp, ph, t, st); break;
      case 5: if (NSMAX >= 5) tile_sparse<(NSMAX >= 5 ? 5 : 1)>(so, S, gp, ph, t, st); break;
      default: if (NSMAX >= 6) tile_sparse<(NSMAX >= 6 ? 6 : 1)>(so, S, gp, ph, t, st); break;
      }
    }
    // counted done at the top of the next iteration, after its barrier
    prev_op = op;
  }
}

}  // namespace tbg
