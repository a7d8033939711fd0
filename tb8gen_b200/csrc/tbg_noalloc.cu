// W-step epilogue that allocates nothing, for callers that cannot allocate
// device memory.
//
// Who needs it: a host whose device memory is entirely owned by someone
// else -- a caching allocator or memory pool that has reserved the HBM for
// the slice bitmaps (PyTorch's allocator, a serving loop that admits work
// against a fixed HBM budget), or a foreign-language host binding the C ABI
// that forbids libraries to allocate behind its back -- and latency-bound
// loops that cannot take the device-wide synchronisation cudaMalloc and
// cudaFree may imply.  tbg_epilogue_W / tbg_epilogue_W_to need tbg_init,
// which allocates a device counter and a status word; this entry point
// needs neither.
//
// Its only scratch is the file-scope array below: one partial popcount per
// 1 MiB chunk of the bitmap plus one total, 8 KiB in all, which every GPU
// that loads this library holds until the process exits.  That caps the
// bitmap at kMaxChunks MiB (1 GiB, 8,589,934,592 positions); larger bitmaps
// are rejected with TBG_ERR_RANGE.  All calls share the array and it keeps
// the last call's contents, so calls that overlap on the GPU (two streams,
// or two host threads) race on it and must not be issued; each call writes
// every partial it later reads, so nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "../../include/tbgpu.h"

namespace {

constexpr int kChunkBytes = 1 << 20;   // one partial per 1 MiB of bitmap
constexpr int kMaxChunks = 1024;       // => at most 1 GiB of bitmap
constexpr int kEpiThreads = 256;

// partials[0 .. kMaxChunks-1], total at [kMaxChunks].
static __device__ __align__(256) unsigned long long g_epi_scratch[kMaxChunks + 1];

// Device address of the scratch array per device ordinal, looked up once.
// It stays valid for the life of the device's primary context: a process
// that calls cudaDeviceReset must not use this entry point afterwards.
constexpr int kMaxDevices = 64;
static std::atomic<void *> g_scratch_addr[kMaxDevices];

// Block b owns bytes [b * kChunkBytes, min((b + 1) * kChunkBytes, bytes)):
// T &= ~wins_in, wins_out = wins_in | T, partial[b] = popcount of T below
// nbits.  wins_in may equal wins_out.
__global__ void __launch_bounds__(kEpiThreads)
k_epilogue_static(uint4 *T, const uint4 *wins_in, uint4 *wins_out, uint64_t bytes,
                  uint64_t nbits, unsigned long long *scratch) {
  const uint64_t begin = (uint64_t)blockIdx.x * (kChunkBytes / 16);
  uint64_t end = begin + kChunkBytes / 16;
  if (end > bytes / 16) end = bytes / 16;
  unsigned long long c = 0;
  for (uint64_t i = begin + threadIdx.x; i < end; i += kEpiThreads) {
    uint4 t = T[i], w = wins_in[i];
    t.x &= ~w.x; t.y &= ~w.y; t.z &= ~w.z; t.w &= ~w.w;
    w.x |= t.x; w.y |= t.y; w.z |= t.z; w.w |= t.w;
    T[i] = t;
    wins_out[i] = w;
    const uint32_t v[4] = {t.x, t.y, t.z, t.w};
    for (int j = 0; j < 4; j++) {
      uint64_t b0 = i * 128 + 32 * j;
      if (b0 >= nbits) break;
      uint32_t m = b0 + 32 <= nbits ? ~0u : (1u << (nbits - b0)) - 1u;
      c += __popc(v[j] & m);
    }
  }
  for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
  __shared__ unsigned long long part[kEpiThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int i = 0; i < kEpiThreads / 32; i++) s += part[i];
    scratch[blockIdx.x] = s;
  }
}

__global__ void k_epilogue_static_total(unsigned long long *scratch, int nchunks) {
  unsigned long long s = 0;
  for (int i = threadIdx.x; i < nchunks; i += blockDim.x) s += scratch[i];
  for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
  __shared__ unsigned long long part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int i = 0; i < (int)(blockDim.x / 32); i++) t += part[i];
    scratch[kMaxChunks] = t;
  }
}

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does the lookup).
int scratch_address(unsigned long long **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return TBG_ERR_CUDA;
  void *p = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    if (cudaGetSymbolAddress(&p, g_epi_scratch) != cudaSuccess || !p) return TBG_ERR_CUDA;
    g_scratch_addr[dev].store(p, std::memory_order_release);
  }
  *out = static_cast<unsigned long long *>(p);
  return TBG_OK;
}

}  // namespace

extern "C" int tbg_epilogue_W_static(void *dev_T, const void *dev_wins_in, void *dev_wins_out,
                                     uint64_t nbits, uint64_t bytes, void *stream,
                                     uint64_t *cnt) {
  if (!dev_T || !dev_wins_in || !dev_wins_out || !cnt) return TBG_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(dev_T) | reinterpret_cast<uintptr_t>(dev_wins_in) |
       reinterpret_cast<uintptr_t>(dev_wins_out)) & 15)
    return TBG_ERR_ARG;
  if (bytes == 0 || (bytes & 15) || nbits > bytes * 8) return TBG_ERR_ARG;
  if (bytes > (uint64_t)kMaxChunks * kChunkBytes) return TBG_ERR_RANGE;
  unsigned long long *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nchunks = (int)((bytes + kChunkBytes - 1) / kChunkBytes);
  // Launched through cudaLaunchKernel, whose status is this launch's own
  // (cudaGetLastError would also return an error left by an earlier,
  // unrelated call of the caller's).
  uint4 *T = static_cast<uint4 *>(dev_T);
  const uint4 *win = static_cast<const uint4 *>(dev_wins_in);
  uint4 *wout = static_cast<uint4 *>(dev_wins_out);
  void *a1[] = {&T, &win, &wout, &bytes, &nbits, &scratch};
  if (cudaLaunchKernel((const void *)k_epilogue_static, dim3(nchunks), dim3(kEpiThreads), a1, 0,
                       st) != cudaSuccess)
    return TBG_ERR_CUDA;
  int nch = nchunks;
  void *a2[] = {&scratch, &nch};
  if (cudaLaunchKernel((const void *)k_epilogue_static_total, dim3(1), dim3(1024), a2, 0, st) !=
      cudaSuccess)
    return TBG_ERR_CUDA;
  unsigned long long total = 0;
  if (cudaMemcpyAsync(&total, scratch + kMaxChunks, sizeof total, cudaMemcpyDeviceToHost, st) !=
      cudaSuccess)
    return TBG_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return TBG_ERR_CUDA;
  *cnt = total;
  return TBG_OK;
}
