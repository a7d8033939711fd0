// Host-side state of the engine: king-slice tables, materials, slot map.
#pragma once

#ifndef TBG_THREADS
#define TBG_THREADS 256
#endif

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "tbg_types.h"

namespace tbg {

// King-pair tables (probe.c:310-539, tb8gen.c:69-89) and king steps.
struct HostTables {
  bool ready = false;
  int kkidx[10][64];
  int kksq[TBG_NSLICES][2];
  int triangle[64];
  int flipdiag[64];
  int mirror[64];
  bool fliptest[64][64];
  int kkmap[64][64];
  uint64_t king[64];
  void build();
};

struct Material {
  DMat d;
  int pt[8];
  int num;
  // Slot map of kslice_slot/kslice_buf/kslice_sub_buf: index s + 1, s = -1
  // is the scratch slot.
  uint8_t *slot[463];
  uint64_t slot_bytes[463];
  uint8_t *sub[463];
  uint64_t sub_len[463];
};


// A recorded batch of ply-step calls (tbg_batch_begin .. tbg_batch_end).
struct Batch {
  bool recording = false;
  bool ready = false;
  std::vector<Op> ops;
  struct Access {
    std::vector<const void *> rd, wplain, wacc;
  };
  // Per buffer: the last op that wrote it outright, and the ops that read it
  // or accumulated into it since.  An op depends on these, not on every
  // earlier op: a dependency wait ends only when all tiles of the awaited
  // op are done, and those waited in turn for theirs.
  struct BufState {
    int writer = -1;
    std::vector<int> readers, accs;
  };
  std::unordered_map<const void *, BufState> bufs;
  std::vector<int> preds;
  int ncounts = 0;
  int nsmax = 1;
  uint64_t total = 0;
  // device copies
  Op *d_ops = nullptr;
  size_t cap_ops = 0;
  int *d_preds = nullptr;
  size_t cap_preds = 0;
  unsigned int *d_done = nullptr;
  size_t cap_done = 0;
  unsigned long long *d_counts = nullptr;
  size_t cap_counts = 0;
  unsigned long long *d_next = nullptr;
  // persistent launch configuration
  int ctas_per_sm = 1024 / TBG_THREADS;
  long long spin_limit = 50000000;

  void clear();
  int add(Op &o);
  int finish();
};

struct Engine {
  bool dev_ready = false;
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  DevStatus *d_status = nullptr;
  unsigned long long *d_cnt = nullptr;
  unsigned long long *h_cnt = nullptr;
  Material mats[TBG_MAX_MATS];
  int nmats = 0;
  int cur = -1;
  uint64_t launches = 0;  // kernels launched by this library
  int scatter_tiles = 0;    // tiles per predecessors work item (tbg_batch_shape; 0: 1)
  int candidate_tiles = 0;  // tiles per candidates work item (0: 4)
  // Recorded batches: kBatchSlots slots, one selected (tbg_batch_select).
  static constexpr int kBatchSlots = 4;
  Batch batches[kBatchSlots];
  int bslot = 0;
  Batch &batch() { return batches[bslot]; }
  // Host-tier copy streams (inbound, outbound) and the event ring behind
  // tickets: ticket t is event t % kTickets until kTickets later ones exist.
  static constexpr uint64_t kTickets = 8192;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaStream_t s_zero = nullptr;  // zero-fills new allocations (tbg_alloc)
  std::vector<cudaEvent_t> tick_ev;
  uint64_t next_ticket = 1;
  // Host-side failure injection: TBG_FAIL_ALLOC_AT=k (read at tbg_init)
  // makes the k-th allocation through tbg_alloc / tbg_host_alloc fail with
  // TBG_ERR_NOMEM, as a failed cudaMalloc or cudaHostAlloc would.
  long fail_alloc_at = 0;
  long alloc_calls = 0;

  int ensure_device();
  bool alloc_refused();
  int add_material(const int *pt, int num);
  int fill_job(SliceJob &J, int stm, int s, bool need_sub);
  int grid_for(uint64_t units, int per_sm);
  int check_launch(const char *what);
  int wait(int timeout_ms);
  int tickets_ready();
  int ticket_event(uint64_t t, cudaEvent_t *e);
  int issue_ticket(cudaStream_t st, uint64_t *t);
};

extern HostTables g_tab;
extern Engine g_eng;

int fail(int code, const char *fmt, ...);

inline uint64_t tbg_host_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace tbg
