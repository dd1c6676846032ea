// Host-side internals shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/meerkat_b200.h"
#include "mk_common.cuh"

namespace mk {

void set_error(const std::string &msg);
mk_status fail(mk_status st, const std::string &msg);
mk_status cuda_fail(cudaError_t e, const char *what);

#define MK_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::mk::cuda_fail(e_, #call); \
  } while (0)

#define MK_CHECK(call)                      \
  do {                                      \
    mk_status s_ = (call);                  \
    if (s_ != MK_OK) return s_;             \
  } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Device buffer that grows on demand (never shrinks).
template <class T>
struct DevBuf {
  T *ptr = nullptr;
  size_t cap = 0;  // elements
  mk_status reserve(size_t n, size_t *bytes_acc = nullptr) {
    if (n <= cap) return MK_OK;
    size_t want = cap ? cap : 1024;
    while (want < n) want *= 2;
    const size_t old = cap;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&ptr, want * sizeof(T));
    if (e != cudaSuccess) {
      ptr = nullptr;
      return cuda_fail(e, "cudaMalloc(scratch)");
    }
    if (bytes_acc) *bytes_acc += (want - old) * sizeof(T);
    cap = want;
    return MK_OK;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

int device_sm_count(int device);

// Scoped device switch (one cudaGetDevice when the device is already current).
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) {
      cudaSetDevice(dev);
      switched = true;
    }
  }
  ~DeviceGuard() {
    if (switched && prev >= 0) cudaSetDevice(prev);
  }
};

// Event pair used by the ms_out timing of the algorithm calls.
struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s = nullptr;
  bool on = false;
  mk_status start(cudaStream_t st, bool enable);
  mk_status stop(float *ms_out);
  ~Timer();
};

// Pinned host staging of small host tables (sources, range tables) for
// stream-ordered uploads: a ring of slots, each reused only once the copy
// that last read it has finished, so an upload never waits for the device
// unless the ring wraps onto a copy still queued.
struct PinnedRing {
  static constexpr int kSlots = 4;
  struct Slot {
    void *host = nullptr;
    size_t cap = 0;
    cudaEvent_t done = nullptr;
    bool used = false;
  };
  Slot slots[kSlots];
  uint32_t next = 0;
  // Copies `bytes` from src into a slot and queues its copy to d_dst on s.
  mk_status upload(void *d_dst, const void *src, size_t bytes, cudaStream_t s);
  void release();
};

// Exclusive scan of n u32 counts into u64 offsets (out has n+1 entries).
mk_status scan_u32_to_u64(const uint32_t *d_in, unsigned long long *d_out,
                          uint32_t n, DevBuf<unsigned long long> &tmp,
                          cudaStream_t s);

// CSR (row offsets, column ids in slab order) of the whole graph into
// buffers that grow to fit; the live edge count comes back to the host
// between the count and the fill (the call synchronises the stream).
mk_status export_csr_grow(mk_graph *g, DevBuf<unsigned long long> &row_ptr, DevBuf<uint32_t> &col,
                          cudaStream_t s, uint64_t *h_edges, size_t *bytes_acc);

// Number of co-resident blocks for a persistent cooperative launch.
int persistent_blocks(const void *kernel, int block, size_t smem, int device);

// Device buffers of a BFS handle that the member solver writes: the packed
// dist << 32 | parent words (one per vertex), the work-item array (one word
// per bucket) and the reached-vertex list (one word per vertex).  For the
// one-launch graph-set step, which runs the member solver itself.
struct TravMemberBufs {
  unsigned long long *dist;
  uint32_t *items;
  uint32_t *found;
};
mk_status trav_member_bufs(mk_traversal *t, TravMemberBufs *out);
// Label array (one word per vertex) of a WCC handle.
uint32_t *wcc_label_buf(mk_wcc *w);

}  // namespace mk

struct mk_graph {
  int device = 0;
  uint32_t V = 0;
  uint32_t weighted = 0;
  uint32_t reverse = 0;
  uint32_t keys_per_slab = 31;
  double load_factor = 0.7;
  uint64_t num_buckets = 0;
  uint64_t pool_cap = 0;
  uint4 *slabs = nullptr;
  uint32_t *boff = nullptr;
  uint32_t *bowner = nullptr;     // owning vertex of every bucket
  uint32_t *deg = nullptr;
  uint32_t *pool_top = nullptr;   // [0] bump pointer; [1] error word
  std::vector<uint32_t> h_boff;
  unsigned long long *counters = nullptr;  // [0] applied count of last update
  // per-batch scratch
  mk::DevBuf<uint8_t> applied;     // per-edge applied flags of the last update
  mk::DevBuf<unsigned long long> scan_tmp;
  mk::DevBuf<uint32_t> bucket_cnt;             // export / orientation scratch
  mk::DevBuf<unsigned long long> bucket_pos;
  uint32_t last_n = 0;
  const uint32_t *last_src = nullptr;
  const uint32_t *last_dst = nullptr;
  int last_op = 0;  // 1 insert, 2 delete
  size_t device_bytes = 0;
  mk_tuning tuning = {0u, 0u, 0u, 0u, 100u, 0u, 0u, 0u};

  // limit of a grid-barrier wait in the persistent kernels (tuning.wait_limit_us)
  unsigned long long wait_limit_ns() const {
    return (tuning.wait_limit_us ? (unsigned long long)tuning.wait_limit_us : 4000000ull) * 1000ull;
  }

  mk::GraphView view() const {
    mk::GraphView v;
    v.slabs = slabs;
    v.boff = boff;
    v.bowner = bowner;
    v.nbuckets = static_cast<uint32_t>(num_buckets);
    v.deg = deg;
    v.pool_top = pool_top;
    v.err = pool_top + 1;
    v.V = V;
    v.pool_cap = static_cast<uint32_t>(pool_cap);
    v.weighted = weighted;
    v.reverse = reverse;
    return v;
  }
  uint32_t *err_word() const { return pool_top + 1; }
};
