// probe.cu -- ceiling of the update path's memory pattern on this device.
//
// Benchmark-only: built into libmk_bench_probe.so, which bench.py alone
// loads; it is not part of libmeerkat_b200.so or its public header.
//
// The update kernels touch, per edge, one random 128-byte slab line (read,
// then a CAS on one of its words), one random word of the bucket-offset
// array (read) and one random word of the degree array (add).  A copy kernel
// measures sequential bandwidth, which random line traffic cannot reach; this
// probe replays the same pattern with no decision logic so the update
// kernels can be judged against what the memory system delivers for it.
//
//   mode 0  random 128-byte line reads
//   mode 1  mode 0 + one CAS per line (the slab read-modify-write)
//   mode 2  mode 1 + a random 4-byte read and a random 4-byte add on two
//           per-vertex arrays of `small_words` words each
//   mode 3  random 32-byte sector reads (one sector of a random line)
//   mode 4  random 64-byte half-line reads
//
// Warp-cooperative: a warp reads the lines of its 32 operations as 32
// coalesced loads, lane j then issues operation j's CAS / add.  Lines and
// words are chosen by a counter-based hash of (seed, operation).
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

__device__ __forceinline__ unsigned long long probe_mix(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void __launch_bounds__(256) k_probe_rmw(uint32_t *__restrict__ lines, uint64_t nlines,
                                                   uint32_t *__restrict__ small_a,
                                                   uint32_t *__restrict__ small_b,
                                                   uint32_t small_words, uint64_t nops,
                                                   uint32_t mode, unsigned long long seed,
                                                   unsigned long long *sink) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  unsigned long long acc = 0;
  if (mode >= 3) {
    // partial-line reads: lane-group g of (2 or 4) lanes reads 32 or 64
    // bytes of operation g's random line (16 bytes per lane)
    const uint32_t per = mode == 3 ? 2u : 4u;  // lanes per operation
    const uint32_t ops_per_warp = 32u / per;
    for (uint64_t base = warp * ops_per_warp; base < nops; base += nwarps * ops_per_warp) {
      const uint64_t op = base + lane / per;
      if (op < nops) {
        const unsigned long long h = probe_mix(seed ^ op);
        const uint64_t line = h % nlines;
        const uint32_t sec = (uint32_t)(h >> 40) & (mode == 3 ? 3u : 1u);  // which 32/64 B of the line
        const uint4 *p = reinterpret_cast<const uint4 *>(lines + line * 32) + sec * per + (lane % per);
        const uint4 q = __ldcg(p);
        acc += q.x ^ q.y ^ q.z ^ q.w;
      }
    }
    if (acc == 0x5EEDull) atomicAdd(sink, acc);
    return;
  }
  for (uint64_t base = warp * 32; base < nops; base += nwarps * 32) {
    const uint64_t op = base + lane;
    const unsigned long long h = probe_mix(seed ^ op);
    const uint64_t line = op < nops ? h % nlines : ~0ull;
    uint32_t v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const uint64_t lj = __shfl_sync(0xFFFFFFFFu, line, j);
      v[j] = lj != ~0ull ? __ldcg(lines + lj * 32 + lane) : 0u;
    }
    uint32_t mine = 0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const uint32_t w5 = __shfl_sync(0xFFFFFFFFu, v[j], 5);
      if (lane == (uint32_t)j) mine = w5;
      acc += v[j];
    }
    if (line != ~0ull && mode >= 1) {
      uint32_t *p = lines + line * 32 + 5;
      acc += atomicCAS(p, mine, mine + 1u);
    }
    if (line != ~0ull && mode >= 2) {
      const uint32_t i = (uint32_t)(h >> 32) % small_words;
      const uint32_t k = (uint32_t)(probe_mix(h) % small_words);
      acc += __ldcg(small_a + i);
      atomicAdd(small_b + k, 1u);
    }
  }
  if (acc == 0x5EEDull) atomicAdd(sink, acc);  // keeps the loads live
}

}  // namespace

// Returns 0 on success, 1 on a bad argument, 2 on a CUDA error.  Synchronises
// and writes the launch's device time to *ms_out (CUDA events on `stream`).
extern "C" int mkb_probe_random_rmw(void *d_lines, uint64_t line_count, void *d_small_a,
                                    void *d_small_b, uint32_t small_words, uint64_t num_ops,
                                    uint32_t mode, uint64_t seed, void *d_sink, void *stream,
                                    float *ms_out) {
  if (!d_lines || !line_count || !d_sink || !ms_out || mode > 4 ||
      (mode == 2 && (!d_small_a || !d_small_b || !small_words)))
    return 1;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 2;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 2;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe_rmw, 256, 0) != cudaSuccess)
    return 2;
  const uint64_t want = (num_ops + 255) / 256;
  const uint64_t cap = (uint64_t)sms * (per_sm > 0 ? per_sm : 1);
  const int blocks = (int)(want < cap ? (want ? want : 1) : cap);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return 2;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return 2;
  }
  int rc = 0;
  cudaEventRecord(e0, s);
  k_probe_rmw<<<blocks, 256, 0, s>>>(static_cast<uint32_t *>(d_lines), line_count,
                                     static_cast<uint32_t *>(d_small_a),
                                     static_cast<uint32_t *>(d_small_b), small_words, num_ops,
                                     mode, seed, static_cast<unsigned long long *>(d_sink));
  if (cudaGetLastError() != cudaSuccess) rc = 2;
  cudaEventRecord(e1, s);
  if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(ms_out, e0, e1) != cudaSuccess)
    rc = 2;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}
