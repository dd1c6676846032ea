// graphset.cu -- many small dynamic graphs served as one.
//
// A graph set concatenates the vertex ranges of its member graphs into one
// slab-hash graph: member m owns the global vertex ids
// [offset[m], offset[m+1]).  Members never share an edge, so one batched
// update, one multi-source traversal (one source per member), or one
// subset connected-components pass serves every member in a single launch,
// instead of one launch chain per graph.  This has no counterpart in the
// reference, whose drivers (src/BFS.cu, src/SSSP.cu) hold one graph per
// process; the per-member results are those of a DynamicGraph holding that
// member alone.
//
// Device generators: R-MAT edges per member (the reference's datasets are
// read from files; the per-member graphs here are synthetic) and random
// update batches per member drawn from a CSR export (deletes of live edges,
// inserts of uniform pairs inside the member).  Random numbers come from the
// SplitMix64 finaliser (Steele, Lea, Flood 2014) applied to a counter, so a
// (seed, index) pair always gives the same edge.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"

namespace mk {

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Uniform double in [0, 1) from the top 53 bits.
__device__ __forceinline__ double unit(unsigned long long h) {
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// Index m with off[m] <= x < off[m + 1] (off ascending, off[0] = 0).
template <typename T>
__device__ __forceinline__ uint32_t owner_of(const T *off, uint32_t n, T x) {
  uint32_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= x)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// One R-MAT edge inside a member of V vertices (V >= 2): recursive quadrant
// choice over `scale` levels; pairs outside [0, V) and self-loops are drawn
// again (32 attempts), then replaced by a uniform pair.
__device__ void rmat_local(uint32_t V, uint32_t scale, double a, double ab, double abc,
                           unsigned long long key, uint32_t &u, uint32_t &v) {
  for (uint32_t t = 0; t < 32; ++t) {
    uint32_t x = 0, y = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      const double r = unit(mix64(key ^ ((unsigned long long)(t * 64u + l) << 40)));
      const uint32_t bu = r >= ab;
      const uint32_t bv = (r >= a && r < ab) || r >= abc;
      x = (x << 1) | bu;
      y = (y << 1) | bv;
    }
    if (x < V && y < V && x != y) {
      u = x;
      v = y;
      return;
    }
  }
  const unsigned long long h = mix64(key ^ 0xA5A5A5A5A5A5A5A5ull);
  u = (uint32_t)(h % V);
  v = (uint32_t)((u + 1 + (h >> 32) % (V - 1)) % V);
}

__global__ void k_gen_rmat_set(const uint32_t *__restrict__ voff, uint32_t G,
                               const unsigned long long *__restrict__ eoff,
                               unsigned long long total, double a, double ab, double abc,
                               unsigned long long seed, uint32_t w_lo, uint32_t w_hi,
                               uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                               uint32_t *__restrict__ w) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < total;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t m = owner_of(eoff, G + 1, i);
    const uint32_t base = voff[m], V = voff[m + 1] - base;
    const unsigned long long key = mix64(seed ^ mix64(i));
    uint32_t u = 0, v = 0;
    if (V >= 2) {
      uint32_t scale = 1;
      while ((1u << scale) < V) ++scale;
      rmat_local(V, scale, a, ab, abc, key, u, v);
    }
    // V == 1 leaves a self-loop, which every update skips
    src[i] = base + u;
    dst[i] = base + v;
    if (w) w[i] = w_lo + (uint32_t)(mix64(key + 1) % ((unsigned long long)w_hi - w_lo + 1));
  }
}

// Deletes: a live edge of the member chosen uniformly from its CSR rows.
__global__ void k_gen_set_deletes(const uint32_t *__restrict__ voff, uint32_t G,
                                  const unsigned long long *__restrict__ row_ptr,
                                  const uint32_t *__restrict__ col,
                                  const unsigned long long *__restrict__ doff,
                                  unsigned long long total, unsigned long long seed,
                                  uint32_t *__restrict__ ds, uint32_t *__restrict__ dd) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < total;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t m = owner_of(doff, G + 1, i);
    const uint32_t lo = voff[m], hi = voff[m + 1];
    const unsigned long long e0 = row_ptr[lo], e1 = row_ptr[hi];
    if (e1 == e0) {  // no edge left: a self-loop is a no-op
      ds[i] = lo;
      dd[i] = lo;
      continue;
    }
    const unsigned long long idx = e0 + mix64(seed ^ mix64(i)) % (e1 - e0);
    const uint32_t row = lo + owner_of(row_ptr + lo, hi - lo + 1, idx);
    ds[i] = row;
    dd[i] = col[idx];
  }
}

// Inserts: a uniform pair of distinct vertices inside the member.
__global__ void k_gen_set_inserts(const uint32_t *__restrict__ voff, uint32_t G,
                                  const unsigned long long *__restrict__ ioff,
                                  unsigned long long total, unsigned long long seed,
                                  uint32_t w_lo, uint32_t w_hi, uint32_t *__restrict__ is,
                                  uint32_t *__restrict__ id, uint32_t *__restrict__ iw) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < total;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t m = owner_of(ioff, G + 1, i);
    const uint32_t base = voff[m], V = voff[m + 1] - base;
    const unsigned long long h = mix64(seed ^ mix64(i ^ 0x5555555555555555ull));
    uint32_t u = 0, v = 0;
    if (V >= 2) {
      u = (uint32_t)(h % V);
      v = (uint32_t)((u + 1 + (h >> 32) % (V - 1)) % V);
    }
    is[i] = base + u;
    id[i] = base + v;
    if (iw) iw[i] = w_lo + (uint32_t)(mix64(h + 7) % ((unsigned long long)w_hi - w_lo + 1));
  }
}

// Bit v of bits = flags[member of v]; one thread per vertex, one ballot per word.
__global__ void k_select_bits(const uint32_t *__restrict__ voff, uint32_t G, uint32_t V,
                              const uint8_t *__restrict__ flags, uint32_t *__restrict__ bits) {
  const uint32_t words = (V + 31) / 32;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < words * 32u;
       base += gridDim.x * blockDim.x) {
    const uint32_t v = base + (threadIdx.x & 31);
    bool on = false;
    if (v < V) on = flags[owner_of(voff, G + 1, v)] != 0;
    const uint32_t word = __ballot_sync(0xFFFFFFFFu, on);
    if ((threadIdx.x & 31) == 0) bits[base >> 5] = word;
  }
}

static int gen_grid(unsigned long long n, int device) {
  return (int)std::max<unsigned long long>(
      1, std::min<unsigned long long>((n + 255) / 256, (unsigned long long)device_sm_count(device) * 16));
}

static mk_status read_total(const unsigned long long *d_off, uint32_t G, cudaStream_t s,
                            unsigned long long *total) {
  MK_CUDA(cudaMemcpyAsync(total, d_off + G, 8, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  return MK_OK;
}

}  // namespace mk

using namespace mk;

struct mk_graphset {
  uint32_t ngraphs = 0;
  mk_graph *g = nullptr;
  std::vector<uint32_t> h_off;
  uint32_t *d_off = nullptr;
};

extern "C" {

mk_status mk_graphset_create(uint32_t num_graphs, const uint32_t *h_num_vertices,
                             const uint32_t *const *h_degree_hints, double load_factor,
                             uint32_t weighted, int32_t device, uint64_t pool_slabs,
                             mk_graphset **out) {
  if (!out || !h_num_vertices) return fail(MK_ERR_INVALID, "mk_graphset_create: null argument");
  *out = nullptr;
  if (num_graphs == 0) return fail(MK_ERR_INVALID, "mk_graphset_create: no member graph");
  std::vector<uint32_t> off((size_t)num_graphs + 1, 0);
  uint64_t total = 0;
  for (uint32_t m = 0; m < num_graphs; ++m) {
    if (h_num_vertices[m] == 0) return fail(MK_ERR_INVALID, "mk_graphset_create: empty member graph");
    total += h_num_vertices[m];
    if (total >= kTombKey) return fail(MK_ERR_INVALID, "mk_graphset_create: too many vertices");
    off[m + 1] = (uint32_t)total;
  }
  std::vector<uint32_t> hints;
  if (h_degree_hints) {
    hints.resize(total, 1u);
    for (uint32_t m = 0; m < num_graphs; ++m)
      if (h_degree_hints[m])
        std::copy(h_degree_hints[m], h_degree_hints[m] + h_num_vertices[m], hints.begin() + off[m]);
  }
  mk_graph_desc d{};
  d.num_vertices = (uint32_t)total;
  d.weighted = weighted ? 1u : 0u;
  d.reverse = 0;
  d.flags = 0;
  d.load_factor = load_factor;
  d.h_degree_hints = h_degree_hints ? hints.data() : nullptr;
  d.device = device;
  d.pool_slabs = pool_slabs;
  mk_graph *g = nullptr;
  MK_CHECK(mk_graph_create(&d, &g));
  DeviceGuard dg(device);
  mk_graphset *s = new mk_graphset();
  s->ngraphs = num_graphs;
  s->g = g;
  s->h_off = std::move(off);
  cudaError_t e = cudaMalloc(&s->d_off, ((size_t)num_graphs + 1) * 4);
  if (e == cudaSuccess)
    e = cudaMemcpy(s->d_off, s->h_off.data(), ((size_t)num_graphs + 1) * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    mk_graphset_destroy(s);
    return cuda_fail(e, "mk_graphset_create");
  }
  g->device_bytes += ((size_t)num_graphs + 1) * 4;
  *out = s;
  return MK_OK;
}

mk_status mk_graphset_destroy(mk_graphset *s) {
  if (!s) return MK_OK;
  if (s->g) {
    DeviceGuard dg(s->g->device);
    if (s->d_off) cudaFree(s->d_off);
    mk_graph_destroy(s->g);
  }
  delete s;
  return MK_OK;
}

mk_status mk_graphset_union(mk_graphset *s, mk_graph **g) {
  if (!s || !g) return fail(MK_ERR_INVALID, "mk_graphset_union: null argument");
  *g = s->g;
  return MK_OK;
}

mk_status mk_graphset_num_graphs(mk_graphset *s, uint32_t *h_num_graphs) {
  if (!s || !h_num_graphs) return fail(MK_ERR_INVALID, "mk_graphset_num_graphs: null argument");
  *h_num_graphs = s->ngraphs;
  return MK_OK;
}

mk_status mk_graphset_offsets(mk_graphset *s, uint32_t *h_offsets) {
  if (!s || !h_offsets) return fail(MK_ERR_INVALID, "mk_graphset_offsets: null argument");
  std::copy(s->h_off.begin(), s->h_off.end(), h_offsets);
  return MK_OK;
}

mk_status mk_graphset_select_bits(mk_graphset *s, const uint8_t *d_graph_flags, uint32_t *d_bits,
                                  void *stream) {
  if (!s || !d_graph_flags || !d_bits)
    return fail(MK_ERR_INVALID, "mk_graphset_select_bits: null argument");
  DeviceGuard dg(s->g->device);
  const uint32_t V = s->g->V;
  const uint32_t words = (V + 31) / 32;
  k_select_bits<<<gen_grid((unsigned long long)words * 32, s->g->device), 256, 0, as_stream(stream)>>>(
      s->d_off, s->ngraphs, V, d_graph_flags, d_bits);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_graphset_offsets_device(mk_graphset *s, const uint32_t **d_offsets) {
  if (!s || !d_offsets) return fail(MK_ERR_INVALID, "mk_graphset_offsets_device: null argument");
  *d_offsets = s->d_off;
  return MK_OK;
}

mk_status mk_gen_rmat_set(const uint32_t *d_vertex_offsets, uint32_t num_graphs,
                          const uint64_t *d_edge_offsets, double a, double b, double c,
                          uint64_t seed, uint32_t w_lo, uint32_t w_hi, uint32_t *d_src,
                          uint32_t *d_dst, uint32_t *d_w, void *stream) {
  if (!d_vertex_offsets || !d_edge_offsets || !d_src || !d_dst)
    return fail(MK_ERR_INVALID, "mk_gen_rmat_set: null argument");
  if (num_graphs == 0) return fail(MK_ERR_INVALID, "mk_gen_rmat_set: no member graph");
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    return fail(MK_ERR_INVALID, "mk_gen_rmat_set: a, b, c must be probabilities with a+b+c <= 1");
  if (w_lo > w_hi) return fail(MK_ERR_INVALID, "mk_gen_rmat_set: w_lo > w_hi");
  int device = 0;
  MK_CUDA(cudaGetDevice(&device));
  cudaStream_t st = as_stream(stream);
  const unsigned long long *eoff = reinterpret_cast<const unsigned long long *>(d_edge_offsets);
  unsigned long long total = 0;
  MK_CHECK(read_total(eoff, num_graphs, st, &total));
  if (total == 0) return MK_OK;
  k_gen_rmat_set<<<gen_grid(total, device), 256, 0, st>>>(
      d_vertex_offsets, num_graphs, eoff, total, a, a + b, a + b + c, seed, w_lo, w_hi, d_src,
      d_dst, d_w);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_gen_set_batches(const uint32_t *d_vertex_offsets, uint32_t num_graphs,
                             const uint64_t *d_row_ptr, const uint32_t *d_col,
                             const uint64_t *d_del_offsets, const uint64_t *d_ins_offsets,
                             uint64_t seed, uint32_t w_lo, uint32_t w_hi, uint32_t *d_del_src,
                             uint32_t *d_del_dst, uint32_t *d_ins_src, uint32_t *d_ins_dst,
                             uint32_t *d_ins_w, void *stream) {
  if (!d_vertex_offsets || !d_row_ptr || !d_col || !d_del_offsets || !d_ins_offsets)
    return fail(MK_ERR_INVALID, "mk_gen_set_batches: null argument");
  if (num_graphs == 0) return fail(MK_ERR_INVALID, "mk_gen_set_batches: no member graph");
  if (w_lo > w_hi) return fail(MK_ERR_INVALID, "mk_gen_set_batches: w_lo > w_hi");
  int device = 0;
  MK_CUDA(cudaGetDevice(&device));
  cudaStream_t st = as_stream(stream);
  const auto *doff = reinterpret_cast<const unsigned long long *>(d_del_offsets);
  const auto *ioff = reinterpret_cast<const unsigned long long *>(d_ins_offsets);
  const auto *rp = reinterpret_cast<const unsigned long long *>(d_row_ptr);
  unsigned long long nd = 0, ni = 0;
  MK_CHECK(read_total(doff, num_graphs, st, &nd));
  MK_CHECK(read_total(ioff, num_graphs, st, &ni));
  if (nd) {
    if (!d_del_src || !d_del_dst) return fail(MK_ERR_INVALID, "mk_gen_set_batches: null delete output");
    k_gen_set_deletes<<<gen_grid(nd, device), 256, 0, st>>>(d_vertex_offsets, num_graphs, rp, d_col,
                                                              doff, nd, seed, d_del_src, d_del_dst);
  }
  if (ni) {
    if (!d_ins_src || !d_ins_dst) return fail(MK_ERR_INVALID, "mk_gen_set_batches: null insert output");
    k_gen_set_inserts<<<gen_grid(ni, device), 256, 0, st>>>(
        d_vertex_offsets, num_graphs, ioff, ni, seed, w_lo, w_hi, d_ins_src, d_ins_dst, d_ins_w);
  }
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

}  // extern "C"
