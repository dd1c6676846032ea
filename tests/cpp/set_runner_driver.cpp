// Batched many-graph step through the C++ shim (meerkat::GraphSet and
// meerkat::GraphSetRunner): a graph set of seeded R-MAT members, one BFS or
// WCC query per member, K steps of a mixed batch per step (deletes of the
// first edges of every member, then inserts of them back, alternating).
// Prints, per member, its query kind and its answer (BFS levels or local WCC
// labels) for the test to compare with the oracle.
//
//   set_runner_driver <members> <steps> <capture 0|1> [single 0|1]
//
// With single = 1 every step is the one-launch form.  The driver exits 5 if
// the runner reports other than four launches per step (two update kernels,
// the member BFS, the member WCC), or one in the one-launch form.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "meerkat_compat.hpp"

static uint32_t *to_device(const std::vector<uint32_t> &h) {
  uint32_t *d = nullptr;
  cudaMalloc(&d, h.size() * 4 + 4);
  cudaMemcpy(d, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
  return d;
}

int main(int argc, char **argv) {
  const uint32_t G = argc > 1 ? (uint32_t)atoi(argv[1]) : 6;
  const uint32_t K = argc > 2 ? (uint32_t)atoi(argv[2]) : 3;
  const bool capture = argc > 3 && atoi(argv[3]) != 0;
  const bool single = argc > 4 && atoi(argv[4]) != 0;
  std::vector<uint32_t> nv(G);
  for (uint32_t m = 0; m < G; ++m) nv[m] = 256u << (m % 4);  // 256 .. 2048 vertices
  meerkat::GraphSet set(nv, /*weighted=*/true);
  const std::vector<uint32_t> off = set.Offsets();
  std::vector<uint32_t> src, dst, wgt, dsrc, ddst;
  std::vector<uint8_t> query(G);
  std::vector<uint32_t> bsrc(G, 0);
  for (uint32_t m = 0; m < G; ++m) {
    uint32_t scale = 0;
    while ((1u << scale) < nv[m]) ++scale;
    const uint64_t E = 6ull * nv[m];
    std::vector<uint32_t> s(E), d(E), w(E);
    meerkat::check(mk_gen_rmat(scale, E, 0.57, 0.19, 0.19, 100 + m, 1, 64, s.data(), d.data(),
                               w.data()), "gen");
    for (uint64_t i = 0; i < E; ++i) {
      src.push_back(s[i] + off[m]);
      dst.push_back(d[i] + off[m]);
      wgt.push_back(w[i]);
      if (i < E / 10) {  // the updated edges: the first tenth of each member
        dsrc.push_back(s[i] + off[m]);
        ddst.push_back(d[i] + off[m]);
      }
    }
    query[m] = (m % 2) ? MK_QUERY_WCC : MK_QUERY_BFS;
    bsrc[m] = s[0];  // a vertex with an out-edge
  }
  uint32_t *dS = to_device(src), *dD = to_device(dst), *dW = to_device(wgt);
  set.InsertEdges(dS, dD, (uint32_t)src.size(), dW);
  std::vector<uint32_t> dw(dsrc.size(), 7);
  uint32_t *uS = to_device(dsrc), *uD = to_device(ddst), *uW = to_device(dw);
  meerkat::check(mk_graph_reserve_batch(set.Union(), (uint32_t)dsrc.size()), "reserve");
  meerkat::GraphSetRunner run(set, query, bsrc);
  if (single) run.SetSingle(true);
  if (run.LaunchesPerStep() != (single ? 1u : 4u)) return 5;
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  // step k deletes the updated edges (k even) or inserts them back with
  // weight 7 (k odd)
  auto step = [&](uint32_t k) {
    if (k % 2 == 0)
      run.Step(uS, uD, (uint32_t)dsrc.size(), nullptr, nullptr, nullptr, 0, st);
    else
      run.Step(nullptr, nullptr, 0, uS, uD, uW, (uint32_t)dsrc.size(), st);
  };
  cudaDeviceSynchronize();
  if (capture && K >= 2) {
    step(0);  // one step outside the capture (first launches load the kernels)
    cudaStreamSynchronize(st);
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    for (uint32_t k = 1; k < K; ++k) step(k);
    if (cudaStreamEndCapture(st, &graph) != cudaSuccess) return 3;
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) return 4;
    cudaGraphLaunch(exec, st);
    cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
  } else {
    for (uint32_t k = 0; k < K; ++k) step(k);
  }
  cudaStreamSynchronize(st);
  uint32_t deverr = 0;
  meerkat::check(mk_graph_sync(set.Union(), st, &deverr), "sync");
  const uint32_t V = off[G];
  std::vector<unsigned long long> packed(V);
  std::vector<uint32_t> labels(V);
  cudaMemcpy(packed.data(), run.BfsPacked(), (size_t)V * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(labels.data(), run.WccLabels(), (size_t)V * 4, cudaMemcpyDeviceToHost);
  for (uint32_t m = 0; m < G; ++m) {
    printf("%u %u %u", m, (unsigned)query[m], bsrc[m]);
    for (uint32_t v = off[m]; v < off[m + 1]; ++v) {
      const uint32_t x = query[m] == MK_QUERY_BFS ? (uint32_t)(packed[v] >> 32) : labels[v] - off[m];
      printf(" %u", x);
    }
    printf("\n");
  }
  return 0;
}
