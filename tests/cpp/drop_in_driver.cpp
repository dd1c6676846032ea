// Reference-style driver on the drop-in shim: the call sequence of
// meerkat-pkd/Meerkat src/BFS.cu:11-131 and src/SSSP.cu (graph from device
// arrays, Static, then per batch: graph update followed by
// Incremental/Decremental with the same device batch), on a seeded R-MAT
// graph instead of text files.  Prints the final BFS and SSSP distances and
// WCC labels as text for the test to compare with the oracle.  With "rev" as
// the second argument the algorithms get reverse graphs of the same edges
// (SetReverse), updated with every batch.
#include <cuda_runtime.h>

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "meerkat_compat.hpp"

static uint32_t *to_device(const std::vector<uint32_t> &h) {
  uint32_t *d = nullptr;
  cudaMalloc(&d, h.size() * 4 + 4);
  cudaMemcpy(d, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
  return d;
}

int main(int argc, char **argv) {
  const uint32_t scale = argc > 1 ? (uint32_t)atoi(argv[1]) : 12;
  const bool rev = argc > 2 && std::string(argv[2]) == "rev";
  const uint64_t E = 8ull << scale;
  const uint32_t V = 1u << scale;
  std::vector<uint32_t> src(E), dst(E), wgt(E);
  meerkat::check(mk_gen_rmat(scale, E, 0.57, 0.19, 0.19, 7, 1, 64, src.data(), dst.data(),
                             wgt.data()), "gen");
  std::vector<uint32_t> hints(V, 1);  // the reference drivers pass hints of 1
  using AllocPolicy = FullAllocatorPolicy<9, 48, 1>;
  using Allocator = typename AllocPolicy::DynamicAllocatorT;
  std::unique_ptr<Allocator> Alloc{new Allocator};
  DynGraph<UnweightedEdgePolicyT<AllocPolicy>> G{V, *Alloc, 0.7, hints.data(), 0};
  DynGraph<WeightedEdgePolicyMapT<AllocPolicy>> GW{V, *Alloc, 0.7, hints.data(), 0};
  uint32_t *dS = to_device(src), *dD = to_device(dst), *dW = to_device(wgt);
  DynGraph<RevUnweightedEdgePolicyT<AllocPolicy>> GR{V, *Alloc, 0.7, hints.data(), 0};
  DynGraph<RevWeightedEdgePolicyMapT<AllocPolicy>> GRW{V, *Alloc, 0.7, hints.data(), 0};
  G.InsertEdges(dS, dD, (uint32_t)E);
  GW.InsertEdges(dS, dD, (uint32_t)E, dW);
  if (rev) {
    GR.InsertEdges(dS, dD, (uint32_t)E);
    GRW.InsertEdges(dS, dD, (uint32_t)E, dW);
  }
  cudaDeviceSynchronize();
  BFS<AllocPolicy> B(G, 0, V);
  SSSP<AllocPolicy> S(GW, 0, V);
  WCC<AllocPolicy> C(G, V);
  if (rev) {
    B.SetReverse(GR);
    S.SetReverse(GRW);
    C.SetReverse(GR);
  }
  B.Static((uint32_t)E);
  S.Static((uint32_t)E);
  C.Static();
  // batch 0: delete the first 1/8 of the edges; batch 1: insert them back
  const uint32_t nb = (uint32_t)(E / 8);
  G.DeleteEdges(dS, dD, nb);
  GW.DeleteEdges(dS, dD, nb);
  if (rev) {
    GR.DeleteEdges(dS, dD, nb);
    GRW.DeleteEdges(dS, dD, nb);
  }
  cudaDeviceSynchronize();
  B.Decremental(dS, dD, nb);
  S.Decremental(dS, dD, dW, nb);
  C.Decremental(dS, dD, nb);
  const uint32_t half = nb / 2;  // re-insert half of them
  G.InsertEdges(dS, dD, half);
  GW.InsertEdges(dS, dD, half, dW);
  if (rev) {
    GR.InsertEdges(dS, dD, half);
    GRW.InsertEdges(dS, dD, half, dW);
  }
  cudaDeviceSynchronize();
  B.Incremental(dS, dD, half);
  S.Incremental(dS, dD, dW, half);
  C.Incremental(dS, dD, half);
  std::vector<uint32_t> db = B.Distances(), ds = S.Distances(), lc = C.Labels();
  printf("V %u E %llu deleted %u reinserted %u\n", V, (unsigned long long)E, nb, half);
  for (uint32_t i = 0; i < V; ++i) printf("%u %u %u\n", db[i], ds[i], lc[i]);
  cudaFree(dS);
  cudaFree(dD);
  cudaFree(dW);
  return 0;
}
