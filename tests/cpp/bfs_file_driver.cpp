// The reference's BFS driver workflow (meerkat-pkd/Meerkat src/BFS.cu:11-131)
// on the drop-in shim, reading the same files:
//   bfs_file_driver <graph file> <op: 0 insert, else delete> <update prefix> <batches>
// Line 1 is the reference's timing line ("<file>,<static ms>,<batch ms>...");
// then the final BFS level of every vertex, one per line, for the test.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "meerkat_compat.hpp"

static uint32_t *to_device(const std::vector<uint32_t> &h) {
  uint32_t *d = nullptr;
  meerkat::check(cudaMalloc(&d, h.size() * 4 + 4) == cudaSuccess ? MK_OK : MK_ERR_CUDA, "cudaMalloc");
  cudaMemcpy(d, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
  return d;
}

int main(int argc, char **argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s <graph> <op> <update prefix> <batches>\n", argv[0]);
    return 2;
  }
  const std::string file = argv[1];
  const bool insertion = std::string(argv[2]) == "0";
  const std::string prefix = argv[3];
  const uint32_t batches = (uint32_t)std::stoul(argv[4]);
  // the reference starts at vertex 2 for wiki-talk and 0 otherwise
  const uint32_t source = std::strstr(file.c_str(), "wiki.txt") ? 2u : 0u;
  std::printf("%s", file.c_str());

  meerkat::EdgeList g = meerkat::ReadGraphFile(file);
  const uint32_t V = g.num_vertices;
  std::vector<uint32_t> hints(V, 1);  // the reference passes hints of 1
  using AllocPolicy = FullAllocatorPolicy<9, 48, 1>;
  using Allocator = typename AllocPolicy::DynamicAllocatorT;
  std::unique_ptr<Allocator> Alloc{new Allocator};
  DynGraph<UnweightedEdgePolicyT<AllocPolicy>> G{V, *Alloc, 0.7, hints.data(), 0};
  uint32_t *dS = to_device(g.src), *dD = to_device(g.dst);
  G.InsertEdges(dS, dD, (uint32_t)g.src.size());
  cudaDeviceSynchronize();
  cudaFree(dS);
  cudaFree(dD);
  BFS<AllocPolicy> B(G, source, V);
  std::printf(",%f", B.Static((uint32_t)g.src.size()));
  for (uint32_t i = 0; i < batches; ++i) {
    meerkat::EdgeList b = meerkat::ReadBatchFile(prefix, i);
    const uint32_t n = (uint32_t)b.src.size();
    uint32_t *bS = to_device(b.src), *bD = to_device(b.dst);
    float ms;
    if (insertion) {
      G.InsertEdges(bS, bD, n);
      ms = B.Incremental(bS, bD, n);
    } else {
      G.DeleteEdges(bS, bD, n);
      ms = B.Decremental(bS, bD, n);
    }
    std::printf(",%f", ms);
    cudaFree(bS);
    cudaFree(bD);
  }
  std::printf("\n");
  for (uint32_t d : B.Distances()) std::printf("%u\n", d);
  return 0;
}
