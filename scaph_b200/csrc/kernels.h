// Host-side entry points of the device kernels (bfs_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"

namespace scaph {

// One BFS level over vertices [vlo, vhi): dir 0 = push (k_push + giant
// chunks over out-edge graph g), dir 1 = pull (k_pull over in-edge graph g).
cudaError_t run_level(int dir, int block, int grid, const GraphDev &g, const BfsDev &s, uint32_t vlo,
                      uint32_t vhi, cudaStream_t st);
// A push or pull pass over a list of vertex ranges (out-of-core page batches;
// push only: the giant chunks they queue run in run_giant).
cudaError_t run_ranges(int dir, int block, int grid, const GraphDev &g, const BfsDev &s, const RangeList &rl,
                       cudaStream_t st);
cudaError_t run_giant(int block, int grid, const GraphDev &g, const BfsDev &s, cudaStream_t st);
// Deferred-claim push levels (BfsDev::push_defer): claims the next frontier
// word by word after the push (and giant-chunk) kernels.
cudaError_t run_push_finalize(int block, int grid, const BfsDev &s, cudaStream_t st);
// k_push_finalize_g(BfsGraphArgs): the graph-mode node, after the giant chunks
const void *push_finalize_graph_kernel(int block);
// k_graph_init(BfsGraphArgs, u32* depth, u32* parent, u32 src, u32 unreached, const u32* dead, u32 nlevels_clear)
// Graph mode: the push, giant-chunk and pull kernels of a level (each leaves
// at once unless the level's direction selects it).
// graph-mode level kernels; giant_pull runs a push level's giant chunks or
// a pull level's pull (one node instead of two)
void level_graph_kernels(int block, const void **push, const void **giant, const void **pull,
                         const void **giant_pull);
const void *graph_init_kernel();
// k_decide(BfsGraphArgs, DecideArgs, handle loop)
const void *decide_kernel();
// k_decide_learned(BfsGraphArgs, DecideArgs, MlpDev, handle loop): 64 threads
const void *decide_learned_kernel();
// Resident CTAs per SM of the level kernel for `dir` at `block` threads.
int level_occupancy(int dir, int block);
cudaError_t fill_u32(uint32_t *p, uint32_t value, unsigned long long n, int grid, cudaStream_t st);
cudaError_t set_source(const BfsDev &s, uint32_t src, uint32_t *front, cudaStream_t st);

}  // namespace scaph
