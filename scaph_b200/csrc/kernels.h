// Host-side entry points of the device kernels (bfs_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"

namespace scaph {

// One BFS level over vertices [vlo, vhi): dir 0 = push (k_push + giant
// chunks over out-edge graph g), dir 1 = pull (k_pull over in-edge graph g).
cudaError_t run_level(int dir, int block, int grid, const GraphDev &g, const BfsDev &s, uint32_t vlo,
                      uint32_t vhi, cudaStream_t st);
// Resident CTAs per SM of the level kernel for `dir` at `block` threads.
int level_occupancy(int dir, int block);
cudaError_t fill_u32(uint32_t *p, uint32_t value, unsigned long long n, int grid, cudaStream_t st);
cudaError_t set_source(const BfsDev &s, uint32_t src, uint32_t *front, cudaStream_t st);

}  // namespace scaph
