// Device helpers shared by the level kernels (bfs_kernels.cu, msbfs.cu).
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"

namespace scaph {
namespace kc {

// Exclusive scan of one u32 per thread over a CTA (total returned too).
// wsum: BLOCK/32 words of shared memory.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t *wsum, uint32_t &total)
{
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < NW ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < NW) wsum[lane] = t;
    }
    __syncthreads();
    uint32_t base = wid ? wsum[wid - 1] : 0u;
    total = wsum[NW - 1];
    __syncthreads();
    return base + inc - x;
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
    return x;
}

// Stages g's page table + coarse index into the given shared arrays when
// they fit (kLutPages / kLutCoarse entries); otherwise uses global memory.
// Caller synchronises the CTA before using the result.
template <int BLOCK>
__device__ __forceinline__ PageLut stage_lut(const GraphDev &g, PageDev *sp, uint32_t *sc)
{
    const uint32_t ncoarse = (g.V >> g.cshift) + 1;
    if (g.npages + 1 <= (uint32_t)kLutPages && ncoarse <= (uint32_t)kLutCoarse) {
        for (uint32_t i = threadIdx.x; i <= g.npages; i += BLOCK) sp[i] = g.pages[i];
        for (uint32_t i = threadIdx.x; i < ncoarse; i += BLOCK) sc[i] = g.coarse[i];
        return PageLut{sp, sc, g.cshift};
    }
    return PageLut{g.pages, g.coarse, g.cshift};
}

// Fire-and-forget global OR (no return value: a reduction, not an atomic
// round trip).  No "memory" clobber: the kernels never read these words in
// the same launch, so loads may be scheduled across the reductions.
__device__ __forceinline__ void red_or(unsigned long long *p, unsigned long long v)
{
    asm volatile("red.global.or.b64 [%0], %1;" ::"l"(p), "l"(v));
}

__device__ __forceinline__ void red_or(uint32_t *p, uint32_t v)
{
    asm volatile("red.global.or.b32 [%0], %1;" ::"l"(p), "r"(v));
}

}  // namespace kc
}  // namespace scaph
