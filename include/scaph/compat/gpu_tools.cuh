// Device helpers that the reference's application hooks call
// (src/gpu_tools.cuh:53-79): atomic min / max of a vertex value that report
// whether they lowered (raised) it.  Part of the App-hook compatibility
// layer: an app's bfs_kernel.cuh / sssp_kernel.cuh / wcc_kernel.cuh includes
// "gpu_tools.cuh" and gets these.
#ifndef SCAPH_COMPAT_GPU_TOOLS_CUH
#define SCAPH_COMPAT_GPU_TOOLS_CUH

// Atomically dst = min(dst, src); true if this call changed dst.
template <typename value_t>
__device__ __forceinline__ bool writeMin(value_t src, value_t &dst)
{
    value_t seen = dst;
    while (src < seen) {
        const value_t prev = atomicCAS(&dst, seen, src);
        if (prev == seen) return true;
        seen = prev;
    }
    return false;
}

// Atomically dst = max(dst, src); true if this call changed dst.
template <typename value_t>
__device__ __forceinline__ bool writeMax(value_t src, value_t &dst)
{
    value_t seen = dst;
    while (seen < src) {
        const value_t prev = atomicCAS(&dst, seen, src);
        if (prev == seen) return true;
        seen = prev;
    }
    return false;
}

#endif
