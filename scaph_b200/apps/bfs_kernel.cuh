// BFS vertex program for the App-hook API: a vertex one hop past a reached
// vertex gets its depth + 1 (the hooks of app/bfs_kernel.cuh:6-16).
#ifndef SCAPH_APPS_BFS_KERNEL_CUH
#define SCAPH_APPS_BFS_KERNEL_CUH
#include "gpu_tools.cuh"

template <typename value_t>
__device__ __forceinline__ bool cond(value_t src_v, value_t dst_v)
{
    return src_v + 1 < dst_v;
}

template <typename value_t>
__device__ __forceinline__ bool update(value_t src_v, value_t &dst_v)
{
    return writeMin<value_t>(src_v + 1, dst_v);
}

template <typename value_t>
__device__ __forceinline__ bool active(value_t new_value, value_t old_value)
{
    return new_value != old_value;
}
#endif
