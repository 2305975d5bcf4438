// Single-source shortest paths for the App-hook API: relax an edge of
// weight w when it shortens the destination's distance (the hooks of
// app/sssp_kernel.cuh:6-16).
#ifndef SCAPH_APPS_SSSP_KERNEL_CUH
#define SCAPH_APPS_SSSP_KERNEL_CUH
#include "gpu_tools.cuh"

template <typename value_t>
__device__ __forceinline__ bool cond(value_t src_v, value_t dst_v, value_t w)
{
    return src_v + w < dst_v;
}

template <typename value_t>
__device__ __forceinline__ bool update(value_t src_v, value_t &dst_v, value_t w)
{
    return writeMin<value_t>(src_v + w, dst_v);
}

template <typename value_t>
__device__ __forceinline__ bool active(value_t new_value, value_t old_value)
{
    return new_value != old_value;
}
#endif
