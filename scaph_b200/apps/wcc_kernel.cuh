// Connected-component labels for the App-hook API: the smallest label
// flows along edges (the hooks of app/wcc_kernel.cuh:5-15).
#ifndef SCAPH_APPS_WCC_KERNEL_CUH
#define SCAPH_APPS_WCC_KERNEL_CUH
#include "gpu_tools.cuh"

template <typename value_t>
__device__ __forceinline__ bool cond(value_t src_v, value_t dst_v)
{
    return src_v < dst_v;
}

template <typename value_t>
__device__ __forceinline__ bool update(value_t src_v, value_t &dst_v)
{
    return writeMin<value_t>(src_v, dst_v);
}

template <typename value_t>
__device__ __forceinline__ bool active(value_t new_value, value_t old_value)
{
    return new_value != old_value;
}
#endif
