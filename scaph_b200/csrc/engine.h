// Engine internals shared by engine.cu and the other device-side modules.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.h"
#include "device.cuh"

namespace scaph {

#define SCAPH_CUDA(call)                                                                      \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            return set_error(SCAPH_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                             cudaGetErrorString(_e));                                         \
    } while (0)

// One paged graph on the device: page pool, page table and coarse index.
struct DeviceGraph {
    uint32_t *pool = nullptr;        // nslots * pagesize words
    PageDev *pages = nullptr;        // npages + 1
    uint32_t *coarse = nullptr;
    std::vector<PageDev> h_pages;    // host mirror of the page table
    std::vector<int> slot_page;      // page held by each pool slot (-1 = free)
    int nslots = 0;
    GraphDev view{};
    const Graph *host = nullptr;

    int build(const Graph &g, int nslots_cap, cudaStream_t st);
    void release();
};

}  // namespace scaph
