// Device-side layout of the paged graph and of the BFS state, shared by the
// level kernels (bfs_kernels.cu) and the engine (engine.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace scaph {

constexpr unsigned long long kNotResident = ~0ull;
constexpr uint32_t kNoParent = 0xFFFFFFFFu;
constexpr int kHistCap = 1024;          // pages histogrammed in shared memory
constexpr uint32_t kGiantEdges = 4096;  // push: adjacency longer than this is split
constexpr int kMaxLevels = 4096;        // hard cap on BFS levels per run

// One page of the device page table.  `base` is the word offset of the page's
// Node array inside the page pool (kNotResident when the page is on the host);
// edges start at base + 3*nodenum (page layout of tools/pagegencsr.cpp:221-242).
struct __align__(16) PageDev {
    unsigned long long base;
    uint32_t left;
    uint32_t nodenum;
};

// Device view of one paged graph (out-edges, or in-edges for pull).
struct GraphDev {
    const uint32_t *pool;      // page pool, 16-byte aligned, slots of pagesize words
    const PageDev *pages;      // npages + 1 entries; pages[npages].left == V
    const uint32_t *coarse;    // coarse[i] = page holding vertex i << cshift
    const uint32_t *zc_pool;   // host pages mapped for zero-copy reads (or null)
    unsigned long long pool_words;  // words addressable through `pool`
    uint32_t cshift;
    uint32_t npages;
    uint32_t V;
    uint32_t pagesize;
};

// Counters of one level, written by that level's kernels.
struct LevelCounters {
    unsigned long long next;        // vertices discovered
    unsigned long long next_edges;  // their out-degree sum
    unsigned long long inspected;   // adjacency entries examined (first-hit for pull)
    unsigned long long headers;     // Node records read
    unsigned int giant;             // giant chunks queued (push)
    unsigned int error;             // nonzero: a kernel saw a bad index / overflow
    unsigned long long zc_words;    // words read zero-copy from host pages
};

struct GiantChunk {
    unsigned long long start;  // first edge word (pool offset)
    uint32_t len;
    uint32_t src;
};

struct BfsDev {
    uint32_t *depth;
    uint32_t *parent;          // may be null
    uint32_t *visited;         // bitmap, V bits
    const uint32_t *front;     // frontier bitmap of this level
    uint32_t *next;            // frontier bitmap of the next level (pre-cleared)
    const uint32_t *degree;    // out-degree per vertex
    LevelCounters *ctr;        // counters of this level
    uint32_t *page_nodes;      // histogram of the next frontier by page (or null)
    uint32_t *page_datas;
    GiantChunk *giant;
    uint32_t giant_cap;
    uint32_t level;            // discovered vertices get depth level+1
    uint32_t V;
    uint32_t weighted_edges;   // 1: pages hold {ngr,wgh} pairs (stride 2)
    GraphDev hg;               // out-edge graph whose pages the histogram counts
};

__device__ __forceinline__ int page_of(const GraphDev &g, uint32_t v)
{
    int p = (int)__ldg(&g.coarse[v >> g.cshift]);
    while (__ldg(&g.pages[p + 1].left) <= v) ++p;
    return p;
}

__device__ __forceinline__ uint4 ld_nc_v4(const uint32_t *p)
{
    return __ldg(reinterpret_cast<const uint4 *>(p));
}

__device__ __forceinline__ uint32_t test_bit(const uint32_t *bm, uint32_t v)
{
    return (__ldg(&bm[v >> 5]) >> (v & 31)) & 1u;
}

// Mask of the vertices of word w that lie in [vlo, vhi).
__device__ __forceinline__ uint32_t range_mask(uint32_t w, uint32_t vlo, uint32_t vhi)
{
    unsigned long long b0 = (unsigned long long)w << 5;
    unsigned long long lo = vlo > b0 ? vlo - b0 : 0;
    unsigned long long hi = vhi < b0 + 32 ? vhi - b0 : 32;
    if (hi <= lo) return 0u;
    uint32_t m = hi >= 32 ? 0xFFFFFFFFu : ((1u << hi) - 1u);
    return m & (0xFFFFFFFFu << lo);
}

}  // namespace scaph
