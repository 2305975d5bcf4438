// scaph_bfs_page_noalloc: single-source BFS over one paged-CSR page that the
// caller already holds in device memory, without allocating anything.
//
// Who needs this: callers that cannot let a library call cudaMalloc.  One
// example is a host process that reserves the GPU's memory up front in its
// own pool and accounts for every byte; an allocation made behind its back
// can fail, or push the pool out of memory.  Another is a latency-critical
// serving path, where cudaMalloc/cudaFree can synchronise the device and
// stall other work.  Such a caller passes its input page and output arrays;
// all other state of the traversal (bitmaps, a degree copy, the level
// counters, the giant-chunk queue and a one-page page table) lives in the
// fixed file-scope array g_noalloc_scratch below.
//
// Limits and rules:
//  * at most SCAPH_NOALLOC_MAX_V vertices and SCAPH_NOALLOC_MAX_E edges;
//    larger graphs are rejected with SCAPH_EINVAL before any GPU work;
//  * the scratch array is about 1.3 MB and is held by every GPU that loads
//    the library, until the process exits;
//  * every call shares that one array and leaves its contents behind; each
//    call clears what must start at zero, but calls whose GPU work overlaps
//    (on different streams, or from different host threads) race on it and
//    give wrong results: serialise them;
//  * pull levels read the same page as in-edges, which is right only when
//    every edge has its reverse: the caller says so with
//    SCAPH_NOALLOC_SYMMETRIC, otherwise every level pushes;
//  * every call looks up the device address of the array with
//    cudaGetSymbolAddress (current device), so nothing is cached across a
//    device reset; the call synchronises its stream once per level.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "engine.h"
#include "kernels.h"

using namespace scaph;

namespace {

constexpr uint32_t kMaxV = SCAPH_NOALLOC_MAX_V;
constexpr uint32_t kMaxE = SCAPH_NOALLOC_MAX_E;
constexpr uint32_t kWords = kMaxV / 32;
constexpr uint32_t kGiantCap = 2 * (kMaxE / kGiantEdges) + 1024;
constexpr uint32_t kCshift = 18;  // kMaxV = 1 << 18: every vertex maps to coarse[0]
static_assert((1u << kCshift) >= kMaxV, "coarse shift must cover kMaxV");

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
// byte offsets of the regions inside the scratch array
constexpr size_t kOffDegree = 0;
constexpr size_t kOffVisited = align256(kOffDegree + 4ull * kMaxV);
constexpr size_t kOffFront0 = align256(kOffVisited + 4ull * kWords);
constexpr size_t kOffFront1 = align256(kOffFront0 + 4ull * kWords);
constexpr size_t kOffCtr = align256(kOffFront1 + 4ull * kWords);
constexpr size_t kOffGiant = align256(kOffCtr + sizeof(LevelCounters));
constexpr size_t kOffPages = align256(kOffGiant + sizeof(GiantChunk) * kGiantCap);
constexpr size_t kOffCoarse = align256(kOffPages + 2 * sizeof(PageDev));
constexpr size_t kScratchBytes = align256(kOffCoarse + 2 * sizeof(uint32_t));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Page table of the one-page graph, the coarse index, the degree copy
// (Node.len), and a check that every Node stays inside the page: a bad
// record sets ctr->error and the traversal is not started.
__global__ void k_noalloc_setup(unsigned char *scratch, const uint32_t *page, uint32_t nodenum,
                                uint32_t edgenum)
{
    uint32_t *degree = reinterpret_cast<uint32_t *>(scratch + kOffDegree);
    LevelCounters *ctr = reinterpret_cast<LevelCounters *>(scratch + kOffCtr);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nodenum; v += stride) {
        const uint32_t vtx = page[3ull * v], pos = page[3ull * v + 1], len = page[3ull * v + 2];
        if (vtx != v || (unsigned long long)pos + len > edgenum) atomicOr(&ctr->error, 16u);
        degree[v] = len;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        PageDev *pages = reinterpret_cast<PageDev *>(scratch + kOffPages);
        uint32_t *coarse = reinterpret_cast<uint32_t *>(scratch + kOffCoarse);
        pages[0].base = 0;
        pages[0].left = 0;
        pages[0].nodenum = nodenum;
        pages[1].base = 0;
        pages[1].left = nodenum;
        pages[1].nodenum = 0;
        coarse[0] = 0;
        coarse[1] = 0;
    }
}

// Device address of g_noalloc_scratch on the current device.  Looked up on
// every call: the lookup is cheap next to the per-level synchronisation, and
// an address cached across a cudaDeviceReset would be stale.
int scratch_address(unsigned char **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return set_error(SCAPH_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
    *out = static_cast<unsigned char *>(p);
    return SCAPH_OK;
}

}  // namespace

extern "C" int scaph_bfs_page_noalloc(const uint32_t *d_page, uint32_t nodenum, uint32_t edgenum, uint32_t src,
                                      uint32_t unreached, int flags, uint32_t *d_depth, uint32_t *d_parent,
                                      scaph_bfs_stats *stats, void *stream)
{
    clear_error();
    if (!d_page || !d_depth) return set_error(SCAPH_EINVAL, "null page or depth pointer");
    if (reinterpret_cast<uintptr_t>(d_page) & 15) return set_error(SCAPH_EINVAL, "page must be 16-byte aligned");
    if (nodenum == 0 || nodenum > kMaxV)
        return set_error(SCAPH_EINVAL, "nodenum %u outside 1..%u (SCAPH_NOALLOC_MAX_V)", nodenum, kMaxV);
    if (edgenum > kMaxE) return set_error(SCAPH_EINVAL, "edgenum %u above %u (SCAPH_NOALLOC_MAX_E)", edgenum, kMaxE);
    if (src >= nodenum) return set_error(SCAPH_EINVAL, "source %u out of range (V=%u)", src, nodenum);
    if (flags & ~SCAPH_NOALLOC_SYMMETRIC) return set_error(SCAPH_EINVAL, "unknown flags 0x%x", flags);
    if (unreached == 0) unreached = 0xFFFFFFFFu;
    if (unreached < 2) return set_error(SCAPH_EINVAL, "unreached sentinel must be >= 2");
    const bool symmetric = (flags & SCAPH_NOALLOC_SYMMETRIC) != 0;
    unsigned char *scr = nullptr;
    int rc = scratch_address(&scr);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    SCAPH_CUDA(cudaGetDevice(&dev));
    SCAPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t V = nodenum, nwords = (V + 31) / 32;
    LevelCounters *ctr = reinterpret_cast<LevelCounters *>(scr + kOffCtr);
    uint32_t *visited = reinterpret_cast<uint32_t *>(scr + kOffVisited);
    uint32_t *bm[2] = {reinterpret_cast<uint32_t *>(scr + kOffFront0), reinterpret_cast<uint32_t *>(scr + kOffFront1)};

    // set-up and validation of the caller's page
    SCAPH_CUDA(cudaMemsetAsync(ctr, 0, sizeof(LevelCounters), st));
    k_noalloc_setup<<<sms * 2, 256, 0, st>>>(scr, d_page, nodenum, edgenum);
    SCAPH_CUDA(cudaGetLastError());
    LevelCounters lc;
    SCAPH_CUDA(cudaMemcpyAsync(&lc, ctr, sizeof(lc), cudaMemcpyDeviceToHost, st));
    SCAPH_CUDA(cudaStreamSynchronize(st));
    if (lc.error) return set_error(SCAPH_EFORMAT, "page records inconsistent with nodenum/edgenum");

    GraphDev g{};
    g.pool = d_page;
    g.pages = reinterpret_cast<const PageDev *>(scr + kOffPages);
    g.coarse = reinterpret_cast<const uint32_t *>(scr + kOffCoarse);
    g.zc_pool = nullptr;
    g.pool_words = ((3ull * nodenum + edgenum) + 3) & ~3ull;
    g.cshift = kCshift;
    g.npages = 1;
    g.V = V;
    g.pagesize = 0;

    BfsDev s{};
    s.depth = d_depth;
    s.parent = d_parent;
    s.visited = visited;
    s.degree = reinterpret_cast<const uint32_t *>(scr + kOffDegree);
    s.page_nodes = s.page_datas = nullptr;
    s.giant = reinterpret_cast<GiantChunk *>(scr + kOffGiant);
    s.giant_cap = kGiantCap;
    s.V = V;
    s.nwords = nwords;
    s.hg = g;

    const int grid_fill = sms * 4;
    SCAPH_CUDA(fill_u32(d_depth, unreached, V, grid_fill, st));
    if (d_parent) SCAPH_CUDA(fill_u32(d_parent, kNoParent, V, grid_fill, st));
    SCAPH_CUDA(cudaMemsetAsync(visited, 0, (size_t)nwords * 4, st));
    SCAPH_CUDA(cudaMemsetAsync(bm[0], 0, (size_t)nwords * 4, st));
    SCAPH_CUDA(set_source(s, src, bm[0], st));

    const int grid_push = std::max(1, level_occupancy(0, 256)) * sms;
    const int grid_pull = std::max(1, level_occupancy(1, 256)) * sms;
    // a one-page graph holding every vertex: its out-edge total is edgenum
    const uint64_t E = edgenum;
    uint32_t deg_src = 0;
    SCAPH_CUDA(cudaMemcpyAsync(&deg_src, s.degree + src, 4, cudaMemcpyDeviceToHost, st));
    SCAPH_CUDA(cudaStreamSynchronize(st));
    uint64_t nf = 1, prev_nf = 0, mf = deg_src, vis_n = 1, vis_e = deg_src, inspected = 0;
    int dir = 0, cur = 0, level = 0, npush = 0, npull = 0;
    // no level cap beyond the sentinel's: the level counters are one record
    // reused every level, and the loop ends once a level discovers nothing
    // (at most V levels)
    for (; nf > 0 && (uint64_t)level + 1 < unreached; level++) {
        if (level > 0 && symmetric) dir = alpha_beta_next(dir, nf, prev_nf, mf, E - vis_e, V, kAlphaDefault,
                                                                   kBetaDefault);
        SCAPH_CUDA(cudaMemsetAsync(ctr, 0, sizeof(LevelCounters), st));
        SCAPH_CUDA(cudaMemsetAsync(bm[cur ^ 1], 0, (size_t)nwords * 4, st));
        s.front = bm[cur];
        s.next = bm[cur ^ 1];
        s.ctr = ctr;
        s.level = (uint32_t)level;
        SCAPH_CUDA(run_level(dir, 256, dir == 0 ? grid_push : grid_pull, g, s, 0, V, st));
        SCAPH_CUDA(cudaMemcpyAsync(&lc, ctr, sizeof(lc), cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
        if (lc.error) return set_error(SCAPH_EDEVICE, "level kernel reported error flags 0x%x", lc.error);
        if (dir == 0) npush++; else npull++;
        inspected += lc.inspected;
        prev_nf = nf;
        nf = lc.next;
        mf = lc.next_edges;
        vis_n += nf;
        vis_e += mf;
        cur ^= 1;
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->levels = level;
        stats->push_levels = npush;
        stats->pull_levels = npull;
        stats->reached = vis_n;
        stats->reached_edges = vis_e;
        stats->edges_inspected = inspected;
        stats->launches = 3 + (d_parent ? 1 : 0) + (uint64_t)npush * 2 + npull;
    }
    return SCAPH_OK;
}
