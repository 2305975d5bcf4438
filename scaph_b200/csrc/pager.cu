// Out-of-core page manager: pages stream from pinned host memory into an HBM
// page pool while the traversal runs.  Replaces PageHandle / VPstat / DPstat
// (src/pagehandle.h:16-474), PageCopy (src/app.cuh:371-393), the CPU
// compaction of cold pages (compress_stat, src/compress.h:18-56) and the host
// queues of src/pipe.h.
//
//  * The host pages of a graph are one buffer registered with
//    cudaHostRegister (pinned + mapped), so a page can be copied with one DMA
//    or read in place by the GPU.
//  * The pool is one device allocation of nslots page slots shared by the
//    out-edge and in-edge graphs.  Each graph has a device page table
//    (PageDev[npages+1], base = slot offset or kNotResident) that the level
//    kernels read; the host mirror decides residency.
//  * For each level the needed pages are known before the level runs: push
//    needs the out-pages holding frontier vertices (the page histogram the
//    previous level's kernels produced, i.e. get_page_info,
//    src/gpu_engine.cuh:397-441), pull needs the in-pages holding unvisited
//    vertices (k_page_unvisited).  Resident pages run at once; pages whose
//    active data is at most compact_threshold/32 of a page are read
//    zero-copy over PCIe (the GPU reads only the active vertices' headers and
//    edges - the bytes the reference's compaction would have copied, without
//    the CPU memcpy); the rest are copied on side streams into free or
//    least-recently-used slots of pages the level does not need, and their
//    kernels start as their copies land.
//  * prefetch() starts copies for pages predicted for the next level (the
//    learned scheduler), overlapping them with the current level.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "engine.h"
#include "kernel_common.cuh"
#include "kernels.h"

namespace scaph {

namespace {

constexpr int kTableBatch = 256;

struct TableUpdate {
    int n;
    uint32_t page[kTableBatch];
    unsigned long long base[kTableBatch];
};

__global__ void k_table_update(PageDev *tab, TableUpdate u)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < u.n) tab[u.page[i]].base = u.base[i];
}

// Per page of graph g: the vertices whose bit is set in bits ^ flip and their
// words sum(deg*ew+3).  flip = 0: active vertices and their out-degrees, i.e.
// get_page_info (src/gpu_engine.cuh:397-441, ew = 2 for weighted pages);
// flip = ~0 over the visited bitmap: unvisited vertices (dead ones start
// visited) with their in-degrees, the pull-side counterpart.
//
// A warp takes a chunk of 32 bitmap words (1024 vertices): one coalesced
// load gives every lane a word; the words are then walked eight at a time,
// lane = vertex, with the eight degree loads issued together, and each lane
// keeps its own count and sum for the chunk's first page.  A chunk rarely
// crosses a page boundary; the vertices past it take the slow path (their
// page looked up, one shared atomic each).  One shared atomic per page per
// warp-chunk, one global atomic per page per CTA.  cnt/datas must be zeroed
// by the caller.
__global__ void k_page_counts(const uint32_t *bits, uint32_t flip, GraphDev g, const uint32_t *deg, uint32_t ew,
                              uint32_t *cnt, uint32_t *datas)
{
    __shared__ uint32_t sc[kHistCap], sd[kHistCap];
    const bool local = g.npages <= (uint32_t)kHistCap;
    if (local)
        for (uint32_t i = threadIdx.x; i < g.npages; i += blockDim.x) sc[i] = sd[i] = 0;
    __syncthreads();
    uint32_t *const pc = local ? sc : cnt;
    uint32_t *const pd = local ? sd : datas;
    const int lane = threadIdx.x & 31;
    const uint32_t nwords = (g.V + 31) / 32;
    const uint32_t nchunks = (nwords + 31) / 32;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t ch = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ch < nchunks; ch += nwarps) {
        const uint32_t w = ch * 32 + lane;
        const uint32_t mine = w < nwords ? (bits[w] ^ flip) & range_mask(w, 0, g.V) : 0u;
        if (!__any_sync(0xFFFFFFFFu, mine != 0)) continue;
        const uint32_t v0 = ch << 10;
        const int p0 = page_of(g, v0);
        const uint32_t lim = __ldg(&g.pages[p0 + 1].left);  // first vertex past page p0
        uint32_t c = 0, dsum = 0;
#pragma unroll 1
        for (int j0 = 0; j0 < 32; j0 += 8) {
            uint32_t m[8], d[8];
#pragma unroll
            for (int k = 0; k < 8; k++) m[k] = __shfl_sync(0xFFFFFFFFu, mine, j0 + k);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t v = v0 + ((uint32_t)(j0 + k) << 5) + lane;
                d[k] = ((m[k] >> lane) & 1u) ? __ldg(&deg[v]) : 0u;
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                if (!((m[k] >> lane) & 1u)) continue;
                const uint32_t v = v0 + ((uint32_t)(j0 + k) << 5) + lane;
                const uint32_t wd = d[k] * ew + 3;
                if (v < lim) {
                    c++;
                    dsum += wd;
                } else {
                    const int p = page_of(g, v);
                    atomicAdd(&pc[p], 1u);
                    atomicAdd(&pd[p], wd);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
            dsum += __shfl_xor_sync(0xFFFFFFFFu, dsum, o);
        }
        if (lane == 0 && c) {
            atomicAdd(&pc[p0], c);
            atomicAdd(&pd[p0], dsum);
        }
    }
    __syncthreads();
    if (local)
        for (uint32_t i = threadIdx.x; i < g.npages; i += blockDim.x) {
            if (sc[i]) {
                atomicAdd(&cnt[i], sc[i]);
                atomicAdd(&datas[i], sd[i]);
            }
        }
}

}  // namespace

int coarse_index(const Graph &g, std::vector<uint32_t> &hc, uint32_t &cshift)
{
    const int np = (int)g.pages.size();
    uint32_t minpage = g.V;
    for (int p = 0; p + 1 < np; p++) minpage = std::min(minpage, g.pages[p].nodenum);
    cshift = 0;
    while (cshift < 24 && (2u << cshift) <= minpage) cshift++;
    const size_t ncoarse = ((size_t)g.V >> cshift) + 1;
    hc.assign(ncoarse, 0);
    int p = 0;
    for (size_t i = 0; i < ncoarse; i++) {
        uint64_t v = (uint64_t)i << cshift;
        while (p + 1 < np && g.pages[p + 1].left <= v) p++;
        hc[i] = (uint32_t)p;
    }
    return SCAPH_OK;
}

struct Pager {
    struct Slot {
        int g = -1, p = -1;
        uint64_t used = 0;
        cudaEvent_t ready = nullptr;     // copy into the slot finished
        cudaEvent_t last_use = nullptr;  // last kernel that read the slot finished
        bool published = false;          // page table entry points here
    };
    struct GState {
        const Graph *host = nullptr;
        std::vector<int> slot_of;
        std::vector<int> protect;  // level stamp: page needed by the level being run
        PageDev *d_tab = nullptr, *d_zc_tab = nullptr;
        uint32_t *d_coarse = nullptr;
        uint32_t *host_dev = nullptr;  // device address of the mapped host pages
        bool registered = false;
        GraphDev view{}, zc{};
        uint32_t *d_cnt = nullptr, *d_datas = nullptr, *h_cnt = nullptr, *h_datas = nullptr;
    };

    uint32_t *pool = nullptr;
    int nslots = 0;
    size_t slot_words = 0;
    std::vector<Slot> slots;
    GState gs[2];
    int ngraphs = 1;
    cudaStream_t cst[4] = {};
    int ncst = 2, next_cst = 0;
    uint32_t *h_rl = nullptr, *d_rl = nullptr;  // range-list staging (pinned, device)
    size_t rl_words = 0, rl_head = 0;
    uint64_t clock = 0;
    int stamp = 0;
    uint32_t pagesize = 0;
    // counters of the current run
    uint64_t h2d_bytes = 0, zc_bytes = 0, faults = 0, prefetched = 0, prefetch_hits = 0;
    uint64_t level_h2d = 0;
    double h2d_gbs = 50.0;  // measured at init

    ~Pager();
    int init(const Graph *g, const Graph *gt, int nslots_, int copy_streams, float link_gbs);
    int setup_graph(int gid, const Graph &g);
    int acquire_slot(int gid, bool for_prefetch);
    int load(int gid, int p, bool prefetch);
    int publish(int gid, const std::vector<int> &pages, cudaStream_t st);
    int launch(int gid, bool zc, const std::vector<int> &pages, const PageLaunch &fn, cudaStream_t st);
    int run_level(int gid, const std::vector<int> &needed, const std::vector<uint32_t> &datas,
                  int compact_threshold, const PageLaunch &fn, cudaStream_t st);
    int prefetch(int gid, const std::vector<int> &pages);
    void evict_all();
};

Pager::~Pager()
{
    for (auto &s : slots) {
        if (s.ready) cudaEventDestroy(s.ready);
        if (s.last_use) cudaEventDestroy(s.last_use);
    }
    for (int i = 0; i < 4; i++)
        if (cst[i]) cudaStreamDestroy(cst[i]);
    for (auto &g : gs) {
        cudaFree(g.d_tab);
        cudaFree(g.d_zc_tab);
        cudaFree(g.d_coarse);
        cudaFree(g.d_cnt);
        cudaFree(g.d_datas);
        cudaFreeHost(g.h_cnt);
        cudaFreeHost(g.h_datas);
    }
    cudaFree(pool);
    cudaFreeHost(h_rl);
    cudaFree(d_rl);
}

void pager_release(Pager *p) { delete p; }

int Pager::setup_graph(int gid, const Graph &g)
{
    GState &G = gs[gid];
    G.host = &g;
    const int np = (int)g.pages.size();
    G.slot_of.assign(np, -1);
    G.protect.assign(np, -1);
    if (!g.pinned) {
        SCAPH_CUDA((cudaError_t)injected_fault(kFaultHostRegister));
        SCAPH_CUDA(cudaHostRegister(g.data, g.data_words * 4, cudaHostRegisterMapped | cudaHostRegisterPortable));
        const_cast<Graph &>(g).pinned = true;  // unregistered by ~Graph
    }
    SCAPH_CUDA(cudaHostGetDevicePointer((void **)&G.host_dev, g.data, 0));
    std::vector<PageDev> tab(np + 1), zt(np + 1);
    for (int p = 0; p < np; p++) {
        tab[p] = PageDev{kNotResident, g.pages[p].left, g.pages[p].nodenum};
        zt[p] = PageDev{(unsigned long long)p * g.pagesize, g.pages[p].left, g.pages[p].nodenum};
    }
    tab[np] = zt[np] = PageDev{0, g.V, 0};
    SCAPH_CUDA(cudaMalloc(&G.d_tab, sizeof(PageDev) * (np + 1)));
    SCAPH_CUDA(cudaMalloc(&G.d_zc_tab, sizeof(PageDev) * (np + 1)));
    SCAPH_CUDA(cudaMemcpy(G.d_tab, tab.data(), sizeof(PageDev) * (np + 1), cudaMemcpyHostToDevice));
    SCAPH_CUDA(cudaMemcpy(G.d_zc_tab, zt.data(), sizeof(PageDev) * (np + 1), cudaMemcpyHostToDevice));
    std::vector<uint32_t> hc;
    uint32_t cshift = 0;
    coarse_index(g, hc, cshift);
    SCAPH_CUDA(cudaMalloc(&G.d_coarse, hc.size() * 4));
    SCAPH_CUDA(cudaMemcpy(G.d_coarse, hc.data(), hc.size() * 4, cudaMemcpyHostToDevice));
    SCAPH_CUDA(cudaMalloc(&G.d_cnt, np * 4));
    SCAPH_CUDA(cudaMalloc(&G.d_datas, np * 4));
    SCAPH_CUDA(cudaMallocHost(&G.h_cnt, np * 4));
    SCAPH_CUDA(cudaMallocHost(&G.h_datas, np * 4));
    GraphDev v{};
    v.pool = pool;
    v.pages = G.d_tab;
    v.coarse = G.d_coarse;
    v.zc_pool = G.host_dev;
    v.pool_words = (unsigned long long)nslots * slot_words;
    v.cshift = cshift;
    v.npages = (uint32_t)np;
    v.V = g.V;
    v.pagesize = g.pagesize;
    G.view = v;
    G.zc = v;
    G.zc.pool = G.host_dev;
    G.zc.pages = G.d_zc_tab;
    G.zc.pool_words = g.data_words;
    return SCAPH_OK;
}

int Pager::init(const Graph *g, const Graph *gt, int nslots_, int copy_streams, float link_gbs)
{
    nslots = nslots_;
    pagesize = g->pagesize;
    slot_words = pagesize;
    if (gt && gt->pagesize != pagesize) return set_error(SCAPH_EINVAL, "out/in graphs need the same page size");
    SCAPH_CUDA(cudaMalloc(&pool, (size_t)nslots * slot_words * 4));
    slots.resize(nslots);
    for (auto &s : slots) {
        SCAPH_CUDA(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
        SCAPH_CUDA(cudaEventCreateWithFlags(&s.last_use, cudaEventDisableTiming));
    }
    ncst = std::max(1, std::min(4, copy_streams));
    for (int i = 0; i < ncst; i++) SCAPH_CUDA(cudaStreamCreateWithFlags(&cst[i], cudaStreamNonBlocking));
    ngraphs = gt ? 2 : 1;
    int rc = setup_graph(0, *g);
    if (rc) return rc;
    if (gt && (rc = setup_graph(1, *gt))) return rc;
    if (link_gbs > 0) {
        h2d_gbs = link_gbs;
    } else {
        // PCIe host->device bandwidth of one pinned page copy
        cudaEvent_t a, b;
        SCAPH_CUDA(cudaEventCreate(&a));
        SCAPH_CUDA(cudaEventCreate(&b));
        const size_t bytes = slot_words * 4;
        SCAPH_CUDA(cudaMemcpyAsync(pool, g->page(0), bytes, cudaMemcpyHostToDevice, cst[0]));
        SCAPH_CUDA(cudaEventRecord(a, cst[0]));
        SCAPH_CUDA(cudaMemcpyAsync(pool, g->page(0), bytes, cudaMemcpyHostToDevice, cst[0]));
        SCAPH_CUDA(cudaEventRecord(b, cst[0]));
        SCAPH_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms > 0) h2d_gbs = bytes / (ms * 1e-3) / 1e9;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    size_t maxp = g->pages.size() + (gt ? gt->pages.size() : 0);
    rl_words = 64 * (3 * maxp + 8);
    SCAPH_CUDA(cudaMallocHost(&h_rl, rl_words * 4));
    SCAPH_CUDA(cudaMalloc(&d_rl, rl_words * 4));
    return SCAPH_OK;
}

void Pager::evict_all()
{
    for (auto &s : slots) {
        if (s.g >= 0) gs[s.g].slot_of[s.p] = -1;
        s.g = s.p = -1;
        s.published = false;
    }
}

// Free slot, else the least recently used slot whose page the running level
// does not need.  -1 when every slot holds a page of the running level.
int Pager::acquire_slot(int gid, bool for_prefetch)
{
    (void)gid;
    int best = -1;
    for (int i = 0; i < nslots; i++) {
        const Slot &s = slots[i];
        if (s.g < 0) return i;
        if (gs[s.g].protect[s.p] == stamp) continue;
        if (for_prefetch) continue;  // prefetches take free slots only
        if (best < 0 || s.used < slots[best].used) best = i;
    }
    return best;
}

// Copies page p of graph gid into a slot; returns the slot, -1 when no slot
// can be had, -2 (error recorded) when the copy could not be issued.
int Pager::load(int gid, int p, bool prefetch_only)
{
    GState &G = gs[gid];
    const int si = acquire_slot(gid, prefetch_only);
    if (si < 0) return -1;
    Slot &s = slots[si];
    // the copy may not overwrite the slot before the kernels that read its
    // previous page are done (a never-recorded event is already complete)
    cudaStream_t cs = cst[next_cst];
    next_cst = (next_cst + 1) % ncst;
    cudaError_t e = cudaStreamWaitEvent(cs, s.last_use, 0);
    if (e == cudaSuccess) e = (cudaError_t)injected_fault(kFaultPageCopy);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(pool + (size_t)si * slot_words, G.host->page(p), slot_words * 4, cudaMemcpyHostToDevice,
                            cs);
    if (e == cudaSuccess) e = cudaEventRecord(s.ready, cs);
    if (e != cudaSuccess) {
        set_error(SCAPH_ECUDA, "page %d of graph %d: copy not issued: %s", p, gid, cudaGetErrorString(e));
        return -2;  // the slot keeps its previous page
    }
    if (s.g >= 0) gs[s.g].slot_of[s.p] = -1;
    s.g = gid;
    s.p = p;
    s.used = clock;
    s.published = false;
    G.slot_of[p] = si;
    h2d_bytes += slot_words * 4;
    level_h2d += slot_words * 4;
    return si;
}

// Makes the device page table of graph gid point at the slots of `pages`
// (after their copies) and marks every page of gid that lost its slot.
int Pager::publish(int gid, const std::vector<int> &pages, cudaStream_t st)
{
    GState &G = gs[gid];
    TableUpdate u;
    u.n = 0;
    auto flush = [&]() -> int {
        if (!u.n) return SCAPH_OK;
        k_table_update<<<(u.n + 127) / 128, 128, 0, st>>>(G.d_tab, u);
        SCAPH_CUDA(cudaGetLastError());
        u.n = 0;
        return SCAPH_OK;
    };
    for (int p : pages) {
        const int si = G.slot_of[p];
        if (si < 0 || slots[si].published) continue;
        SCAPH_CUDA(cudaStreamWaitEvent(st, slots[si].ready, 0));
        u.page[u.n] = (uint32_t)p;
        u.base[u.n] = (unsigned long long)si * slot_words;
        u.n++;
        slots[si].published = true;
        if (u.n == kTableBatch) {
            int rc = flush();
            if (rc) return rc;
        }
    }
    return flush();
}

int Pager::launch(int gid, bool zc, const std::vector<int> &pages, const PageLaunch &fn, cudaStream_t st)
{
    if (pages.empty()) return SCAPH_OK;
    GState &G = gs[gid];
    // ranges: consecutive pages merge into one range
    std::vector<uint32_t> lo, hi;
    std::vector<int> sorted = pages;
    std::sort(sorted.begin(), sorted.end());
    for (size_t i = 0; i < sorted.size(); i++) {
        const scaph_page_info &pi = G.host->pages[sorted[i]];
        if (!lo.empty() && hi.back() == pi.left) hi.back() = pi.right + 1;
        else {
            lo.push_back(pi.left);
            hi.push_back(pi.right + 1);
        }
    }
    const uint32_t n = (uint32_t)lo.size();
    if (rl_head + 3 * n + 1 > rl_words) rl_head = 0;  // ring: the host loop syncs every level
    uint32_t *h = h_rl + rl_head;
    uint32_t t = 0;
    for (uint32_t i = 0; i < n; i++) {
        h[i] = lo[i];
        h[n + i] = hi[i];
        h[2 * n + i] = t;
        t += ((hi[i] + 31) / 32 - lo[i] / 32 + 127) / 128;
    }
    h[3 * n] = t;
    uint32_t *d = d_rl + rl_head;
    SCAPH_CUDA(cudaMemcpyAsync(d, h, (3 * n + 1) * 4, cudaMemcpyHostToDevice, st));
    rl_head += 3 * n + 1;
    RangeList rl{d, d + n, d + 2 * n, n};
    int rc = fn.run(zc ? G.zc : G.view, gid, rl, t, st);
    if (rc) return rc;
    if (!zc) {
        for (int p : pages) {
            const int si = G.slot_of[p];
            if (si < 0) continue;
            slots[si].used = clock;
            SCAPH_CUDA(cudaEventRecord(slots[si].last_use, st));
        }
    }
    return SCAPH_OK;
}

int Pager::run_level(int gid, const std::vector<int> &needed, const std::vector<uint32_t> &datas,
                     int compact_threshold, const PageLaunch &fn, cudaStream_t st)
{
    GState &G = gs[gid];
    clock++;
    stamp++;
    level_h2d = 0;
    const uint64_t thresh = (uint64_t)compact_threshold * (pagesize / 32);
    std::vector<int> resident, zcp, fetch;
    for (int p : needed) G.protect[p] = stamp;
    for (int p : needed) {
        if (G.slot_of[p] >= 0) {
            resident.push_back(p);
            if (!slots[G.slot_of[p]].published) prefetch_hits++;
        } else if (datas[p] <= thresh) {
            zcp.push_back(p);
        } else {
            fetch.push_back(p);
        }
    }
    int rc = publish(gid, resident, st);
    if (rc) return rc;
    if ((rc = launch(gid, false, resident, fn, st))) return rc;
    if ((rc = launch(gid, true, zcp, fn, st))) return rc;
    for (int p : zcp) zc_bytes += (uint64_t)datas[p] * 4;
    // demand fetches, in batches that start as soon as their copies land
    std::vector<int> done_pages = resident;
    size_t i = 0;
    const size_t batch = std::max<size_t>(1, std::min<size_t>(8, (size_t)nslots / 4 + 1));
    while (i < fetch.size()) {
        std::vector<int> b;
        while (b.size() < batch && i < fetch.size()) {
            const int si = load(gid, fetch[i], false);
            if (si == -2) return SCAPH_ECUDA;
            if (si < 0) break;
            b.push_back(fetch[i]);
            faults++;
            i++;
        }
        if (b.empty()) {
            // every slot holds a page of this level: the pages already
            // processed may now be evicted
            if (done_pages.empty()) return set_error(SCAPH_EUNSUPPORTED, "page pool too small for one page");
            for (int p : done_pages) G.protect[p] = -1;
            done_pages.clear();
            continue;
        }
        if ((rc = publish(gid, b, st))) return rc;
        if ((rc = launch(gid, false, b, fn, st))) return rc;
        done_pages.insert(done_pages.end(), b.begin(), b.end());
    }
    return SCAPH_OK;
}

int Pager::prefetch(int gid, const std::vector<int> &pages)
{
    GState &G = gs[gid];
    for (int p : pages) {
        if (p < 0 || p >= (int)G.slot_of.size() || G.slot_of[p] >= 0) continue;
        const int si = load(gid, p, true);
        if (si == -2) return SCAPH_ECUDA;
        if (si < 0) break;
        prefetched++;
    }
    return SCAPH_OK;
}

// ---------------------------------------------------------------------------
// engine glue
// ---------------------------------------------------------------------------
int pager_create(const Graph *g, const Graph *gt, int nslots, int copy_streams, float link_gbs, Pager **out)
{
    Pager *p = new Pager();
    int rc = p->init(g, gt, nslots, copy_streams > 0 ? copy_streams : 2, link_gbs);
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return SCAPH_OK;
}

const GraphDev &pager_view(const Pager *p, int gid) { return p->gs[gid].view; }

// Pages the coming level needs, with their active words.
int pager_needs(scaph_engine *e, Pager *pg, int dir, int level, uint32_t src, std::vector<int> &needed,
                std::vector<uint32_t> &datas)
{
    needed.clear();
    const int gid = (dir == 0 || pg->ngraphs == 1) ? 0 : 1;
    Pager::GState &G = pg->gs[gid];
    const int np = (int)G.host->pages.size();
    datas.assign(np, 0);
    if (dir == 0) {
        if (level == 0) {
            int p = 0;
            while (p + 1 < np && G.host->pages[p + 1].left <= src) p++;
            needed.push_back(p);
            datas[p] = e->g->degree[src] + 3;
            return SCAPH_OK;
        }
        // frontier of this level = vertices discovered by the previous one
        const uint32_t *h = e->d_hist + (size_t)(level - 1) * 2 * np;
        SCAPH_CUDA(cudaMemcpyAsync(G.h_cnt, h, np * 4, cudaMemcpyDeviceToHost, e->st));
        SCAPH_CUDA(cudaMemcpyAsync(G.h_datas, h + np, np * 4, cudaMemcpyDeviceToHost, e->st));
    } else {
        SCAPH_CUDA(page_unvisited(G.view, e->d_visited, e->d_indeg, G.d_cnt, G.d_datas, e->num_sms * 8, e->st));
        SCAPH_CUDA(cudaMemcpyAsync(G.h_cnt, G.d_cnt, np * 4, cudaMemcpyDeviceToHost, e->st));
        SCAPH_CUDA(cudaMemcpyAsync(G.h_datas, G.d_datas, np * 4, cudaMemcpyDeviceToHost, e->st));
    }
    SCAPH_CUDA(cudaStreamSynchronize(e->st));
    for (int p = 0; p < np; p++) {
        if (G.h_cnt[p]) {
            needed.push_back(p);
            datas[p] = G.h_datas[p];
        }
    }
    return SCAPH_OK;
}

int pager_run_level(scaph_engine *e, Pager *pg, int dir, const BfsDev &s, const std::vector<int> &needed,
                    const std::vector<uint32_t> &datas)
{
    const int gid = (dir == 0 || pg->ngraphs == 1) ? 0 : 1;
    PageLaunch fn;
    fn.run = [&](const GraphDev &gv, int, const RangeList &rl, uint32_t, cudaStream_t st) -> int {
        const int grid = dir == 0 ? e->grid_push : e->grid_pull;
        SCAPH_CUDA(run_ranges(dir, e->block, grid, gv, s, rl, st));
        if (dir == 0) {
            // the giant chunks reference this view's pool: run them now,
            // then reset the chunk count for the next batch
            SCAPH_CUDA(run_giant(e->block, grid, gv, s, st));
            SCAPH_CUDA(cudaMemsetAsync(&s.ctr->giant, 0, sizeof(unsigned int), st));
        }
        return SCAPH_OK;
    };
    return pg->run_level(gid, needed, datas, e->cfg.compact_threshold, fn, e->st);
}

int pager_run_level(Pager *pg, int gid, const std::vector<int> &needed, const std::vector<uint32_t> &datas,
                    int compact_threshold, const PageLaunch &fn, cudaStream_t st)
{
    return pg->run_level(gid, needed, datas, compact_threshold, fn, st);
}

int pager_prefetch(scaph_engine *, Pager *pg, int gid, const std::vector<int> &pages)
{
    return pg->prefetch(gid, pages);
}

int pager_page_counts(Pager *pg, int gid, const uint32_t *bits, bool invert, const uint32_t *deg, uint32_t ew,
                      int grid, cudaStream_t st, std::vector<int> &needed, std::vector<uint32_t> &datas,
                      std::vector<uint32_t> *counts)
{
    Pager::GState &G = pg->gs[gid];
    const int np = (int)G.host->pages.size();
    SCAPH_CUDA(page_counts(G.view, bits, invert, deg, ew, G.d_cnt, G.d_datas, grid, st));
    SCAPH_CUDA(cudaMemcpyAsync(G.h_cnt, G.d_cnt, np * 4, cudaMemcpyDeviceToHost, st));
    SCAPH_CUDA(cudaMemcpyAsync(G.h_datas, G.d_datas, np * 4, cudaMemcpyDeviceToHost, st));
    SCAPH_CUDA(cudaStreamSynchronize(st));
    needed.clear();
    datas.assign(np, 0);
    for (int p = 0; p < np; p++)
        if (G.h_cnt[p]) {
            needed.push_back(p);
            datas[p] = G.h_datas[p];
        }
    if (counts) counts->assign(G.h_cnt, G.h_cnt + np);
    return SCAPH_OK;
}

void pager_counters(const Pager *pg, uint64_t *h2d, uint64_t *zc, uint64_t *faults, uint64_t *prefetched,
                    uint64_t *hits, uint64_t *level_h2d)
{
    *h2d = pg->h2d_bytes;
    *zc = pg->zc_bytes;
    *faults = pg->faults;
    *prefetched = pg->prefetched;
    *hits = pg->prefetch_hits;
    *level_h2d = pg->level_h2d;
}

void pager_reset_counters(Pager *pg)
{
    pg->h2d_bytes = pg->zc_bytes = pg->faults = pg->prefetched = pg->prefetch_hits = 0;
}

void pager_evict_all(Pager *pg) { pg->evict_all(); }

int pager_nslots(const Pager *pg) { return pg->nslots; }

int pager_free_slots(const Pager *pg)
{
    int n = 0;
    for (const auto &s : pg->slots) n += s.g < 0;
    return n;
}

bool pager_is_resident(const Pager *pg, int gid, int p) { return pg->gs[gid].slot_of[p] >= 0; }

float pager_resident_fraction(const Pager *pg, int gid, const std::vector<int> *pages)
{
    const Pager::GState &G = pg->gs[gid];
    if (pages) {
        if (pages->empty()) return 1.f;
        int r = 0;
        for (int p : *pages) r += G.slot_of[p] >= 0 ? 1 : 0;
        return (float)r / (float)pages->size();
    }
    int r = 0;
    for (int s : G.slot_of) r += s >= 0 ? 1 : 0;
    return G.slot_of.empty() ? 1.f : (float)r / (float)G.slot_of.size();
}

uint64_t pager_missing_words(const Pager *pg, int gid, const std::vector<int> &needed,
                             const std::vector<uint32_t> &datas)
{
    // a page prefetched for this level and not yet used by any level counts
    // as missing: the link still had to carry it for this level
    const Pager::GState &G = pg->gs[gid];
    uint64_t w = 0;
    for (int p : needed)
        if (G.slot_of[p] < 0 || !pg->slots[G.slot_of[p]].published) w += datas[p];
    return w;
}

double pager_transfer_ms(const Pager *pg, int gid, const uint32_t *cnt, const uint32_t *datas, int npages,
                         int compact_threshold)
{
    const Pager::GState &G = pg->gs[gid];
    const uint64_t thresh = (uint64_t)compact_threshold * (pg->pagesize / 32);
    double bytes = 0;
    for (int p = 0; p < npages && p < (int)G.slot_of.size(); p++) {
        if (!cnt[p] || G.slot_of[p] >= 0) continue;
        bytes += datas[p] <= thresh ? 4.0 * datas[p] : 4.0 * pg->slot_words;
    }
    return bytes / (pg->h2d_gbs * 1e9) * 1e3;
}

cudaError_t page_counts(const GraphDev &g, const uint32_t *bits, bool invert, const uint32_t *deg, uint32_t ew,
                        uint32_t *cnt, uint32_t *datas, int grid, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * g.npages, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(datas, 0, sizeof(uint32_t) * g.npages, st);
    if (e != cudaSuccess) return e;
    k_page_counts<<<grid, 256, 0, st>>>(bits, invert ? ~0u : 0u, g, deg, ew, cnt, datas);
    return cudaGetLastError();
}

cudaError_t page_unvisited(const GraphDev &g, const uint32_t *visited, const uint32_t *indeg, uint32_t *cnt,
                           uint32_t *datas, int grid, cudaStream_t st)
{
    return page_counts(g, visited, true, indeg, 1, cnt, datas, grid, st);
}

}  // namespace scaph
