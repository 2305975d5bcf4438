// The BFS engine: device page pool + page table, per-vertex state, and the
// level loop with the direction switch.  Replaces App (src/app.cuh:72-345)
// for the BFS application: App::load_graph's allocations and pool fill
// (src/app.cuh:267-345), App::run's round loop (:220-265) and iter_init's
// per-round D2H of the whole stat array (:188-207).  Here the round loop is
// a level-synchronous BFS; the only per-level host traffic is one 48-byte
// counter record.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "engine.h"
#include "kernels.h"

using namespace scaph;

namespace scaph {

int DeviceGraph::build(const Graph &g, int nslots_cap, cudaStream_t st)
{
    host = &g;
    const int np = (int)g.pages.size();
    nslots = nslots_cap <= 0 ? np : std::min(np, nslots_cap);
    if (nslots < 1) return set_error(SCAPH_EINVAL, "page pool must hold at least one page");
    const size_t slot_words = g.pagesize;  // multiple of 4 (16-byte aligned slots)
    SCAPH_CUDA(cudaMalloc(&pool, (size_t)nslots * slot_words * 4));
    SCAPH_CUDA(cudaMalloc(&pages, sizeof(PageDev) * ((size_t)np + 1)));
    h_pages.assign((size_t)np + 1, PageDev{kNotResident, 0, 0});
    slot_page.assign(nslots, -1);
    for (int p = 0; p < np; p++) {
        h_pages[p].left = g.pages[p].left;
        h_pages[p].nodenum = g.pages[p].nodenum;
    }
    h_pages[np].left = g.V;
    h_pages[np].base = 0;
    // the first nslots pages are loaded now (the reference pre-loads the
    // first pool_size pages too, src/app.cuh:330-338)
    for (int s = 0; s < nslots; s++) {
        SCAPH_CUDA(cudaMemcpyAsync(pool + (size_t)s * slot_words, g.page(s), slot_words * 4,
                                   cudaMemcpyHostToDevice, st));
        h_pages[s].base = (unsigned long long)s * slot_words;
        slot_page[s] = s;
    }
    SCAPH_CUDA(cudaMemcpyAsync(pages, h_pages.data(), sizeof(PageDev) * h_pages.size(), cudaMemcpyHostToDevice, st));
    // coarse index: bucket size = largest power of two not above the
    // smallest page (last page excluded), so page_of steps at most twice.
    uint32_t minpage = g.V;
    for (int p = 0; p + 1 < np; p++) minpage = std::min(minpage, g.pages[p].nodenum);
    uint32_t cshift = 0;
    while (cshift < 24 && (2u << cshift) <= minpage) cshift++;
    const size_t ncoarse = ((size_t)g.V >> cshift) + 1;
    std::vector<uint32_t> hc(ncoarse);
    int p = 0;
    for (size_t i = 0; i < ncoarse; i++) {
        uint64_t v = (uint64_t)i << cshift;
        while (p + 1 < np && g.pages[p + 1].left <= v) p++;
        hc[i] = (uint32_t)p;
    }
    SCAPH_CUDA(cudaMalloc(&coarse, ncoarse * 4));
    SCAPH_CUDA(cudaMemcpyAsync(coarse, hc.data(), ncoarse * 4, cudaMemcpyHostToDevice, st));
    SCAPH_CUDA(cudaStreamSynchronize(st));
    view.pool = pool;
    view.pages = pages;
    view.coarse = coarse;
    view.zc_pool = nullptr;
    view.pool_words = (unsigned long long)nslots * slot_words;
    view.cshift = cshift;
    view.npages = (uint32_t)np;
    view.V = g.V;
    view.pagesize = g.pagesize;
    return SCAPH_OK;
}

void DeviceGraph::release()
{
    cudaFree(pool);
    cudaFree(pages);
    cudaFree(coarse);
    pool = nullptr;
    pages = nullptr;
    coarse = nullptr;
}

int alpha_beta_next(int cur_dir, uint64_t nf, uint64_t prev_nf, uint64_t mf, uint64_t mu, uint64_t V,
                    float alpha, float beta)
{
    if (cur_dir == 0) return (double)mf > (double)mu / alpha ? 1 : 0;
    return ((double)nf < (double)V / beta && nf < prev_nf) ? 0 : 1;
}

}  // namespace scaph

struct scaph_engine {
    scaph_config cfg{};
    int device = 0;
    int num_sms = 148;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    const Graph *g = nullptr;
    const Graph *gt = nullptr;
    DeviceGraph dout, din;
    bool symmetric = true;
    uint32_t V = 0, nwords = 0;
    uint64_t E = 0;
    uint32_t unreached = 0xFFFFFFFFu;
    int block = 256, grid_push = 0, grid_pull = 0;

    uint32_t *d_depth = nullptr, *d_parent = nullptr, *d_visited = nullptr, *d_bm[2] = {nullptr, nullptr};
    uint32_t *d_degree = nullptr;
    LevelCounters *d_ctr = nullptr, *h_ctr = nullptr;
    uint32_t *d_hist = nullptr;  // [kHistLevels][2][npages]
    GiantChunk *d_giant = nullptr;
    uint32_t giant_cap = 0;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    std::vector<cudaEvent_t> ev_level;

    std::vector<scaph_level_trace> trace;
    int last_levels = 0;

    static constexpr int kHistLevels = 256;

    const GraphDev &gin() const { return symmetric ? dout.view : din.view; }
    int create(const Graph *g_, const Graph *gt_, const scaph_config *c);
    void destroy();
    int bfs(uint32_t src, uint32_t *depths, uint32_t *parents, int out_on_device, scaph_bfs_stats *stats);
};

int scaph_engine::create(const Graph *g_, const Graph *gt_, const scaph_config *c)
{
    if (c) cfg = *c;
    g = g_;
    gt = gt_;
    symmetric = gt == nullptr;
    V = g->V;
    E = g->E;
    nwords = (V + 31) / 32;
    unreached = cfg.unreached ? cfg.unreached : 0xFFFFFFFFu;
    if (cfg.alpha <= 0) cfg.alpha = 14.0f;
    if (cfg.beta <= 0) cfg.beta = 24.0f;
    block = cfg.block_size == 128 || cfg.block_size == 512 ? cfg.block_size : 256;
    device = cfg.device;
    if (g->weighted) return set_error(SCAPH_EUNSUPPORTED, "BFS engine needs unweighted pages");
    if (gt && (gt->V != V || gt->E != E || gt->weighted))
        return set_error(SCAPH_EINVAL, "transposed graph does not match");
    if (V == 0) return set_error(SCAPH_EINVAL, "empty graph");
    SCAPH_CUDA(cudaSetDevice(device));
    SCAPH_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    if (cfg.stream) {
        st = (cudaStream_t)cfg.stream;
    } else {
        SCAPH_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        own_stream = true;
    }
    int nslots = 0;
    if (cfg.pool_bytes > 0) {
        const int64_t per = (int64_t)g->pagesize * 4;
        nslots = (int)std::max<int64_t>(1, cfg.pool_bytes / per);
        if (nslots < (int)g->pages.size() || (gt && nslots < (int)gt->pages.size()))
            return set_error(SCAPH_EUNSUPPORTED, "pool of %d pages smaller than the graph: use scaph_ooc_create", nslots);
    }
    int rc = dout.build(*g, nslots, st);
    if (rc) return rc;
    if (gt && (rc = din.build(*gt, nslots, st))) return rc;

    SCAPH_CUDA(cudaMalloc(&d_depth, (size_t)V * 4));
    SCAPH_CUDA(cudaMalloc(&d_parent, (size_t)V * 4));
    SCAPH_CUDA(cudaMalloc(&d_visited, (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&d_bm[0], (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&d_bm[1], (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&d_degree, (size_t)V * 4));
    SCAPH_CUDA(cudaMemcpyAsync(d_degree, g->degree.data(), (size_t)V * 4, cudaMemcpyHostToDevice, st));
    SCAPH_CUDA(cudaMalloc(&d_ctr, sizeof(LevelCounters) * kMaxLevels));
    SCAPH_CUDA(cudaMallocHost(&h_ctr, sizeof(LevelCounters) * kMaxLevels));
    const size_t np = g->pages.size();
    SCAPH_CUDA(cudaMalloc(&d_hist, sizeof(uint32_t) * 2 * np * kHistLevels));
    giant_cap = (uint32_t)std::min<uint64_t>(0xFFFFFFF0u, 2 * (E / kGiantEdges) + 1024);
    SCAPH_CUDA(cudaMalloc(&d_giant, sizeof(GiantChunk) * (size_t)giant_cap));
    SCAPH_CUDA(cudaEventCreate(&ev_start));
    SCAPH_CUDA(cudaEventCreate(&ev_stop));
    ev_level.resize(2 * kMaxLevels);
    for (auto &e : ev_level) SCAPH_CUDA(cudaEventCreate(&e));
    int occ_push = std::max(1, level_occupancy(0, block));
    int occ_pull = std::max(1, level_occupancy(1, block));
    grid_push = cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm * num_sms : occ_push * num_sms;
    grid_pull = cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm * num_sms : occ_pull * num_sms;
    SCAPH_CUDA(cudaStreamSynchronize(st));
    return SCAPH_OK;
}

void scaph_engine::destroy()
{
    if (st) cudaStreamSynchronize(st);
    dout.release();
    din.release();
    cudaFree(d_depth);
    cudaFree(d_parent);
    cudaFree(d_visited);
    cudaFree(d_bm[0]);
    cudaFree(d_bm[1]);
    cudaFree(d_degree);
    cudaFree(d_ctr);
    cudaFreeHost(h_ctr);
    cudaFree(d_hist);
    cudaFree(d_giant);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    for (auto &e : ev_level) if (e) cudaEventDestroy(e);
    if (own_stream && st) cudaStreamDestroy(st);
}

int scaph_engine::bfs(uint32_t src, uint32_t *depths, uint32_t *parents, int out_on_device, scaph_bfs_stats *stats)
{
    if (src >= V) return set_error(SCAPH_EINVAL, "source %u out of range (V=%u)", src, V);
    SCAPH_CUDA(cudaSetDevice(device));
    uint32_t *dd = (out_on_device && depths) ? depths : d_depth;
    uint32_t *dp = (out_on_device && parents) ? parents : (parents ? d_parent : nullptr);
    const int fill_grid = num_sms * 4;
    const size_t np = g->pages.size();
    trace.clear();

    SCAPH_CUDA(cudaEventRecord(ev_start, st));
    // bfs_init + setsrc (app/bfs.cu:20-37)
    SCAPH_CUDA(fill_u32(dd, unreached, V, fill_grid, st));
    if (dp) SCAPH_CUDA(fill_u32(dp, kNoParent, V, fill_grid, st));
    SCAPH_CUDA(cudaMemsetAsync(d_visited, 0, (size_t)nwords * 4, st));
    SCAPH_CUDA(cudaMemsetAsync(d_bm[0], 0, (size_t)nwords * 4, st));
    SCAPH_CUDA(cudaMemsetAsync(d_ctr, 0, sizeof(LevelCounters) * kMaxLevels, st));
    SCAPH_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(uint32_t) * 2 * np * kHistLevels, st));

    BfsDev s{};
    s.depth = dd;
    s.parent = dp;
    s.visited = d_visited;
    s.degree = d_degree;
    s.giant = d_giant;
    s.giant_cap = giant_cap;
    s.V = V;
    s.weighted_edges = 0;
    s.hg = dout.view;
    SCAPH_CUDA(set_source(s, src, d_bm[0], st));

    uint64_t nf = 1, prev_nf = 0, mf = g->degree[src];
    uint64_t vis_n = 1, vis_e = mf;
    uint64_t insp_total = 0, alg_total = 0;
    uint64_t launches = dp ? 3 : 2;  // fills + set_source
    int dir = 0, cur = 0, level = 0, npush = 0, npull = 0;
    uint32_t err = 0;
    while (nf > 0 && level < kMaxLevels && (uint64_t)level + 1 < unreached) {
        const uint64_t mu = E - vis_e;
        switch (cfg.direction) {
        case SCAPH_DIR_PUSH: dir = 0; break;
        case SCAPH_DIR_PULL: dir = level == 0 ? 0 : 1; break;
        default: dir = level == 0 ? 0 : alpha_beta_next(dir, nf, prev_nf, mf, mu, V, cfg.alpha, cfg.beta); break;
        }
        uint32_t *next = d_bm[cur ^ 1];
        SCAPH_CUDA(cudaEventRecord(ev_level[2 * level], st));
        SCAPH_CUDA(cudaMemsetAsync(next, 0, (size_t)nwords * 4, st));
        s.front = d_bm[cur];
        s.next = next;
        s.ctr = d_ctr + level;
        s.level = (uint32_t)level;
        if (level < kHistLevels) {
            s.page_nodes = d_hist + (size_t)level * 2 * np;
            s.page_datas = s.page_nodes + np;
        } else {
            s.page_nodes = s.page_datas = nullptr;
        }
        const GraphDev &gv = dir == 0 ? dout.view : gin();
        SCAPH_CUDA(run_level(dir, block, dir == 0 ? grid_push : grid_pull, gv, s, 0, V, st));
        SCAPH_CUDA(cudaEventRecord(ev_level[2 * level + 1], st));
        SCAPH_CUDA(cudaMemcpyAsync(h_ctr + level, d_ctr + level, sizeof(LevelCounters), cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
        const LevelCounters &lc = h_ctr[level];
        err |= lc.error;
        scaph_level_trace t{};
        t.level = level;
        t.direction = dir;
        t.frontier = nf;
        t.frontier_edges = mf;
        t.unvisited = V - vis_n;
        t.unvisited_edges = mu;
        t.next = lc.next;
        t.edges_inspected = lc.inspected;
        trace.push_back(t);
        // algorithmic bytes (push: headers + adjacency of the frontier;
        // pull: headers of unvisited vertices + in-edges up to the first
        // frontier hit; both: a V/8 bitmap pass and depth+parent writes)
        const uint64_t state_w = lc.next * (dp ? 8 : 4) + (uint64_t)nwords * 4;
        const uint64_t alg = dir == 0 ? nf * 12 + mf * 4 + state_w : (V - vis_n) * 12 + lc.inspected * 4 + state_w;
        trace.back().alg_bytes = alg;
        alg_total += alg;
        if (dir == 0) {
            npush++;
            launches += 2;
        } else {
            npull++;
            launches += 1;
        }
        insp_total += lc.inspected;
        prev_nf = nf;
        nf = lc.next;
        mf = lc.next_edges;
        vis_n += nf;
        vis_e += mf;
        cur ^= 1;
        level++;
        if (err) break;
    }
    SCAPH_CUDA(cudaEventRecord(ev_stop, st));
    SCAPH_CUDA(cudaEventSynchronize(ev_stop));
    last_levels = level;
    for (int l = 0; l < level; l++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_level[2 * l], ev_level[2 * l + 1]);
        trace[l].ms = ms;
    }
    if (err) return set_error(SCAPH_EDEVICE, "level kernel reported error flags 0x%x", err);
    if (!out_on_device) {
        if (depths) SCAPH_CUDA(cudaMemcpyAsync(depths, dd, (size_t)V * 4, cudaMemcpyDeviceToHost, st));
        if (parents) SCAPH_CUDA(cudaMemcpyAsync(parents, dp, (size_t)V * 4, cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_start, ev_stop);
        stats->ms = ms;
        stats->levels = level;
        stats->push_levels = npush;
        stats->pull_levels = npull;
        stats->reached = vis_n;
        stats->reached_edges = vis_e;
        stats->edges_inspected = insp_total;
        stats->alg_bytes = alg_total;
        stats->launches = launches;
    }
    return SCAPH_OK;
}

extern "C" {

int scaph_engine_create(const scaph_graph *g, const scaph_graph *gt, const scaph_config *cfg, scaph_engine **e)
{
    clear_error();
    if (!g || !e) return set_error(SCAPH_EINVAL, "null argument");
    *e = nullptr;
    std::unique_ptr<scaph_engine> eng(new scaph_engine());
    int rc = eng->create(g, gt, cfg);
    if (rc) {
        eng->destroy();
        return rc;
    }
    *e = eng.release();
    return SCAPH_OK;
}

int scaph_engine_destroy(scaph_engine *e)
{
    if (!e) return SCAPH_OK;
    e->destroy();
    delete e;
    return SCAPH_OK;
}

int scaph_bfs(scaph_engine *e, uint32_t src, uint32_t *depths, uint32_t *parents, int out_on_device,
              scaph_bfs_stats *stats)
{
    clear_error();
    if (!e) return set_error(SCAPH_EINVAL, "null engine");
    return e->bfs(src, depths, parents, out_on_device, stats);
}

int scaph_bfs_trace(const scaph_engine *e, scaph_level_trace *out, int cap)
{
    if (!e || (!out && cap > 0)) return set_error(SCAPH_EINVAL, "null argument");
    int n = std::min<int>(cap, (int)e->trace.size());
    for (int i = 0; i < n; i++) out[i] = e->trace[i];
    return n;
}

int scaph_bfs_page_hist(const scaph_engine *e, int level, uint32_t *nodes, uint32_t *datas, int npages)
{
    if (!e || !nodes || !datas) return set_error(SCAPH_EINVAL, "null argument");
    const int np = (int)e->g->pages.size();
    if (npages < np) return set_error(SCAPH_EINVAL, "need %d pages", np);
    // histogram slot `level` holds the frontier discovered BY level; the
    // frontier AT level L is slot L-1 (level 0 is the source alone)
    if (level < 0 || level > e->last_levels || level > scaph_engine::kHistLevels)
        return set_error(SCAPH_EINVAL, "level %d not recorded", level);
    if (level == 0) {
        memset(nodes, 0, sizeof(uint32_t) * np);
        memset(datas, 0, sizeof(uint32_t) * np);
        return SCAPH_OK;  // caller knows the source; kept simple
    }
    const uint32_t *h = e->d_hist + (size_t)(level - 1) * 2 * np;
    SCAPH_CUDA(cudaMemcpy(nodes, h, sizeof(uint32_t) * np, cudaMemcpyDeviceToHost));
    SCAPH_CUDA(cudaMemcpy(datas, h + np, sizeof(uint32_t) * np, cudaMemcpyDeviceToHost));
    return SCAPH_OK;
}

void *scaph_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        set_error(SCAPH_ENOMEM, "cudaMallocHost(%zu)", bytes);
        return nullptr;
    }
    return p;
}

void scaph_host_free(void *p) { cudaFreeHost(p); }

int scaph_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

}  // extern "C"
