// The BFS engine: device page pool + page table, per-vertex state, and the
// level loop with the direction switch.  Replaces App (src/app.cuh:72-345)
// for the BFS application: App::load_graph's allocations and pool fill
// (src/app.cuh:267-345), App::run's round loop (:220-265) and iter_init's
// per-round D2H of the whole stat array (:188-207).
//
// Two ways to run the level loop:
//  * graph mode (default when the whole graph is resident): one CUDA-graph
//    launch per BFS.  Its level loop is a conditional WHILE node whose body
//    is push -> giant -> pull -> decide (the level kernels the level's
//    direction does not select leave at once); the decide kernel applies the
//    direction rule on the device and sets the loop's condition, so a BFS
//    never returns to the host between levels;
//  * host loop: one launch per level and a 64-byte counter read-back,
//    with CUDA events around every level (per-level kernel timing) - used
//    for out-of-core page batches and for the roofline pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <utility>

#include "engine.h"

// the pull's CTA tiles read the phase-A arrays of the live vertices only
#ifndef SCAPH_PULL_LIVE
#define SCAPH_PULL_LIVE 1
#endif
// ... and the warp-centric pull reads the records of the live vertices
#ifndef SCAPH_PULL_LIVE_REC
#define SCAPH_PULL_LIVE_REC 1
#endif
// graph mode runs a level's giant chunks and pull in one kernel node
#ifndef SCAPH_GRAPH_GIANT_PULL
#define SCAPH_GRAPH_GIANT_PULL 1
#endif
#include "kernels.h"

using namespace scaph;

// Pull phase A's first probes: 0 = the first in-edges, read from the pages;
// 1 = the same edges from dense per-vertex rows (16 B per vertex of device
// memory); 2 = dense rows of the in-neighbours with the largest out-degree.
#ifndef SCAPH_PULL_HEAD
#define SCAPH_PULL_HEAD 2
#endif

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

}  // namespace scaph

const GraphDev &scaph_engine::out_view() const { return pager ? pager_view(pager, 0) : dout.view; }

const GraphDev &scaph_engine::gin() const
{
    if (pager) return pager_view(pager, symmetric ? 0 : 1);
    return symmetric ? dout.view : din.view;
}

BfsDev scaph_engine::base_state(uint32_t *dd, uint32_t *dp) const
{
    BfsDev s{};
    s.depth = dd;
    s.parent = dp;
    s.visited = d_visited;
    s.degree = d_degree;
    s.giant = d_giant;
    s.giant_cap = giant_cap;
    s.V = V;
    s.nwords = nwords;
    s.hg = out_view();
    s.head = d_head;
    s.indeg = d_indeg;
    s.head_ranked = head_ranked ? 1u : 0u;
    s.prec = d_prec;
    s.prow = cfg.pull_rows == 1 && head_ranked ? d_prow : nullptr;  // phase B rescans ranked rows from 0
    s.live_rank = d_live_rank;
    s.dead = d_dead;
    s.live_head = d_live_head;
    s.live_indeg = d_live_indeg;
    s.live_deg = d_live_deg;
    s.live_prec = d_live_prec;
    s.push_sparse = push_use_sparse(cfg.push_sparse_ratio, 1, V) ? 1u : 0u;  // level 0
    s.giant_edges = (uint32_t)cfg.giant_edges;
    s.pull_warp = cfg.pull_warp == 3 ? 0u : (uint32_t)cfg.pull_warp;  // kernel: 0 tiles, 1 warp, 2 lanes
    return s;
}

// The pull's phase-A arrays over the live vertices only (in-degree > 0, the
// vertices a traversal can discover), indexed by live rank: rank(v) =
// live_rank[v / 32] + the live vertices below v in its word.  On RMAT-24
// 56% of the vertices have no edge; in the V-entry arrays their entries
// share every sector with live ones, so the small-frontier pull level read
// 44 bytes of sectors per unvisited vertex for 24 bytes of fields.
static __global__ void k_build_live(const uint32_t *dead, const uint32_t *rank, const uint32_t *head,
                                    const uint32_t *indeg, const uint32_t *deg, const uint2 *prec, uint4 *lhead,
                                    uint32_t *lindeg, uint32_t *ldeg, uint2 *lprec, uint32_t V)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t w = v >> 5, live = ~dead[w];
        if (!((live >> (v & 31)) & 1u)) continue;
        const uint32_t r = rank[w] + __popc(live & ((1u << (v & 31)) - 1u));
        lhead[r] = reinterpret_cast<const uint4 *>(head)[v];
        lindeg[r] = indeg[v];
        ldeg[r] = deg[v];
        if (lprec) lprec[r] = prec[v];
    }
}

int scaph_engine::build_live(const std::vector<uint32_t> &dead)
{
    if (!d_head || !d_prec || !head_ranked) return SCAPH_OK;
    std::vector<uint32_t> rank(nwords + 1);
    uint32_t n = 0;
    for (uint32_t w = 0; w < nwords; w++) {
        rank[w] = n;
        const uint32_t valid = (w + 1) * 32ull <= V ? 0xFFFFFFFFu : ((1u << (V & 31)) - 1u);
        n += __builtin_popcount(~dead[w] & valid);
    }
    rank[nwords] = n;
    if (n != V - n_dead) return set_error(SCAPH_EINVAL, "live vertex count %u != %u", n, (unsigned)(V - n_dead));
    SCAPH_CUDA(cudaMalloc(&d_live_rank, (size_t)(nwords + 1) * 4));
    SCAPH_CUDA(cudaMemcpyAsync(d_live_rank, rank.data(), (size_t)(nwords + 1) * 4, cudaMemcpyHostToDevice, st));
    const size_t nl = std::max<uint32_t>(n, 1);
    SCAPH_CUDA(cudaMalloc(&d_live_head, nl * sizeof(uint4)));
    SCAPH_CUDA(cudaMalloc(&d_live_indeg, nl * 4));
    SCAPH_CUDA(cudaMalloc(&d_live_deg, nl * 4));
#if SCAPH_PULL_LIVE_REC
    SCAPH_CUDA(cudaMalloc(&d_live_prec, nl * sizeof(uint2)));
#endif
    k_build_live<<<num_sms * 8, 256, 0, st>>>(d_dead, d_live_rank, d_head, d_indeg, d_degree, d_prec, d_live_head,
                                              d_live_indeg, d_live_deg, d_live_prec, V);
    SCAPH_CUDA(cudaGetLastError());
    SCAPH_CUDA(cudaStreamSynchronize(st));  // rank lives on the host stack until here
    return SCAPH_OK;
}

// The 16-byte pull rows (scaph_config.pull_rows = 1): the first three ranked
// in-neighbours of the head row and the records' degree word, one load per
// vertex instead of the in-degree, the head row and the out-degree.  Built
// on the device from those two arrays when first asked for.
static __global__ void k_build_prow(const uint32_t *head, const uint2 *prec, uint4 *prow, uint32_t V)
{
    static_assert(kPullHead == 4, "the rows keep three of the four head entries");
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint4 h = reinterpret_cast<const uint4 *>(head)[v];
        prow[v] = make_uint4(h.x, h.y, h.z, prec[v].y);
    }
}

int scaph_engine::build_prow()
{
    if (d_prow || !d_head || !d_prec) return SCAPH_OK;
    SCAPH_CUDA(cudaMalloc(&d_prow, (size_t)V * sizeof(uint4)));
    k_build_prow<<<num_sms * 8, 256, 0, st>>>(d_head, d_prec, d_prow, V);
    SCAPH_CUDA(cudaGetLastError());
    SCAPH_CUDA(cudaStreamSynchronize(st));
    return SCAPH_OK;
}

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
    if (unreached < 2) return set_error(SCAPH_EINVAL, "unreached sentinel must be >= 2");
    if (cfg.alpha <= 0) cfg.alpha = kAlphaDefault;
    if (cfg.beta <= 0) cfg.beta = kBetaDefault;
    block = cfg.block_size == 128 || cfg.block_size == 512 ? cfg.block_size : 256;
    if (cfg.giant_edges == 0) cfg.giant_edges = (int32_t)kGiantEdges;
    if (cfg.giant_edges < 128 || cfg.giant_edges > 65536)
        return set_error(SCAPH_EINVAL, "giant_edges %d outside 128..65536", cfg.giant_edges);
    if (cfg.pull_gather_ratio <= 0) cfg.pull_gather_ratio = (int32_t)kPullGatherRatio;
    if (cfg.ms_compact_l2_div <= 0) cfg.ms_compact_l2_div = 3;
    if (cfg.ms_compact_min_deg <= 0) cfg.ms_compact_min_deg = 16;
    if (cfg.push_defer_edges == 0) cfg.push_defer_edges = kDeferEdgesDefault;
    if (cfg.pull_records < 0 || cfg.pull_records > 2) cfg.pull_records = 0;
    if (cfg.pull_warp < 1 || cfg.pull_warp > 3) cfg.pull_warp = 1;
    if (cfg.pull_rows < 0 || cfg.pull_rows > 2) cfg.pull_rows = 0;
    if (cfg.push_sparse_ratio == 0) cfg.push_sparse_ratio = (int32_t)kPushSparseRatio;
    if (cfg.pull_runs < 0 || cfg.pull_runs > 2) cfg.pull_runs = 0;
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
    int rc;
    const size_t total_pages = g->pages.size() + (gt ? gt->pages.size() : 0);
    const int64_t per = (int64_t)g->pagesize * 4;
    const int nslots = cfg.pool_bytes > 0 ? (int)std::max<int64_t>(1, cfg.pool_bytes / per) : 0;
    if (nslots > 0 && (size_t)nslots < total_pages) {
        // out-of-core: pages stream through a pool of nslots page slots
        if ((rc = pager_create(g, gt, nslots, cfg.copy_streams, cfg.link_gbs, &pager))) return rc;
    } else {
        if ((rc = dout.build(*g, 0, st))) return rc;
        if (gt && (rc = din.build(*gt, 0, st))) return rc;
    }
    {
        const std::vector<uint32_t> &indeg = gt ? gt->degree : g->degree;
        SCAPH_CUDA(cudaMalloc(&d_indeg, (size_t)V * 4));
        SCAPH_CUDA(cudaMemcpyAsync(d_indeg, indeg.data(), (size_t)V * 4, cudaMemcpyHostToDevice, st));
        const size_t npi = (gt ? gt->pages.size() : g->pages.size()) + 1;
        SCAPH_CUDA(cudaMalloc(&d_pcnt, npi * 4));
        SCAPH_CUDA(cudaMalloc(&d_pdatas, npi * 4));
    }

    if (SCAPH_PULL_HEAD) {
        // pull phase A's dense rows: the first in-edges of every vertex
        // in-neighbours of largest out-degree first: the likeliest to be in
        // a frontier (hubs join it early), so most vertices settle on the
        // first probe
        const Graph &gi = gt ? *gt : *g;
        std::vector<uint32_t> head((size_t)V * kPullHead);
        adjacency_heads(gi, kPullHead, head.data(), SCAPH_PULL_HEAD == 2 ? g->degree.data() : nullptr);
        head_ranked = SCAPH_PULL_HEAD == 2;
        SCAPH_CUDA(cudaMalloc(&d_head, head.size() * 4));
        SCAPH_CUDA(cudaMemcpy(d_head, head.data(), head.size() * 4, cudaMemcpyHostToDevice));
        // the 8-byte records phase A reads first: the top-ranked in-neighbour,
        // and the in- and out-degree in one word (pull_meta)
        const std::vector<uint32_t> &indeg = gt ? gt->degree : g->degree;
        std::vector<uint2> prec(V);
        #pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < (int64_t)V; v++)
            prec[v] = make_uint2(head[(size_t)v * kPullHead], pull_meta(indeg[v], g->degree[v]));
        SCAPH_CUDA(cudaMalloc(&d_prec, (size_t)V * sizeof(uint2)));
        SCAPH_CUDA(cudaMemcpy(d_prec, prec.data(), (size_t)V * sizeof(uint2), cudaMemcpyHostToDevice));
        if (cfg.pull_rows == 1 && (rc = build_prow())) return rc;
    }

    // vertices no edge reaches (in-degree 0) are never discovered: they start
    // out "visited" so pull levels skip them
    const std::vector<uint32_t> &indeg = gt ? gt->degree : g->degree;
    std::vector<uint32_t> dead(nwords, 0);
    for (uint32_t v = 0; v < V; v++) {
        if (indeg[v] == 0) {
            dead[v >> 5] |= 1u << (v & 31);
            n_dead++;
            dead_edges += g->degree[v];
        }
    }
    SCAPH_CUDA(cudaMalloc(&d_dead, (size_t)nwords * 4));
    SCAPH_CUDA(cudaMemcpyAsync(d_dead, dead.data(), (size_t)nwords * 4, cudaMemcpyHostToDevice, st));

    SCAPH_CUDA((cudaError_t)injected_fault(kFaultDeviceAlloc));
    SCAPH_CUDA(cudaMalloc(&d_depth, (size_t)V * 4));
    SCAPH_CUDA(cudaMalloc(&d_parent, (size_t)V * 4));
    SCAPH_CUDA(cudaMalloc(&d_visited, (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&d_bm3, (size_t)nwords * 4 * 3));
    SCAPH_CUDA(cudaMalloc(&d_degree, (size_t)V * 4));
    SCAPH_CUDA(cudaMemcpyAsync(d_degree, g->degree.data(), (size_t)V * 4, cudaMemcpyHostToDevice, st));
#if SCAPH_PULL_LIVE
    if ((rc = build_live(dead))) return rc;
#endif
    SCAPH_CUDA(cudaMalloc(&d_ctr, sizeof(LevelCounters) * kMaxLevels));
    SCAPH_CUDA(cudaMallocHost(&h_ctr, sizeof(LevelCounters) * kMaxLevels));
    SCAPH_CUDA(cudaMalloc(&d_ctl, sizeof(BfsCtl)));
    SCAPH_CUDA(cudaMallocHost(&h_ctl, sizeof(BfsCtl)));
    const size_t np = g->pages.size();
    SCAPH_CUDA(cudaMalloc(&d_hist, sizeof(uint32_t) * 2 * np * kHistLevels));
    // sum of ceil(len / cut) over one level's lists of more than cut edges is
    // at most 2 E / cut; the multi-source kernels cut at kGiantEdges
    const uint64_t cut = std::min<uint64_t>((uint64_t)cfg.giant_edges, kGiantEdges);
    giant_cap = (uint32_t)std::min<uint64_t>(0xFFFFFFF0u, 2 * (E / cut) + 1024);
    SCAPH_CUDA(cudaMalloc(&d_giant, sizeof(GiantChunk) * (size_t)giant_cap));
    SCAPH_CUDA(cudaEventCreate(&ev_start));
    SCAPH_CUDA(cudaEventCreate(&ev_stop));
    SCAPH_CUDA(cudaEventCreate(&ev_dual[0]));
    SCAPH_CUDA(cudaEventCreate(&ev_dual[1]));
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
    if (copy_st) {
        cudaStreamSynchronize(copy_st);
        cudaStreamDestroy(copy_st);
        copy_st = nullptr;
    }
    for (int i = 0; i < 2; i++) {
        cudaFree(d_pipe[i]);
        d_pipe[i] = nullptr;
        if (ev_run[i]) cudaEventDestroy(ev_run[i]);
        if (ev_copied[i]) cudaEventDestroy(ev_copied[i]);
        ev_run[i] = ev_copied[i] = nullptr;
    }
    ms_release(ms);
    ms = nullptr;
    pager_release(pager);
    pager = nullptr;
    cudaFree(d_indeg);
    cudaFree(d_head);
    cudaFree(d_prec);
    cudaFree(d_prow);
    cudaFree(d_live_rank);
    cudaFree(d_live_head);
    cudaFree(d_live_indeg);
    cudaFree(d_live_deg);
    cudaFree(d_live_prec);
    cudaFree(d_snap);
    cudaFree(d_pcnt);
    cudaFree(d_pdatas);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (cap_st) cudaStreamDestroy(cap_st);
    dout.release();
    din.release();
    cudaFree(d_depth);
    cudaFree(d_parent);
    cudaFree(d_visited);
    cudaFree(d_bm3);
    cudaFree(d_degree);
    cudaFree(d_dead);
    cudaFree(d_ctr);
    cudaFreeHost(h_ctr);
    cudaFree(d_ctl);
    cudaFreeHost(h_ctl);
    cudaFree(d_hist);
    cudaFree(d_giant);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    for (auto &ev : ev_dual)
        if (ev) cudaEventDestroy(ev);
    for (auto &e : ev_level) if (e) cudaEventDestroy(e);
    cudaFreeHost(h_fstage);
    cudaFreeHost(h_inc);
    cudaFree(d_hist_in);
    if (own_stream && st) cudaStreamDestroy(st);
}

// The first ten scheduler features of a level (layout in scaph.h), shared
// by the single- and multi-source loops and by k_decide_learned.
void scaph::sched_globals(float *f, uint64_t nf, uint64_t mf, uint64_t unvis, uint64_t mu, uint32_t V, uint64_t E,
                          int level, int prev_dir)
{
    auto lg = [](double x, double d) { return (float)(std::log2(1.0 + x) / d); };
    f[0] = lg((double)nf, 32);
    f[1] = lg((double)mf, 40);
    f[2] = lg((double)unvis, 32);
    f[3] = lg((double)mu, 40);
    f[4] = (float)((double)nf / V);
    f[5] = (float)std::min(1.0, (double)mf / std::max<uint64_t>(1, E));
    f[6] = (float)((double)unvis / V);
    f[7] = (float)std::min(1.0, (double)mu / std::max<uint64_t>(1, E));
    f[8] = (float)level / 32.f;
    f[9] = (float)prev_dir;
}

// Scheduler features of the coming level (layout in scaph.h): 16 globals,
// then the frontier's share of every out-edge page.  The frontier histogram
// and the pull-side page counts come from the incremental copies the host
// loop keeps (inc_hist / inc_pull) when they are current, else from the
// device.
int scaph_engine::features(int level, uint32_t src, uint64_t nf, uint64_t mf, uint64_t unvis, uint64_t mu,
                           int prev_dir, int ab_dir, float *f, std::vector<uint32_t> &pull_cnt,
                           std::vector<uint32_t> &hist)
{
    const size_t np = g->pages.size();
    const GraphDev &gi = gin();
    const int npi = (int)gi.npages;
    // frontier histogram over out-pages, counts then active words (level 0:
    // the source alone)
    // both read-backs land in pinned staging and wait on one synchronisation
    if (!h_fstage) {
        SCAPH_CUDA((cudaError_t)injected_fault(kFaultPinnedAlloc));
        SCAPH_CUDA(cudaMallocHost(&h_fstage, sizeof(uint32_t) * 2 * (np + (size_t)npi)));
    }
    uint32_t *hh = h_fstage, *hp = h_fstage + 2 * np;
    const bool hist_inc = level > 0 && inc_hist_level == level;
    const bool hist_dev = level > 0 && level - 1 < kHistLevels && !hist_inc;
    if (hist_dev)
        SCAPH_CUDA(cudaMemcpyAsync(hh, d_hist + (size_t)(level - 1) * 2 * np, 2 * np * 4, cudaMemcpyDeviceToHost, st));
    // unvisited vertices per in-edge page (only needed out of core, for the
    // residency features, and for training traces)
    const bool pull_inc = inc_pull_valid;
    const bool pull_dev = (pager || cfg.record_features) && !pull_inc;
    if (pull_dev) {
        SCAPH_CUDA(page_unvisited(gi, d_visited, d_indeg, d_pcnt, d_pdatas, num_sms * 8, st));
        SCAPH_CUDA(cudaMemcpyAsync(hp, d_pcnt, npi * 4, cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaMemcpyAsync(hp + npi, d_pdatas, npi * 4, cudaMemcpyDeviceToHost, st));
    }
    if (hist_dev || pull_dev) SCAPH_CUDA(cudaStreamSynchronize(st));
    hist.assign(2 * np, 0);
    if (level == 0) {
        size_t p = 0;
        while (p + 1 < np && g->pages[p + 1].left <= src) p++;
        hist[p] = 1;
        hist[np + p] = g->degree[src] + 3;
    } else if (hist_inc) {
        hist.assign(inc_hist.begin(), inc_hist.end());
    } else if (hist_dev) {
        hist.assign(hh, hh + 2 * np);
    }
    pull_cnt.assign(2 * (size_t)npi, 0);  // counts, then active words
    if (pull_inc) pull_cnt.assign(inc_pull.begin(), inc_pull.end());
    else if (pull_dev) pull_cnt.assign(hp, hp + 2 * (size_t)npi);
    sched_globals(f, nf, mf, unvis, mu, V, E, level, prev_dir);
    float res_out = 1.f, res_in = 1.f, res_push = 1.f, res_pull = 1.f;
    if (pager) {
        std::vector<int> push_pages, pull_pages;
        for (size_t p = 0; p < np; p++)
            if (hist[p]) push_pages.push_back((int)p);
        for (int p = 0; p < npi; p++)
            if (pull_cnt[p]) pull_pages.push_back(p);  // counts are the first npi entries
        const int gid_in = symmetric ? 0 : 1;
        res_out = pager_resident_fraction(pager, 0, nullptr);
        res_in = pager_resident_fraction(pager, gid_in, nullptr);
        res_push = pager_resident_fraction(pager, 0, &push_pages);
        res_pull = pager_resident_fraction(pager, gid_in, &pull_pages);
    }
    f[10] = res_out;
    f[11] = res_in;
    f[12] = res_push;
    f[13] = res_pull;
    f[14] = (float)ab_dir;
    f[15] = 1.f;
    for (size_t p = 0; p < np; p++) f[SCAPH_SCHED_GLOBALS + p] = (float)hist[p] / (float)std::max(1u, g->pages[p].nodenum);
    return SCAPH_OK;
}

// Host-driven level loop (one launch + one counter read-back per level).
int scaph_engine::run_host_loop(uint32_t src, uint32_t *dd, uint32_t *dp)
{
    const int fill_grid = num_sms * 4;
    const size_t np = g->pages.size();
    // The pool holds the in-edge pages with half the out-edge pages beside
    // them: what a level brings in stays for later levels and traversals.
    const bool keep_pool = pager && !symmetric && 2 * gin().npages + np <= 2 * (size_t)pager_nslots(pager);
    // The network's direction output models the resident level kernels'
    // time (its labels come from timing both directions on a resident
    // graph); the paged kernels cost differently (config 3, pool kept, warm:
    // same bytes moved, its directions 0.81x of alpha/beta).  Out of core it
    // names pages to prefetch, and only where pages do not stay in the pool
    // (in one that keeps them, demand paging already reads a single
    // traversal's sparse pages zero-copy and keeps the dense ones): a pool
    // that keeps pages runs the plain loop.
    const bool learned = cfg.direction == SCAPH_DIR_LEARNED && sched && !keep_pool;
    const bool want_feat = learned || cfg.record_features;
    const bool dual = cfg.dual_timing && !pager;
    // per-level page histograms (get_page_info's counts) cost a shared-memory
    // atomic pair per discovered vertex: recorded only where something reads
    // them (pager, learned features, record_features)
    const bool hist_on = host_records_hist();
    SCAPH_CUDA(fill_u32(dd, unreached, V, fill_grid, st));
    if (dp) SCAPH_CUDA(fill_u32(dp, kNoParent, V, fill_grid, st));
    SCAPH_CUDA(cudaMemcpyAsync(d_visited, d_dead, (size_t)nwords * 4, cudaMemcpyDeviceToDevice, st));
    SCAPH_CUDA(cudaMemsetAsync(d_bm3, 0, (size_t)nwords * 4, st));
    SCAPH_CUDA(cudaMemsetAsync(d_ctr, 0, sizeof(LevelCounters) * kMaxLevels, st));
    SCAPH_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(uint32_t) * 2 * np * kHistLevels, st));
    BfsDev s = base_state(dd, dp);
    uint32_t *bm[2] = {d_bm3, d_bm3 + nwords};
    SCAPH_CUDA(set_source(s, src, bm[0], st));
    level_h2d.clear();
    pcie_alg = 0;
    dual_ms.clear();
    feat_log.clear();
    pull_log.clear();
    feat_dim = SCAPH_SCHED_GLOBALS + (int)np;
    if (pager) pager_reset_counters(pager);
    if (dual && !d_snap) SCAPH_CUDA(cudaMalloc(&d_snap, (size_t)nwords * 4));
    const bool src_dead = (gt ? gt->degree[src] : g->degree[src]) == 0;

    uint64_t nf = 1, prev_nf = 0, mf = g->degree[src];
    uint64_t vis_n = 1, vis_e = mf;
    int dir = 0, cur = 0, level = 0;
    std::vector<float> f(feat_dim), y;
    if (learned) {
        int rc = mlp_host_snapshot(sched, sched_host);
        if (rc) return rc;
    }
    // out of core, the learned scheduler's per-level page counts are kept
    // incrementally: the pull side starts from one pass over the vertices
    // and loses each level's discoveries (the in-page histogram the level
    // kernels record), the push side is the level's out-page histogram; both
    // arrive with the level's counters, so a level needs no extra pass
    const bool incr = pager && learned && !dual;
    const GraphDev &gview_in = gin();
    const size_t npi = gview_in.npages;
    inc_pull_valid = false;
    inc_hist_level = -1;
    if (incr) {
        if (!h_inc) SCAPH_CUDA(cudaMallocHost(&h_inc, sizeof(uint32_t) * 2 * (np + npi)));
        if (!symmetric && !d_hist_in) SCAPH_CUDA(cudaMalloc(&d_hist_in, sizeof(uint32_t) * 2 * npi * kHistLevels));
        if (d_hist_in) SCAPH_CUDA(cudaMemsetAsync(d_hist_in, 0, sizeof(uint32_t) * 2 * npi * kHistLevels, st));
        SCAPH_CUDA(page_unvisited(gview_in, d_visited, d_indeg, d_pcnt, d_pdatas, num_sms * 8, st));
        SCAPH_CUDA(cudaMemcpyAsync(h_inc, d_pcnt, npi * 4, cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaMemcpyAsync(h_inc + npi, d_pdatas, npi * 4, cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
        inc_pull.assign(h_inc, h_inc + 2 * npi);
        inc_pull_valid = true;
    }
    // page counts of the last feature pass, reused by the pager
    std::vector<uint32_t> feat_pc, feat_hist;
    while (nf > 0 && level < kMaxLevels && (uint64_t)level + 1 < unreached) {
        const uint64_t used = vis_e + dead_edges;
        const uint64_t mu = E > used ? E - used : 0;
        const int ab = level == 0 ? 0 : alpha_beta_next(dir, nf, prev_nf, mf, mu, V, cfg.alpha, cfg.beta);
        const int prev_dir = dir;
        switch (cfg.direction) {
        case SCAPH_DIR_PUSH: dir = 0; break;
        case SCAPH_DIR_PULL: dir = level == 0 ? 0 : 1; break;
        default: dir = ab; break;
        }
        std::vector<int> prefetch_pages;
        if (want_feat) {
            std::vector<uint32_t> pc, hist;
            const uint64_t unvis = (uint64_t)V - n_dead - vis_n + (src_dead ? 1 : 0);
            int rc = features(level, src, nf, mf, unvis, mu, prev_dir, ab, f.data(), pc, hist);
            if (rc) return rc;
            feat_log.insert(feat_log.end(), f.begin(), f.end());
            if (learned) {
                int in = 0, out = 0;
                mlp_dims(sched, &in, &out);
                y.resize(out);
                mlp_forward_host(sched_host, f.data(), y.data());
                if (level > 0 && !pager) {
                    dir = y[0] > 0.f ? 1 : 0;
                    // far from the alpha/beta threshold the rule decides
                    const int sure = alpha_beta_confident(prev_dir, nf, mf, mu, V, cfg.alpha, cfg.beta);
                    if (sure >= 0) dir = sure;
                } else if (level > 0) {
                    // out of core (a pool that does not keep pages): the page
                    // traffic each direction would cause is known exactly; a
                    // direction whose traffic is more than twice the other's
                    // (and 1 ms more) is turned around
                    const int npc = (int)pc.size() / 2;
                    const double t_push = pager_transfer_ms(pager, 0, hist.data(), hist.data() + np, (int)np,
                                                            cfg.compact_threshold);
                    const double t_pull = pager_transfer_ms(pager, symmetric ? 0 : 1, pc.data(), pc.data() + npc,
                                                            npc, cfg.compact_threshold);
                    if (t_push > 2 * t_pull + 1.0) dir = 1;
                    else if (t_pull > 2 * t_push + 1.0) dir = 0;
                }
                // prefetch only pages the network is confident about (into
                // free slots; never at the expense of resident pages)
                if (pager)
                    for (int p = 0; p + 1 < out && p < (int)np; p++)
                        if (y[1 + p] > 2.f) prefetch_pages.push_back(p);
            }
            feat_pc = pc;
            feat_hist = std::move(hist);
            pull_log.push_back(std::move(pc));
        }
        uint32_t *next = bm[cur ^ 1];
        s.front = bm[cur];
        s.next = next;
        s.ctr = d_ctr + level;
        s.level = (uint32_t)level;
        if (hist_on && level < kHistLevels) {
            s.page_nodes = d_hist + (size_t)level * 2 * np;
            s.page_datas = s.page_nodes + np;
        } else {
            s.page_nodes = s.page_datas = nullptr;
        }
        {
            const uint64_t unv_now = (uint64_t)V - n_dead - vis_n + (src_dead ? 1 : 0);
            s.pull_gather = unv_now * (uint64_t)cfg.pull_gather_ratio < V ? (cfg.pull_runs == 2 ? 1u : 2u) : 0u;
            s.prec = pull_use_records(cfg.pull_records, nf, unv_now) ? d_prec : nullptr;
        }
        // deferred claims on big push levels (resident graphs, no parents)
        s.push_defer = !pager && !dp && !dual && cfg.push_defer_edges > 0 && mf >= (uint64_t)cfg.push_defer_edges
                           ? 1u : 0u;
        s.push_sparse = push_use_sparse(cfg.push_sparse_ratio, nf, V) ? 1u : 0u;
        s.page_nodes_in = s.page_datas_in = nullptr;
        if (incr && d_hist_in && level < kHistLevels) {
            s.page_nodes_in = d_hist_in + (size_t)level * 2 * npi;
            s.page_datas_in = s.page_nodes_in + npi;
            s.hgi = gview_in;
        }
        double dual_push = 0, dual_pull = 0;
        if (dual && level > 0) {
            // both directions from the same state: push first, then the
            // state is restored and pull runs (both discover the same set)
            SCAPH_CUDA(cudaMemcpyAsync(d_snap, d_visited, (size_t)nwords * 4, cudaMemcpyDeviceToDevice, st));
            SCAPH_CUDA(cudaMemsetAsync(next, 0, (size_t)nwords * 4, st));
            SCAPH_CUDA(cudaEventRecord(ev_dual[0], st));
            SCAPH_CUDA(run_level(0, block, grid_push, dout.view, s, 0, V, st));
            SCAPH_CUDA(cudaEventRecord(ev_dual[1], st));
            SCAPH_CUDA(cudaEventSynchronize(ev_dual[1]));
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_dual[0], ev_dual[1]);
            dual_push = ms;
            SCAPH_CUDA(cudaMemcpyAsync(d_visited, d_snap, (size_t)nwords * 4, cudaMemcpyDeviceToDevice, st));
            SCAPH_CUDA(cudaMemsetAsync(d_ctr + level, 0, sizeof(LevelCounters), st));
            if (s.page_nodes) SCAPH_CUDA(cudaMemsetAsync(s.page_nodes, 0, sizeof(uint32_t) * 2 * np, st));
        }
        SCAPH_CUDA(cudaEventRecord(ev_level[2 * level], st));
        SCAPH_CUDA(cudaMemsetAsync(next, 0, (size_t)nwords * 4, st));
        const int run_dir = (dual && level > 0) ? 1 : dir;
        if (pager) {
            std::vector<int> needed;
            std::vector<uint32_t> datas;
            int rc = SCAPH_OK;
            if (want_feat && (run_dir == 0 ? !feat_hist.empty() : !feat_pc.empty())) {
                // the feature pass of this level already counted these pages
                const std::vector<uint32_t> &c = run_dir == 0 ? feat_hist : feat_pc;
                const size_t n = c.size() / 2;
                datas.assign(n, 0);
                for (size_t p = 0; p < n; p++)
                    if (c[p]) {
                        needed.push_back((int)p);
                        datas[p] = c[n + p];
                    }
            } else {
                rc = pager_needs(this, pager, run_dir, level, src, needed, datas);
            }
            if (!rc) pcie_alg += 4 * pager_missing_words(pager, run_dir == 0 || symmetric ? 0 : 1, needed, datas);
            if (!rc) rc = pager_run_level(this, pager, run_dir, s, needed, datas);
            if (!rc && !prefetch_pages.empty() && run_dir == 0) rc = pager_prefetch(this, pager, 0, prefetch_pages);
            if (rc) return rc;
            uint64_t h2d, zc, ff, pf, hits, lh;
            pager_counters(pager, &h2d, &zc, &ff, &pf, &hits, &lh);
            level_h2d.push_back(lh);
        } else {
            const GraphDev &gv = run_dir == 0 ? dout.view : gin();
            SCAPH_CUDA(run_level(run_dir, block, run_dir == 0 ? grid_push : grid_pull, gv, s, 0, V, st));
            if (run_dir == 0 && s.push_defer) SCAPH_CUDA(run_push_finalize(block, num_sms * 4, s, st));
        }
        SCAPH_CUDA(cudaEventRecord(ev_level[2 * level + 1], st));
        SCAPH_CUDA(cudaMemcpyAsync(h_ctr + level, d_ctr + level, sizeof(LevelCounters), cudaMemcpyDeviceToHost, st));
        const bool inc_now = incr && level < kHistLevels;
        if (inc_now) {
            SCAPH_CUDA(cudaMemcpyAsync(h_inc, d_hist + (size_t)level * 2 * np, 2 * np * 4, cudaMemcpyDeviceToHost, st));
            if (d_hist_in)
                SCAPH_CUDA(cudaMemcpyAsync(h_inc + 2 * np, d_hist_in + (size_t)level * 2 * npi, 2 * npi * 4,
                                           cudaMemcpyDeviceToHost, st));
        }
        SCAPH_CUDA(cudaStreamSynchronize(st));
        if (inc_now) {
            inc_hist.assign(h_inc, h_inc + 2 * np);
            inc_hist_level = level + 1;
            const uint32_t *hin = d_hist_in ? h_inc + 2 * np : h_inc;  // symmetric: in-pages are the out-pages
            for (size_t p = 0; p < 2 * npi; p++) inc_pull[p] -= hin[p];
        } else if (incr) {
            inc_pull_valid = false;
            inc_hist_level = -1;
        }
        if (dual) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_level[2 * level], ev_level[2 * level + 1]);
            dual_pull = level > 0 ? ms : 0;
            if (level == 0) dual_push = ms;
            dual_ms.push_back({dual_push, dual_pull});
        }
        h_ctr[level].dir = dir;
        if (h_ctr[level].error) {
            level++;
            break;
        }
        prev_nf = nf;
        nf = h_ctr[level].next;
        mf = h_ctr[level].next_edges;
        vis_n += nf;
        vis_e += mf;
        cur ^= 1;
        level++;
    }
    last_levels = level;
    if (nf > 0 && level == kMaxLevels && (uint64_t)level + 1 < unreached)
        return set_error(SCAPH_EUNSUPPORTED, "traversal deeper than %d levels", kMaxLevels);
    return SCAPH_OK;
}

int scaph_engine::build_graph()
{
    SCAPH_CUDA(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h_loop;
    SCAPH_CUDA(cudaGraphConditionalHandleCreate(&h_loop, graph, 1, cudaGraphCondAssignDefault));

    const size_t np = g->pages.size();
    gargs.base = base_state(d_depth, nullptr);
    gargs.bm3 = d_bm3;
    gargs.ctr0 = d_ctr;
    // the per-page histogram of each level's discoveries (get_page_info's
    // counts) costs ~3% of a resident traversal: recorded in graph mode only
    // for the learned direction (its features) or on request
    gargs.hist0 = graph_records_hist() ? d_hist : nullptr;
    gargs.hist_levels = kHistLevels;
    gargs.npages_h = (uint32_t)np;
    gargs.ctl = d_ctl;
    dargs.E = E;
    dargs.dead_edges = dead_edges;
    dargs.dead = n_dead;
    dargs.dead_bm = d_dead;
    dargs.V = V;
    dargs.unreached = unreached;
    dargs.mode = cfg.direction == SCAPH_DIR_PUSH ? 1 : cfg.direction == SCAPH_DIR_PULL ? 2 : 0;
    dargs.alpha = cfg.alpha;
    dargs.beta = cfg.beta;
    dargs.max_levels = kMaxLevels;
    dargs.gather_ratio = (uint32_t)cfg.pull_gather_ratio;
    dargs.defer_edges = cfg.push_defer_edges > 0 ? (unsigned long long)cfg.push_defer_edges : 0ull;
    dargs.pull_records = cfg.pull_records;
    dargs.push_sparse_ratio = cfg.push_sparse_ratio;
    dargs.pull_gather_mode = cfg.pull_runs == 2 ? 1u : 2u;

    // init (run inputs are this node's arguments, replaced per launch)
    uint32_t *depth0 = d_depth, *parent0 = nullptr, src0 = 0, unr = unreached, nclear = kMaxLevels;
    const uint32_t *dead = d_dead;
    void *init_args[] = {&gargs, &depth0, &parent0, &src0, &unr, &dead, &nclear};
    cudaKernelNodeParams kp{};
    kp.func = const_cast<void *>(graph_init_kernel());
    kp.gridDim = dim3(num_sms * 4);
    kp.blockDim = dim3(256);
    kp.kernelParams = init_args;
    // (the init node also writes the source's depth, parent and bits)
    SCAPH_CUDA(cudaGraphAddKernelNode(&n_init, graph, nullptr, 0, &kp));

    // WHILE(loop) { push; giant; pull; decide }: the level kernel the level's
    // direction does not select leaves at once (cheaper than IF nodes)
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h_loop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t n_while;
    SCAPH_CUDA(cudaGraphAddNode(&n_while, graph, &n_init, 1, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];

    const void *f_push, *f_giant, *f_pull, *f_giant_pull;
    level_graph_kernels(block, &f_push, &f_giant, &f_pull, &f_giant_pull);
    GraphDev gout = dout.view, gpull = gin();
    void *push_args[] = {&gout, &gargs};
    cudaGraphNode_t n_push, n_pull;
    cudaKernelNodeParams lp{};
    lp.func = const_cast<void *>(f_push);
    lp.gridDim = dim3(grid_push);
    lp.blockDim = dim3(block);
    lp.kernelParams = push_args;
    SCAPH_CUDA(cudaGraphAddKernelNode(&n_push, body, nullptr, 0, &lp));
    void *fin_args[] = {&gargs};
    cudaKernelNodeParams fp{};
    fp.func = const_cast<void *>(push_finalize_graph_kernel(block));
    fp.gridDim = dim3(num_sms * 4);
    fp.blockDim = dim3(block);
    fp.kernelParams = fin_args;
    const bool learned = cfg.direction == SCAPH_DIR_LEARNED && sched;
#if SCAPH_GRAPH_GIANT_PULL
    // push; giant chunks or pull (one node); [finalize of deferred claims]
    void *giant_pull_args[] = {&gout, &gpull, &gargs};
    lp.func = const_cast<void *>(f_giant_pull);
    lp.gridDim = dim3(std::max(grid_push, grid_pull));
    lp.kernelParams = giant_pull_args;
    SCAPH_CUDA(cudaGraphAddKernelNode(&n_pull, body, &n_push, 1, &lp));
    if (cfg.push_defer_edges > 0) {
        cudaGraphNode_t n_fin;
        SCAPH_CUDA(cudaGraphAddKernelNode(&n_fin, body, &n_pull, 1, &fp));
        n_pull = n_fin;
    }
    (void)f_giant;
    (void)f_pull;
#else
    // push; giant chunks; [finalize of deferred claims]; pull
    (void)f_giant_pull;
    void *pull_args[] = {&gpull, &gargs};
    cudaGraphNode_t n_giant;
    lp.func = const_cast<void *>(f_giant);
    SCAPH_CUDA(cudaGraphAddKernelNode(&n_giant, body, &n_push, 1, &lp));
    cudaGraphNode_t n_before_pull = n_giant;
    if (cfg.push_defer_edges > 0) {
        cudaGraphNode_t n_fin;
        SCAPH_CUDA(cudaGraphAddKernelNode(&n_fin, body, &n_giant, 1, &fp));
        n_before_pull = n_fin;
    }
    lp.func = const_cast<void *>(f_pull);
    lp.gridDim = dim3(grid_pull);
    lp.kernelParams = pull_args;
    SCAPH_CUDA(cudaGraphAddKernelNode(&n_pull, body, &n_before_pull, 1, &lp));
#endif

    MlpDev net{};
    if (learned) mlp_device_view(sched, &net);
    void *dec_args[] = {&gargs, &dargs, &h_loop};
    void *dec_learned_args[] = {&gargs, &dargs, &net, &h_loop};
    cudaKernelNodeParams dp{};
    dp.func = const_cast<void *>(learned ? decide_learned_kernel() : decide_kernel());
    dp.gridDim = dim3(1);
    dp.blockDim = dim3(learned ? 64 : 1);
    dp.kernelParams = learned ? dec_learned_args : dec_args;
    cudaGraphNode_t n_decide;
    SCAPH_CUDA(cudaGraphAddKernelNode(&n_decide, body, &n_pull, 1, &dp));
    SCAPH_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
    return SCAPH_OK;
}

void scaph_engine::drop_graph()
{
    if (st) cudaStreamSynchronize(st);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (cap_st) cudaStreamDestroy(cap_st);
    gexec = nullptr;
    graph = nullptr;
    cap_st = nullptr;
}

int scaph_engine::launch_graph(uint32_t src, uint32_t *dd, uint32_t *dp)
{
    if (!gexec) {
        int rc = build_graph();
        if (rc) return rc;
    }
    uint32_t unr = unreached, nclear = kMaxLevels;
    const uint32_t *dead = d_dead;
    void *init_args[] = {&gargs, &dd, &dp, &src, &unr, &dead, &nclear};
    cudaKernelNodeParams kp{};
    kp.func = const_cast<void *>(graph_init_kernel());
    kp.gridDim = dim3(num_sms * 4);
    kp.blockDim = dim3(256);
    kp.kernelParams = init_args;
    SCAPH_CUDA(cudaGraphExecKernelNodeSetParams(gexec, n_init, &kp));
    SCAPH_CUDA(cudaGraphLaunch(gexec, st));
    return SCAPH_OK;
}

// Reads back the counters of the last run and rebuilds trace + stats.
int scaph_engine::collect(bool from_graph)
{
    const size_t np = g->pages.size();
    (void)np;
    if (from_graph) {
        SCAPH_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
        last_levels = (int)h_ctl->level + 1;
        SCAPH_CUDA(cudaMemcpyAsync(h_ctr, d_ctr, sizeof(LevelCounters) * last_levels, cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
    }
    const uint32_t src = pending_src;
    const bool dp = pending_parent;
    trace.clear();
    uint64_t nf = 1, mf = g->degree[src], vis_n = 1, vis_e = mf, insp = 0, alg = 0, launches = 0;
    int npush = 0, npull = 0;
    uint32_t err = 0;
    const bool src_dead = gt ? gt->degree[src] == 0 : g->degree[src] == 0;
    unsigned long long tprev = from_graph ? h_ctl->t_start : 0;
    launches = from_graph ? 1 : (dp ? 3 : 2);
    for (int l = 0; l < last_levels; l++) {
        const LevelCounters &lc = h_ctr[l];
        err |= lc.error;
        scaph_level_trace t{};
        t.level = l;
        t.direction = lc.dir;
        t.frontier = nf;
        t.frontier_edges = mf;
        const uint64_t used = vis_e + dead_edges;
        t.unvisited = (uint64_t)V - n_dead - vis_n + (src_dead ? 1 : 0);
        t.unvisited_edges = E > used ? E - used : 0;
        t.next = lc.next;
        t.edges_inspected = lc.inspected;
        // algorithmic bytes (push: headers + adjacency of the frontier;
        // pull: headers of unvisited vertices + in-edges up to the first
        // frontier hit; both: a V/8 bitmap pass and depth (+parent) writes)
        const uint64_t state_w = lc.next * (dp ? 8 : 4) + (uint64_t)nwords * 4;
        t.alg_bytes = lc.dir == 0 ? nf * 12 + mf * 4 + state_w : t.unvisited * 12 + lc.inspected * 4 + state_w;
        if (from_graph) {
            t.ms = (double)(lc.t_end - tprev) * 1e-6;
            tprev = lc.t_end;
            // push, giant + pull (one node), the finalize node when deferred
            // claims are on, and decide run every level; the unselected ones
            // leave at once
            launches += 1 + (SCAPH_GRAPH_GIANT_PULL ? 1 : 2) + (cfg.push_defer_edges > 0 ? 1 : 0) + 1;
        } else {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_level[2 * l], ev_level[2 * l + 1]);
            t.ms = ms;
            launches += (lc.dir == 0 ? 2 : 1) + lc.deferred;
            if ((size_t)l < level_h2d.size()) t.h2d_bytes = level_h2d[l];
            if ((size_t)l < dual_ms.size()) {
                t.push_ms = dual_ms[l].first;
                t.pull_ms = dual_ms[l].second;
            }
        }
        trace.push_back(t);
        alg += t.alg_bytes;
        insp += lc.inspected;
        if (lc.dir == 0) npush++; else npull++;
        nf = lc.next;
        mf = lc.next_edges;
        vis_n += nf;
        vis_e += mf;
    }
    memset(&last_stats, 0, sizeof(last_stats));
    last_stats.levels = last_levels;
    last_stats.push_levels = npush;
    last_stats.pull_levels = npull;
    last_stats.reached = vis_n;
    last_stats.reached_edges = vis_e;
    last_stats.edges_inspected = insp;
    last_stats.alg_bytes = alg;
    last_stats.launches = launches;
    if (pager && !from_graph) {
        uint64_t h2d, zc, f, pf, hits, lh;
        pager_counters(pager, &h2d, &zc, &f, &pf, &hits, &lh);
        last_stats.h2d_bytes = h2d;
        last_stats.zc_bytes = zc;
        last_stats.page_faults = f;
        last_stats.prefetched = pf;
        last_stats.pcie_alg_bytes = pcie_alg;
    }
    pending = false;
    if (err) return set_error(SCAPH_EDEVICE, "level kernel reported error flags 0x%x", err);
    // the level loop stops at kMaxLevels (the per-level counter records);
    // a frontier still left there means deeper vertices were not reached
    if (last_levels == kMaxLevels && nf > 0 && (uint64_t)last_levels + 1 < unreached)
        return set_error(SCAPH_EUNSUPPORTED, "traversal deeper than %d levels", kMaxLevels);
    return SCAPH_OK;
}

int scaph_engine::bfs(uint32_t src, uint32_t *depths, uint32_t *parents, int out_on_device, scaph_bfs_stats *stats)
{
    if (src >= V) return set_error(SCAPH_EINVAL, "source %u out of range (V=%u)", src, V);
    SCAPH_CUDA(cudaSetDevice(device));
    uint32_t *dd = (out_on_device && depths) ? depths : d_depth;
    uint32_t *dp = (out_on_device && parents) ? parents : (parents ? d_parent : nullptr);
    pending_src = src;
    pending_parent = dp != nullptr;
    const bool use_graph = graph_mode();
    last_hist = use_graph ? graph_records_hist() : host_records_hist();
    SCAPH_CUDA(cudaEventRecord(ev_start, st));
    int rc = use_graph ? launch_graph(src, dd, dp) : run_host_loop(src, dd, dp);
    if (rc) return rc;
    SCAPH_CUDA(cudaEventRecord(ev_stop, st));
    if (!out_on_device) {
        if (depths) SCAPH_CUDA(cudaMemcpyAsync(depths, dd, (size_t)V * 4, cudaMemcpyDeviceToHost, st));
        if (parents) SCAPH_CUDA(cudaMemcpyAsync(parents, dp, (size_t)V * 4, cudaMemcpyDeviceToHost, st));
    }
    if (use_graph && out_on_device && !stats) {
        pending = true;  // asynchronous: trace/stats read back on demand
        return SCAPH_OK;
    }
    rc = collect(use_graph);
    SCAPH_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        *stats = last_stats;
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_start, ev_stop);
        stats->ms = ms;
    }
    return rc;
}

// Pipelined traversal into host memory: run i writes device buffer i % 2 on
// the engine stream; its copy to the host runs on a second stream after the
// run, so it overlaps run i+1; run i+2 reuses the buffer once that copy is
// done.  Graph mode only (the traversal is one launch).
int scaph_engine::enqueue(uint32_t src, uint32_t *host_depths)
{
    if (src >= V) return set_error(SCAPH_EINVAL, "source %u out of range (V=%u)", src, V);
    if (!host_depths) return set_error(SCAPH_EINVAL, "null output");
    if (!graph_mode()) return set_error(SCAPH_EUNSUPPORTED, "pipelined runs need graph mode (resident graph)");
    SCAPH_CUDA(cudaSetDevice(device));
    if (!copy_st) {
        SCAPH_CUDA(cudaStreamCreateWithFlags(&copy_st, cudaStreamNonBlocking));
        for (int i = 0; i < 2; i++) {
            SCAPH_CUDA(cudaMalloc(&d_pipe[i], (size_t)V * 4));
            SCAPH_CUDA(cudaEventCreateWithFlags(&ev_run[i], cudaEventDisableTiming));
            SCAPH_CUDA(cudaEventCreateWithFlags(&ev_copied[i], cudaEventDisableTiming));
        }
    }
    const int b = (int)(pipe_runs & 1);
    SCAPH_CUDA(cudaStreamWaitEvent(st, ev_copied[b], 0));  // the buffer's previous copy is done
    pending_src = src;
    pending_parent = false;
    last_hist = graph_records_hist();
    int rc = launch_graph(src, d_pipe[b], nullptr);
    if (rc) return rc;
    pending = true;
    SCAPH_CUDA(cudaEventRecord(ev_run[b], st));
    SCAPH_CUDA(cudaStreamWaitEvent(copy_st, ev_run[b], 0));
    SCAPH_CUDA(cudaMemcpyAsync(host_depths, d_pipe[b], (size_t)V * 4, cudaMemcpyDeviceToHost, copy_st));
    SCAPH_CUDA(cudaEventRecord(ev_copied[b], copy_st));
    pipe_runs++;
    return SCAPH_OK;
}

extern "C" {

int scaph_bfs_enqueue(scaph_engine *e, uint32_t src, uint32_t *host_depths)
{
    clear_error();
    if (!e) return set_error(SCAPH_EINVAL, "null engine");
    return e->enqueue(src, host_depths);
}

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

int scaph_engine_set_scheduler(scaph_engine *e, scaph_mlp *m)
{
    if (!e) return set_error(SCAPH_EINVAL, "null engine");
    if (m) {
        int in = 0, out = 0;
        mlp_dims(m, &in, &out);
        const int np = (int)e->g->pages.size();
        if (in != SCAPH_SCHED_GLOBALS + np || out != 1 + np)
            return set_error(SCAPH_EINVAL, "scheduler network must be %d -> %d for this graph (is %d -> %d)",
                             SCAPH_SCHED_GLOBALS + np, 1 + np, in, out);
    }
    if (e->sched != m) e->drop_graph();  // the decide node embeds the network
    e->sched = m;
    return SCAPH_OK;
}

int scaph_bfs_features(scaph_engine *e, float *out, int cap, int *dim)
{
    if (!e) return set_error(SCAPH_EINVAL, "null engine");
    const int rows = e->feat_dim ? (int)(e->feat_log.size() / e->feat_dim) : 0;
    if (dim) *dim = e->feat_dim;
    if (out && cap > 0) memcpy(out, e->feat_log.data(), sizeof(float) * (size_t)std::min(cap, rows) * e->feat_dim);
    return rows;
}

int scaph_bfs_pull_pages(scaph_engine *e, int level, uint32_t *cnt, uint32_t *datas, int npages)
{
    if (!e || !cnt) return set_error(SCAPH_EINVAL, "null argument");
    if (level < 0 || level >= (int)e->pull_log.size()) return set_error(SCAPH_EINVAL, "level %d not recorded", level);
    const auto &v = e->pull_log[level];
    const int n = (int)v.size() / 2;
    if (npages < n) return set_error(SCAPH_EINVAL, "need %d pages", n);
    memcpy(cnt, v.data(), (size_t)n * 4);
    if (datas) memcpy(datas, v.data() + n, (size_t)n * 4);
    return n;
}

int scaph_engine_tune(scaph_engine *e, const scaph_config *c)
{
    clear_error();
    if (!e || !c) return set_error(SCAPH_EINVAL, "null argument");
    const int ge = c->giant_edges ? c->giant_edges : (int)kGiantEdges;
    if (ge < 128 || ge > 65536) return set_error(SCAPH_EINVAL, "giant_edges %d outside 128..65536", ge);
    if (c->block_size && c->block_size != 128 && c->block_size != 256 && c->block_size != 512)
        return set_error(SCAPH_EINVAL, "block_size %d not 128, 256 or 512", c->block_size);
    SCAPH_CUDA(cudaSetDevice(e->device));
    SCAPH_CUDA(cudaStreamSynchronize(e->st));
    e->drop_graph();  // the graph bakes in grid sizes and decision arguments
    scaph_config &k = e->cfg;
    k.alpha = c->alpha > 0 ? c->alpha : kAlphaDefault;
    k.beta = c->beta > 0 ? c->beta : kBetaDefault;
    k.giant_edges = ge;
    k.pull_gather_ratio = c->pull_gather_ratio > 0 ? c->pull_gather_ratio : (int32_t)kPullGatherRatio;
    k.ms_compact_l2_div = c->ms_compact_l2_div > 0 ? c->ms_compact_l2_div : 3;
    k.ms_compact_min_deg = c->ms_compact_min_deg > 0 ? c->ms_compact_min_deg : 16;
    k.ctas_per_sm = c->ctas_per_sm;
    k.push_defer_edges = c->push_defer_edges == 0 ? kDeferEdgesDefault : c->push_defer_edges;
    k.pull_warp = c->pull_warp >= 1 && c->pull_warp <= 3 ? c->pull_warp : 1;
    k.pull_records = c->pull_records >= 0 && c->pull_records <= 2 ? c->pull_records : 0;
    k.pull_rows = c->pull_rows >= 0 && c->pull_rows <= 2 ? c->pull_rows : 0;
    if (k.pull_rows == 1) {
        const int rc = e->build_prow();
        if (rc) return rc;
    }
    k.push_sparse_ratio = c->push_sparse_ratio == 0 ? (int32_t)kPushSparseRatio : c->push_sparse_ratio;
    k.pull_runs = c->pull_runs >= 0 && c->pull_runs <= 2 ? c->pull_runs : 0;
    e->block = c->block_size ? c->block_size : 256;
    const int occ_push = std::max(1, level_occupancy(0, e->block)), occ_pull = std::max(1, level_occupancy(1, e->block));
    e->grid_push = k.ctas_per_sm > 0 ? k.ctas_per_sm * e->num_sms : occ_push * e->num_sms;
    e->grid_pull = k.ctas_per_sm > 0 ? k.ctas_per_sm * e->num_sms : occ_pull * e->num_sms;
    const uint64_t cut = std::min<uint64_t>((uint64_t)ge, kGiantEdges);
    const uint32_t cap = (uint32_t)std::min<uint64_t>(0xFFFFFFF0u, 2 * (e->E / cut) + 1024);
    if (cap > e->giant_cap) {
        cudaFree(e->d_giant);
        e->d_giant = nullptr;
        e->giant_cap = 0;
        SCAPH_CUDA(cudaMalloc(&e->d_giant, sizeof(scaph::GiantChunk) * (size_t)cap));
        e->giant_cap = cap;
    }
    return SCAPH_OK;
}

int scaph_engine_evict_all(scaph_engine *e)
{
    if (!e) return set_error(SCAPH_EINVAL, "null engine");
    if (e->pager) {
        SCAPH_CUDA(cudaStreamSynchronize(e->st));
        pager_evict_all(e->pager);
    }
    return SCAPH_OK;
}

int scaph_engine_sync(scaph_engine *e)
{
    if (!e) return set_error(SCAPH_EINVAL, "null engine");
    SCAPH_CUDA(cudaStreamSynchronize(e->st));
    if (e->copy_st) SCAPH_CUDA(cudaStreamSynchronize(e->copy_st));
    return SCAPH_OK;
}

int scaph_bfs_trace(scaph_engine *e, scaph_level_trace *out, int cap)
{
    if (!e || (!out && cap > 0)) return set_error(SCAPH_EINVAL, "null argument");
    if (e->pending) {
        int rc = e->collect(true);
        if (rc) return rc;
    }
    int n = std::min<int>(cap, (int)e->trace.size());
    for (int i = 0; i < n; i++) out[i] = e->trace[i];
    return n;
}

int scaph_bfs_page_hist(scaph_engine *e, int level, uint32_t *nodes, uint32_t *datas, int npages)
{
    if (!e || !nodes || !datas) return set_error(SCAPH_EINVAL, "null argument");
    if (e->pending) {
        int rc = e->collect(true);
        if (rc) return rc;
    }
    const int np = (int)e->g->pages.size();
    if (npages < np) return set_error(SCAPH_EINVAL, "need %d pages", np);
    if (!e->last_hist)
        return set_error(SCAPH_EUNSUPPORTED, "resident runs record page histograms only with record_features "
                                             "or the learned direction");
    // histogram slot L holds the frontier discovered BY level L, i.e. the
    // frontier AT level L+1 (level 0's frontier is the source alone)
    if (level < 0 || level > e->last_levels || level > scaph_engine::kHistLevels)
        return set_error(SCAPH_EINVAL, "level %d not recorded", level);
    if (level == 0) {
        memset(nodes, 0, sizeof(uint32_t) * np);
        memset(datas, 0, sizeof(uint32_t) * np);
        return SCAPH_OK;
    }
    const uint32_t *h = e->d_hist + (size_t)(level - 1) * 2 * np;
    SCAPH_CUDA(cudaMemcpy(nodes, h, sizeof(uint32_t) * np, cudaMemcpyDeviceToHost));
    SCAPH_CUDA(cudaMemcpy(datas, h + np, sizeof(uint32_t) * np, cudaMemcpyDeviceToHost));
    return SCAPH_OK;
}

void *scaph_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (injected_fault(kFaultPinnedAlloc) != cudaSuccess || cudaMallocHost(&p, bytes) != cudaSuccess) {
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
