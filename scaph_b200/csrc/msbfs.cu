// Multi-source BFS (scaph_msbfs): up to 128 single-source BFS traversals
// share one pass over the edges, one bit per source in per-vertex masks (the
// device side is in ms_kernels.cuh).  No reference counterpart: the
// reference runs one source per App::run (src/app.cuh:220-265,
// app/bfs.cu:137-140).  This file is the host loop: one launch per phase and
// level, the direction rule between levels, depths unpacked at the end into
// u32 depth[i][V], bit-exact with single-source BFS.
#include <chrono>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.h"
#include "kernel_common.cuh"

#include "ms_kernels.cuh"

namespace scaph {

struct MsState {
    int nw = 0;
    uint32_t V = 0;
    unsigned long long *sa = nullptr, *visit[2] = {nullptr, nullptr};
    unsigned long long *planes[kMsPlanes] = {};
    uint32_t *act[2] = {nullptr, nullptr}, *touched = nullptr, *inc = nullptr, *inc0 = nullptr;
    uint2 *actrank = nullptr;            // pull levels: {act word, rank} per bitmap word
    unsigned long long *fmask = nullptr;  // pull levels: the frontier masks in rank order
    uint32_t *rank_sums = nullptr;        // frontier vertices per run of bitmap words
    MsCounters *d_ctr = nullptr, *h_ctr = nullptr;
    uint32_t *d_src = nullptr;  // the batch's sources (SCAPH_MSBFS_MAX entries)
    uint32_t *out = nullptr;  // internal depth output [128][V] when the caller wants host memory
    size_t out_words = 0;
    std::vector<scaph_level_trace> trace;
    std::vector<uint64_t> h2d;  // out of core: page bytes copied or read zero-copy per level
    uint32_t *d_pc = nullptr, *h_pc = nullptr;  // resident page census: counts then words, per graph
};

void ms_release(MsState *m)
{
    if (!m) return;
    cudaFree(m->sa);
    cudaFree(m->visit[0]);
    cudaFree(m->visit[1]);
    for (auto p : m->planes) cudaFree(p);
    cudaFree(m->act[0]);
    cudaFree(m->act[1]);
    cudaFree(m->touched);
    cudaFree(m->inc);
    cudaFree(m->inc0);
    cudaFree(m->actrank);
    cudaFree(m->fmask);
    cudaFree(m->rank_sums);
    cudaFree(m->d_ctr);
    cudaFreeHost(m->h_ctr);
    cudaFree(m->d_src);
    cudaFree(m->out);
    cudaFree(m->d_pc);
    cudaFreeHost(m->h_pc);
    delete m;
}

}  // namespace scaph

using namespace scaph;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

int ms_alloc(scaph_engine *e, int nw)
{
    MsState *m = e->ms;
    if (m && m->nw >= nw) return SCAPH_OK;
    if (m) {
        ms_release(m);
        e->ms = nullptr;
    }
    m = new MsState();
    e->ms = m;
    m->nw = nw;
    m->V = e->V;
    const size_t mw = (size_t)e->V * nw * 8;
    SCAPH_CUDA(cudaMalloc(&m->sa, 2 * mw));
    SCAPH_CUDA(cudaMalloc(&m->visit[0], mw));
    SCAPH_CUDA(cudaMalloc(&m->visit[1], mw));
    SCAPH_CUDA(cudaMalloc(&m->act[0], (size_t)e->nwords * 4));
    SCAPH_CUDA(cudaMalloc(&m->act[1], (size_t)e->nwords * 4));
    SCAPH_CUDA(cudaMalloc(&m->touched, (size_t)e->nwords * 4));
    SCAPH_CUDA(cudaMemset(m->touched, 0, (size_t)e->nwords * 4));
    SCAPH_CUDA(cudaMalloc(&m->inc, (size_t)e->nwords * 4));
    SCAPH_CUDA(cudaMalloc(&m->inc0, (size_t)e->nwords * 4));
    SCAPH_CUDA(cudaMalloc(&m->actrank, (size_t)e->nwords * sizeof(uint2)));
    SCAPH_CUDA(cudaMalloc(&m->fmask, mw));
    SCAPH_CUDA(cudaMalloc(&m->rank_sums, ((size_t)e->nwords / kRankWordsPerCta + 1) * 4));
    // vertices that can be incomplete: everything except the ones no edge
    // reaches (those only ever hold their own source bit)
    std::vector<uint32_t> dead(e->nwords);
    SCAPH_CUDA(cudaMemcpy(dead.data(), e->d_dead, (size_t)e->nwords * 4, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < e->nwords; i++) dead[i] = ~dead[i];
    if (e->V & 31) dead[e->nwords - 1] &= (1u << (e->V & 31)) - 1u;
    SCAPH_CUDA(cudaMemcpy(m->inc0, dead.data(), (size_t)e->nwords * 4, cudaMemcpyHostToDevice));
    SCAPH_CUDA(cudaMalloc(&m->d_src, sizeof(uint32_t) * SCAPH_MSBFS_MAX));
    SCAPH_CUDA(cudaMalloc(&m->d_ctr, sizeof(MsCounters) * kMaxLevels));
    SCAPH_CUDA(cudaMallocHost(&m->h_ctr, sizeof(MsCounters) * kMaxLevels));
    const size_t npmax = std::max(e->g->pages.size(), e->gt ? e->gt->pages.size() : 0) + 1;
    SCAPH_CUDA(cudaMalloc(&m->d_pc, 2 * npmax * 4));
    SCAPH_CUDA(cudaMallocHost(&m->h_pc, 2 * npmax * 4));
    return SCAPH_OK;
}

}  // namespace

// Page census of one multi-source level: the out-pages holding frontier
// vertices (what a push reads) and the in-pages holding incomplete vertices
// (what a pull reads), with counts and active words sum(deg+3).
struct MsLevelPages {
    std::vector<int> push_need, pull_need;
    std::vector<uint32_t> push_datas, pull_datas, push_cnt, pull_cnt;
    uint64_t incomplete = 0;
};

// Resident graphs count on the engine's own buffers; out of core the pager
// counts (and later reuses the result for the level it runs).
static int ms_level_pages(scaph_engine *e, const uint32_t *act, const uint32_t *inc, int grid, MsLevelPages &lp)
{
    const int gin = e->symmetric ? 0 : 1;
    for (int d = 0; d < 2; d++) {
        const uint32_t *bits = d == 0 ? act : inc;
        const uint32_t *deg = d == 0 || !e->d_indeg ? e->d_degree : e->d_indeg;
        std::vector<int> &need = d == 0 ? lp.push_need : lp.pull_need;
        std::vector<uint32_t> &datas = d == 0 ? lp.push_datas : lp.pull_datas;
        std::vector<uint32_t> &cnt = d == 0 ? lp.push_cnt : lp.pull_cnt;
        if (e->pager) {
            int rc = pager_page_counts(e->pager, d == 0 ? 0 : gin, bits, false, deg, 1, grid, e->st, need, datas, &cnt);
            if (rc) return rc;
        } else {
            const GraphDev &gv = d == 0 ? e->dout.view : e->gin();
            const int np = (int)gv.npages;
            MsState *m = e->ms;
            SCAPH_CUDA(page_counts(gv, bits, false, deg, 1, m->d_pc, m->d_pc + np, grid, e->st));
            SCAPH_CUDA(cudaMemcpyAsync(m->h_pc, m->d_pc, 2ull * np * 4, cudaMemcpyDeviceToHost, e->st));
            SCAPH_CUDA(cudaStreamSynchronize(e->st));
            cnt.assign(m->h_pc, m->h_pc + np);
            datas.assign(m->h_pc + np, m->h_pc + 2 * np);
            need.clear();
            for (int p = 0; p < np; p++)
                if (cnt[p]) need.push_back(p);
        }
    }
    lp.incomplete = 0;
    for (uint32_t c : lp.pull_cnt) lp.incomplete += c;
    return SCAPH_OK;
}

// Page traffic (ms at the link bandwidth) of a push and of a pull level.
static void ms_transfer_ms(scaph_engine *e, const MsLevelPages &lp, double &t_push, double &t_pull)
{
    const int gin = e->symmetric ? 0 : 1;
    t_push = pager_transfer_ms(e->pager, 0, lp.push_cnt.data(), lp.push_datas.data(), (int)lp.push_cnt.size(),
                               e->cfg.compact_threshold);
    t_pull = pager_transfer_ms(e->pager, gin, lp.pull_cnt.data(), lp.pull_datas.data(), (int)lp.pull_cnt.size(),
                               e->cfg.compact_threshold);
}

// One out-of-core level: push sends from the pages holding frontier
// vertices (giant chunks after each page batch, whose pool they address),
// then one finalize; pull reads the in-pages holding incomplete vertices.
template <int NW>
static int ms_ooc_level(scaph_engine *e, const MsDev &s, int dir, int level, int grid, uint64_t &launches,
                        std::vector<uint64_t> &h2d, const MsLevelPages *lp)
{
    cudaStream_t st = e->st;
    const int gid = (dir == 0 || e->symmetric) ? 0 : 1;
    std::vector<int> needed;
    std::vector<uint32_t> datas;
    int rc = SCAPH_OK;
    if (lp) {
        needed = dir == 0 ? lp->push_need : lp->pull_need;
        datas = dir == 0 ? lp->push_datas : lp->pull_datas;
    } else {
        rc = pager_page_counts(e->pager, gid, dir == 0 ? s.act_cur : s.inc, false,
                               dir == 0 || !e->d_indeg ? e->d_degree : e->d_indeg, 1, grid, st, needed, datas);
        if (rc) return rc;
    }
    PageLaunch fn;
    fn.run = [&](const GraphDev &gv, int, const RangeList &rl, uint32_t, cudaStream_t cs) -> int {
        if (dir == 0) {
            k_ms_push<NW><<<grid, kMsBlock, 0, cs>>>(gv, s, rl);
            k_ms_push_giant<NW><<<grid, kMsBlock, 0, cs>>>(gv, s);
            SCAPH_CUDA(cudaMemsetAsync(&s.ctr->giant, 0, sizeof(unsigned int), cs));
            launches += 2;
        } else {
            k_ms_pull<NW><<<grid, kMsBlock, 0, cs>>>(gv, s, rl);
            launches += 1;
        }
        SCAPH_CUDA(cudaGetLastError());
        return SCAPH_OK;
    };
    e->pcie_alg += 4 * pager_missing_words(e->pager, gid, needed, datas);
    uint64_t h0, z0, f0, pf, hits, lh;
    pager_counters(e->pager, &h0, &z0, &f0, &pf, &hits, &lh);
    if ((rc = pager_run_level(e->pager, gid, needed, datas, e->cfg.compact_threshold, fn, st))) return rc;
    if (dir == 0) {
        k_ms_finalize<NW><<<grid, kMsBlock, 0, st>>>(s);
        launches += 1;
    }
    uint64_t h1, z1, f1;
    pager_counters(e->pager, &h1, &z1, &f1, &pf, &hits, &lh);
    if ((size_t)level >= h2d.size()) h2d.resize(level + 1, 0);
    h2d[level] = (h1 - h0) + (z1 - z0);
    return SCAPH_OK;
}

template <int NW>
static int ms_run(scaph_engine *e, const uint32_t *srcs, int nsrc, uint32_t *out, scaph_bfs_stats *stats)
{
    MsState *m = e->ms;
    cudaStream_t st = e->st;
    const uint32_t V = e->V;
    const size_t mw = (size_t)V * NW * 8;
    MsDev s{};
    s.sa = m->sa;
    s.touched = m->touched;
    s.inc = m->inc;
    s.degree = e->d_degree;
    s.giant = e->d_giant;
    s.giant_cap = e->giant_cap;
    s.V = V;
    s.nwords = e->nwords;
    s.all[0] = nsrc >= 64 ? ~0ull : ((1ull << nsrc) - 1);
    s.all[1] = nsrc > 64 ? (nsrc >= 128 ? ~0ull : ((1ull << (nsrc - 64)) - 1)) : 0ull;
    s.head = e->d_head;
    s.indeg = e->d_indeg;
    s.head_ranked = e->head_ranked ? 1u : 0u;
    s.dyn_tiles = e->pager ? 0u : 1u;  // resident: one pull launch per level
    for (int k = 0; k < kMsPlanes; k++) s.planes[k] = m->planes[k];

    uint32_t *d_src = m->d_src;
    SCAPH_CUDA(cudaEventRecord(e->ev_start, st));
    SCAPH_CUDA(cudaMemcpyAsync(d_src, srcs, (size_t)nsrc * 4, cudaMemcpyHostToDevice, st));
    SCAPH_CUDA(cudaMemsetAsync(m->sa, 0, 2 * mw, st));
    SCAPH_CUDA(cudaMemsetAsync(m->act[0], 0, (size_t)e->nwords * 4, st));
    SCAPH_CUDA(cudaMemcpyAsync(m->inc, m->inc0, (size_t)e->nwords * 4, cudaMemcpyDeviceToDevice, st));
    SCAPH_CUDA(cudaMemsetAsync(m->d_ctr, 0, sizeof(MsCounters) * kMaxLevels, st));
    s.visit_cur = m->visit[0];
    s.act_cur = m->act[0];
    s.ctr = m->d_ctr;
    k_ms_clear_sources<NW><<<(nsrc + 127) / 128, 128, 0, st>>>(s, d_src, nsrc);
    k_ms_sources<NW><<<(nsrc + 127) / 128, 128, 0, st>>>(s, d_src, nsrc);
    SCAPH_CUDA(cudaGetLastError());

    const int grid = e->num_sms * 4;
    const float alpha = e->cfg.alpha, beta = e->cfg.beta;
    int l2_attr = 0;
    cudaDeviceGetAttribute(&l2_attr, cudaDevAttrL2CacheSize, e->device);
    const uint64_t l2_bytes = l2_attr > 0 ? (uint64_t)l2_attr : (126ull << 20);
    uint64_t nf = 0, prev_nf = 0, mf = 0, done_e = e->dead_edges;
    {
        // frontier of level 0: the distinct sources
        std::vector<uint32_t> hs(srcs, srcs + nsrc);
        std::sort(hs.begin(), hs.end());
        hs.erase(std::unique(hs.begin(), hs.end()), hs.end());
        nf = hs.size();
        for (uint32_t v : hs) mf += e->g->degree[v];
    }
    uint64_t pairs = (uint64_t)nsrc, insp = 0, alg = 0, launches = 2;
    int dir = 0, cur = 0, level = 0, npush = 0, npull = 0, planes_used = 0;
    uint32_t err = 0;
    m->trace.clear();
    m->h2d.clear();
    if (e->pager) pager_reset_counters(e->pager);
    e->pcie_alg = 0;
    // The learned scheduler (SCAPH_DIR_LEARNED with a network set): before
    // every level the same feature row as the single-source loop (16 globals,
    // then the frontier's share of every out-page, counted over the union of
    // the batch's frontiers) goes through the network.  Out of core its
    // direction logit marks the push levels that lead into the pull levels,
    // during which the in-pages the first pull level reads are prefetched
    // into free pool slots.  Without a network, the exact page traffic of
    // either direction overrides alpha/beta where one side clearly
    // dominates.  The rows are kept (scaph_bfs_features) with
    // record_features.
    const bool learned = e->cfg.direction == SCAPH_DIR_LEARNED;
    const bool net_on = learned && e->sched;
    const bool want_feat = net_on || e->cfg.record_features;
    const size_t np = e->g->pages.size();
    const int feat_dim = SCAPH_SCHED_GLOBALS + (int)np;
    std::vector<float> f(feat_dim), y;
    e->feat_log.clear();
    e->feat_dim = want_feat ? feat_dim : 0;
    if (net_on) {
        int rc = mlp_host_snapshot(e->sched, e->sched_host);
        if (rc) return rc;
        int in = 0, out_dim = 0;
        mlp_dims(e->sched, &in, &out_dim);
        y.resize(out_dim);
    }
    uint64_t npref = 0;
    std::vector<double> host_ms;  // per level: census and decisions on the host
    while (nf > 0 && level < kMaxLevels && (uint64_t)level + 1 < e->unreached) {
        const auto h0 = std::chrono::steady_clock::now();
        const uint64_t mu = e->E > done_e ? e->E - done_e : 0;
        const int prev_dir = dir;
        const int ab = level == 0 ? 0 : alpha_beta_next(dir, nf, prev_nf, mf, mu, V, alpha, beta);
        switch (e->cfg.direction) {
        case SCAPH_DIR_PUSH: dir = 0; break;
        case SCAPH_DIR_PULL: dir = level == 0 ? 0 : 1; break;
        default: dir = ab; break;
        }
        MsLevelPages lp;
        const bool census = want_feat || (e->pager && learned && level > 0);
        std::vector<int> prefetch_pages;
        if (census) {
            int rc = ms_level_pages(e, m->act[cur], m->inc, grid, lp);
            if (rc) return rc;
            launches += 2;
        }
        if (want_feat) {
            sched_globals(f.data(), nf, mf, lp.incomplete, mu, V, e->E, level, prev_dir);
            float res_out = 1.f, res_in = 1.f, res_push = 1.f, res_pull = 1.f;
            if (e->pager) {
                const int gin = e->symmetric ? 0 : 1;
                res_out = pager_resident_fraction(e->pager, 0, nullptr);
                res_in = pager_resident_fraction(e->pager, gin, nullptr);
                res_push = pager_resident_fraction(e->pager, 0, &lp.push_need);
                res_pull = pager_resident_fraction(e->pager, gin, &lp.pull_need);
            }
            f[10] = res_out;
            f[11] = res_in;
            f[12] = res_push;
            f[13] = res_pull;
            f[14] = (float)ab;
            f[15] = 1.f;
            for (size_t p = 0; p < np; p++)
                f[SCAPH_SCHED_GLOBALS + p] = (float)lp.push_cnt[p] / (float)std::max(1u, e->g->pages[p].nodenum);
            e->feat_log.insert(e->feat_log.end(), f.begin(), f.end());
        }
        if (net_on) {
            // the network's direction output is trained on single-source
            // level costs, which a batch's levels do not share (a pull level
            // serves every source at once): the batch keeps alpha/beta for
            // direction and reads the logit as a sign that pull is near
            mlp_forward_host(e->sched_host, f.data(), y.data());
        }
        if (e->pager && learned && !net_on && level > 0) {
            // the exact page traffic each direction would cause overrides
            // the kernel-time choice when one side clearly dominates (not
            // with the network's prefetch: prefetched pages make a direction
            // look free of traffic - measured on config 5 with out-page
            // prefetch: 8 push levels, 0.77x of alpha/beta cold)
            double tp = 0, tq = 0;
            ms_transfer_ms(e, lp, tp, tq);
            if (tp > 2 * tq + 1.0) dir = 1;
            else if (tq > 2 * tp + 1.0) dir = 0;
        }
        if (net_on && e->pager && dir == 0) {
            // during a push level that leads into the pull levels: the
            // in-pages holding incomplete vertices (every one of them is
            // read whole by the first pull level) are copied into free
            // slots while this level runs, so that the link is busy during
            // the push levels.  The pull is expected next when the network
            // rates this level pull-worthy (its direction logit, trained on
            // single-source levels) or when alpha/beta, run on the frontier
            // grown at its last rate, would switch.  Out-pages the network
            // names are not prefetched: a batch's push levels read their
            // sparse out-pages zero-copy, so whole-page copies of them went
            // unused (config 5 cold: 189 pages, 7.9 GB moved for nothing,
            // 0.74x of alpha/beta)
            const double grow = prev_nf ? (double)nf / (double)prev_nf : 1.0;
            const double mf_next = (double)mf * std::max(1.0, grow);
            const double mu_next = std::max(0.0, (double)mu - mf_next);
            const bool pull_soon = y[0] > 0.f || mf_next * alpha > mu_next;
            if (pull_soon) {
                const int gin = e->symmetric ? 0 : 1;
                long long room = (long long)pager_free_slots(e->pager);
                for (int p : lp.push_need)
                    if (!pager_is_resident(e->pager, 0, p)) room--;
                for (int p : lp.pull_need) {
                    if (room <= 0) break;
                    if (pager_is_resident(e->pager, gin, p)) continue;
                    prefetch_pages.push_back(p);
                    room--;
                }
            }
        }
        const uint32_t d = (uint32_t)level + 1;
        for (int k = 0; k < kMsPlanes; k++) {
            if (!((d >> k) & 1u) || k < planes_used) continue;
            if (!m->planes[k]) SCAPH_CUDA(cudaMalloc(&m->planes[k], mw));
            SCAPH_CUDA(cudaMemsetAsync(m->planes[k], 0, mw, st));
            s.planes[k] = m->planes[k];
            planes_used = k + 1;
        }
        host_ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count());
        SCAPH_CUDA(cudaEventRecord(e->ev_level[2 * level], st));
        SCAPH_CUDA(cudaMemsetAsync(m->act[cur ^ 1], 0, (size_t)e->nwords * 4, st));
        s.visit_cur = m->visit[cur];
        s.visit_nxt = m->visit[cur ^ 1];
        s.act_cur = m->act[cur];
        s.act_nxt = m->act[cur ^ 1];
        s.ctr = m->d_ctr + level;
        s.level = (uint32_t)level;
        const RangeList whole{nullptr, nullptr, nullptr, 0};
        s.actrank = nullptr;
        s.fmask = nullptr;
        s.all_active = SCAPH_MS_ALL_ACTIVE && level > 0 && nf == V ? 1u : 0u;
        // the frontier's masks compacted in rank order, when that pays: they
        // fit a third of L2 (frontier vertices spread over the V-entry mask
        // array keep a sector each, which does not stay there), and the
        // frontier has 16+ out-edges per vertex, so that the pull looks masks
        // up many times per mask gathered (RMAT-25, 64 sources: the first
        // pull level 7.95 -> 6.19 ms; the larger frontiers after it lost)
        const bool compact = dir == 1 && nf * NW * 8 <= l2_bytes / (uint64_t)e->cfg.ms_compact_l2_div &&
                             mf >= (uint64_t)e->cfg.ms_compact_min_deg * nf;
        if (compact) {
            const uint32_t nb = (e->nwords + kRankWordsPerCta - 1) / kRankWordsPerCta;
            k_ms_rank_sums<<<nb, kMsBlock, 0, st>>>(s.act_cur, e->nwords, m->rank_sums);
            k_ms_rank_scan<<<1, kMsBlock, 0, st>>>(m->rank_sums, nb);
            k_ms_rank_gather<NW><<<nb, kMsBlock, 0, st>>>(s.act_cur, e->nwords, m->rank_sums, s.visit_cur,
                                                          m->actrank, m->fmask);
            SCAPH_CUDA(cudaGetLastError());
            s.actrank = m->actrank;
            s.fmask = m->fmask;
            s.all_active = 0u;  // the compacted masks are read by rank
            launches += 3;
        }
        if (e->pager) {
            // out of core: the pages holding frontier vertices (push) or
            // incomplete vertices (pull), in batches the pager makes ready
            // (resident, zero-copy, demand copies)
            int rc = ms_ooc_level<NW>(e, s, dir, level, grid, launches, m->h2d, census ? &lp : nullptr);
            if (rc) return rc;
            if (dir == 0) npush++; else npull++;
            if (!prefetch_pages.empty()) {
                // copies into free slots on the copy streams, behind this
                // level's own copies in the queue of the link
                if ((rc = pager_prefetch(e, e->pager, e->symmetric ? 0 : 1, prefetch_pages))) return rc;
                npref += prefetch_pages.size();
            }
        } else if (dir == 0) {
            k_ms_push<NW><<<grid, kMsBlock, 0, st>>>(e->dout.view, s, whole);
            k_ms_push_giant<NW><<<grid, kMsBlock, 0, st>>>(e->dout.view, s);
            k_ms_finalize<NW><<<grid, kMsBlock, 0, st>>>(s);
            launches += 3;
            npush++;
        } else {
            k_ms_pull<NW><<<grid, kMsBlock, 0, st>>>(e->gin(), s, whole);
            launches += 1;
            npull++;
        }
        SCAPH_CUDA(cudaGetLastError());
        SCAPH_CUDA(cudaEventRecord(e->ev_level[2 * level + 1], st));
        SCAPH_CUDA(cudaMemcpyAsync(m->h_ctr + level, m->d_ctr + level, sizeof(MsCounters), cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
        const MsCounters &c = m->h_ctr[level];
        err |= c.error;
        scaph_level_trace t{};
        t.level = level;
        t.direction = dir;
        t.frontier = nf;
        t.frontier_edges = mf;
        t.unvisited_edges = mu;
        t.next = c.active;
        t.edges_inspected = c.inspected;
        // algorithmic bytes of an MS-BFS level: headers + adjacency of the
        // vertices with a nonzero frontier mask (push) or the in-edges read
        // (pull), plus a read and a write of a mask per vertex
        t.alg_bytes = dir == 0 ? nf * 12 + mf * 4 + 2ull * NW * 8 * V : c.inspected * 4 + 2ull * NW * 8 * V;
        if ((size_t)level < m->h2d.size()) t.h2d_bytes = m->h2d[level];
        m->trace.push_back(t);
        alg += t.alg_bytes;
        insp += c.inspected;
        pairs += c.pairs;
        prev_nf = nf;
        nf = c.active;
        mf = c.active_edges;
        done_e += c.completed_edges;
        cur ^= 1;
        level++;
        if (err) break;
    }
    {
        uint32_t unr = e->unreached;
        int ns = nsrc;
        void *args[] = {&s, &out, &ns, &unr};
        SCAPH_CUDA(cudaLaunchKernel(ms_unpack_kernel<NW>(planes_used), dim3(grid), dim3(kMsBlock), args, 0, st));
    }
    launches += 1;
    SCAPH_CUDA(cudaEventRecord(e->ev_stop, st));
    SCAPH_CUDA(cudaEventSynchronize(e->ev_stop));
    for (int l = 0; l < level; l++) {
        float ms = 0, gap = 0;
        cudaEventElapsedTime(&ms, e->ev_level[2 * l], e->ev_level[2 * l + 1]);
        if (l > 0) cudaEventElapsedTime(&gap, e->ev_level[2 * l - 1], e->ev_level[2 * l]);
        m->trace[l].ms = ms;
        m->trace[l].push_ms = gap;
        m->trace[l].pull_ms = (size_t)l < host_ms.size() ? host_ms[l] : 0.0;
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev_start, e->ev_stop);
        stats->ms = ms;
        if (e->pager) {
            uint64_t h2d, zc, faults, pf, hits, lh;
            pager_counters(e->pager, &h2d, &zc, &faults, &pf, &hits, &lh);
            stats->h2d_bytes = h2d;
            stats->zc_bytes = zc;
            stats->page_faults = faults;
            stats->prefetched = pf;
            stats->pcie_alg_bytes = e->pcie_alg;
        }
        stats->levels = level;
        stats->push_levels = npush;
        stats->pull_levels = npull;
        stats->reached = pairs;
        stats->edges_inspected = insp;
        stats->alg_bytes = alg;
        stats->launches = launches;
    }
    if (err) return set_error(SCAPH_EDEVICE, "multi-source kernels reported error flags 0x%x", err);
    if (nf > 0 && level == kMaxLevels && (uint64_t)level + 1 < e->unreached)
        return set_error(SCAPH_EUNSUPPORTED, "traversal deeper than %d levels", kMaxLevels);
    return SCAPH_OK;
}

extern "C" int scaph_msbfs(scaph_engine *e, const uint32_t *srcs, int nsrc, uint32_t *depths, int out_on_device,
                           scaph_bfs_stats *stats)
{
    clear_error();
    if (!e || !srcs || !depths) return set_error(SCAPH_EINVAL, "null argument");
    if (nsrc < 1 || nsrc > SCAPH_MSBFS_MAX) return set_error(SCAPH_EINVAL, "nsrc %d outside 1..%d", nsrc, SCAPH_MSBFS_MAX);
    for (int i = 0; i < nsrc; i++)
        if (srcs[i] >= e->V) return set_error(SCAPH_EINVAL, "source %u out of range (V=%u)", srcs[i], e->V);
    SCAPH_CUDA(cudaSetDevice(e->device));
    const int nw = nsrc > 64 ? 2 : 1;
    int rc = ms_alloc(e, nw);
    if (rc) return rc;
    MsState *m = e->ms;
    uint32_t *out = depths;
    if (!out_on_device) {
        const size_t need = (size_t)nsrc * e->V;
        if (m->out_words < need) {
            cudaFree(m->out);
            m->out = nullptr;
            SCAPH_CUDA(cudaMalloc(&m->out, need * 4));
            m->out_words = need;
        }
        out = m->out;
    }
    rc = m->nw == 2 ? ms_run<2>(e, srcs, nsrc, out, stats) : ms_run<1>(e, srcs, nsrc, out, stats);
    if (rc) return rc;
    if (!out_on_device) {
        SCAPH_CUDA(cudaMemcpyAsync(depths, out, (size_t)nsrc * e->V * 4, cudaMemcpyDeviceToHost, e->st));
        SCAPH_CUDA(cudaStreamSynchronize(e->st));
    }
    return SCAPH_OK;
}

extern "C" int scaph_msbfs_trace(scaph_engine *e, scaph_level_trace *out, int cap)
{
    if (!e || (!out && cap > 0)) return set_error(SCAPH_EINVAL, "null argument");
    if (!e->ms) return 0;
    const int n = std::min<int>(cap, (int)e->ms->trace.size());
    for (int i = 0; i < n; i++) out[i] = e->ms->trace[i];
    return n;
}
