// Page store for App-hook engines: a paged graph (weighted or not) on the
// device for applications that bring their own vertex program - the
// cond/update hooks of the reference's apps (app/bfs_kernel.cuh,
// app/sssp_kernel.cuh, app/wcc_kernel.cuh) compiled into the application's
// own kernels by the compat App<> (include/scaph/compat/app.cuh).
//
// This replaces the part of App::load_graph / App::gpu_push_batch /
// App::PageCopy (src/app.cuh:267-468) that decides which pages a round needs
// and brings them into HBM: the store computes, from the device bitmap of
// active vertices, the pages holding them (get_page_info,
// src/gpu_engine.cuh:397-441) and hands the application batches of pages
// that are ready to read - all of them at once when the graph is resident,
// otherwise resident pages first, then sparse pages read zero-copy, then
// pages copied on demand (the same pager as the BFS engine).
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>

#include "engine.h"

using namespace scaph;

static_assert(sizeof(scaph_page_dev) == sizeof(PageDev), "scaph_page_dev mirrors PageDev");
static_assert(offsetof(scaph_page_dev, left) == offsetof(PageDev, left), "scaph_page_dev mirrors PageDev");

struct scaph_store {
    const Graph *g = nullptr;
    int device = 0;
    int compact_threshold = 3;
    int num_sms = 148;
    cudaStream_t st = nullptr;  // setup
    DeviceGraph dev;            // resident graph
    Pager *pager = nullptr;     // out of core
    uint32_t *d_deg = nullptr;
    uint32_t *d_full = nullptr;  // the single range [0, V) of a resident level
    uint64_t h2d = 0, zc = 0, faults = 0;

    ~scaph_store()
    {
        if (st) cudaStreamSynchronize(st);
        pager_release(pager);
        dev.release();
        cudaFree(d_deg);
        cudaFree(d_full);
        if (st) cudaStreamDestroy(st);
    }

    scaph_page_view to_view(const GraphDev &v) const
    {
        scaph_page_view o{};
        o.pool = v.pool;
        o.pages = reinterpret_cast<const scaph_page_dev *>(v.pages);
        o.coarse = v.coarse;
        o.cshift = v.cshift;
        o.npages = v.npages;
        o.V = v.V;
        o.pagesize = v.pagesize;
        o.weighted = (uint32_t)g->weighted;
        return o;
    }
};

extern "C" {

int scaph_store_create(const scaph_graph *g, int64_t pool_bytes, int compact_threshold, int copy_streams,
                       int device, scaph_store **out)
{
    clear_error();
    if (!g || !out) return set_error(SCAPH_EINVAL, "null argument");
    if (g->pages.empty() || g->V == 0) return set_error(SCAPH_EINVAL, "empty graph");
    *out = nullptr;
    SCAPH_CUDA(cudaSetDevice(device));
    std::unique_ptr<scaph_store> s(new scaph_store());
    s->g = g;
    s->device = device;
    s->compact_threshold = compact_threshold > 0 ? compact_threshold : 3;
    SCAPH_CUDA(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device));
    SCAPH_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
    const int np = (int)g->pages.size();
    const int64_t page_bytes = (int64_t)g->pagesize * 4;
    int nslots = np;
    if (pool_bytes > 0) nslots = (int)std::min<int64_t>(np, pool_bytes / page_bytes);
    if (nslots < 1) return set_error(SCAPH_EINVAL, "pool_bytes holds no page");
    SCAPH_CUDA(cudaMalloc(&s->d_deg, (size_t)g->V * 4));
    SCAPH_CUDA(cudaMemcpyAsync(s->d_deg, g->degree.data(), (size_t)g->V * 4, cudaMemcpyHostToDevice, s->st));
    SCAPH_CUDA(cudaMalloc(&s->d_full, 4 * 4));
    const uint32_t full[4] = {0, g->V, 0, ((g->V + 31) / 32 + 127) / 128};
    SCAPH_CUDA(cudaMemcpyAsync(s->d_full, full, sizeof(full), cudaMemcpyHostToDevice, s->st));
    int rc;
    if (nslots >= np) {
        if ((rc = s->dev.build(*g, np, s->st))) return rc;
    } else if ((rc = pager_create(g, nullptr, nslots, copy_streams, 0.f, &s->pager))) {
        return rc;
    }
    SCAPH_CUDA(cudaStreamSynchronize(s->st));
    *out = s.release();
    return SCAPH_OK;
}

int scaph_store_destroy(scaph_store *s)
{
    delete s;
    return SCAPH_OK;
}

int scaph_store_resident(const scaph_store *s) { return s && !s->pager ? 1 : 0; }

int scaph_store_view(const scaph_store *s, scaph_page_view *out)
{
    clear_error();
    if (!s || !out) return set_error(SCAPH_EINVAL, "null argument");
    if (s->pager) return set_error(SCAPH_EUNSUPPORTED, "out-of-core store: pages are handed out per level");
    *out = s->to_view(s->dev.view);
    return SCAPH_OK;
}

const uint32_t *scaph_store_degree(const scaph_store *s) { return s ? s->d_deg : nullptr; }

int scaph_store_level(scaph_store *s, const uint32_t *d_active, scaph_batch_fn fn, void *user, void *stream)
{
    clear_error();
    if (!s || !d_active || !fn) return set_error(SCAPH_EINVAL, "null argument");
    SCAPH_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!s->pager) {
        const uint32_t tiles = ((s->g->V + 31) / 32 + 127) / 128;
        const scaph_ranges r{s->d_full, s->d_full + 1, s->d_full + 2, 1, tiles};
        const scaph_page_view v = s->to_view(s->dev.view);
        const int rc = fn(user, &v, &r, stream);
        return rc ? set_error(rc, "batch callback failed (%d)", rc) : SCAPH_OK;
    }
    std::vector<int> needed;
    std::vector<uint32_t> datas;
    int rc = pager_page_counts(s->pager, 0, d_active, false, s->d_deg, s->g->weighted ? 2 : 1, s->num_sms * 4, st,
                               needed, datas);
    if (rc) return rc;
    if (needed.empty()) return SCAPH_OK;
    PageLaunch pl;
    pl.run = [&](const GraphDev &gv, int, const RangeList &rl, uint32_t tiles, cudaStream_t cs) -> int {
        const scaph_ranges r{rl.lo, rl.hi, rl.tile0, rl.n, tiles};
        const scaph_page_view v = s->to_view(gv);
        const int frc = fn(user, &v, &r, cs);
        return frc ? set_error(frc, "batch callback failed (%d)", frc) : SCAPH_OK;
    };
    uint64_t h0, z0, f0, pf, hits, lh;
    pager_counters(s->pager, &h0, &z0, &f0, &pf, &hits, &lh);
    rc = pager_run_level(s->pager, 0, needed, datas, s->compact_threshold, pl, st);
    uint64_t h1, z1, f1;
    pager_counters(s->pager, &h1, &z1, &f1, &pf, &hits, &lh);
    s->h2d += h1 - h0;
    s->zc += z1 - z0;
    s->faults += f1 - f0;
    return rc;
}

int scaph_store_counters(const scaph_store *s, uint64_t *h2d_bytes, uint64_t *zc_bytes, uint64_t *page_faults)
{
    if (!s) return set_error(SCAPH_EINVAL, "null argument");
    if (h2d_bytes) *h2d_bytes = s->h2d;
    if (zc_bytes) *zc_bytes = s->zc;
    if (page_faults) *page_faults = s->faults;
    return SCAPH_OK;
}

}  // extern "C"
