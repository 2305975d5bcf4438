// Engine internals shared by engine.cu and the other device-side modules.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <functional>
#include <vector>

#include "common.h"
#include "mlp_host.h"
#include "device.cuh"
#include "scaph/scaph.h"

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

struct MsState;  // multi-source BFS state (msbfs.cu)
void ms_release(MsState *m);

struct Pager;  // out-of-core page manager (pager.cu)
int coarse_index(const Graph &g, std::vector<uint32_t> &hc, uint32_t &cshift);

}  // namespace scaph

namespace scaph {
// Runs the kernels of one batch of resident (or zero-copy) pages: `view` is
// the graph's page table as the kernels must read it, `rl` the batch's
// vertex ranges; range i owns the tiles tile0[i].. of 128 bitmap words
// counted from its first word (`tiles` in all, see range_of_tile).
struct PageLaunch {
    std::function<int(const GraphDev &view, int gid, const RangeList &rl, uint32_t tiles, cudaStream_t st)> run;
};
int pager_create(const Graph *g, const Graph *gt, int nslots, int copy_streams, float link_gbs, Pager **out);
void pager_release(Pager *p);
const GraphDev &pager_view(const Pager *p, int gid);
int pager_needs(scaph_engine *e, Pager *pg, int dir, int level, uint32_t src, std::vector<int> &needed,
                std::vector<uint32_t> &datas);
int pager_run_level(scaph_engine *e, Pager *pg, int dir, const BfsDev &s, const std::vector<int> &needed,
                    const std::vector<uint32_t> &datas);
int pager_run_level(Pager *pg, int gid, const std::vector<int> &needed, const std::vector<uint32_t> &datas,
                    int compact_threshold, const PageLaunch &fn, cudaStream_t st);
int pager_prefetch(scaph_engine *e, Pager *pg, int gid, const std::vector<int> &pages);
// Pages of graph gid holding set bits of `bits` (invert: clear bits), with
// their words sum(deg*ew+3); synchronises st.
int pager_page_counts(Pager *pg, int gid, const uint32_t *bits, bool invert, const uint32_t *deg, uint32_t ew,
                      int grid, cudaStream_t st, std::vector<int> &needed, std::vector<uint32_t> &datas,
                      std::vector<uint32_t> *counts = nullptr);
void pager_counters(const Pager *pg, uint64_t *h2d, uint64_t *zc, uint64_t *faults, uint64_t *prefetched,
                    uint64_t *hits, uint64_t *level_h2d);
void pager_reset_counters(Pager *pg);
void pager_evict_all(Pager *pg);
int pager_nslots(const Pager *pg);
// Slots holding no page.
int pager_free_slots(const Pager *pg);
float pager_resident_fraction(const Pager *pg, int gid, const std::vector<int> *pages);
// Page p of graph gid holds a pool slot (copied, or being copied).
bool pager_is_resident(const Pager *pg, int gid, int p);
// Active words sum(deg*ew+3) of the needed pages that are not resident: the
// least a level must bring over the link (get_page_info's `datas`,
// src/gpu_engine.cuh:413-419, over the pages the pool lacks).
uint64_t pager_missing_words(const Pager *pg, int gid, const std::vector<int> &needed,
                             const std::vector<uint32_t> &datas);
// Page traffic (ms at the measured PCIe bandwidth) a level would cause on
// graph gid: per page with cnt > 0, nothing if resident, its active words
// if sparse enough for zero-copy reads, else a full page copy.
double pager_transfer_ms(const Pager *pg, int gid, const uint32_t *cnt, const uint32_t *datas, int npages,
                         int compact_threshold);
cudaError_t page_unvisited(const GraphDev &g, const uint32_t *visited, const uint32_t *indeg, uint32_t *cnt,
                           uint32_t *datas, int grid, cudaStream_t st);
cudaError_t page_counts(const GraphDev &g, const uint32_t *bits, bool invert, const uint32_t *deg, uint32_t ew,
                        uint32_t *cnt, uint32_t *datas, int grid, cudaStream_t st);
void sched_globals(float *f, uint64_t nf, uint64_t mf, uint64_t unvis, uint64_t mu, uint32_t V, uint64_t E, int level,
                   int prev_dir);
int mlp_forward_device(scaph_mlp *m, const float *hX, int n, float *hY);
int mlp_dims(const scaph_mlp *m, int *in, int *out);
int mlp_device_view(const scaph_mlp *m, MlpDev *v);
int mlp_forward1(scaph_mlp *m, const float *hX, float *hY, cudaStream_t st);
int mlp_host_snapshot(const scaph_mlp *m, MlpHost &h);
}  // namespace scaph

// The engine behind the opaque C-ABI handle.
struct scaph_engine {
    using DeviceGraph = scaph::DeviceGraph;
    using Graph = scaph::Graph;
    using LevelCounters = scaph::LevelCounters;
    using GiantChunk = scaph::GiantChunk;
    using BfsCtl = scaph::BfsCtl;
    using BfsGraphArgs = scaph::BfsGraphArgs;
    using DecideArgs = scaph::DecideArgs;
    using BfsDev = scaph::BfsDev;
    using GraphDev = scaph::GraphDev;

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

    uint32_t *d_depth = nullptr, *d_parent = nullptr, *d_visited = nullptr, *d_bm3 = nullptr;
    uint32_t *d_degree = nullptr, *d_dead = nullptr;
    uint64_t n_dead = 0, dead_edges = 0;
    LevelCounters *d_ctr = nullptr, *h_ctr = nullptr;
    uint32_t *d_hist = nullptr;  // [kHistLevels][2][npages]
    GiantChunk *d_giant = nullptr;
    uint32_t giant_cap = 0;
    BfsCtl *d_ctl = nullptr, *h_ctl = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_dual[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> ev_level;

    // graph mode
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraphNode_t n_init = nullptr;
    cudaStream_t cap_st = nullptr;
    BfsGraphArgs gargs{};
    DecideArgs dargs{};

    // last run
    std::vector<scaph_level_trace> trace;
    int last_levels = 0;
    bool pending = false;  // a graph-mode run whose trace has not been read back
    uint32_t pending_src = 0;
    bool pending_parent = false;
    scaph_bfs_stats last_stats{};

    scaph::MsState *ms = nullptr;  // allocated by the first scaph_msbfs call
    scaph::Pager *pager = nullptr;  // out-of-core mode: pool smaller than the graph
    uint32_t *d_indeg = nullptr;    // in-degree per vertex (pull page statistics)
    uint32_t *d_head = nullptr;     // kPullHead in-edges per vertex (pull phase A)
    uint2 *d_prec = nullptr;        // 8-byte pull record per vertex (pull phase A)
    uint4 *d_prow = nullptr;        // 16-byte pull row per vertex (phase A without records)
    uint32_t *d_live_rank = nullptr;  // live vertices before each bitmap word (nwords + 1)
    uint4 *d_live_head = nullptr;     // head rows of the live vertices, by live rank
    uint32_t *d_live_indeg = nullptr; // in-degrees of the live vertices, by live rank
    uint32_t *d_live_deg = nullptr;   // out-degrees of the live vertices, by live rank
    uint2 *d_live_prec = nullptr;     // 8-byte pull records of the live vertices, by live rank
    bool head_ranked = false;       // d_head holds the top in-neighbours by out-degree
    std::vector<uint64_t> level_h2d;  // page bytes copied per level of the last run
    uint64_t pcie_alg = 0;            // algorithmic link bytes of the last run
    scaph_bfs_stats pager_stats{};
    // learned scheduler / training traces
    scaph_mlp *sched = nullptr;
    scaph::MlpHost sched_host;  // snapshot of sched taken at each host-loop run
    std::vector<float> feat_log;                    // levels x feat_dim
    int feat_dim = 0;
    std::vector<std::vector<uint32_t>> pull_log;    // unvisited per in-page, per level
    std::vector<std::pair<double, double>> dual_ms; // (push, pull) per level
    uint32_t *d_snap = nullptr, *d_pcnt = nullptr, *d_pdatas = nullptr;
    uint32_t *h_fstage = nullptr;  // pinned: the feature pass's page counts
    // pipelined host output (scaph_bfs_enqueue): two device depth buffers,
    // a copy stream, and per buffer "traversal done" / "copy done" events
    uint32_t *d_pipe[2] = {nullptr, nullptr};
    cudaStream_t copy_st = nullptr;
    cudaEvent_t ev_run[2] = {nullptr, nullptr}, ev_copied[2] = {nullptr, nullptr};
    uint64_t pipe_runs = 0;
    int enqueue(uint32_t src, uint32_t *host_depths);
    bool last_hist = true;  // the last run recorded per-level page histograms
    bool graph_records_hist() const
    {
        return (cfg.direction == SCAPH_DIR_LEARNED && sched) || cfg.record_features;
    }
    // the host loop also needs them out of core (the pager reads the pages
    // holding the frontier from them)
    bool host_records_hist() const { return pager != nullptr || graph_records_hist(); }
    // incremental page counts of the learned host loop (out of core)
    uint32_t *d_hist_in = nullptr;  // [kHistLevels][2][in-pages]: discoveries by in-page
    uint32_t *h_inc = nullptr;      // pinned read-back of a level's histograms
    std::vector<uint32_t> inc_hist, inc_pull;
    int inc_hist_level = -1;        // level whose frontier histogram inc_hist holds
    bool inc_pull_valid = false;

    static constexpr int kHistLevels = 256;

    const GraphDev &out_view() const;
    const GraphDev &gin() const;
    bool graph_mode() const
    {
        return cfg.use_graph != 2 && !pager && !cfg.record_features && !cfg.dual_timing &&
               (cfg.direction != SCAPH_DIR_LEARNED || sched);
    }
    void drop_graph();
    int create(const Graph *g_, const Graph *gt_, const scaph_config *c);
    void destroy();
    int bfs(uint32_t src, uint32_t *depths, uint32_t *parents, int out_on_device, scaph_bfs_stats *stats);
    int run_host_loop(uint32_t src, uint32_t *dd, uint32_t *dp);
    int build_prow();
    int build_live(const std::vector<uint32_t> &dead);
    int features(int level, uint32_t src, uint64_t nf, uint64_t mf, uint64_t unvis, uint64_t mu, int prev_dir,
                 int ab_dir, float *f, std::vector<uint32_t> &pull_cnt, std::vector<uint32_t> &hist);
    int build_graph();
    int launch_graph(uint32_t src, uint32_t *dd, uint32_t *dp);
    int collect(bool from_graph);
    BfsDev base_state(uint32_t *dd, uint32_t *dp) const;
};

