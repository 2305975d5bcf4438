// Mixed query batches: many single-source BFS queries over many graphs of
// uneven size in ONE launch of a CUDA graph.  No reference counterpart (the
// reference runs one source of one graph per App::run, src/app.cuh:220-265).
//
//  * The graphs are laid side by side as one disjoint union (graph g owns the
//    vertex ids lo[g] .. lo[g+1]-1), paged and uploaded once.
//  * Queries on the same graph share a traversal bit-parallel (multi-source
//    BFS, ms_kernels.cuh), one bit each; bits are reused across graphs, since
//    no edge joins two graphs.  A graph with k queries uses bits 0..k-1 and
//    its vertices start with the other bits already "seen", so a vertex is
//    complete once its own graph's queries have reached it and every graph
//    finishes independently inside the shared level loop.
//  * The whole traversal is one CUDA graph: state resets (memset nodes), an
//    init kernel, the sources, then WHILE(levels) { IF(push){push, giant,
//    finalize} IF(pull){pull} decide } with the direction rule evaluated on
//    the device by `decide`, then the unpack of depths per query.  The level
//    kernels read their state through a device pointer that `decide`
//    rotates, so one instantiated graph replays for any batch of the same
//    size class.
//  * Block size, CTAs per SM and the alpha/beta thresholds are parameters
//    (scaph_batch_set_params) that the autotuner (scaph_b200/autotune.py)
//    picks by timing candidates.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "engine.h"
#include "ms_kernels.cuh"

using namespace scaph;

namespace scaph {
namespace {

constexpr int kBatchMaxGraphs = 1024;
constexpr int kBatchPlanes = 5;  // depths up to 31 in one launch; deeper -> relaunch with more

struct BatchCtl {
    unsigned long long nf, prev_nf, mf, done_e, E, V;
    unsigned long long pairs, inspected, alg;
    MsCounters *ctr0;
    unsigned long long *visit[2];
    uint32_t *act[3];
    uint32_t level, dir, npush, npull, max_level, overflow, err, mode;
    float alpha, beta;
    unsigned long long t_start;
};

struct BatchLevel {
    unsigned long long nf, mf, t_end;
    uint32_t dir, pad;
};

struct BatchArgs {
    const uint32_t *lo;            // ngraphs + 1 vertex offsets
    const unsigned long long *pad; // per graph, NW words: bits not used by its queries
    const uint32_t *qstart;        // ngraphs + 1: the graph's queries are slots qstart[g]..
    const uint32_t *qv;            // per slot: union vertex id of the source
    const unsigned long long *qoff;// per slot: output offset (words) of the query's depth row
    const uint32_t *inc0;          // vertices some edge reaches (the rest start complete)
    const uint32_t *dead;          // dead vertices (no in-edge)
    const uint32_t *degree;
    int ngraphs, nq;
};

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// graph holding union vertex u (lo staged in shared memory)
__device__ __forceinline__ int graph_of(const uint32_t *slo, int n, uint32_t u)
{
    int a = 0, b = n - 1;
    while (a < b) {
        const int m = (a + b + 1) >> 1;
        if (slo[m] <= u) a = m; else b = m - 1;
    }
    return a;
}

// seen = the padding bits of u's graph, acc = 0; incomplete = reachable
// vertices of graphs with queries; edges that will never be explored (dead
// vertices, graphs without queries) count as done for the direction rule.
template <int NW>
__global__ void k_bt_init(MsDev *ps, BatchCtl *ctl, BatchArgs a)
{
    __shared__ uint32_t slo[kBatchMaxGraphs + 1], sq[kBatchMaxGraphs];
    for (int i = threadIdx.x; i <= a.ngraphs; i += blockDim.x) slo[i] = a.lo[i];
    for (int i = threadIdx.x; i < a.ngraphs; i += blockDim.x) sq[i] = a.qstart[i + 1] - a.qstart[i];
    __syncthreads();
    const MsDev s = *ps;
    const int lane = threadIdx.x & 31;
    unsigned long long done = 0;
    const uint32_t wstride = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < s.nwords; w += wstride) {
        const uint32_t u = (w << 5) + lane;
        bool live = false;
        if (u < s.V) {
            const int g = graph_of(slo, a.ngraphs, u);
            ulonglong2 *p = reinterpret_cast<ulonglong2 *>(s.sa + 2ull * NW * u);
            if constexpr (NW == 1) {
                p[0] = make_ulonglong2(a.pad[g], 0ull);
            } else {
                p[0] = make_ulonglong2(a.pad[2 * g], a.pad[2 * g + 1]);
                p[1] = make_ulonglong2(0ull, 0ull);
            }
            live = sq[g] > 0;
            const bool dead = (__ldg(&a.dead[w]) >> lane) & 1u;
            if (!live || dead) done += __ldg(&a.degree[u]);
        }
        const uint32_t lm = __ballot_sync(0xFFFFFFFFu, live);
        if (lane == 0) s.inc[w] = a.inc0[w] & lm;
    }
    done = kc::warp_sum64(done);
    if (lane == 0 && done) atomicAdd(&ctl->done_e, done);
}

// the sources' frontier masks may hold bits of an earlier batch
template <int NW>
__global__ void k_bt_clear_sources(MsDev *ps, BatchArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nq) return;
    const MsDev s = *ps;
#pragma unroll
    for (int j = 0; j < NW; j++) s.visit_cur[(size_t)a.qv[i] * NW + j] = 0ull;
}

// slot i of graph g is bit i - qstart[g] of the vertices of g
template <int NW>
__global__ void k_bt_sources(MsDev *ps, BatchCtl *ctl, BatchArgs a)
{
    __shared__ uint32_t slo[kBatchMaxGraphs + 1];
    for (int i = threadIdx.x; i <= a.ngraphs; i += blockDim.x) slo[i] = a.lo[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nq) return;
    const MsDev s = *ps;
    const uint32_t v = a.qv[i];
    if (v >= s.V) {
        atomicOr(&ctl->err, 32u);
        return;
    }
    const int g = graph_of(slo, a.ngraphs, v);
    const uint32_t b = (uint32_t)i - a.qstart[g];
    const int word = (int)(b >> 6);
    const unsigned long long bit = 1ull << (b & 63);
    atomicOr(s.sa + 2ull * NW * v + word, bit);
    atomicOr(s.visit_cur + (size_t)v * NW + word, bit);
    const uint32_t old = atomicOr(&s.act_cur[v >> 5], 1u << (v & 31));
    if (!((old >> (v & 31)) & 1u)) {
        atomicAdd(&ctl->nf, 1ull);
        atomicAdd(&ctl->mf, (unsigned long long)a.degree[v]);
    }
}

// zero the act bitmap two levels ahead (read two levels ago, written next
// level); grid-stride, before the level body
__device__ __forceinline__ void clear_ahead(const MsDev &s, uint32_t *buf)
{
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < s.nwords; w += gridDim.x * blockDim.x) buf[w] = 0;
}

template <int NW, int B>
__global__ void __launch_bounds__(B) k_bt_push(GraphDev g, const MsDev *ps, const BatchCtl *ctl)
{
    const MsDev s = *ps;
    clear_ahead(s, ctl->act[(ctl->level + 2) % 3]);
    ms_push_body<NW, B>(g, s, RangeList{nullptr, nullptr, nullptr, 0});
}

template <int NW, int B>
__global__ void __launch_bounds__(B) k_bt_push_giant(GraphDev g, const MsDev *ps)
{
    const MsDev s = *ps;
    ms_push_giant_body<NW, B>(g, s);
}

template <int NW, int B>
__global__ void __launch_bounds__(B) k_bt_finalize(const MsDev *ps)
{
    const MsDev s = *ps;
    ms_finalize_body<NW, B>(s);
}

template <int NW, int B>
__global__ void __launch_bounds__(B) k_bt_pull(GraphDev g, const MsDev *ps, const BatchCtl *ctl)
{
    const MsDev s = *ps;
    clear_ahead(s, ctl->act[(ctl->level + 2) % 3]);
    ms_pull_body<NW, B>(g, s, RangeList{nullptr, nullptr, nullptr, 0});
}

// End of a level: counters -> next direction, state rotation, loop control.
__global__ void k_bt_decide(MsDev *ps, BatchCtl *ctl, BatchLevel *info, cudaGraphConditionalHandle h_loop,
                            cudaGraphConditionalHandle h_push, cudaGraphConditionalHandle h_pull)
{
    BatchCtl &c = *ctl;
    MsDev &s = *ps;
    const MsCounters k = *s.ctr;
    const uint32_t L = c.level;
    const int NWb = (int)(s.all[1] != 0ull) + 1;
    info[L].nf = c.nf;
    info[L].mf = c.mf;
    info[L].dir = c.dir;
    info[L].t_end = gtimer();
    c.pairs += k.pairs;
    c.inspected += k.inspected;
    c.alg += c.dir == 0 ? c.nf * 12 + c.mf * 4 + 2ull * NWb * 8 * s.V : k.inspected * 4 + 2ull * NWb * 8 * s.V;
    c.err |= k.error;
    if (c.dir == 0) c.npush++; else c.npull++;
    c.prev_nf = c.nf;
    c.nf = k.active;
    c.mf = k.active_edges;
    c.done_e += k.completed_edges;
    c.level = L + 1;
    bool go = c.nf > 0 && !c.err && c.level < c.max_level;
    if (c.nf > 0 && c.level >= c.max_level) c.overflow = 1;
    if (go) {
        const unsigned long long mu = c.E > c.done_e ? c.E - c.done_e : 0ull;
        if (c.mode == 1) c.dir = 0;
        else if (c.mode == 2) c.dir = 1;
        else c.dir = alpha_beta_next((int)c.dir, c.nf, c.prev_nf, c.mf, mu, c.V, c.alpha, c.beta);
        // rotate: visit cur <-> next; act cur <- next <- (cleared) <- cur
        unsigned long long *vt = s.visit_cur;
        s.visit_cur = s.visit_nxt;
        s.visit_nxt = vt;
        s.act_cur = c.act[(L + 1) % 3];
        s.act_nxt = c.act[(L + 2) % 3];
        s.ctr = c.ctr0 + c.level;
        s.level = c.level;
    }
    cudaGraphSetConditional(h_loop, go ? 1u : 0u);
    cudaGraphSetConditional(h_push, go && c.dir == 0 ? 1u : 0u);
    cudaGraphSetConditional(h_pull, go && c.dir == 1 ? 1u : 0u);
}

// Resets the control block and the rotating state for a launch.
__global__ void k_bt_start(MsDev *ps, MsDev base, BatchCtl *ctl, BatchCtl c0)
{
    c0.t_start = gtimer();
    *ctl = c0;
    *ps = base;
}

// depth rows: for each query slot of u's graph, the depth of u (bit planes),
// or `unreached`; NP (the depth bit planes) is a template argument so that
// the planes stay in registers
template <int NW, int NP>
__global__ void k_bt_unpack(const MsDev *ps, BatchArgs a, uint32_t *out, uint32_t unreached)
{
    __shared__ uint32_t slo[kBatchMaxGraphs + 1], sqs[kBatchMaxGraphs + 1];
    for (int i = threadIdx.x; i <= a.ngraphs; i += blockDim.x) {
        slo[i] = a.lo[i];
        sqs[i] = a.qstart[i];
    }
    __syncthreads();
    const MsDev s = *ps;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t uu = (size_t)blockIdx.x * blockDim.x + threadIdx.x; uu < s.V; uu += stride) {
        const uint32_t u = (uint32_t)uu;
        const int g = graph_of(slo, a.ngraphs, u);
        const uint32_t q0 = sqs[g], q1 = sqs[g + 1];
        if (q0 == q1) continue;
        const Mask<NW> sn = ld_seen<NW>(s.sa, u);
        Mask<NW> pl[NP];
#pragma unroll
        for (int k = 0; k < NP; k++) pl[k] = ld_mask<NW>(s.planes[k], u);
        const uint32_t local = u - slo[g];
        for (uint32_t j = q0; j < q1; j++) {
            const uint32_t b = j - q0;
            const bool hi = b >= 64;
            const int bit = (int)(b & 63);
            uint32_t d = unreached;
            if ((mask_word<NW>(sn, hi) >> bit) & 1ull) {
                d = 0;
#pragma unroll
                for (int k = 0; k < NP; k++) d |= (uint32_t)((mask_word<NW>(pl[k], hi) >> bit) & 1ull) << k;
            }
            out[a.qoff[j] + local] = d;
        }
    }
}

// The k_bt_unpack instantiation for the batch's plane counts (kBatchPlanes,
// then three more per relaunch, up to kMsPlanes).
template <int NW>
const void *bt_unpack_kernel(int nplanes)
{
    switch (nplanes) {
    case kBatchPlanes: return (const void *)k_bt_unpack<NW, kBatchPlanes>;
    case kBatchPlanes + 3: return (const void *)k_bt_unpack<NW, kBatchPlanes + 3>;
    case kBatchPlanes + 6: return (const void *)k_bt_unpack<NW, kBatchPlanes + 6>;
    default: return (const void *)k_bt_unpack<NW, kMsPlanes>;
    }
}
static_assert(kBatchPlanes + 6 < kMsPlanes, "plane counts of a batch: 5, 8, 11, then 12");

}  // namespace
}  // namespace scaph

struct scaph_batch {
    int device = 0;
    int ngraphs = 0;
    std::vector<uint32_t> lo;        // ngraphs + 1
    std::vector<uint64_t> edges;     // per graph
    std::unique_ptr<scaph_graph> ug, ugt;
    scaph_engine *e = nullptr;
    scaph_batch_params params{256, 4, 14.f, 24.f, 0};

    // multi-source state (sized for nw words, nq_cap query slots)
    int nw = 0, nq_cap = 0, nplanes = kBatchPlanes;
    unsigned long long *sa = nullptr, *visit[2] = {nullptr, nullptr};
    unsigned long long *planes[kMsPlanes] = {};
    uint32_t *act[3] = {nullptr, nullptr, nullptr}, *touched = nullptr, *inc = nullptr, *inc0 = nullptr;
    MsCounters *d_ctr = nullptr;
    MsDev *d_s = nullptr;
    BatchCtl *d_ctl = nullptr, *h_ctl = nullptr;
    BatchLevel *d_info = nullptr, *h_info = nullptr;
    uint32_t *d_lo = nullptr, *d_qstart = nullptr, *d_qv = nullptr;
    unsigned long long *d_pad = nullptr, *d_qoff = nullptr;
    uint32_t *d_out = nullptr;
    size_t out_words = 0;

    // the instantiated graph and what it was built for
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraphNode_t n_start = nullptr;
    int g_nw = 0, g_block = 0, g_ctas = 0, g_nq = 0, g_planes = 0;
    uint32_t *g_out = nullptr;
    MsDev base{};
    BatchCtl c0{};
    BatchArgs args{};
    std::vector<scaph_level_trace> trace;

    ~scaph_batch()
    {
        drop_graph();
        free_state();
        cudaFree(d_lo);
        cudaFree(d_out);
        if (e) scaph_engine_destroy(e);
    }
    void drop_graph()
    {
        if (e && e->st) cudaStreamSynchronize(e->st);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    }
    void free_state()
    {
        cudaFree(sa);
        cudaFree(visit[0]);
        cudaFree(visit[1]);
        for (auto &p : planes) {
            cudaFree(p);
            p = nullptr;
        }
        for (auto &p : act) {
            cudaFree(p);
            p = nullptr;
        }
        cudaFree(touched);
        cudaFree(inc);
        cudaFree(inc0);
        cudaFree(d_ctr);
        cudaFree(d_s);
        cudaFree(d_ctl);
        cudaFreeHost(h_ctl);
        cudaFree(d_info);
        cudaFreeHost(h_info);
        cudaFree(d_qstart);
        cudaFree(d_qv);
        cudaFree(d_pad);
        cudaFree(d_qoff);
        sa = visit[0] = visit[1] = nullptr;
        touched = inc = inc0 = nullptr;
        d_ctr = nullptr;
        d_s = nullptr;
        d_ctl = h_ctl = nullptr;
        d_info = h_info = nullptr;
        d_qstart = d_qv = nullptr;
        d_pad = d_qoff = nullptr;
        nw = nq_cap = 0;
    }
    int alloc_state(int nw_, int nq_);
    int build_graph(uint32_t *out);
};

int scaph_batch::alloc_state(int nw_, int nq_)
{
    if (nw >= nw_ && nq_cap >= nq_ && sa) return SCAPH_OK;
    drop_graph();
    free_state();
    nw = nw_;
    nq_cap = std::max(nq_, 64);
    const uint32_t V = e->V, nwords = e->nwords;
    const size_t mw = (size_t)V * nw * 8;
    SCAPH_CUDA(cudaMalloc(&sa, 2 * mw));
    SCAPH_CUDA(cudaMalloc(&visit[0], mw));
    SCAPH_CUDA(cudaMalloc(&visit[1], mw));
    for (int i = 0; i < 3; i++) SCAPH_CUDA(cudaMalloc(&act[i], (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&touched, (size_t)nwords * 4));
    SCAPH_CUDA(cudaMemset(touched, 0, (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&inc, (size_t)nwords * 4));
    SCAPH_CUDA(cudaMalloc(&inc0, (size_t)nwords * 4));
    {
        std::vector<uint32_t> live(nwords);
        SCAPH_CUDA(cudaMemcpy(live.data(), e->d_dead, (size_t)nwords * 4, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < nwords; i++) live[i] = ~live[i];
        if (V & 31) live[nwords - 1] &= (1u << (V & 31)) - 1u;
        SCAPH_CUDA(cudaMemcpy(inc0, live.data(), (size_t)nwords * 4, cudaMemcpyHostToDevice));
    }
    SCAPH_CUDA(cudaMalloc(&d_ctr, sizeof(MsCounters) * kMaxLevels));
    SCAPH_CUDA(cudaMalloc(&d_s, sizeof(MsDev)));
    SCAPH_CUDA(cudaMalloc(&d_ctl, sizeof(BatchCtl)));
    SCAPH_CUDA(cudaMallocHost(&h_ctl, sizeof(BatchCtl)));
    SCAPH_CUDA(cudaMalloc(&d_info, sizeof(BatchLevel) * kMaxLevels));
    SCAPH_CUDA(cudaMallocHost(&h_info, sizeof(BatchLevel) * kMaxLevels));
    SCAPH_CUDA(cudaMalloc(&d_qstart, sizeof(uint32_t) * (ngraphs + 1)));
    SCAPH_CUDA(cudaMalloc(&d_qv, sizeof(uint32_t) * nq_cap));
    SCAPH_CUDA(cudaMalloc(&d_pad, sizeof(unsigned long long) * 2 * ngraphs));
    SCAPH_CUDA(cudaMalloc(&d_qoff, sizeof(unsigned long long) * nq_cap));
    return SCAPH_OK;
}

// state resets, init, sources, WHILE(levels), unpack - one graph
int scaph_batch::build_graph(uint32_t *out)
{
    drop_graph();
    const int B = params.block_size;
    const int grid = e->num_sms * params.ctas_per_sm;
    const uint32_t V = e->V, nwords = e->nwords;
    const size_t mw = (size_t)V * nw * 8;
    for (int k = 0; k < nplanes; k++)
        if (!planes[k]) SCAPH_CUDA(cudaMalloc(&planes[k], mw));

    base = MsDev{};
    base.sa = sa;
    base.visit_cur = visit[0];
    base.visit_nxt = visit[1];
    for (int k = 0; k < kMsPlanes; k++) base.planes[k] = planes[k];
    base.act_cur = act[0];
    base.act_nxt = act[1];
    base.touched = touched;
    base.inc = inc;
    base.degree = e->d_degree;
    base.ctr = d_ctr;
    base.giant = e->d_giant;
    base.giant_cap = e->giant_cap;
    base.V = V;
    base.nwords = nwords;
    base.level = 0;
    base.all[0] = ~0ull;
    base.all[1] = nw == 2 ? ~0ull : 0ull;
    base.head = e->d_head;
    base.indeg = e->d_indeg;
    base.head_ranked = e->head_ranked ? 1u : 0u;

    SCAPH_CUDA(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h_loop, h_push, h_pull;
    SCAPH_CUDA(cudaGraphConditionalHandleCreate(&h_loop, graph, 1, cudaGraphCondAssignDefault));
    SCAPH_CUDA(cudaGraphConditionalHandleCreate(&h_push, graph, 1, cudaGraphCondAssignDefault));
    SCAPH_CUDA(cudaGraphConditionalHandleCreate(&h_pull, graph, 0, cudaGraphCondAssignDefault));

    std::vector<cudaGraphNode_t> deps;
    auto memset_node = [&](void *ptr, size_t bytes) -> int {
        cudaMemsetParams m{};
        m.dst = ptr;
        m.value = 0;
        m.elementSize = 4;
        m.width = bytes / 4;
        m.height = 1;
        m.pitch = 0;
        cudaGraphNode_t n;
        SCAPH_CUDA(cudaGraphAddMemsetNode(&n, graph, nullptr, 0, &m));
        deps.push_back(n);
        return SCAPH_OK;
    };
    int rc;
    if ((rc = memset_node(d_ctr, sizeof(MsCounters) * kMaxLevels))) return rc;
    for (int i = 0; i < 2; i++)
        if ((rc = memset_node(act[i], (size_t)nwords * 4))) return rc;
    for (int k = 0; k < nplanes; k++)
        if ((rc = memset_node(planes[k], mw))) return rc;

    auto kernel_node = [&](cudaGraph_t gr, const void *fn, dim3 gd, dim3 bd, void **kargs,
                           const std::vector<cudaGraphNode_t> &dep, cudaGraphNode_t *outn) -> int {
        cudaKernelNodeParams kp{};
        kp.func = const_cast<void *>(fn);
        kp.gridDim = gd;
        kp.blockDim = bd;
        kp.kernelParams = kargs;
        SCAPH_CUDA(cudaGraphAddKernelNode(outn, gr, dep.data(), dep.size(), &kp));
        return SCAPH_OK;
    };
    MsDev *ps = d_s;
    BatchCtl *pc = d_ctl;
    void *start_args[] = {&ps, &base, &pc, &c0};
    rc = kernel_node(graph, (const void *)k_bt_start, dim3(1), dim3(1), start_args, deps, &n_start);
    if (rc) return rc;
    cudaGraphNode_t n_init, n_clear, n_src;
    void *init_args[] = {&ps, &pc, &args};
    const void *f_init = nw == 2 ? (const void *)k_bt_init<2> : (const void *)k_bt_init<1>;
    rc = kernel_node(graph, f_init, dim3(grid), dim3(256), init_args, {n_start}, &n_init);
    if (rc) return rc;
    void *clr_args[] = {&ps, &args};
    const void *f_clr = nw == 2 ? (const void *)k_bt_clear_sources<2> : (const void *)k_bt_clear_sources<1>;
    rc = kernel_node(graph, f_clr, dim3((args.nq + 127) / 128), dim3(128), clr_args, {n_init}, &n_clear);
    if (rc) return rc;
    void *src_args[] = {&ps, &pc, &args};
    const void *f_src = nw == 2 ? (const void *)k_bt_sources<2> : (const void *)k_bt_sources<1>;
    rc = kernel_node(graph, f_src, dim3((args.nq + 127) / 128), dim3(128), src_args, {n_clear}, &n_src);
    if (rc) return rc;

    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h_loop;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t n_while;
    SCAPH_CUDA(cudaGraphAddNode(&n_while, graph, &n_src, 1, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    cudaGraphNodeParams ip{};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = h_push;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t n_ifpush;
    SCAPH_CUDA(cudaGraphAddNode(&n_ifpush, body, nullptr, 0, &ip));
    cudaGraph_t bpush = ip.conditional.phGraph_out[0];
    cudaGraphNodeParams iq{};
    iq.type = cudaGraphNodeTypeConditional;
    iq.conditional.handle = h_pull;
    iq.conditional.type = cudaGraphCondTypeIf;
    iq.conditional.size = 1;
    cudaGraphNode_t n_ifpull;
    SCAPH_CUDA(cudaGraphAddNode(&n_ifpull, body, &n_ifpush, 1, &iq));
    cudaGraph_t bpull = iq.conditional.phGraph_out[0];
    cudaGraphNode_t n_dec;
    BatchLevel *pinfo = d_info;
    void *dec_args[] = {&ps, &pc, &pinfo, &h_loop, &h_push, &h_pull};
    rc = kernel_node(body, (const void *)k_bt_decide, dim3(1), dim3(1), dec_args, {n_ifpull}, &n_dec);
    if (rc) return rc;

    GraphDev gout = e->dout.view, gin = e->gin();
    const void *f_push, *f_giant, *f_fin, *f_pull;
#define SCAPH_BT_PICK(NWv, Bv)                                   \
    do {                                                         \
        f_push = (const void *)k_bt_push<NWv, Bv>;               \
        f_giant = (const void *)k_bt_push_giant<NWv, Bv>;        \
        f_fin = (const void *)k_bt_finalize<NWv, Bv>;            \
        f_pull = (const void *)k_bt_pull<NWv, Bv>;               \
    } while (0)
    if (nw == 1 && B == 256) SCAPH_BT_PICK(1, 256);
    else if (nw == 1) SCAPH_BT_PICK(1, 512);
    else if (B == 256) SCAPH_BT_PICK(2, 256);
    else SCAPH_BT_PICK(2, 512);
#undef SCAPH_BT_PICK
    const BatchCtl *pcc = d_ctl;
    const MsDev *psc = d_s;
    void *push_args[] = {&gout, &psc, &pcc};
    void *giant_args[] = {&gout, &psc};
    void *fin_args[] = {&psc};
    void *pull_args[] = {&gin, &psc, &pcc};
    cudaGraphNode_t n1, n2, n3, n4;
    rc = kernel_node(bpush, f_push, dim3(grid), dim3(B), push_args, {}, &n1);
    if (rc) return rc;
    rc = kernel_node(bpush, f_giant, dim3(grid), dim3(B), giant_args, {n1}, &n2);
    if (rc) return rc;
    rc = kernel_node(bpush, f_fin, dim3(grid), dim3(B), fin_args, {n2}, &n3);
    if (rc) return rc;
    rc = kernel_node(bpull, f_pull, dim3(grid), dim3(B), pull_args, {}, &n4);
    if (rc) return rc;

    cudaGraphNode_t n_unpack;
    uint32_t unr = e->unreached;
    void *unp_args[] = {&psc, &args, &out, &unr};
    const void *f_unp = nw == 2 ? bt_unpack_kernel<2>(nplanes) : bt_unpack_kernel<1>(nplanes);
    rc = kernel_node(graph, f_unp, dim3(e->num_sms * 8), dim3(256), unp_args, {n_while}, &n_unpack);
    if (rc) return rc;
    SCAPH_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
    g_nw = nw;
    g_block = B;
    g_ctas = params.ctas_per_sm;
    g_nq = args.nq;
    g_planes = nplanes;
    g_out = out;
    return SCAPH_OK;
}

extern "C" {

int scaph_batch_create(const scaph_csr *graphs, int ngraphs, const scaph_csr *transposed, uint32_t pagesize_words,
                       const scaph_config *cfg, scaph_batch **out)
{
    clear_error();
    if (!graphs || !out || ngraphs < 1) return set_error(SCAPH_EINVAL, "null argument or no graphs");
    if (ngraphs > kBatchMaxGraphs) return set_error(SCAPH_EINVAL, "at most %d graphs per batch", kBatchMaxGraphs);
    if (cfg && cfg->pool_bytes > 0) return set_error(SCAPH_EUNSUPPORTED, "query batches need the graphs resident");
    *out = nullptr;
    std::unique_ptr<scaph_batch> b(new scaph_batch());
    b->ngraphs = ngraphs;
    b->lo.assign(ngraphs + 1, 0);
    b->edges.assign(ngraphs, 0);
    uint64_t V = 0, E = 0;
    for (int i = 0; i < ngraphs; i++) {
        if (!graphs[i].idx || (graphs[i].E && !graphs[i].ngh)) return set_error(SCAPH_EINVAL, "graph %d empty", i);
        if (transposed && (transposed[i].V != graphs[i].V || transposed[i].E != graphs[i].E))
            return set_error(SCAPH_EINVAL, "transposed graph %d does not match", i);
        b->lo[i] = (uint32_t)V;
        b->edges[i] = graphs[i].E;
        V += graphs[i].V;
        E += graphs[i].E;
        if (V >= 0xFFFFFFFFull) return set_error(SCAPH_EINVAL, "the graphs hold 2^32 or more vertices together");
    }
    b->lo[ngraphs] = (uint32_t)V;
    // disjoint union, vertex ids of graph i shifted by lo[i]
    auto concat = [&](const scaph_csr *parts, scaph_csr *u) -> int {
        memset(u, 0, sizeof(*u));
        u->V = (uint32_t)V;
        u->E = E;
        u->idx = (uint64_t *)malloc(sizeof(uint64_t) * (V + 1));
        u->ngh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(E, 1));
        if (!u->idx || !u->ngh) {
            scaph_csr_free(u);
            return set_error(SCAPH_ENOMEM, "union allocation");
        }
        uint64_t eo = 0;
        for (int i = 0; i < ngraphs; i++) {
            const scaph_csr &p = parts[i];
            const uint32_t lo = b->lo[i];
            for (uint32_t v = 0; v < p.V; v++) u->idx[lo + v] = eo + p.idx[v];
            #pragma omp parallel for schedule(static)
            for (int64_t k = 0; k < (int64_t)p.E; k++) u->ngh[eo + k] = p.ngh[k] + lo;
            eo += p.E;
        }
        u->idx[V] = eo;
        return SCAPH_OK;
    };
    scaph_csr u;
    int rc = concat(graphs, &u);
    if (rc) return rc;
    scaph_graph *g = nullptr;
    rc = scaph_graph_from_csr(&u, pagesize_words, 0, &g);
    scaph_csr_free(&u);
    if (rc) return rc;
    b->ug.reset(g);
    if (transposed) {
        if ((rc = concat(transposed, &u))) return rc;
        rc = scaph_graph_from_csr(&u, pagesize_words, 0, &g);
        scaph_csr_free(&u);
        if (rc) return rc;
        b->ugt.reset(g);
    }
    scaph_config c{};
    if (cfg) c = *cfg;
    c.pool_bytes = 0;
    c.use_graph = 0;
    if ((rc = scaph_engine_create(b->ug.get(), b->ugt.get(), &c, &b->e))) return rc;
    b->device = b->e->device;
    b->params.alpha = b->e->cfg.alpha;
    b->params.beta = b->e->cfg.beta;
    SCAPH_CUDA(cudaMalloc(&b->d_lo, sizeof(uint32_t) * (ngraphs + 1)));
    SCAPH_CUDA(cudaMemcpy(b->d_lo, b->lo.data(), sizeof(uint32_t) * (ngraphs + 1), cudaMemcpyHostToDevice));
    *out = b.release();
    return SCAPH_OK;
}

int scaph_batch_destroy(scaph_batch *b)
{
    delete b;
    return SCAPH_OK;
}

int scaph_batch_graph_range(const scaph_batch *b, int graph, uint32_t *first_vertex, uint32_t *nvertices)
{
    if (!b || graph < 0 || graph >= b->ngraphs) return set_error(SCAPH_EINVAL, "graph %d out of range", graph);
    if (first_vertex) *first_vertex = b->lo[graph];
    if (nvertices) *nvertices = b->lo[graph + 1] - b->lo[graph];
    return SCAPH_OK;
}

int scaph_batch_set_params(scaph_batch *b, const scaph_batch_params *p)
{
    clear_error();
    if (!b || !p) return set_error(SCAPH_EINVAL, "null argument");
    if (p->block_size != 256 && p->block_size != 512) return set_error(SCAPH_EINVAL, "block_size must be 256 or 512");
    if (p->ctas_per_sm < 1 || p->ctas_per_sm > 16) return set_error(SCAPH_EINVAL, "ctas_per_sm outside 1..16");
    if (!(p->alpha > 0.f) || !(p->beta > 0.f)) return set_error(SCAPH_EINVAL, "alpha and beta must be positive");
    if (p->block_size != b->params.block_size || p->ctas_per_sm != b->params.ctas_per_sm) b->drop_graph();
    b->params = *p;
    return SCAPH_OK;
}

int scaph_batch_get_params(const scaph_batch *b, scaph_batch_params *p)
{
    if (!b || !p) return set_error(SCAPH_EINVAL, "null argument");
    *p = b->params;
    return SCAPH_OK;
}

int scaph_batch_run(scaph_batch *b, const scaph_query *q, int nq, uint32_t *depths, int out_on_device,
                    scaph_bfs_stats *stats)
{
    clear_error();
    if (!b || !q || !depths || nq < 1) return set_error(SCAPH_EINVAL, "null argument or no queries");
    SCAPH_CUDA(cudaSetDevice(b->device));
    scaph_engine *e = b->e;
    const int G = b->ngraphs;
    // slots: queries grouped by graph (stable), bit = rank within the graph
    std::vector<uint32_t> cnt(G + 1, 0);
    uint64_t total_out = 0;
    for (int i = 0; i < nq; i++) {
        if ((int)q[i].graph < 0 || (int)q[i].graph >= G) return set_error(SCAPH_EINVAL, "query %d: graph out of range", i);
        const uint32_t n = b->lo[q[i].graph + 1] - b->lo[q[i].graph];
        if (q[i].source >= n) return set_error(SCAPH_EINVAL, "query %d: source %u out of range", i, q[i].source);
        cnt[q[i].graph + 1]++;
        total_out += n;
    }
    uint32_t maxq = 0;
    for (int g = 1; g <= G; g++) maxq = std::max(maxq, cnt[g]);
    if (maxq > 128) return set_error(SCAPH_EINVAL, "%u queries on one graph (at most 128 per launch)", maxq);
    const int nw = maxq > 64 ? 2 : 1;
    std::vector<uint32_t> qstart(G + 1, 0);
    for (int g = 0; g < G; g++) qstart[g + 1] = qstart[g] + cnt[g + 1];
    std::vector<uint32_t> qv(nq);
    std::vector<unsigned long long> qoff(nq), pad(2 * G);
    std::vector<uint32_t> fill(qstart.begin(), qstart.end() - 1);
    uint64_t off = 0;
    for (int i = 0; i < nq; i++) {
        const uint32_t g = q[i].graph, slot = fill[g]++;
        qv[slot] = b->lo[g] + q[i].source;
        qoff[slot] = off;
        off += b->lo[g + 1] - b->lo[g];
    }
    for (int g = 0; g < G; g++) {
        const uint32_t k = cnt[g + 1];
        for (int w = 0; w < 2; w++) {
            const uint32_t used = k > 64u * w ? std::min<uint32_t>(64, k - 64 * w) : 0;
            pad[2 * g + w] = used >= 64 ? 0ull : ~((1ull << used) - 1ull);
        }
    }
    int rc = b->alloc_state(nw, nq);
    if (rc) return rc;
    if (b->nw == 1)
        for (int g = 0; g < G; g++) pad[g] = pad[2 * g];  // one word per graph
    cudaStream_t st = e->st;
    SCAPH_CUDA(cudaMemcpyAsync(b->d_qstart, qstart.data(), sizeof(uint32_t) * (G + 1), cudaMemcpyHostToDevice, st));
    SCAPH_CUDA(cudaMemcpyAsync(b->d_qv, qv.data(), sizeof(uint32_t) * nq, cudaMemcpyHostToDevice, st));
    SCAPH_CUDA(cudaMemcpyAsync(b->d_qoff, qoff.data(), sizeof(unsigned long long) * nq, cudaMemcpyHostToDevice, st));
    SCAPH_CUDA(cudaMemcpyAsync(b->d_pad, pad.data(), sizeof(unsigned long long) * 2 * G, cudaMemcpyHostToDevice, st));
    uint32_t *out = depths;
    if (!out_on_device) {
        if (b->out_words < total_out) {
            cudaFree(b->d_out);
            b->d_out = nullptr;
            SCAPH_CUDA(cudaMalloc(&b->d_out, total_out * 4));
            b->out_words = total_out;
        }
        out = b->d_out;
    }
    b->args.lo = b->d_lo;
    b->args.pad = b->d_pad;
    b->args.qstart = b->d_qstart;
    b->args.qv = b->d_qv;
    b->args.qoff = b->d_qoff;
    b->args.inc0 = b->inc0;
    b->args.dead = e->d_dead;
    b->args.degree = e->d_degree;
    b->args.ngraphs = G;
    b->args.nq = nq;
    BatchCtl &c0 = b->c0;
    memset(&c0, 0, sizeof(c0));
    c0.E = e->E;
    c0.V = e->V;
    c0.ctr0 = b->d_ctr;
    c0.visit[0] = b->visit[0];
    c0.visit[1] = b->visit[1];
    for (int i = 0; i < 3; i++) c0.act[i] = b->act[i];
    c0.mode = e->cfg.direction == SCAPH_DIR_PUSH ? 1 : e->cfg.direction == SCAPH_DIR_PULL ? 2 : 0;
    c0.alpha = b->params.alpha;
    c0.beta = b->params.beta;
    // the level cap comes from the depth planes, or from the sentinel (the
    // loop assigns depths below `unreached` only); stopping at the
    // sentinel's cap is the traversal's end, not an overflow
    bool unr_bound = false;
    for (int attempt = 0; attempt < 3; attempt++) {
        c0.max_level = std::min<uint32_t>((1u << b->nplanes) - 1, kMaxLevels);
        unr_bound = (uint64_t)c0.max_level + 1 > e->unreached;
        if (unr_bound) c0.max_level = e->unreached - 1;
        // the graph bakes in pointers, sizes and the start state: rebuild
        // when any of them changed
        if (!b->gexec || b->g_nw != b->nw || b->g_block != b->params.block_size || b->g_ctas != b->params.ctas_per_sm ||
            b->g_nq != nq || b->g_planes != b->nplanes || b->g_out != out) {
            if ((rc = b->build_graph(out))) return rc;
        } else {
            // refresh the start state (alpha/beta may have changed)
            MsDev *ps = b->d_s;
            BatchCtl *pc = b->d_ctl;
            void *start_args[] = {&ps, &b->base, &pc, &c0};
            cudaKernelNodeParams kp{};
            kp.func = (void *)k_bt_start;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(1);
            kp.kernelParams = start_args;
            SCAPH_CUDA(cudaGraphExecKernelNodeSetParams(b->gexec, b->n_start, &kp));
        }
        SCAPH_CUDA(cudaEventRecord(e->ev_start, st));
        SCAPH_CUDA(cudaGraphLaunch(b->gexec, st));
        SCAPH_CUDA(cudaEventRecord(e->ev_stop, st));
        SCAPH_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
        if (!b->h_ctl->overflow || unr_bound) break;
        // deeper than the planes can hold: more planes, run again
        b->nplanes = std::min(kMsPlanes, b->nplanes + 3);
        b->drop_graph();
    }
    const BatchCtl &c = *b->h_ctl;
    if (c.overflow && !unr_bound) return set_error(SCAPH_EUNSUPPORTED, "traversal deeper than %d levels", (1 << kMsPlanes) - 1);
    if (c.err) return set_error(SCAPH_EDEVICE, "batch kernels reported error flags 0x%x", c.err);
    const int levels = (int)c.level;
    b->trace.clear();
    if (levels > 0) {
        SCAPH_CUDA(cudaMemcpy(b->h_info, b->d_info, sizeof(BatchLevel) * levels, cudaMemcpyDeviceToHost));
        unsigned long long tprev = c.t_start;
        for (int l = 0; l < levels; l++) {
            scaph_level_trace t{};
            t.level = l;
            t.direction = (int32_t)b->h_info[l].dir;
            t.frontier = b->h_info[l].nf;
            t.frontier_edges = b->h_info[l].mf;
            t.next = l + 1 < levels ? b->h_info[l + 1].nf : 0;
            t.ms = (double)(b->h_info[l].t_end - tprev) * 1e-6;
            tprev = b->h_info[l].t_end;
            b->trace.push_back(t);
        }
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        float ms = 0;
        cudaEventElapsedTime(&ms, e->ev_start, e->ev_stop);
        stats->ms = ms;
        stats->levels = levels;
        stats->push_levels = (int32_t)c.npush;
        stats->pull_levels = (int32_t)c.npull;
        stats->reached = c.pairs + nq;
        stats->edges_inspected = c.inspected;
        stats->alg_bytes = c.alg;
        stats->launches = 1;
    }
    if (!out_on_device) {
        SCAPH_CUDA(cudaMemcpyAsync(depths, out, total_out * 4, cudaMemcpyDeviceToHost, st));
        SCAPH_CUDA(cudaStreamSynchronize(st));
    }
    return SCAPH_OK;
}

int scaph_batch_trace(const scaph_batch *b, scaph_level_trace *out, int cap)
{
    if (!b || (!out && cap > 0)) return set_error(SCAPH_EINVAL, "null argument");
    const int n = std::min<int>(cap, (int)b->trace.size());
    for (int i = 0; i < n; i++) out[i] = b->trace[i];
    return (int)b->trace.size();
}

}  // extern "C"
