// App-hook compatibility layer: a drop-in for the reference's src/app.cuh.
//
// The reference's applications (app/bfs.cu, app/sssp.cu, app/wcc.cu)
// subclass `App<vertex_t, index_t, value_t>`, initialise d_value / d_stat in
// gpu_init(), and supply a vertex program as device hooks
// (cond / update in app/<name>_kernel.cuh, picked by -DAPPBFS, -DAPPWCC or
// -DAPPSSSP).  They build unchanged against this header: put this directory
// where the reference's src/ was (or on the include path) next to the app's
// own directory, compile with -DAPP<NAME>, link -lscaph.
//
// What runs instead of the reference engine (src/app.cuh:188-468,
// src/gpu_engine.cuh:41-169):
//  * The graph is the same paged CSR (<p>page<N>, <p>page.info,
//    <p>graph.info), loaded by libscaph; csr_idx / csr_ngh / csr_deg /
//    csr_wgh (which the apps' check() reads) are rebuilt from the pages, so
//    the flat <p>_csr.* files are optional.
//  * Generic path (every app): rounds over a device bitmap of active
//    vertices; each round runs the app's hooks over the active vertices'
//    edges with one edge-balanced kernel per batch of pages the libscaph page
//    store hands out (all pages when the graph fits the memory budget,
//    otherwise resident pages, zero-copy sparse pages and demand-copied
//    pages).  A vertex whose value a hook lowered is active in the next
//    round; the run ends when a round activates nothing.  For monotone hooks
//    (the min-updates of BFS, SSSP and WCC) this reaches the same fixed point
//    as the reference's asynchronous page rounds.
//  * BFS (-DAPPBFS): when gpu_init() left exactly one active vertex s and
//    every other vertex at one common value M > value[s] - the shape of a
//    single-source BFS - run() uses the direction-optimising BFS engine and
//    writes value[v] = min(M, value[s] + depth(v)), which is the fixed point
//    of the BFS hooks from that state (a vertex at value[s] + depth >= M is
//    never lowered).  Other initial states take the generic path.
//
// Flags are plain globals as in src/app.cuh:38-52; the constructor also
// parses gflags-style --name=value arguments (the reference's constructor
// ignores argv, its gflags call is commented out, src/app.cuh:140-141):
// --graphfile=<prefix> --src=N --check --max_memory=MB --threshold=N
// --num_stream=N --device=N.  Errors print a message and exit, as H_ERR does
// (src/gpu_engine.cuh:28-39).
#ifndef SCAPH_COMPAT_APP_CUH
#define SCAPH_COMPAT_APP_CUH
// The reference header's own include guard: an application that includes
// the reference's src/app.cuh by relative path (app/sssp.cu:1) after this
// header was force-included (-include scaph/compat/app.cuh) gets nothing
// from that file.
#ifndef __APP_CUH__
#define __APP_CUH__
#endif

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <type_traits>
#include <vector>

#include "scaph/scaph.h"
#include "gpu_tools.cuh"
#include "tools.h"

#if defined(APPBFS)
#include "bfs_kernel.cuh"
#elif defined(APPWCC)
#include "wcc_kernel.cuh"
#elif defined(APPSSSP)
#include "sssp_kernel.cuh"
#ifndef WEIGHT
#define WEIGHT
#endif
#else
#error "compile the application with -DAPPBFS, -DAPPWCC or -DAPPSSSP"
#endif

// The reference's app.cuh opens namespace std for its applications, and
// their code relies on it (vector, cout, endl unqualified).
using namespace std;

// Flags of src/app.cuh:38-52 (defaults as there).
inline int FLAGS_pagesize = 10;
inline int FLAGS_max_memory = 4096;  // MiB of device memory for vertex data + page pool
inline int FLAGS_multi = 1;
inline int FLAGS_num_stream = 5;
inline int FLAGS_num_blks = 256;
inline int FLAGS_num_thds = 256;
inline int FLAGS_threshold = 8;      // pages with active data <= threshold/32 are read zero-copy
inline bool FLAGS_check = false;
inline int FLAGS_tricknum = 0;
inline int FLAGS_src = 0;
inline double Total_throughput = 0;
inline std::string FLAGS_graphfile;
inline int FLAGS_device = 0;         // CUDA device (no reference counterpart)

namespace scaph_compat {

[[noreturn]] inline void die(const char *what, int rc)
{
    fprintf(stderr, "scaph: %s failed (%d): %s\n", what, rc, scaph_last_error());
    exit(EXIT_FAILURE);
}

#define SCAPH_COMPAT_CHECK(call)                         \
    do {                                                 \
        const int rc_ = (call);                          \
        if (rc_ < 0) scaph_compat::die(#call, rc_);      \
    } while (0)

#define SCAPH_COMPAT_CUDA(call)                                                                  \
    do {                                                                                         \
        const cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                                 \
            fprintf(stderr, "scaph: %s at %s:%d: %s\n", #call, __FILE__, __LINE__,               \
                    cudaGetErrorString(e_));                                                     \
            exit(EXIT_FAILURE);                                                                  \
        }                                                                                        \
    } while (0)

// Applies one --name=value (or --name value, --name / --noname for bools).
inline bool set_flag(const std::string &name, const char *value)
{
    auto as_int = [&](int &dst) { dst = atoi(value); return true; };
    if (name == "graphfile") { FLAGS_graphfile = value; return true; }
    if (name == "src") return as_int(FLAGS_src);
    if (name == "max_memory") return as_int(FLAGS_max_memory);
    if (name == "threshold") return as_int(FLAGS_threshold);
    if (name == "num_stream") return as_int(FLAGS_num_stream);
    if (name == "num_blks") return as_int(FLAGS_num_blks);
    if (name == "num_thds") return as_int(FLAGS_num_thds);
    if (name == "pagesize") return as_int(FLAGS_pagesize);
    if (name == "multi") return as_int(FLAGS_multi);
    if (name == "tricknum") return as_int(FLAGS_tricknum);
    if (name == "device") return as_int(FLAGS_device);
    if (name == "check") {
        FLAGS_check = !(value && (!strcmp(value, "false") || !strcmp(value, "0")));
        return true;
    }
    return false;
}

inline void parse_flags(int argc, char **argv)
{
    for (int i = 1; i < argc && argv; i++) {
        const char *a = argv[i];
        if (!a || a[0] != '-') continue;
        while (*a == '-') a++;
        std::string name(a);
        const char *value = nullptr;
        const size_t eq = name.find('=');
        std::string vbuf;
        if (eq != std::string::npos) {
            vbuf = name.substr(eq + 1);
            name = name.substr(0, eq);
            value = vbuf.c_str();
        }
        if (name == "check" || name == "nocheck") {
            FLAGS_check = name == "check" && !(value && (!strcmp(value, "false") || !strcmp(value, "0")));
            continue;
        }
        if (!value) {
            if (i + 1 >= argc) {
                fprintf(stderr, "scaph: flag --%s needs a value\n", name.c_str());
                continue;
            }
            value = argv[++i];
        }
        if (!set_flag(name, value)) fprintf(stderr, "scaph: unknown flag --%s ignored\n", name.c_str());
    }
}

// ---------------------------------------------------------------------------
// device side: the hooked round
// ---------------------------------------------------------------------------
constexpr int kBlock = 256;

struct Round {
    const uint32_t *cur;           // active bitmap of this round
    uint32_t *next;                // vertices a hook changed (next round)
    unsigned long long *activated; // += vertices newly set in next
};

__device__ __forceinline__ uint32_t page_of(const scaph_page_view &g, uint32_t v)
{
    uint32_t p = __ldg(&g.coarse[v >> g.cshift]);
    while (__ldg(&g.pages[p + 1].left) <= v) ++p;
    return p;
}

// Exclusive scan of one value per thread over a 256-thread block; also
// returns the total.  Uses s_warp[0..8].
__device__ __forceinline__ uint32_t block_scan(uint32_t x, uint32_t *s_warp, uint32_t &total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < kBlock / 32 ? s_warp[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < kBlock / 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kBlock / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
        if (lane == kBlock / 32 - 1) s_warp[kBlock / 32] = wi;
    }
    __syncthreads();
    total = s_warp[kBlock / 32];
    return inc - x + s_warp[wid];
}

// One round of the app's hooks over the active vertices of a batch of
// pages.  Each CTA takes tiles of 4096 vertices (128 bitmap words) of the
// batch's ranges, 256 vertices at a time: a thread per vertex loads the
// Node record of an active vertex (its page found through the coarse index)
// and its value, a block scan lays the 256 adjacency lists end to end, and
// the CTA walks the concatenated edges with every thread on consecutive
// edges (coalesced edge loads; the owner of edge i found by binary search
// over the scanned offsets).  This is gpu_push_csr's relaxation
// (src/gpu_engine.cuh:95-160) with the CTA/warp/thread tiers replaced by
// one edge-balanced loop.
template <typename value_t, bool W>
__global__ void __launch_bounds__(kBlock) k_hook_round(scaph_page_view g, scaph_ranges rl, value_t *value, Round r)
{
    __shared__ uint32_t s_off[kBlock];
    __shared__ unsigned long long s_start[kBlock];
    __shared__ value_t s_val[kBlock];
    __shared__ uint32_t s_warp[kBlock / 32 + 1];
    constexpr uint32_t ew = W ? 2u : 1u;
    uint32_t activated = 0;
    for (uint32_t tile = blockIdx.x; tile < rl.tiles; tile += gridDim.x) {
        uint32_t lo = 0, hi = rl.n - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&rl.tile0[mid]) <= tile) lo = mid; else hi = mid - 1;
        }
        const uint32_t rlo = __ldg(&rl.lo[lo]), rhi = __ldg(&rl.hi[lo]);
        const uint64_t w0 = (uint64_t)(rlo >> 5) + 128ull * (tile - __ldg(&rl.tile0[lo]));
        for (uint32_t sub = 0; sub < 16; sub++) {
            const uint64_t base = (w0 + 8ull * sub) * 32ull;
            if (base >= rhi) break;  // uniform across the CTA
            const uint32_t v = (uint32_t)(base + threadIdx.x);
            const bool act = base + threadIdx.x < rhi && v >= rlo && ((__ldg(&r.cur[v >> 5]) >> (v & 31)) & 1u);
            if (!__syncthreads_or(act)) continue;
            uint32_t len = 0;
            unsigned long long start = 0;
            value_t sv{};
            if (act) {
                const uint32_t p = page_of(g, v);
                const scaph_page_dev pg = g.pages[p];
                const uint32_t *node = g.pool + pg.base + 3ull * (v - pg.left);
                len = node[2];
                start = pg.base + 3ull * pg.nodenum + (unsigned long long)node[1] * ew;
                sv = value[v];
            }
            uint32_t total;
            const uint32_t off = block_scan(len, s_warp, total);
            s_off[threadIdx.x] = off;
            s_start[threadIdx.x] = start;
            s_val[threadIdx.x] = sv;
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < total; i += kBlock) {
                uint32_t a = 0, b = kBlock - 1;
                while (a < b) {
                    const uint32_t m = (a + b + 1) >> 1;
                    if (s_off[m] <= i) a = m; else b = m - 1;
                }
                const uint32_t *e = g.pool + s_start[a] + (unsigned long long)(i - s_off[a]) * ew;
                const uint32_t u = e[0];
                const value_t src = s_val[a];
                bool hit;
#ifdef WEIGHT
                const value_t w = (value_t)e[1];
                hit = cond<value_t>(src, value[u], w) && update<value_t>(src, value[u], w);
#else
                hit = cond<value_t>(src, value[u]) && update<value_t>(src, value[u]);
#endif
                if (hit) {
                    const uint32_t bit = 1u << (u & 31);
                    if (!(atomicOr(&r.next[u >> 5], bit) & bit)) activated++;
                }
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) activated += __shfl_xor_sync(0xFFFFFFFFu, activated, o);
    if ((threadIdx.x & 31) == 0 && activated) atomicAdd(r.activated, (unsigned long long)activated);
}

// bool stat[V] (the apps' active flags) -> bitmap, one thread per word.
__global__ void k_stat_to_bits(const bool *stat, uint32_t V, uint32_t *bits)
{
    const uint32_t nw = (V + 31) / 32;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
        uint32_t m = 0;
        const uint32_t v0 = w * 32;
        for (uint32_t k = 0; k < 32 && v0 + k < V; k++) m |= (stat[v0 + k] ? 1u : 0u) << k;
        bits[w] = m;
    }
}

struct Shape {
    unsigned long long active;  // vertices with stat set
    unsigned int first;         // smallest of them
    unsigned int vmin, vmax;    // values of the others
};

// Is the state gpu_init() left a single-source BFS start?  Counts the
// active vertices and the range of the other vertices' values.
__global__ void k_bfs_shape(const unsigned int *value, const bool *stat, uint32_t V, Shape *out)
{
    unsigned long long n = 0;
    unsigned int first = 0xFFFFFFFFu, vmin = 0xFFFFFFFFu, vmax = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        if (stat[v]) {
            n++;
            first = min(first, v);
        } else {
            const unsigned int x = value[v];
            vmin = min(vmin, x);
            vmax = max(vmax, x);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
        first = min(first, __shfl_xor_sync(0xFFFFFFFFu, first, o));
        vmin = min(vmin, __shfl_xor_sync(0xFFFFFFFFu, vmin, o));
        vmax = max(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (n) atomicAdd(&out->active, n);
        atomicMin(&out->first, first);
        atomicMin(&out->vmin, vmin);
        atomicMax(&out->vmax, vmax);
    }
}

// value[v] = min(M, vs + depth[v]) for v != s (unreached: M); stat cleared.
__global__ void k_bfs_merge(unsigned int *value, bool *stat, const uint32_t *depth, uint32_t s, unsigned int vs,
                            unsigned int M, uint32_t V)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        stat[v] = false;
        if (v == s) continue;
        const uint32_t d = depth[v];
        value[v] = (d != 0xFFFFFFFFu && (unsigned long long)vs + d < M) ? vs + d : M;
    }
}

}  // namespace scaph_compat

// ---------------------------------------------------------------------------
// App<vertex_t, index_t, value_t>  (src/app.cuh:66-135)
// ---------------------------------------------------------------------------
template <typename vertex_t, typename index_t, typename value_t>
class App
{
    static_assert(sizeof(vertex_t) == 4, "paged CSR vertex ids are 32-bit");
    static_assert(sizeof(value_t) == 4, "vertex values are 32-bit words");

public:
    int64_t gpu_memsize = 0;
    vertex_t vert_count = 0;
    index_t edge_count = 0;

    vertex_t pagesize = 0;
    vertex_t chunksize = 0;
    vertex_t threshold = 0;

    cudaStream_t *execstream = nullptr;
    cudaStream_t copystream = nullptr;

    int list_size = 0, pool_size = 0;
    int num_blks = 0, num_thds = 0, num_stream = 0;

    bool *h_stat = nullptr, *d_stat = nullptr;
    value_t *h_value = nullptr, *d_value = nullptr;
    vertex_t *h_degree = nullptr, *d_degree = nullptr;

    std::string graphfile;
    index_t *csr_idx = nullptr;
    vertex_t *csr_ngh = nullptr;
    vertex_t *csr_deg = nullptr;
    value_t *csr_wgh = nullptr;

    // of the last run(): device seconds, rounds of the generic path (0 when
    // the BFS engine ran), and whether the BFS engine ran
    double last_seconds = 0;
    int last_rounds = 0;
    bool last_used_bfs_engine = false;
    // page traffic of the last run(): bytes copied host->HBM, bytes read
    // zero-copy, demand page copies
    uint64_t last_h2d_bytes = 0, last_zc_bytes = 0, last_page_faults = 0;

    App(int argc, char **argv);
    App(const App &) = delete;
    App &operator=(const App &) = delete;
    virtual ~App();
    void load_graph();
    void run();
    virtual void gpu_init() = 0;
    virtual bool check();

private:
    scaph_graph *graph_ = nullptr, *graph_t_ = nullptr;
    scaph_store *store_ = nullptr;
    scaph_engine *bfs_ = nullptr;
    int64_t pool_bytes_ = 0;
    int num_sms_ = 148;
    uint32_t *d_bits_[2] = {nullptr, nullptr};
    unsigned long long *d_cnt_ = nullptr, *h_cnt_ = nullptr;
    uint32_t *d_depth_ = nullptr;
    scaph_compat::Shape *d_shape_ = nullptr, *h_shape_ = nullptr;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    bool loaded_ = false;

    bool run_bfs_engine(cudaStream_t st);
    void run_hooks(cudaStream_t st);
    static int batch(void *user, const scaph_page_view *view, const scaph_ranges *ranges, void *stream);
};

template <typename vertex_t, typename index_t, typename value_t>
App<vertex_t, index_t, value_t>::App(int argc, char **argv)
{
    scaph_compat::parse_flags(argc, argv);
    graphfile = FLAGS_graphfile;
    num_stream = std::max(1, FLAGS_num_stream);
    num_blks = FLAGS_num_blks;
    num_thds = FLAGS_num_thds;
    pagesize = (vertex_t)FLAGS_pagesize * 1024 * 1024;
    chunksize = pagesize / 32;
    threshold = (vertex_t)FLAGS_threshold * chunksize;
    gpu_memsize = (int64_t)FLAGS_max_memory * 1024 * 1024;
}

template <typename vertex_t, typename index_t, typename value_t>
App<vertex_t, index_t, value_t>::~App()
{
    if (loaded_) cudaDeviceSynchronize();
    if (bfs_) scaph_engine_destroy(bfs_);
    if (store_) scaph_store_destroy(store_);
    if (graph_t_) scaph_graph_close(graph_t_);
    if (graph_) scaph_graph_close(graph_);
    cudaFree(d_value);
    cudaFree(d_stat);
    cudaFree(d_degree);
    cudaFree(d_bits_[0]);
    cudaFree(d_bits_[1]);
    cudaFree(d_cnt_);
    cudaFree(d_depth_);
    cudaFree(d_shape_);
    cudaFreeHost(h_value);
    cudaFreeHost(h_stat);
    cudaFreeHost(h_cnt_);
    cudaFreeHost(h_shape_);
    for (cudaEvent_t e : ev_)
        if (e) cudaEventDestroy(e);
    if (execstream) {
        for (int i = 0; i < num_stream; i++) cudaStreamDestroy(execstream[i]);
        delete[] execstream;
    }
    if (copystream) cudaStreamDestroy(copystream);
    delete[] csr_idx;
    delete[] csr_ngh;
    delete[] csr_deg;
    delete[] csr_wgh;
}

// Loads the paged graph <graphfile>page* (fetch_graph, src/graph.h:24-108),
// allocates the vertex arrays and puts the pages on the device within
// FLAGS_max_memory (src/app.cuh:267-345).
template <typename vertex_t, typename index_t, typename value_t>
void App<vertex_t, index_t, value_t>::load_graph()
{
    if (loaded_) return;
    SCAPH_COMPAT_CUDA(cudaSetDevice(FLAGS_device));
    SCAPH_COMPAT_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, FLAGS_device));
    if (graphfile.empty()) {
        fprintf(stderr, "scaph: no graph: pass --graphfile=<prefix of the paged CSR files>\n");
        exit(EXIT_FAILURE);
    }
#ifdef WEIGHT
    const int weighted = 1;
#else
    const int weighted = 0;
#endif
    SCAPH_COMPAT_CHECK(scaph_graph_open(graphfile.c_str(), weighted, &graph_));
    scaph_graph_info gi;
    SCAPH_COMPAT_CHECK(scaph_graph_get_info(graph_, &gi));
    vert_count = gi.V;
    edge_count = (index_t)gi.E;
    if ((uint64_t)edge_count != gi.E) {
        fprintf(stderr, "scaph: %llu edges do not fit index_t\n", (unsigned long long)gi.E);
        exit(EXIT_FAILURE);
    }
    list_size = gi.npages;
    pagesize = gi.pagesize;
    chunksize = pagesize / 32;
    threshold = (vertex_t)FLAGS_threshold * chunksize;

    scaph_csr csr;
    SCAPH_COMPAT_CHECK(scaph_graph_to_csr(graph_, &csr));
    const size_t V = vert_count, E = gi.E;
    csr_idx = new index_t[V + 1];
    csr_ngh = new vertex_t[std::max<size_t>(E, 1)];
    csr_deg = new vertex_t[std::max<size_t>(V, 1)];
    for (size_t v = 0; v <= V; v++) csr_idx[v] = (index_t)csr.idx[v];
    memcpy(csr_ngh, csr.ngh, E * sizeof(vertex_t));
    memcpy(csr_deg, scaph_graph_degree(graph_), V * sizeof(vertex_t));
    if (csr.wgh) {
        csr_wgh = new value_t[std::max<size_t>(E, 1)];
        for (size_t e = 0; e < E; e++) csr_wgh[e] = (value_t)csr.wgh[e];
    }
    h_degree = csr_deg;

    execstream = new cudaStream_t[num_stream];
    for (int i = 0; i < num_stream; i++) SCAPH_COMPAT_CUDA(cudaStreamCreate(&execstream[i]));
    SCAPH_COMPAT_CUDA(cudaStreamCreate(&copystream));
    for (cudaEvent_t &e : ev_) SCAPH_COMPAT_CUDA(cudaEventCreate(&e));

    // vertex data first, the page pool gets the rest of the budget
    const int64_t vbytes = (int64_t)V * (sizeof(value_t) + sizeof(bool) + sizeof(vertex_t) + 2 * 4 + 4);
    gpu_memsize -= vbytes;
    const int64_t page_bytes = (int64_t)pagesize * 4;
    if (gpu_memsize < page_bytes) {
        fprintf(stderr, "scaph: vertex data leaves no room for one page within --max_memory=%d MiB\n",
                FLAGS_max_memory);
        exit(EXIT_FAILURE);
    }
    SCAPH_COMPAT_CUDA(cudaMalloc(&d_value, sizeof(value_t) * std::max<size_t>(V, 1)));
    SCAPH_COMPAT_CUDA(cudaMalloc(&d_stat, sizeof(bool) * std::max<size_t>(V, 1)));
    SCAPH_COMPAT_CUDA(cudaMalloc(&d_degree, sizeof(vertex_t) * std::max<size_t>(V, 1)));
    SCAPH_COMPAT_CUDA(cudaMemcpy(d_degree, csr_deg, sizeof(vertex_t) * V, cudaMemcpyHostToDevice));
    SCAPH_COMPAT_CUDA(cudaMallocHost(&h_value, sizeof(value_t) * std::max<size_t>(V, 1)));
    SCAPH_COMPAT_CUDA(cudaMallocHost(&h_stat, sizeof(bool) * std::max<size_t>(V, 1)));
    SCAPH_COMPAT_CUDA(cudaMalloc(&d_cnt_, sizeof(unsigned long long)));
    SCAPH_COMPAT_CUDA(cudaMallocHost(&h_cnt_, sizeof(unsigned long long)));
    SCAPH_COMPAT_CUDA(cudaMalloc(&d_shape_, sizeof(scaph_compat::Shape)));
    SCAPH_COMPAT_CUDA(cudaMallocHost(&h_shape_, sizeof(scaph_compat::Shape)));

#ifdef APPBFS
    // the BFS engine pulls over in-edges: directed graphs need the
    // transposed pages
    const int sym = scaph_csr_symmetric(&csr);
    if (sym < 0) scaph_compat::die("scaph_csr_symmetric", sym);
    int64_t need = (int64_t)list_size * page_bytes;
    if (!sym) {
        scaph_csr t;
        SCAPH_COMPAT_CHECK(scaph_csr_transpose(&csr, &t));
        SCAPH_COMPAT_CHECK(scaph_graph_from_csr(&t, pagesize, 0, &graph_t_));
        scaph_csr_free(&t);
        scaph_graph_info ti;
        SCAPH_COMPAT_CHECK(scaph_graph_get_info(graph_t_, &ti));
        need += (int64_t)ti.npages * page_bytes;
    }
    pool_bytes_ = need <= gpu_memsize ? 0 : gpu_memsize;
    pool_size = pool_bytes_ ? (int)(pool_bytes_ / page_bytes) : list_size;
    SCAPH_COMPAT_CUDA(cudaMalloc(&d_depth_, sizeof(uint32_t) * std::max<size_t>(V, 1)));
    scaph_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.pool_bytes = pool_bytes_;
    cfg.direction = SCAPH_DIR_ALPHABETA;
    cfg.compact_threshold = FLAGS_threshold;
    cfg.copy_streams = std::min(4, num_stream);
    cfg.device = FLAGS_device;
    cfg.stream = execstream[0];
    SCAPH_COMPAT_CHECK(scaph_engine_create(graph_, graph_t_, &cfg, &bfs_));
#else
    pool_bytes_ = (int64_t)list_size * page_bytes <= gpu_memsize ? 0 : gpu_memsize;
    pool_size = pool_bytes_ ? (int)(pool_bytes_ / page_bytes) : list_size;
    SCAPH_COMPAT_CHECK(scaph_store_create(graph_, pool_bytes_, FLAGS_threshold, std::min(4, num_stream),
                                          FLAGS_device, &store_));
#endif
    gpu_memsize -= (int64_t)pool_size * page_bytes;
    scaph_csr_free(&csr);
    loaded_ = true;
}

template <typename vertex_t, typename index_t, typename value_t>
int App<vertex_t, index_t, value_t>::batch(void *user, const scaph_page_view *view, const scaph_ranges *ranges,
                                           void *stream)
{
    App *a = static_cast<App *>(user);
    if (!ranges->tiles) return 0;
    const int grid = (int)std::min<uint32_t>(ranges->tiles, (uint32_t)a->num_sms_ * 8);
    scaph_compat::Round r{a->d_bits_[0], a->d_bits_[1], a->d_cnt_};
#ifdef WEIGHT
    constexpr bool W = true;
#else
    constexpr bool W = false;
#endif
    scaph_compat::k_hook_round<value_t, W>
        <<<grid, scaph_compat::kBlock, 0, static_cast<cudaStream_t>(stream)>>>(*view, *ranges, a->d_value, r);
    return cudaGetLastError() == cudaSuccess ? 0 : SCAPH_ECUDA;
}

// The generic path: rounds of the app's hooks until none changes a value.
template <typename vertex_t, typename index_t, typename value_t>
void App<vertex_t, index_t, value_t>::run_hooks(cudaStream_t st)
{
    const uint32_t V = vert_count, nw = (V + 31) / 32;
    if (!store_) {
        SCAPH_COMPAT_CHECK(scaph_store_create(graph_, pool_bytes_, FLAGS_threshold, std::min(4, num_stream),
                                              FLAGS_device, &store_));
    }
    if (!d_bits_[0]) {
        SCAPH_COMPAT_CUDA(cudaMalloc(&d_bits_[0], 4 * (size_t)std::max<uint32_t>(nw, 1)));
        SCAPH_COMPAT_CUDA(cudaMalloc(&d_bits_[1], 4 * (size_t)std::max<uint32_t>(nw, 1)));
    }
    uint64_t h0 = 0, z0 = 0, f0 = 0;
    SCAPH_COMPAT_CHECK(scaph_store_counters(store_, &h0, &z0, &f0));
    const int grid = num_sms_ * 4;
    scaph_compat::k_stat_to_bits<<<grid, 256, 0, st>>>(d_stat, V, d_bits_[0]);
    SCAPH_COMPAT_CUDA(cudaGetLastError());
    SCAPH_COMPAT_CUDA(cudaMemsetAsync(d_bits_[1], 0, 4 * (size_t)nw, st));
    last_rounds = 0;
    for (;;) {
        SCAPH_COMPAT_CUDA(cudaMemsetAsync(d_cnt_, 0, sizeof(unsigned long long), st));
        SCAPH_COMPAT_CHECK(scaph_store_level(store_, d_bits_[0], &App::batch, this, st));
        SCAPH_COMPAT_CUDA(cudaMemcpyAsync(h_cnt_, d_cnt_, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        SCAPH_COMPAT_CUDA(cudaMemsetAsync(d_bits_[0], 0, 4 * (size_t)nw, st));
        std::swap(d_bits_[0], d_bits_[1]);
        SCAPH_COMPAT_CUDA(cudaStreamSynchronize(st));
        last_rounds++;
        if (*h_cnt_ == 0) break;
        if ((uint64_t)last_rounds > (uint64_t)V + 1) {
            // monotone hooks settle within V rounds
            fprintf(stderr, "scaph: the application's hooks did not converge after %d rounds\n", last_rounds);
            exit(EXIT_FAILURE);
        }
    }
    SCAPH_COMPAT_CUDA(cudaMemsetAsync(d_stat, 0, sizeof(bool) * V, st));
    uint64_t h1 = 0, z1 = 0, f1 = 0;
    SCAPH_COMPAT_CHECK(scaph_store_counters(store_, &h1, &z1, &f1));
    last_h2d_bytes = h1 - h0;
    last_zc_bytes = z1 - z0;
    last_page_faults = f1 - f0;
}

// BFS-shaped start -> the direction-optimising engine (see the file header).
template <typename vertex_t, typename index_t, typename value_t>
bool App<vertex_t, index_t, value_t>::run_bfs_engine(cudaStream_t st)
{
    if constexpr (!std::is_same<value_t, unsigned int>::value) {
        return false;
    } else {
        if (!bfs_ || vert_count == 0) return false;
        const uint32_t V = vert_count;
        h_shape_->active = 0;
        h_shape_->first = 0xFFFFFFFFu;
        h_shape_->vmin = 0xFFFFFFFFu;
        h_shape_->vmax = 0;
        SCAPH_COMPAT_CUDA(cudaMemcpyAsync(d_shape_, h_shape_, sizeof(*h_shape_), cudaMemcpyHostToDevice, st));
        scaph_compat::k_bfs_shape<<<num_sms_ * 4, 256, 0, st>>>(d_value, d_stat, V, d_shape_);
        SCAPH_COMPAT_CUDA(cudaGetLastError());
        SCAPH_COMPAT_CUDA(cudaMemcpyAsync(h_shape_, d_shape_, sizeof(*h_shape_), cudaMemcpyDeviceToHost, st));
        SCAPH_COMPAT_CUDA(cudaStreamSynchronize(st));
        if (h_shape_->active != 1 || V < 2 || h_shape_->vmin != h_shape_->vmax) return false;
        const uint32_t s = h_shape_->first;
        const unsigned int M = h_shape_->vmin;
        unsigned int vs = 0;
        SCAPH_COMPAT_CUDA(cudaMemcpy(&vs, d_value + s, sizeof(vs), cudaMemcpyDeviceToHost));
        if (vs >= M) return false;
        scaph_bfs_stats stats;
        SCAPH_COMPAT_CHECK(scaph_bfs(bfs_, s, d_depth_, nullptr, 1, &stats));
        last_h2d_bytes = stats.h2d_bytes;
        last_zc_bytes = stats.zc_bytes;
        last_page_faults = stats.page_faults;
        scaph_compat::k_bfs_merge<<<num_sms_ * 4, 256, 0, st>>>(d_value, d_stat, d_depth_, s, vs, M, V);
        SCAPH_COMPAT_CUDA(cudaGetLastError());
        return true;
    }
}

// App::run (src/app.cuh:220-265): gpu_init(), the traversal, timing.
template <typename vertex_t, typename index_t, typename value_t>
void App<vertex_t, index_t, value_t>::run()
{
    if (!loaded_) load_graph();
    gpu_init();
    SCAPH_COMPAT_CUDA(cudaStreamSynchronize(copystream));
    cudaStream_t st = execstream[0];
    SCAPH_COMPAT_CUDA(cudaEventRecord(ev_[0], st));
    last_used_bfs_engine = false;
    last_rounds = 0;
#ifdef APPBFS
    last_used_bfs_engine = run_bfs_engine(st);
#endif
    if (!last_used_bfs_engine) run_hooks(st);
    SCAPH_COMPAT_CUDA(cudaEventRecord(ev_[1], st));
    SCAPH_COMPAT_CUDA(cudaEventSynchronize(ev_[1]));
    float ms = 0;
    SCAPH_COMPAT_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    last_seconds = ms * 1e-3;
    const double gteps = last_seconds > 0 ? (double)edge_count / last_seconds / 1e9 : 0.0;
    Total_throughput += gteps;
    printf("scaph: run %.8f s, %.6f GTEPS (%s)\n", last_seconds, gteps,
           last_used_bfs_engine ? "BFS engine" : "hook rounds");
    if (FLAGS_check) {
        SCAPH_COMPAT_CUDA(cudaMemcpy(h_value, d_value, sizeof(value_t) * vert_count, cudaMemcpyDeviceToHost));
        SCAPH_COMPAT_CUDA(cudaMemcpy(h_stat, d_stat, sizeof(bool) * vert_count, cudaMemcpyDeviceToHost));
    }
}

template <typename vertex_t, typename index_t, typename value_t>
bool App<vertex_t, index_t, value_t>::check()
{
    return true;
}

#endif  // SCAPH_COMPAT_APP_CUH
