// PageRank over the paged CSR, on the library's page store (scaph_store_*).
//
//   pr --graphfile=<prefix> [--iters=N] [--damping=D] [--max_memory=MB]
//      [--threshold=N] [--weighted] [--out=<file>]
//
// The reference ships app/pr.cu but it does not build (it is a copy of
// app/sssp.cu naming members that exist nowhere: scv, cpu_iteration,
// vertexSubset), and its hooks (app/pr_kernel.cuh) are SSSP's relax-by-min,
// which cannot express a rank sum.  This program is the PageRank that
// directory names, on the same pages and the same page store the other apps
// use: every iteration pushes each vertex's share of rank along its
// out-edges, page batch by page batch (all pages resident when the graph
// fits --max_memory, else resident, zero-copy and demand-copied batches from
// the pool), then applies
//     rank'(v) = (1 - d) / V + d * (sum over in-edges u->v of rank(u)/outdeg(u)
//                                  + (rank held by vertices without out-edges) / V)
// FP32 values with FP32 atomic accumulation, so the last bits depend on the
// order of the additions; the tests compare with a float64 power iteration
// within a stated tolerance.  --out writes the final ranks (f32[V]); the last
// line printed gives the iterations, the final L1 change and the page
// traffic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "scaph/scaph.h"

namespace {

constexpr int kBlock = 256;

#define PR_CUDA(call)                                                                                 \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #call, cudaGetErrorString(e_));    \
            exit(EXIT_FAILURE);                                                                       \
        }                                                                                             \
    } while (0)
#define PR_CHECK(call)                                                                                \
    do {                                                                                              \
        int rc_ = (call);                                                                             \
        if (rc_ != SCAPH_OK) {                                                                        \
            fprintf(stderr, "%s:%d %s: %d %s\n", __FILE__, __LINE__, #call, rc_, scaph_last_error()); \
            exit(EXIT_FAILURE);                                                                       \
        }                                                                                             \
    } while (0)

__device__ __forceinline__ uint32_t page_of(const scaph_page_view &g, uint32_t v)
{
    uint32_t p = __ldg(&g.coarse[v >> g.cshift]);
    while (__ldg(&g.pages[p + 1].left) <= v) ++p;
    return p;
}

// contrib[v] = rank[v] / outdeg[v]; the rank of vertices without out-edges
// summed into *dangling (FP64)
__global__ void k_contrib(const float *rank, const uint32_t *deg, uint32_t V, float *contrib, double *dangling)
{
    double local = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t d = deg[v];
        contrib[v] = d ? rank[v] / (float)d : 0.f;
        if (!d) local += rank[v];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local != 0.0) atomicAdd(dangling, local);
}

// Every vertex of the batch's ranges adds contrib[v] to acc[u] for each
// out-edge v->u: 256 vertices at a time, their lists laid end to end by a
// block scan and walked edge-balanced (consecutive edges per thread).
__global__ void __launch_bounds__(kBlock) k_push(scaph_page_view g, scaph_ranges rl, const float *contrib, float *acc)
{
    __shared__ uint32_t s_off[kBlock + 1];
    __shared__ unsigned long long s_start[kBlock];
    __shared__ float s_c[kBlock];
    __shared__ uint32_t s_warp[kBlock / 32];
    const uint32_t ew = g.weighted ? 2u : 1u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
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
            const bool mine = base + threadIdx.x < rhi && v >= rlo;
            uint32_t len = 0;
            unsigned long long start = 0;
            float c = 0.f;
            if (mine) {
                const uint32_t p = page_of(g, v);
                const scaph_page_dev pg = g.pages[p];
                const uint32_t *node = g.pool + pg.base + 3ull * (v - pg.left);
                len = node[2];
                start = pg.base + 3ull * pg.nodenum + (unsigned long long)node[1] * ew;
                c = contrib[v];
                if (c == 0.f) len = 0;
            }
            // exclusive block scan of len
            uint32_t inc = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane == 31) s_warp[wid] = inc;
            __syncthreads();
            if (wid == 0) {
                uint32_t w = lane < kBlock / 32 ? s_warp[lane] : 0, wi = w;
#pragma unroll
                for (int o = 1; o < kBlock / 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
                    if (lane >= o) wi += y;
                }
                if (lane < kBlock / 32) s_warp[lane] = wi - w;
                if (lane == kBlock / 32 - 1) s_off[kBlock] = wi;
            }
            __syncthreads();
            s_off[threadIdx.x] = inc - len + s_warp[wid];
            s_start[threadIdx.x] = start;
            s_c[threadIdx.x] = c;
            __syncthreads();
            const uint32_t total = s_off[kBlock];
            for (uint32_t i = threadIdx.x; i < total; i += kBlock) {
                uint32_t a = 0, b = kBlock - 1;
                while (a < b) {
                    const uint32_t m = (a + b + 1) >> 1;
                    if (s_off[m] <= i) a = m; else b = m - 1;
                }
                const uint32_t u = g.pool[s_start[a] + (unsigned long long)(i - s_off[a]) * ew];
                if (u < g.V) atomicAdd(&acc[u], s_c[a]);
            }
            __syncthreads();
        }
    }
}

// rank = (1-d)/V + d * (acc + dangling/V); acc cleared; |change| summed
__global__ void k_apply(float *rank, float *acc, uint32_t V, float damping, const double *dangling, double *l1)
{
    const float base = (1.f - damping) / (float)V;
    const float dang = (float)(*dangling / (double)V);
    double local = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const float r = base + damping * (acc[v] + dang);
        local += fabs((double)r - (double)rank[v]);
        rank[v] = r;
        acc[v] = 0.f;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31) == 0 && local != 0.0) atomicAdd(l1, local);
}

__global__ void k_fill(float *x, uint32_t V, float value)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) x[v] = value;
}

struct PushArgs {
    const float *contrib;
    float *acc;
    int grid;
};

int push_batch(void *user, const scaph_page_view *view, const scaph_ranges *ranges, void *stream)
{
    const PushArgs *a = static_cast<const PushArgs *>(user);
    if (!ranges->tiles) return SCAPH_OK;
    const int grid = (int)std::min<uint32_t>(ranges->tiles, (uint32_t)a->grid);
    k_push<<<grid, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(*view, *ranges, a->contrib, a->acc);
    return cudaGetLastError() == cudaSuccess ? SCAPH_OK : SCAPH_ECUDA;
}

}  // namespace

int main(int argc, char **argv)
{
    std::string prefix, out;
    int iters = 20, threshold = 3, device = 0, weighted = 0;
    double damping = 0.85;
    long long max_memory_mb = 0;
    for (int i = 1; i < argc; i++) {
        const std::string a(argv[i]);
        auto val = [&](const char *k) { return a.substr(strlen(k)); };
        if (a.rfind("--graphfile=", 0) == 0) prefix = val("--graphfile=");
        else if (a.rfind("--out=", 0) == 0) out = val("--out=");
        else if (a.rfind("--iters=", 0) == 0) iters = atoi(val("--iters=").c_str());
        else if (a.rfind("--damping=", 0) == 0) damping = atof(val("--damping=").c_str());
        else if (a.rfind("--max_memory=", 0) == 0) max_memory_mb = atoll(val("--max_memory=").c_str());
        else if (a.rfind("--threshold=", 0) == 0) threshold = atoi(val("--threshold=").c_str());
        else if (a.rfind("--device=", 0) == 0) device = atoi(val("--device=").c_str());
        else if (a == "--weighted") weighted = 1;
        else {
            fprintf(stderr, "unknown argument %s\n", argv[i]);
            return 2;
        }
    }
    if (prefix.empty() || iters < 1 || damping <= 0.0 || damping >= 1.0) {
        fprintf(stderr, "usage: pr --graphfile=<prefix> [--iters=N] [--damping=D in (0,1)] [--max_memory=MB] "
                        "[--threshold=N] [--weighted] [--out=<file>]\n");
        return 2;
    }
    PR_CUDA(cudaSetDevice(device));
    scaph_graph *g = nullptr;
    PR_CHECK(scaph_graph_open(prefix.c_str(), weighted, &g));
    scaph_graph_info info;
    PR_CHECK(scaph_graph_get_info(g, &info));
    const uint32_t V = info.V, nw = (V + 31) / 32;
    scaph_store *store = nullptr;
    PR_CHECK(scaph_store_create(g, max_memory_mb * (1ll << 20), threshold, 2, device, &store));
    int sms = 148;
    PR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));

    float *rank, *contrib, *acc;
    uint32_t *active;
    double *scal;  // dangling, l1
    PR_CUDA(cudaMalloc(&rank, 4ull * V));
    PR_CUDA(cudaMalloc(&contrib, 4ull * V));
    PR_CUDA(cudaMalloc(&acc, 4ull * V));
    PR_CUDA(cudaMalloc(&active, 4ull * nw));
    PR_CUDA(cudaMalloc(&scal, 2 * sizeof(double)));
    // every vertex pushes every iteration: all pages are needed
    std::vector<uint32_t> ones(nw, 0xFFFFFFFFu);
    if (V & 31) ones[nw - 1] = (1u << (V & 31)) - 1u;
    PR_CUDA(cudaMemcpy(active, ones.data(), 4ull * nw, cudaMemcpyHostToDevice));
    cudaStream_t st;
    PR_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const int grid = sms * 4;
    k_fill<<<grid, kBlock, 0, st>>>(rank, V, 1.f / (float)V);
    PR_CUDA(cudaMemsetAsync(acc, 0, 4ull * V, st));
    uint64_t h0 = 0, z0 = 0, f0 = 0;
    PR_CHECK(scaph_store_counters(store, &h0, &z0, &f0));
    PushArgs pa{contrib, acc, sms * 8};
    double l1 = 0.0;
    cudaEvent_t e0, e1;
    PR_CUDA(cudaEventCreate(&e0));
    PR_CUDA(cudaEventCreate(&e1));
    PR_CUDA(cudaEventRecord(e0, st));
    for (int it = 0; it < iters; it++) {
        PR_CUDA(cudaMemsetAsync(scal, 0, 2 * sizeof(double), st));
        k_contrib<<<grid, kBlock, 0, st>>>(rank, scaph_store_degree(store), V, contrib, scal);
        PR_CHECK(scaph_store_level(store, active, &push_batch, &pa, st));
        k_apply<<<grid, kBlock, 0, st>>>(rank, acc, V, (float)damping, scal, scal + 1);
        PR_CUDA(cudaGetLastError());
    }
    PR_CUDA(cudaEventRecord(e1, st));
    PR_CUDA(cudaMemcpyAsync(&l1, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    PR_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    PR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    uint64_t h1 = 0, z1 = 0, f1 = 0;
    PR_CHECK(scaph_store_counters(store, &h1, &z1, &f1));
    if (!out.empty()) {
        std::vector<float> h(V);
        PR_CUDA(cudaMemcpy(h.data(), rank, 4ull * V, cudaMemcpyDeviceToHost));
        FILE *f = fopen(out.c_str(), "wb");
        if (!f || fwrite(h.data(), 4, V, f) != V) {
            fprintf(stderr, "cannot write %s\n", out.c_str());
            return 2;
        }
        fclose(f);
    }
    printf("pagerank iters=%d l1=%.6e ms=%.3f resident=%d h2d=%llu zc=%llu faults=%llu\n", iters, l1, ms,
           scaph_store_resident(store), (unsigned long long)(h1 - h0), (unsigned long long)(z1 - z0),
           (unsigned long long)(f1 - f0));
    cudaFree(rank);
    cudaFree(contrib);
    cudaFree(acc);
    cudaFree(active);
    cudaFree(scal);
    cudaStreamDestroy(st);
    scaph_store_destroy(store);
    scaph_graph_close(g);
    return 0;
}
