// Level kernels of the level-synchronous BFS, written for sm_100a.
//
// push (top-down): replaces gpu_push_csr (src/gpu_engine.cuh:41-169).  The
//   reference walks every Node of a page with a static vertex split per CTA
//   and a CAS min per edge.  Here a CTA takes a tile of frontier-bitmap
//   words, compacts the set bits into a shared-memory queue (popc + block
//   scan), reads the queued vertices' page headers, and expands their
//   adjacency with 128-bit loads, edge-balanced across the CTA by a scan over
//   16-byte quads.  Visited marking is one atomicOr on the visited bitmap
//   (the winner writes depth/parent and the next-frontier bit), so depths are
//   exact.  Adjacency longer than kGiantEdges is cut into chunks that a
//   second kernel spreads over the whole GPU.
// pull (bottom-up): has no reference counterpart (gpu_pull_iteration is a
//   stub, src/app.cuh:365-369).  A warp owns one word (32 vertices) of the
//   visited bitmap, so visited/next words are written without atomics; each
//   unvisited vertex scans its in-edges against the frontier bitmap and
//   stops at the first hit (thread-per-vertex for the first few edges, then
//   warp-cooperative with ballot).
// Both fold the per-page frontier statistics of get_page_info
// (src/gpu_engine.cuh:397-441) into their epilogue: a shared-memory
// histogram of the next frontier by page, flushed once per CTA.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace scaph {

namespace {

template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t *wsum, uint32_t &total)
{
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < NW ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < NW) wsum[lane] = t;
    }
    __syncthreads();
    uint32_t base = wid ? wsum[wid - 1] : 0u;
    total = wsum[NW - 1];
    __syncthreads();
    return base + inc - x;
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
    return x;
}

// Per-CTA accumulators flushed once at kernel exit.
struct CtaAcc {
    unsigned long long next, next_edges, inspected, headers;
};

template <int BLOCK>
__device__ __forceinline__ void flush_acc(CtaAcc *acc, unsigned long long next, unsigned long long next_edges,
                                          unsigned long long inspected, unsigned long long headers,
                                          LevelCounters *ctr)
{
    next = warp_sum64(next);
    next_edges = warp_sum64(next_edges);
    inspected = warp_sum64(inspected);
    headers = warp_sum64(headers);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc->next, next);
        atomicAdd(&acc->next_edges, next_edges);
        atomicAdd(&acc->inspected, inspected);
        atomicAdd(&acc->headers, headers);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (acc->next) atomicAdd(&ctr->next, acc->next);
        if (acc->next_edges) atomicAdd(&ctr->next_edges, acc->next_edges);
        if (acc->inspected) atomicAdd(&ctr->inspected, acc->inspected);
        if (acc->headers) atomicAdd(&ctr->headers, acc->headers);
    }
}

// Adds vertex u (out-degree + 3 words, the reference's `datas` unit) to the
// next-frontier histogram over the pages of the out-edge graph s.hg.
__device__ __forceinline__ void hist_add(uint32_t *hn, uint32_t *hd, const BfsDev &s, uint32_t u, uint32_t datas)
{
    if (!s.page_nodes) return;
    const int p = page_of(s.hg, u);
    if (p < kHistCap) {
        atomicAdd(&hn[p], 1u);
        atomicAdd(&hd[p], datas);
    } else {
        atomicAdd(&s.page_nodes[p], 1u);
        atomicAdd(&s.page_datas[p], datas);
    }
}

template <int BLOCK>
__device__ __forceinline__ void hist_init(uint32_t *hn, uint32_t *hd, const BfsDev &s)
{
    if (!s.page_nodes) return;
    const int n = s.hg.npages < (uint32_t)kHistCap ? (int)s.hg.npages : kHistCap;
    for (int i = threadIdx.x; i < n; i += BLOCK) { hn[i] = 0; hd[i] = 0; }
}

template <int BLOCK>
__device__ __forceinline__ void hist_flush(const uint32_t *hn, const uint32_t *hd, const BfsDev &s)
{
    if (!s.page_nodes) return;
    const int n = s.hg.npages < (uint32_t)kHistCap ? (int)s.hg.npages : kHistCap;
    for (int i = threadIdx.x; i < n; i += BLOCK) {
        if (hn[i]) {
            atomicAdd(&s.page_nodes[i], hn[i]);
            atomicAdd(&s.page_datas[i], hd[i]);
        }
    }
}

// Claims vertex u for the next frontier.  Returns true for the one thread that
// flips its visited bit.
__device__ __forceinline__ bool claim(const BfsDev &s, uint32_t u, uint32_t src)
{
    const uint32_t w = u >> 5, bit = 1u << (u & 31);
    if (*((volatile const uint32_t *)&s.visited[w]) & bit) return false;
    const uint32_t old = atomicOr(&s.visited[w], bit);
    if (old & bit) return false;
    s.depth[u] = s.level + 1;
    if (s.parent) s.parent[u] = src;
    atomicOr(&s.next[w], bit);
    return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// push level
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push(GraphDev g, BfsDev s, uint32_t vlo, uint32_t vhi)
{
    constexpr int TW = BLOCK < 256 ? BLOCK : 256;  // bitmap words per tile
    __shared__ uint32_t q[TW * 32];
    __shared__ unsigned long long ebase[BLOCK];
    __shared__ uint32_t elen[BLOCK];
    __shared__ uint32_t qoff[BLOCK];
    __shared__ uint32_t wsum[BLOCK / 32];
    __shared__ uint32_t hn[kHistCap], hd[kHistCap];
    __shared__ CtaAcc acc;

    if (threadIdx.x == 0) acc = CtaAcc{0, 0, 0, 0};
    hist_init<BLOCK>(hn, hd, s);
    __syncthreads();

    unsigned long long my_next = 0, my_edges = 0, my_insp = 0, my_hdr = 0;
    const uint32_t ew = s.weighted_edges ? 2u : 1u;
    const uint32_t wlo = vlo >> 5, whi = (uint32_t)(((unsigned long long)vhi + 31) >> 5);
    const uint32_t ntiles = (whi - wlo + TW - 1) / TW;

    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t w = wlo + tile * TW + threadIdx.x;
        uint32_t f = 0;
        if (threadIdx.x < TW && w < whi) f = s.front[w] & range_mask(w, vlo, vhi);
        uint32_t total;
        uint32_t off = block_exclusive_scan<BLOCK>(__popc(f), wsum, total);
        if (total == 0) continue;
        while (f) {
            q[off++] = (w << 5) + (__ffs(f) - 1);
            f &= f - 1;
        }
        __syncthreads();
        for (uint32_t c0 = 0; c0 < total; c0 += BLOCK) {
            const uint32_t k = c0 + threadIdx.x;
            uint32_t nq = 0;
            if (k < total) {
                const uint32_t v = q[k];
                const int p = page_of(g, v);
                const PageDev pd = g.pages[p];
                uint32_t len = 0;
                unsigned long long st = 0;
                if (pd.base != kNotResident) {
                    const uint32_t *node = g.pool + pd.base + 3ull * (v - pd.left);
                    const uint32_t pos = node[1];
                    len = node[2];
                    st = pd.base + 3ull * pd.nodenum + (unsigned long long)pos * ew;
                    my_hdr++;
                    my_insp += len;
                    if (len > kGiantEdges && ew == 1) {
                        const uint32_t nch = (len + kGiantEdges - 1) / kGiantEdges;
                        const uint32_t at = atomicAdd(&s.ctr->giant, nch);
                        if (at + nch <= s.giant_cap) {
                            for (uint32_t c = 0; c < nch; c++) {
                                GiantChunk gc;
                                gc.start = st + (unsigned long long)c * kGiantEdges;
                                gc.len = min(kGiantEdges, len - c * kGiantEdges);
                                gc.src = v;
                                s.giant[at + c] = gc;
                            }
                            len = 0;
                        } else {
                            atomicOr(&s.ctr->error, 2u);  // giant queue overflow: expand here
                        }
                    }
                } else {
                    atomicOr(&s.ctr->error, 4u);  // frontier vertex on a non-resident page
                }
                ebase[threadIdx.x] = st;
                elen[threadIdx.x] = len * ew;
                nq = len ? (uint32_t)(((st + (unsigned long long)len * ew + 3) >> 2) - (st >> 2)) : 0u;
            }
            uint32_t tq;
            const uint32_t qo = block_exclusive_scan<BLOCK>(nq, wsum, tq);
            qoff[threadIdx.x] = qo;
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < tq; i += BLOCK) {
                int lo = 0, hi = BLOCK - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (qoff[mid] <= i) lo = mid; else hi = mid - 1;
                }
                const unsigned long long st = ebase[lo];
                const unsigned long long en = st + elen[lo];
                const unsigned long long quad = (st >> 2) + (i - qoff[lo]);
                const uint4 val = ld_nc_v4(g.pool + quad * 4);
                const uint32_t src = q[c0 + lo];
                const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const unsigned long long word = quad * 4 + j;
                    if (word >= st && word < en && ((word - st) % ew) == 0) {
                        const uint32_t u = vals[j];
                        if (u < s.V && claim(s, u, src)) {
                            my_next++;
                            const uint32_t du = __ldg(&s.degree[u]);
                            my_edges += du;
                            hist_add(hn, hd, s, u, du + 3);
                        } else if (u >= s.V) {
                            atomicOr(&s.ctr->error, 1u);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    __syncthreads();
    flush_acc<BLOCK>(&acc, my_next, my_edges, my_insp, my_hdr, s.ctr);
    hist_flush<BLOCK>(hn, hd, s);
}

// Giant adjacency chunks queued by k_push: one CTA per chunk, grid-stride.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_giant(GraphDev g, BfsDev s)
{
    __shared__ uint32_t hn[kHistCap], hd[kHistCap];
    __shared__ CtaAcc acc;
    if (threadIdx.x == 0) acc = CtaAcc{0, 0, 0, 0};
    hist_init<BLOCK>(hn, hd, s);
    __syncthreads();
    unsigned long long my_next = 0, my_edges = 0;
    const uint32_t n = min(*((volatile uint32_t *)&s.ctr->giant), s.giant_cap);
    for (uint32_t c = blockIdx.x; c < n; c += gridDim.x) {
        const GiantChunk gc = s.giant[c];
        if (gc.len > kGiantEdges || gc.start + gc.len > g.pool_words || gc.src >= s.V) {
            if (threadIdx.x == 0) atomicOr(&s.ctr->error, 8u);  // corrupt chunk record
            continue;
        }
        const unsigned long long st = gc.start, en = gc.start + gc.len;
        const unsigned long long q0 = st >> 2, q1 = (en + 3) >> 2;
        for (unsigned long long qd = q0 + threadIdx.x; qd < q1; qd += BLOCK) {
            const uint4 val = ld_nc_v4(g.pool + qd * 4);
            const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const unsigned long long word = qd * 4 + j;
                if (word >= st && word < en) {
                    const uint32_t u = vals[j];
                    if (u < s.V && claim(s, u, gc.src)) {
                        my_next++;
                        const uint32_t du = __ldg(&s.degree[u]);
                        my_edges += du;
                        hist_add(hn, hd, s, u, du + 3);
                    } else if (u >= s.V) {
                        atomicOr(&s.ctr->error, 1u);
                    }
                }
            }
        }
    }
    __syncthreads();
    flush_acc<BLOCK>(&acc, my_next, my_edges, 0, 0, s.ctr);
    hist_flush<BLOCK>(hn, hd, s);
}

// ---------------------------------------------------------------------------
// pull level (g = in-edge graph)
// ---------------------------------------------------------------------------
constexpr uint32_t kPullSerial = 4;  // edges each lane tries alone before the warp helps

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pull(GraphDev g, BfsDev s, uint32_t vlo, uint32_t vhi)
{
    __shared__ uint32_t hn[kHistCap], hd[kHistCap];
    __shared__ CtaAcc acc;
    if (threadIdx.x == 0) acc = CtaAcc{0, 0, 0, 0};
    hist_init<BLOCK>(hn, hd, s);
    __syncthreads();

    unsigned long long my_next = 0, my_edges = 0, my_insp = 0, my_hdr = 0;
    const int lane = threadIdx.x & 31;
    const uint32_t ew = s.weighted_edges ? 2u : 1u;
    const uint32_t wlo = vlo >> 5, whi = (uint32_t)(((unsigned long long)vhi + 31) >> 5);
    const uint32_t wstride = (gridDim.x * BLOCK) >> 5;

    for (uint32_t w = wlo + ((blockIdx.x * BLOCK + threadIdx.x) >> 5); w < whi; w += wstride) {
        const uint32_t vis = s.visited[w];
        const uint32_t unv = ~vis & range_mask(w, vlo, vhi);
        if (!unv) continue;
        const uint32_t v = (w << 5) + lane;
        const bool mine = (unv >> lane) & 1u;
        uint32_t len = 0, found = 0, par = kNoParent, k = 0;
        unsigned long long st = 0;
        if (mine) {
            const int p = page_of(g, v);
            const PageDev pd = g.pages[p];
            if (pd.base != kNotResident) {
                const uint32_t *node = g.pool + pd.base + 3ull * (v - pd.left);
                const uint32_t pos = node[1];
                len = node[2];
                st = pd.base + 3ull * pd.nodenum + (unsigned long long)pos * ew;
                my_hdr++;
                const uint32_t lim = min(len, kPullSerial);
                for (; k < lim; k++) {
                    const uint32_t u = __ldg(&g.pool[st + (unsigned long long)k * ew]);
                    if (u < s.V && test_bit(s.front, u)) {
                        found = 1;
                        par = u;
                        k++;
                        break;
                    }
                }
                my_insp += k;
            } else {
                atomicOr(&s.ctr->error, 4u);
            }
        }
        // warp-cooperative scan of the lanes that still have edges left
        uint32_t need = __ballot_sync(0xFFFFFFFFu, mine && !found && len > kPullSerial);
        while (need) {
            const int leader = __ffs(need) - 1;
            need &= need - 1;
            const unsigned long long lst = __shfl_sync(0xFFFFFFFFu, st, leader);
            const uint32_t llen = __shfl_sync(0xFFFFFFFFu, len, leader);
            uint32_t hit_par = kNoParent, scanned = llen - kPullSerial;
            for (uint32_t j0 = kPullSerial; j0 < llen; j0 += 32) {
                const uint32_t j = j0 + lane;
                uint32_t u = 0;
                bool hit = false;
                if (j < llen) {
                    u = __ldg(&g.pool[lst + (unsigned long long)j * ew]);
                    hit = u < s.V && test_bit(s.front, u);
                }
                const uint32_t b = __ballot_sync(0xFFFFFFFFu, hit);
                if (b) {
                    const int first = __ffs(b) - 1;
                    hit_par = __shfl_sync(0xFFFFFFFFu, u, first);
                    scanned = j0 + first + 1 - kPullSerial;
                    break;
                }
            }
            if (lane == leader) {
                my_insp += scanned;
                if (hit_par != kNoParent) { found = 1; par = hit_par; }
            }
        }
        const uint32_t fmask = __ballot_sync(0xFFFFFFFFu, found);
        if (found) {
            s.depth[v] = s.level + 1;
            if (s.parent) s.parent[v] = par;
            const uint32_t dv = __ldg(&s.degree[v]);
            my_next++;
            my_edges += dv;
            hist_add(hn, hd, s, v, dv + 3);
        }
        if (lane == 0 && fmask) {
            s.visited[w] = vis | fmask;
            s.next[w] = fmask;
        }
    }
    __syncthreads();
    flush_acc<BLOCK>(&acc, my_next, my_edges, my_insp, my_hdr, s.ctr);
    hist_flush<BLOCK>(hn, hd, s);
}

// ---------------------------------------------------------------------------
// state init: depth = unreached, parent = none, bitmaps cleared, then the
// source (bfs_init + setsrc of app/bfs.cu:20-37)
// ---------------------------------------------------------------------------
__global__ void k_fill_u32_scalar(uint32_t *p, uint32_t value, unsigned long long n)
{
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n; i += stride)
        p[i] = value;
}

// p must be 16-byte aligned (fill_u32 checks)
__global__ void k_fill_u32(uint32_t *p, uint32_t value, unsigned long long n)
{
    const unsigned long long n4 = n / 4;
    uint4 v4 = make_uint4(value, value, value, value);
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n4; i += stride)
        reinterpret_cast<uint4 *>(p)[i] = v4;
    for (unsigned long long i = n4 * 4 + blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n; i += stride)
        p[i] = value;
}

__global__ void k_set_source(BfsDev s, uint32_t src, uint32_t *front)
{
    s.depth[src] = 0;
    if (s.parent) s.parent[src] = src;
    s.visited[src >> 5] |= 1u << (src & 31);
    front[src >> 5] |= 1u << (src & 31);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// The push kernel's static shared memory (tile queue + page histogram) caps
// it at 256 threads; 512-thread configurations run push at 256.
template <int BLOCK>
static cudaError_t launch_level(int dir, int grid, const GraphDev &g, const BfsDev &s, uint32_t vlo, uint32_t vhi,
                                cudaStream_t st)
{
    constexpr int PB = BLOCK > 256 ? 256 : BLOCK;
    if (dir == 0) {
        k_push<PB><<<grid, PB, 0, st>>>(g, s, vlo, vhi);
        k_push_giant<PB><<<grid, PB, 0, st>>>(g, s);
    } else {
        k_pull<BLOCK><<<grid, BLOCK, 0, st>>>(g, s, vlo, vhi);
    }
    return cudaGetLastError();
}

cudaError_t run_level(int dir, int block, int grid, const GraphDev &g, const BfsDev &s, uint32_t vlo, uint32_t vhi,
                      cudaStream_t st)
{
    switch (block) {
    case 128: return launch_level<128>(dir, grid, g, s, vlo, vhi, st);
    case 512: return launch_level<512>(dir, grid, g, s, vlo, vhi, st);
    default: return launch_level<256>(dir, grid, g, s, vlo, vhi, st);
    }
}

int level_occupancy(int dir, int block)
{
    int n = 0;
    switch (block) {
    case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dir ? (const void *)k_pull<128> : (const void *)k_push<128>, 128, 0); break;
    case 512:
        if (dir) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void *)k_pull<512>, 512, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void *)k_push<256>, 256, 0);
        break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dir ? (const void *)k_pull<256> : (const void *)k_push<256>, 256, 0); break;
    }
    return n;
}

cudaError_t fill_u32(uint32_t *p, uint32_t value, unsigned long long n, int grid, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    if (reinterpret_cast<uintptr_t>(p) & 15) k_fill_u32_scalar<<<grid, 256, 0, st>>>(p, value, n);
    else k_fill_u32<<<grid, 256, 0, st>>>(p, value, n);
    return cudaGetLastError();
}

cudaError_t set_source(const BfsDev &s, uint32_t src, uint32_t *front, cudaStream_t st)
{
    k_set_source<<<1, 1, 0, st>>>(s, src, front);
    return cudaGetLastError();
}

}  // namespace scaph
