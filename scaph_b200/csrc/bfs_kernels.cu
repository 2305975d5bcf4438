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
//   stub, src/app.cuh:365-369).  A CTA takes a tile of visited-bitmap words
//   and compacts the tile's unvisited vertices into a shared queue.  Phase A:
//   each thread takes two of them at a time, reads their in-degrees and
//   dense head rows (in-neighbours ranked by out-degree) with all loads
//   issued before any frontier probe, and probes the top-ranked neighbour
//   first.  Vertices still unresolved are scanned by groups of eight lanes,
//   32 in-edges per step with 128-bit loads, up to the first frontier hit
//   (phase B).  Found vertices are collected in a shared bitmap and written
//   back once per tile word.
// Both stage the page table and coarse index in shared memory, and fold the
// per-page frontier statistics of get_page_info (src/gpu_engine.cuh:397-441)
// into their epilogue: a shared-memory histogram of the next frontier by
// page, flushed once per CTA.
//
// Two entry points per level kernel: one takes the level's state as kernel
// arguments (host-driven loop, out-of-core page batches), the other reads it
// from a device control block (graph mode: a whole BFS is one CUDA-graph
// launch whose level loop is a conditional WHILE node, see engine.cu).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace scaph {

namespace {

#ifndef SCAPH_PULL_SERIAL
#define SCAPH_PULL_SERIAL 4
#endif
constexpr int kPushTileWords = 128;                  // frontier-bitmap words per push tile
#ifndef SCAPH_PULL_DEFER_B
#define SCAPH_PULL_DEFER_B 1  // pull phase B waits for several rounds' vertices (see pull_body)
#endif
#ifndef SCAPH_PULL_FIRST_PROBE
#define SCAPH_PULL_FIRST_PROBE 1
#endif
#ifndef SCAPH_PULL_PER_THREAD
#define SCAPH_PULL_PER_THREAD 2
#endif
#ifndef SCAPH_PULL_GROUP
#define SCAPH_PULL_GROUP 8  // lanes per unresolved vertex in pull phase B
#endif
#ifndef SCAPH_PULL_MINB
#define SCAPH_PULL_MINB 1024
#endif
constexpr int kPullPerThread = SCAPH_PULL_PER_THREAD;  // unvisited vertices each thread takes per pull round
constexpr int kPullTileWords = 128;                  // visited-bitmap words per pull tile (the range-list tile)
constexpr int kPullMinThreads = SCAPH_PULL_MINB;     // resident threads per SM the pull kernel is compiled for
#ifndef SCAPH_PUSH_MINB
#define SCAPH_PUSH_MINB 1024
#endif
// resident threads per SM the push kernels are compiled for: 4 CTAs of 256
// threads get 64 registers (the graph-mode kernel's level-state setup
// spilled at the 48 registers that 5 CTAs allow)
constexpr int kPushMinThreads = SCAPH_PUSH_MINB;
constexpr uint32_t kPullSerial = SCAPH_PULL_SERIAL;  // in-edges each lane probes before the warp helps
static_assert(kPullSerial == kPullHead, "phase A reads one dense head row of in-edges");

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

// per-thread counts stay below 2^32: a level touches each vertex once and
// each of the < 2^32 edges of a paged graph at most once
struct ThreadAcc {
    uint32_t next = 0, next_edges = 0, inspected = 0, headers = 0;
};

template <int BLOCK>
__device__ __forceinline__ void flush_acc(CtaAcc *acc, ThreadAcc t, LevelCounters *ctr)
{
    const unsigned long long n = warp_sum64(t.next), ne = warp_sum64(t.next_edges);
    const unsigned long long in = warp_sum64(t.inspected), h = warp_sum64(t.headers);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc->next, n);
        atomicAdd(&acc->next_edges, ne);
        atomicAdd(&acc->inspected, in);
        atomicAdd(&acc->headers, h);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (acc->next) atomicAdd(&ctr->next, acc->next);
        if (acc->next_edges) atomicAdd(&ctr->next_edges, acc->next_edges);
        if (acc->inspected) atomicAdd(&ctr->inspected, acc->inspected);
        if (acc->headers) atomicAdd(&ctr->headers, acc->headers);
    }
}

// Shared-memory working set common to the level kernels.
constexpr int kHistInCap = 256;  // in-pages counted in shared memory (the rest: global atomics)

struct LevelSmem {
    uint32_t hn[kHistCap], hd[kHistCap];
    uint32_t hni[kHistInCap], hdi[kHistInCap];  // in-page histogram (page_nodes_in)
    PageDev lut_pages[kLutPages];
    uint32_t lut_coarse[kLutCoarse];
    CtaAcc acc;
};

// Stages g's page table + coarse index in shared memory when they fit.
template <int BLOCK>
__device__ __forceinline__ PageLut stage_lut(const GraphDev &g, LevelSmem &sm)
{
    const uint32_t ncoarse = (g.V >> g.cshift) + 1;
    if (g.npages + 1 <= (uint32_t)kLutPages && ncoarse <= (uint32_t)kLutCoarse) {
        for (uint32_t i = threadIdx.x; i <= g.npages; i += BLOCK) sm.lut_pages[i] = g.pages[i];
        for (uint32_t i = threadIdx.x; i < ncoarse; i += BLOCK) sm.lut_coarse[i] = g.coarse[i];
        return PageLut{sm.lut_pages, sm.lut_coarse, g.cshift};
    }
    return PageLut{g.pages, g.coarse, g.cshift};
}

template <int BLOCK>
__device__ __forceinline__ void level_prologue(LevelSmem &sm, const BfsDev &s)
{
    if (threadIdx.x == 0) sm.acc = CtaAcc{0, 0, 0, 0};
    if (s.page_nodes) {
        const int n = s.hg.npages < (uint32_t)kHistCap ? (int)s.hg.npages : kHistCap;
        for (int i = threadIdx.x; i < n; i += BLOCK) {
            sm.hn[i] = 0;
            sm.hd[i] = 0;
        }
    }
    if (s.page_nodes_in) {
        const int n = s.hgi.npages < (uint32_t)kHistInCap ? (int)s.hgi.npages : kHistInCap;
        for (int i = threadIdx.x; i < n; i += BLOCK) {
            sm.hni[i] = 0;
            sm.hdi[i] = 0;
        }
    }
}

template <int BLOCK>
__device__ __forceinline__ void level_epilogue(LevelSmem &sm, const BfsDev &s, const ThreadAcc &t)
{
    __syncthreads();
    flush_acc<BLOCK>(&sm.acc, t, s.ctr);
    if (s.page_nodes) {
        const int n = s.hg.npages < (uint32_t)kHistCap ? (int)s.hg.npages : kHistCap;
        for (int i = threadIdx.x; i < n; i += BLOCK) {
            if (sm.hn[i]) {
                atomicAdd(&s.page_nodes[i], sm.hn[i]);
                atomicAdd(&s.page_datas[i], sm.hd[i]);
            }
        }
    }
    if (s.page_nodes_in) {
        const int n = s.hgi.npages < (uint32_t)kHistInCap ? (int)s.hgi.npages : kHistInCap;
        for (int i = threadIdx.x; i < n; i += BLOCK) {
            if (sm.hni[i]) {
                atomicAdd(&s.page_nodes_in[i], sm.hni[i]);
                atomicAdd(&s.page_datas_in[i], sm.hdi[i]);
            }
        }
    }
}

// Adds a discovered vertex (page p of the histogram graph; out-degree + 3
// words, the reference's `datas` unit) to the next-frontier histogram.
__device__ __forceinline__ void hist_add(LevelSmem &sm, const BfsDev &s, int p, uint32_t datas)
{
    if (p < kHistCap) {
        atomicAdd(&sm.hn[p], 1u);
        atomicAdd(&sm.hd[p], datas);
    } else {
        atomicAdd(&s.page_nodes[p], 1u);
        atomicAdd(&s.page_datas[p], datas);
    }
}

// Adds discovered vertex v to the in-page histogram (in-degree + 3 words).
__device__ __forceinline__ void hist_in_add(LevelSmem &sm, const BfsDev &s, uint32_t v)
{
    if (!s.page_nodes_in) return;
    const int p = page_of(s.hgi, v);
    const uint32_t d = __ldg(&s.indeg[v]) + 3;
    if (p < kHistInCap) {
        atomicAdd(&sm.hni[p], 1u);
        atomicAdd(&sm.hdi[p], d);
    } else {
        atomicAdd(&s.page_nodes_in[p], 1u);
        atomicAdd(&s.page_datas_in[p], d);
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

// Visits up to four neighbours of `src` (in[j] marks the valid ones): the
// four visited words are read first, all at once, and only neighbours whose
// bit is still clear go on to the atomic claim.
__device__ __forceinline__ void visit4(LevelSmem &sm, const BfsDev &s, ThreadAcc &t, const uint32_t (&u)[4],
                                       const bool (&in)[4], uint32_t src, bool hist_same, const PageLut &lut)
{
    uint32_t vw[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        vw[j] = (in[j] && u[j] < s.V) ? *((volatile const uint32_t *)&s.visited[u[j] >> 5]) : 0xFFFFFFFFu;
    if (s.push_defer) {
        // deferred claims: visited does not change during the level, so an
        // unvisited neighbour's bit goes straight into the next frontier
        // (fire-and-forget reduction); k_push_finalize does the rest
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (!in[j]) continue;
            if (u[j] >= s.V) {
                atomicOr(&s.ctr->error, 1u);
                continue;
            }
            if (!((vw[j] >> (u[j] & 31)) & 1u))
                atomicOr(s.next + (u[j] >> 5), 1u << (u[j] & 31));  // result unused: a reduction
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (!in[j]) continue;
        if (u[j] >= s.V) {
            atomicOr(&s.ctr->error, 1u);
            continue;
        }
        if ((vw[j] >> (u[j] & 31)) & 1u) continue;
        if (!claim(s, u[j], src)) continue;
        t.next++;
        const uint32_t du = __ldg(&s.degree[u[j]]);
        t.next_edges += du;
        if (s.page_nodes) hist_add(sm, s, hist_same ? lut.of(u[j]) : page_of(s.hg, u[j]), du + 3);
        hist_in_add(sm, s, u[j]);
    }
}

// ---------------------------------------------------------------------------
// bodies
// ---------------------------------------------------------------------------
template <int BLOCK>
__device__ __forceinline__ void push_body(const GraphDev &g, const BfsDev &s, uint32_t vlo, uint32_t vhi,
                                          const RangeList &rl)
{
    __shared__ LevelSmem sm;
    __shared__ uint32_t q[kPushTileWords * 32];
    __shared__ unsigned long long ebase[BLOCK];
    __shared__ uint32_t elen[BLOCK];
    __shared__ uint32_t qoff[BLOCK];
    __shared__ uint32_t wsum[BLOCK / 32];

    level_prologue<BLOCK>(sm, s);
    const PageLut lut = stage_lut<BLOCK>(g, sm);
    const bool hist_same = s.hg.pages == g.pages;
    __syncthreads();

    ThreadAcc t;
    const uint32_t ntiles = rl.n ? rl.tile0[rl.n]
                                 : (((uint32_t)(((unsigned long long)vhi + 31) >> 5)) - (vlo >> 5) + kPushTileWords - 1) /
                                       kPushTileWords;

    // expands the frontier vertices q[0, total), BLOCK at a time (every
    // thread of the CTA calls it)
    auto run_queue = [&](uint32_t total) {
        for (uint32_t c0 = 0; c0 < total; c0 += BLOCK) {
            const uint32_t k = c0 + threadIdx.x;
            uint32_t nq = 0;
            if (k < total) {
                const uint32_t v = q[k];
                const int p = lut.of(v);
                const PageDev pd = lut.pages[p];
                uint32_t len = 0;
                unsigned long long st = 0;
                if (pd.base != kNotResident) {
                    const uint32_t *node = g.pool + pd.base + 3ull * (v - pd.left);
                    const uint32_t pos = node[1];
                    len = node[2];
                    st = pd.base + 3ull * pd.nodenum + pos;
                    t.headers++;
                    t.inspected += len;
                    const uint32_t ge = s.giant_edges ? s.giant_edges : kGiantEdges;
                    if (len > ge) {
                        const uint32_t nch = (len + ge - 1) / ge;
                        const uint32_t at = atomicAdd(&s.ctr->giant, nch);
                        if (at + nch <= s.giant_cap) {
                            for (uint32_t c = 0; c < nch; c++) {
                                GiantChunk gc;
                                gc.start = st + (unsigned long long)c * ge;
                                gc.len = min(ge, len - c * ge);
                                gc.src = v;
                                s.giant[at + c] = gc;
                            }
                            len = 0;
                        } else {
                            atomicOr(&s.ctr->error, 2u);  // cannot happen: the queue holds 2E/4096+1024
                        }
                    }
                } else {
                    atomicOr(&s.ctr->error, 4u);  // frontier vertex on a non-resident page
                }
                ebase[threadIdx.x] = st;
                elen[threadIdx.x] = len;
                nq = len ? (uint32_t)(((st + len + 3) >> 2) - (st >> 2)) : 0u;
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
                bool in[4];
#pragma unroll
                for (int j = 0; j < 4; j++) in[j] = quad * 4 + j >= st && quad * 4 + j < en;
                visit4(sm, s, t, vals, in, src, hist_same, lut);
            }
            __syncthreads();
        }
    };

    if (s.push_sparse && rl.n == 0) {
        // ---- sparse level: the CTA owns one contiguous run of frontier
        // words and reads it BLOCK*4 words per round (each thread four
        // coalesced words), so that its few frontier vertices are found with
        // one round trip and expanded together, not one tile after another
        const uint32_t wlo = vlo >> 5, whi = (uint32_t)(((unsigned long long)vhi + 31) >> 5);
        const uint32_t per = (whi - wlo + gridDim.x - 1) / gridDim.x;
        const uint32_t w0 = wlo + blockIdx.x * per, w1 = min(whi, w0 + per);
        constexpr uint32_t kCap = kPushTileWords * 32;  // q's capacity
        for (uint32_t cw = w0; cw < w1; cw += 4 * BLOCK) {
            uint32_t f[4], n = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t w = cw + k * BLOCK + threadIdx.x;
                f[k] = w < w1 ? s.front[w] & range_mask(w, vlo, vhi) : 0u;
                n += __popc(f[k]);
            }
            if (!__syncthreads_or(n != 0)) continue;
            uint32_t total;
            const uint32_t off = block_exclusive_scan<BLOCK>(n, wsum, total);
            // more vertices than q holds (a dense run): windows of kCap
            for (uint32_t lo = 0; lo < total; lo += kCap) {
                uint32_t at = off;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    uint32_t m = f[k];
                    const uint32_t base = (cw + k * BLOCK + threadIdx.x) << 5;
                    while (m) {
                        if (at >= lo && at < lo + kCap) q[at - lo] = base + (__ffs(m) - 1);
                        at++;
                        m &= m - 1;
                    }
                }
                __syncthreads();
                run_queue(min(kCap, total - lo));
            }
        }
    } else {
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            uint32_t rlo = vlo, rhi = vhi, local;
            range_of_tile(rl, tile, rlo, rhi, local);
            const uint32_t rwhi = (uint32_t)(((unsigned long long)rhi + 31) >> 5);
            const uint32_t w = (rlo >> 5) + local * kPushTileWords + threadIdx.x;
            uint32_t f = 0;
            if (threadIdx.x < kPushTileWords && w < rwhi) f = s.front[w] & range_mask(w, rlo, rhi);
            if (!__syncthreads_or(f != 0)) continue;
            uint32_t total;
            uint32_t off = block_exclusive_scan<BLOCK>(__popc(f), wsum, total);
            if (total == 0) continue;
            while (f) {
                q[off++] = (w << 5) + (__ffs(f) - 1);
                f &= f - 1;
            }
            __syncthreads();
            run_queue(total);
        }
    }
    level_epilogue<BLOCK>(sm, s, t);
}

// sm: the level's shared state, declared by the calling kernel (one copy
// in a kernel that runs either of two bodies)
template <int BLOCK>
__device__ __forceinline__ void giant_body(const GraphDev &g, const BfsDev &s, LevelSmem &sm)
{
    const uint32_t n = min(*((volatile uint32_t *)&s.ctr->giant), s.giant_cap);
    if (blockIdx.x >= n) return;  // whole CTA: no chunk for it
    level_prologue<BLOCK>(sm, s);
    const PageLut lut = stage_lut<BLOCK>(s.hg, sm);
    __syncthreads();
    ThreadAcc t;
    for (uint32_t c = blockIdx.x; c < n; c += gridDim.x) {
        const GiantChunk gc = s.giant[c];
        if (gc.len > (s.giant_edges ? s.giant_edges : kGiantEdges) || gc.start + gc.len > g.pool_words ||
            gc.src >= s.V) {
            if (threadIdx.x == 0) atomicOr(&s.ctr->error, 8u);  // corrupt chunk record
            continue;
        }
        const unsigned long long st = gc.start, en = gc.start + gc.len;
        const unsigned long long q0 = st >> 2, q1 = (en + 3) >> 2;
        for (unsigned long long qd = q0 + threadIdx.x; qd < q1; qd += BLOCK) {
            const uint4 val = ld_nc_v4(g.pool + qd * 4);
            const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
            bool in[4];
#pragma unroll
            for (int j = 0; j < 4; j++) in[j] = qd * 4 + j >= st && qd * 4 + j < en;
            visit4(sm, s, t, vals, in, gc.src, true, lut);
        }
    }
    level_epilogue<BLOCK>(sm, s, t);
}

template <int BLOCK>
__device__ __forceinline__ void pull_body(const GraphDev &g, const BfsDev &s, uint32_t vlo, uint32_t vhi,
                                          const RangeList &rl, LevelSmem &sm)
{
    // A CTA takes a tile of kPullTileWords visited-bitmap words, compacts the
    // tile's unvisited vertices into q, and runs them one per thread (phase
    // A: header, the first kPullSerial in-edges and their frontier probes, all
    // issued back to back).  Vertices still unresolved go to bq and are
    // scanned by groups of kGroup lanes, 4*kGroup in-edges per step with
    // 128-bit loads, up to the first frontier hit (phase B).  Found vertices
    // are collected in a shared bitmap and the tile's visited/next words are
    // then written once, without global atomics.
    constexpr int kGroup = SCAPH_PULL_GROUP;
    constexpr int kGroups = BLOCK / kGroup;
    __shared__ uint32_t q[kPullTileWords * 32];
    __shared__ uint32_t fnd[kPullTileWords];
    // the tile's live ranks and live words (BfsDev::live_rank), for phase A
    __shared__ uint32_t t_rank[kPullTileWords], t_live[kPullTileWords];
    constexpr int kPPT = BLOCK >= 512 ? 1 : kPullPerThread;  // shared memory bounds the 512-thread CTA
    // phase-B queue: with SCAPH_PULL_DEFER_B the vertices of several rounds
    // wait here and phase B runs once they would overflow it (or at the end
    // of the queue), so that a CTA waits for its longest in-list once per
    // few rounds instead of once per round
    constexpr uint32_t kBq = (SCAPH_PULL_DEFER_B ? 3 : 2) * kPPT * BLOCK / 2;  // static shared memory: 48 KB
    __shared__ uint32_t bq_v[kBq], bq_len[kBq];
    __shared__ unsigned long long bq_st[kBq];
    __shared__ uint32_t wsum[BLOCK / 32];

    level_prologue<BLOCK>(sm, s);
    const PageLut lut = stage_lut<BLOCK>(g, sm);
    const bool hist_same = s.hg.pages == g.pages;
    const int lane = threadIdx.x & 31;
    const int grp = threadIdx.x / kGroup, glane = threadIdx.x % kGroup;
    const int gshift = (lane / kGroup) * kGroup;  // bit offset of this group in a warp ballot
    __syncthreads();

    ThreadAcc t;
    const uint32_t ntiles = rl.n ? rl.tile0[rl.n]
                                 : (((uint32_t)(((unsigned long long)vhi + 31) >> 5)) - (vlo >> 5) + kPullTileWords - 1) /
                                       kPullTileWords;

    // where vertex v's in-list lives (false: its page is missing)
    auto list_start_w = [&](uint32_t v, int &p, unsigned long long &st) -> bool {
        p = lut.of(v);
        const PageDev pd = lut.pages[p];
        if (pd.base == kNotResident) {
            atomicOr(&s.ctr->error, 4u);
            return false;
        }
        st = pd.base + 3ull * pd.nodenum + g.pool[pd.base + 3ull * (v - pd.left) + 1];
        t.headers++;
        return true;
    };

    // Runs phases A and B over q[0, total): found vertices go to the tile's
    // shared bitmap fnd (tbase = the tile's first word), or, gathering
    // several sparse tiles, straight to the visited / next words.
    auto run_queue = [&](uint32_t total, uint32_t tbase, bool gathered) {
        auto mark_found = [&](uint32_t v) {
            const uint32_t bit = 1u << (v & 31);
            if (gathered) {
                atomicOr(&s.visited[v >> 5], bit);
                atomicOr(&s.next[v >> 5], bit);
            } else {
                atomicOr(&fnd[(v >> 5) - tbase], bit);
            }
        };
        // a vertex found by phase A: depth, parent, the found bitmaps, the
        // counters and the page histograms (p < 0: page looked up here)
        auto found = [&](uint32_t v, uint32_t par, uint32_t dv, int p) {
            s.depth[v] = s.level + 1;
            if (s.parent) s.parent[v] = par;
            mark_found(v);
            t.next++;
            t.next_edges += dv;
            if (s.page_nodes) {
                if (p < 0 || !hist_same) p = hist_same ? lut.of(v) : page_of(s.hg, v);
                hist_add(sm, s, p, dv + 3);
            }
            hist_in_add(sm, s, v);
        };
        // phase B needs where vertex v's in-list lives (false: page missing)
        auto list_start = [&](uint32_t v, int &p, unsigned long long &st) -> bool {
            p = lut.of(v);
            const PageDev pd = lut.pages[p];
            if (pd.base == kNotResident) {
                atomicOr(&s.ctr->error, 4u);
                return false;
            }
            st = pd.base + 3ull * pd.nodenum + g.pool[pd.base + 3ull * (v - pd.left) + 1];
            t.headers++;
            return true;
        };
        // the same with the in-list's length read from the header
        auto list_start_len = [&](uint32_t v, int &p, unsigned long long &st, uint32_t &len) -> bool {
            p = lut.of(v);
            const PageDev pd = lut.pages[p];
            if (pd.base == kNotResident) {
                atomicOr(&s.ctr->error, 4u);
                return false;
            }
            const uint32_t *node = g.pool + pd.base + 3ull * (v - pd.left);
            st = pd.base + 3ull * pd.nodenum + node[1];
            len = node[2];
            t.headers++;
            return true;
        };
        // ---- phase B over bq[0, nb): groups of kGroup lanes, one vertex per group
        auto phase_b = [&](uint32_t nb) {
            for (uint32_t e0 = 0; e0 < nb; e0 += kGroups) {
                const uint32_t e = e0 + grp;
                const bool mine = e < nb;
                unsigned long long a = 0, b = 0;
                if (mine) {
                    a = bq_st[e] + (s.head_ranked ? 0u : kPullSerial);
                    b = bq_st[e] + bq_len[e];
                }
                const unsigned long long qa = a >> 2, qb = (b + 3) >> 2;
                unsigned long long qd = qa + glane;
                bool active = mine;
                uint32_t hit_par = kNoParent;
                unsigned long long hit_word = b;
                while (__any_sync(0xFFFFFFFFu, active)) {
                    uint32_t myhit = 0, vals[4] = {0, 0, 0, 0};
                    if (active && qd < qb) {
                        const uint4 val = ld_nc_v4(g.pool + qd * 4);
                        vals[0] = val.x;
                        vals[1] = val.y;
                        vals[2] = val.z;
                        vals[3] = val.w;
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const unsigned long long word = qd * 4 + j;
                            if (word >= a && word < b && vals[j] < s.V && test_bit(s.front, vals[j])) myhit |= 1u << j;
                        }
                    }
                    // every lane runs the same ballot/shuffles (warp stays converged)
                    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, myhit != 0);
                    const uint32_t gb = (bal >> gshift) & ((1u << kGroup) - 1u);
                    const int first = gb ? __ffs(gb) - 1 : 0;  // group lane holding the first hit
                    const uint32_t fh = __shfl_sync(0xFFFFFFFFu, myhit, gshift + first);
                    const int j = __ffs(fh | 0x10u) - 1;       // 4 when the group has no hit
                    const uint32_t pick = j == 0 ? vals[0] : j == 1 ? vals[1] : j == 2 ? vals[2] : vals[3];
                    const uint32_t hp = __shfl_sync(0xFFFFFFFFu, pick, gshift + first);
                    if (active) {
                        if (gb) {
                            hit_par = hp;
                            hit_word = (qd - glane + first) * 4 + j;
                            active = false;
                        } else {
                            qd += kGroup;
                            if (qd - glane >= qb) active = false;
                        }
                    }
                }
                if (mine && glane == 0) {
                    t.inspected += (uint32_t)(hit_word - a) + (hit_par != kNoParent ? 1u : 0u);
                    if (hit_par != kNoParent) {
                        const uint32_t vv = bq_v[e];
                        s.depth[vv] = s.level + 1;
                        if (s.parent) s.parent[vv] = hit_par;
                        mark_found(vv);
                        const uint32_t dv = __ldg(&s.degree[vv]);
                        t.next++;
                        t.next_edges += dv;
                        if (s.page_nodes) hist_add(sm, s, hist_same ? lut.of(vv) : page_of(s.hg, vv), dv + 3);
                        hist_in_add(sm, s, vv);
                    }
                }
            }
        };
        uint32_t nbq = 0;  // vertices waiting in bq for phase B (uniform across the CTA)
        for (uint32_t c0 = 0; c0 < total; c0 += kPPT * BLOCK) {
            uint32_t vv[kPPT], len[kPPT], need[kPPT], dg[kPPT];
            unsigned long long st[kPPT];
            int p[kPPT];
            uint32_t u[kPPT][kPullSerial];
            bool ok[kPPT];
#pragma unroll
            for (int i = 0; i < kPPT; i++) {
                const uint32_t k = c0 + i * BLOCK + threadIdx.x;
                vv[i] = 0;
                dg[i] = 0;
                len[i] = 0;
                need[i] = 0;
                st[i] = 0;
                p[i] = -1;
                ok[i] = k < total;
#pragma unroll
                for (uint32_t j = 0; j < kPullSerial; j++) u[i][j] = 0xFFFFFFFFu;
                if (ok[i]) vv[i] = q[k];
            }
            if (s.prec) {
                // ---- phase A from the 8-byte records: the top-ranked
                // in-neighbour settles most vertices (frontier hubs), and the
                // in-degree field ends those with no other in-edge; only the
                // rest read the in-degree and the row of ranked in-neighbours
                uint2 rec[kPPT];
#pragma unroll
                for (int i = 0; i < kPPT; i++) rec[i] = ok[i] ? ld_nc_v2(s.prec + vv[i]) : make_uint2(0xFFFFFFFFu, 0u);
                bool slow[kPPT];
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    slow[i] = false;
                    if (!ok[i]) continue;
                    const uint32_t h0 = rec[i].x, nin = rec[i].y >> 28;
                    dg[i] = rec[i].y & kPrecDegMax;
                    if (h0 < s.V && test_bit(s.front, h0)) {
                        t.inspected += 1;
                        found(vv[i], h0, dg[i] == kPrecDegMax ? __ldg(&s.degree[vv[i]]) : dg[i], -1);
                    } else if (nin <= 1) {
                        t.inspected += nin;
                    } else {
                        slow[i] = true;
                    }
                }
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    if (!slow[i]) continue;
                    len[i] = __ldg(&s.indeg[vv[i]]);
                    const uint4 h = ld_nc_v4(s.head + (size_t)kPullHead * vv[i]);
                    u[i][1] = h.y;
                    u[i][2] = h.z;
                    u[i][3] = h.w;
                    if (dg[i] == kPrecDegMax) dg[i] = __ldg(&s.degree[vv[i]]);
                }
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    if (!slow[i]) continue;
                    uint32_t hit = 0;
#pragma unroll
                    for (uint32_t j = 1; j < kPullSerial; j++)
                        if (u[i][j] < s.V && test_bit(s.front, u[i][j])) hit |= 1u << j;
                    if (hit) {
                        const uint32_t j = __ffs(hit) - 1;
                        t.inspected += j + 1;
                        found(vv[i], j == 1 ? u[i][1] : j == 2 ? u[i][2] : u[i][3], dg[i], -1);
                    } else {
                        t.inspected += min(len[i], kPullSerial);
                        need[i] = len[i] > kPullSerial && list_start(vv[i], p[i], st[i]);
                    }
                }
            } else if (s.prow) {
                // ---- phase A from the 16-byte rows: one load per vertex
                // brings the three top-ranked in-neighbours and the degrees;
                // the top one is probed first, the other two on a miss.  An
                // in-degree of three or less is then decided; the rest read
                // their whole in-list in phase B (its length from the header)
                uint4 r[kPPT];
#pragma unroll
                for (int i = 0; i < kPPT; i++)
                    r[i] = ok[i] ? ld_nc_v4(reinterpret_cast<const uint32_t *>(s.prow + vv[i])) : make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u);
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    if (!ok[i]) continue;
                    const uint32_t nin = r[i].w >> 28;
                    dg[i] = r[i].w & kPrecDegMax;
                    uint32_t hit = 0;
                    if (r[i].x < s.V && test_bit(s.front, r[i].x)) {
                        hit = 1u;
                    } else {
                        if (r[i].y < s.V && test_bit(s.front, r[i].y)) hit |= 2u;
                        if (r[i].z < s.V && test_bit(s.front, r[i].z)) hit |= 4u;
                    }
                    if (hit) {
                        const uint32_t j = __ffs(hit) - 1;
                        t.inspected += j + 1;
                        if (dg[i] == kPrecDegMax) dg[i] = __ldg(&s.degree[vv[i]]);
                        found(vv[i], j == 0 ? r[i].x : j == 1 ? r[i].y : r[i].z, dg[i], -1);
                    } else {
                        t.inspected += min(nin, 3u);
                        need[i] = nin > 3 && list_start_len(vv[i], p[i], st[i], len[i]);
                    }
                }
            } else {
                // ---- phase A: kPPT unvisited vertices per thread, all
                // their row (or header and first in-edge) loads issued before
                // any of their frontier probes
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    if (!ok[i]) continue;
                    const uint32_t v = vv[i];
                    if (s.head && s.live_rank && !gathered) {
                        // the live vertices' arrays: v's live rank from the
                        // tile's staged rank and live word
                        const uint32_t wi = (v >> 5) - tbase;
                        const uint32_t r = t_rank[wi] + __popc(t_live[wi] & ((1u << (v & 31)) - 1u));
                        dg[i] = __ldg(&s.live_deg[r]);
                        len[i] = __ldg(&s.live_indeg[r]);
                        const uint4 h = ld_nc_v4(reinterpret_cast<const uint32_t *>(s.live_head + r));
                        u[i][0] = h.x;
                        u[i][1] = h.y;
                        u[i][2] = h.z;
                        u[i][3] = h.w;
                    } else if (s.head) {
                        // dense rows: the in-degree and the first in-edges of
                        // consecutive vertices, independent coalesced loads; the
                        // page is read only if these do not decide
                        dg[i] = __ldg(&s.degree[v]);  // travels with the row loads (needed if v is found)
                        len[i] = __ldg(&s.indeg[v]);
                        const uint4 h = ld_nc_v4(s.head + (size_t)kPullHead * v);
                        u[i][0] = h.x;
                        u[i][1] = h.y;
                        u[i][2] = h.z;
                        u[i][3] = h.w;
                    } else {
                        dg[i] = __ldg(&s.degree[v]);
                        p[i] = lut.of(v);
                        const PageDev pd = lut.pages[p[i]];
                        if (pd.base != kNotResident) {
                            const uint32_t *node = g.pool + pd.base + 3ull * (v - pd.left);
                            len[i] = node[2];
                            st[i] = pd.base + 3ull * pd.nodenum + node[1];
                            t.headers++;
#pragma unroll
                            for (uint32_t j = 0; j < kPullSerial; j++)
                                u[i][j] = j < len[i] ? __ldg(&g.pool[st[i] + j]) : 0xFFFFFFFFu;
                        } else {
                            atomicOr(&s.ctr->error, 4u);
                            ok[i] = false;
                        }
                    }
                }
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    if (!ok[i]) continue;
                    const uint32_t v = vv[i];
                    uint32_t hit = 0;
#if SCAPH_PULL_FIRST_PROBE
                    // ranked rows: the top in-neighbour alone first (it settles
                    // most vertices), the other three only on a miss
                    if (s.head_ranked) {
                        if (u[i][0] < s.V && test_bit(s.front, u[i][0])) hit = 1u;
                        else {
#pragma unroll
                            for (uint32_t j = 1; j < kPullSerial; j++)
                                if (u[i][j] < s.V && test_bit(s.front, u[i][j])) hit |= 1u << j;
                        }
                    } else
#endif
                    {
#pragma unroll
                        for (uint32_t j = 0; j < kPullSerial; j++)
                            if (u[i][j] < s.V && test_bit(s.front, u[i][j])) hit |= 1u << j;
                    }
                    if (hit) {
                        const uint32_t j = __ffs(hit) - 1;
                        t.inspected += j + 1;
                        static_assert(kPullSerial == 4, "the parent select below names four probes");
                        const uint32_t par = j == 0 ? u[i][0] : j == 1 ? u[i][1] : j == 2 ? u[i][2] : u[i][3];
                        found(v, par, dg[i], s.head ? -1 : p[i]);
                    } else {
                        t.inspected += min(len[i], kPullSerial);
                        need[i] = len[i] > kPullSerial;
                        if (need[i] && s.head) need[i] = list_start(v, p[i], st[i]);
                    }
                }
            }
            uint32_t nneed = 0;
#pragma unroll
            for (int i = 0; i < kPPT; i++) nneed += need[i];
            uint32_t nb;
            uint32_t bo = block_exclusive_scan<BLOCK>(nneed, wsum, nb);
            if (nbq + nb > kBq) {
                // the waiting vertices first (block_exclusive_scan ended
                // with a barrier, so their entries are visible)
                phase_b(nbq);
                __syncthreads();
                nbq = 0;
            }
            bo += nbq;
#pragma unroll
            for (int i = 0; i < kPPT; i++) {
                if (!need[i]) continue;
                bq_v[bo] = vv[i];
                bq_st[bo] = st[i];
                bq_len[bo] = len[i];
                bo++;
            }
            nbq += nb;
            if (!SCAPH_PULL_DEFER_B) {
                __syncthreads();
                phase_b(nbq);
                __syncthreads();
                nbq = 0;
            }
        }
        if (nbq) {
            __syncthreads();
            phase_b(nbq);
            __syncthreads();
        }
    };
    // Warp-centric variant (s.pull_warp, 8-byte records present): every
    // warp owns chunks of 16 bitmap words (512 vertices) on its own -
    // compaction by warp scan into its 512-entry slice of q, found bits in
    // its 16-word slice of fnd, phase B by the whole warp - so no CTA
    // barrier stands between a warp and its next chunk.
    // Vertex-parallel variant (s.pull_warp == 2, records present): a warp
    // takes kDenseWords bitmap words at a time and lane i handles bit i of
    // each, so the record loads and depth stores of a word are one coalesced
    // 256- or 128-byte access, the found bits are a warp ballot (one atomic
    // per word), and there is no queue, scan or barrier at all; lanes whose
    // vertex is visited idle instead.
    if (s.pull_warp == 2 && s.prec) {
        constexpr uint32_t kDenseWords = 4, kGroups = kPullTileWords / kDenseWords;
        const int warp = threadIdx.x >> 5;
        const uint32_t ngroups = ntiles * kGroups, warps = gridDim.x * (BLOCK / 32);
        for (uint32_t gi = blockIdx.x * (BLOCK / 32) + warp; gi < ngroups; gi += warps) {
            uint32_t rlo = vlo, rhi = vhi, local;
            range_of_tile(rl, gi / kGroups, rlo, rhi, local);
            const uint32_t rwhi = (uint32_t)(((unsigned long long)rhi + 31) >> 5);
            const uint32_t w0 = (rlo >> 5) + local * kPullTileWords + (gi % kGroups) * kDenseWords;
            uint32_t unv[kDenseWords];
            uint32_t any = 0;
#pragma unroll
            for (uint32_t j = 0; j < kDenseWords; j++) {
                const uint32_t w = w0 + j;
                unv[j] = w < rwhi ? ~s.visited[w] & range_mask(w, rlo, rhi) : 0u;
                any |= unv[j];
            }
            if (!any) continue;  // uniform: every lane read the same words
            uint2 rec[kDenseWords];
            uint32_t stat = 0;  // bit j: lane's vertex of word j is unvisited
#pragma unroll
            for (uint32_t j = 0; j < kDenseWords; j++) {
                const bool act = (unv[j] >> lane) & 1u;
                stat |= act ? 1u << j : 0u;
                rec[j] = act ? ld_nc_v2(s.prec + (((w0 + j) << 5) + lane)) : make_uint2(0xFFFFFFFFu, 0u);
            }
            uint32_t found = 0, slow = 0, par[kDenseWords], dgs[kDenseWords];
#pragma unroll
            for (uint32_t j = 0; j < kDenseWords; j++) {
                par[j] = kNoParent;
                dgs[j] = rec[j].y & kPrecDegMax;
                if (!((stat >> j) & 1u)) continue;
                const uint32_t h0 = rec[j].x, nin = rec[j].y >> 28;
                if (h0 < s.V && test_bit(s.front, h0)) {
                    t.inspected += 1;
                    par[j] = h0;
                    found |= 1u << j;
                } else if (nin <= 1) {
                    t.inspected += nin;
                } else {
                    slow |= 1u << j;
                }
            }
            // the rest: in-degree and ranked head row, then (rarely) the
            // whole in-list, scanned by the warp
#pragma unroll
            for (uint32_t j = 0; j < kDenseWords; j++) {
                const uint32_t v = ((w0 + j) << 5) + lane;
                uint32_t need = 0, len = 0;
                unsigned long long st = 0;
                if ((slow >> j) & 1u) {
                    len = __ldg(&s.indeg[v]);
                    const uint4 h = ld_nc_v4(s.head + (size_t)kPullHead * v);
                    uint32_t jj = 0;
                    if (h.y < s.V && test_bit(s.front, h.y)) par[j] = h.y, jj = 2;
                    else if (h.z < s.V && test_bit(s.front, h.z)) par[j] = h.z, jj = 3;
                    else if (h.w < s.V && test_bit(s.front, h.w)) par[j] = h.w, jj = 4;
                    if (jj) {
                        t.inspected += jj;
                        found |= 1u << j;
                    } else {
                        t.inspected += min(len, kPullSerial);
                        int pg = -1;
                        need = len > kPullSerial && list_start_w(v, pg, st) ? 1u : 0u;
                    }
                }
                uint32_t todo = __ballot_sync(0xFFFFFFFFu, need);
                while (todo) {
                    const int src_lane = __ffs(todo) - 1;
                    todo &= todo - 1;
                    const uint32_t n = __shfl_sync(0xFFFFFFFFu, len, src_lane);
                    const unsigned long long a = __shfl_sync(0xFFFFFFFFu, st, src_lane);
                    const unsigned long long b = a + n, qa = a >> 2, qb = (b + 3) >> 2;
                    uint32_t hit_par = kNoParent;
                    unsigned long long hit_word = b;
                    for (unsigned long long q0 = qa; q0 < qb; q0 += 32) {
                        const unsigned long long qd = q0 + lane;
                        uint32_t myhit = 0;
                        uint4 val = make_uint4(0, 0, 0, 0);
                        if (qd < qb) {
                            val = ld_nc_v4(g.pool + qd * 4);
                            const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
                            for (int k = 0; k < 4; k++) {
                                const unsigned long long word = qd * 4 + k;
                                if (word >= a && word < b && vals[k] < s.V && test_bit(s.front, vals[k]))
                                    myhit |= 1u << k;
                            }
                        }
                        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, myhit != 0);
                        if (bal) {
                            const int first = __ffs(bal) - 1;
                            const uint32_t fh = __shfl_sync(0xFFFFFFFFu, myhit, first);
                            const int k = __ffs(fh) - 1;
                            const uint32_t pick = k == 0 ? val.x : k == 1 ? val.y : k == 2 ? val.z : val.w;
                            hit_par = __shfl_sync(0xFFFFFFFFu, pick, first);
                            hit_word = (q0 + first) * 4 + k;
                            break;
                        }
                    }
                    if (lane == src_lane) {
                        t.inspected += (uint32_t)(hit_word - a) + (hit_par != kNoParent ? 1u : 0u);
                        if (hit_par != kNoParent) {
                            par[j] = hit_par;
                            found |= 1u << j;
                        }
                    }
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < kDenseWords; j++) {
                const uint32_t v = ((w0 + j) << 5) + lane;
                const bool f = (found >> j) & 1u;
                const uint32_t mask = __ballot_sync(0xFFFFFFFFu, f);
                if (!mask) continue;
                if (f) {
                    s.depth[v] = s.level + 1;
                    if (s.parent) s.parent[v] = par[j];
                    const uint32_t dv = dgs[j] == kPrecDegMax ? __ldg(&s.degree[v]) : dgs[j];
                    t.next++;
                    t.next_edges += dv;
                    if (s.page_nodes) hist_add(sm, s, hist_same ? lut.of(v) : page_of(s.hg, v), dv + 3);
                    hist_in_add(sm, s, v);
                }
                if (lane == 0) {
                    // a word at a range boundary may belong to two ranges
                    atomicOr(&s.visited[w0 + j], mask);
                    atomicOr(&s.next[w0 + j], mask);
                }
            }
        }
        level_epilogue<BLOCK>(sm, s, t);
        return;
    }

    // (levels without the records keep the CTA tiles: RMAT-24's level 2,
    // frontier 0.19 M, 7.2 M unvisited, ran 201 us tiled and 210 us here)
    if (BLOCK <= 256 && s.pull_warp == 1 && s.prec) {
        constexpr uint32_t kChunkWords = 16, kChunks = kPullTileWords / kChunkWords;
        static_assert(kChunkWords * 32 * (256 / 32) <= kPullTileWords * 32, "per-warp queues fit q");
        const int warp = threadIdx.x >> 5;
        // records by live rank (BfsDev::live_prec): each lane of the first 16
        // holds its word's live rank and live bits, the others shuffle them
        const bool live = s.live_prec != nullptr;
        uint32_t *qw = q + warp * (kChunkWords * 32);
        uint32_t *fw = fnd + warp * kChunkWords;
        const uint32_t nchunks = ntiles * kChunks, warps = gridDim.x * (BLOCK / 32);
        for (uint32_t c = blockIdx.x * (BLOCK / 32) + warp; c < nchunks; c += warps) {
            uint32_t rlo = vlo, rhi = vhi, local;
            range_of_tile(rl, c / kChunks, rlo, rhi, local);
            const uint32_t rwhi = (uint32_t)(((unsigned long long)rhi + 31) >> 5);
            const uint32_t wbase = (rlo >> 5) + local * kPullTileWords + (c % kChunks) * kChunkWords;
            const uint32_t w = wbase + lane;
            uint32_t unv = 0, wl_rank = 0, wl_live = 0;
            if (lane < (int)kChunkWords) {
                fw[lane] = 0;
                if (w < rwhi) unv = ~s.visited[w] & range_mask(w, rlo, rhi);
                if (live && w < rwhi) {
                    wl_rank = s.live_rank[w];
                    wl_live = ~s.dead[w];
                }
            }
            const uint32_t cnt = __popc(unv);
            uint32_t inc = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
                if (lane >= o) inc += y;
            }
            const uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
            if (total == 0) continue;
            {
                uint32_t at = inc - cnt, m = unv;
                while (m) {
                    qw[at++] = (w << 5) + (__ffs(m) - 1);
                    m &= m - 1;
                }
            }
            __syncwarp();
            auto found_w = [&](uint32_t v, uint32_t par, uint32_t dv) {
                s.depth[v] = s.level + 1;
                if (s.parent) s.parent[v] = par;
                atomicOr(&fw[(v >> 5) - wbase], 1u << (v & 31));
                t.next++;
                t.next_edges += dv;
                if (s.page_nodes) hist_add(sm, s, hist_same ? lut.of(v) : page_of(s.hg, v), dv + 3);
                hist_in_add(sm, s, v);
            };
            for (uint32_t k0 = 0; k0 < total; k0 += 32 * kPPT) {
                uint32_t vv[kPPT], dg[kPPT], rr[kPPT];
                uint2 rec[kPPT];
                bool slow[kPPT];
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    const uint32_t k = k0 + i * 32 + lane;
                    vv[i] = k < total ? qw[k] : 0xFFFFFFFFu;
                    rr[i] = 0;
                    if (live) {  // uniform: every lane shuffles
                        const int wi = (int)(((vv[i] >> 5) - wbase) & 31u);
                        const uint32_t base = __shfl_sync(0xFFFFFFFFu, wl_rank, wi);
                        const uint32_t lw = __shfl_sync(0xFFFFFFFFu, wl_live, wi);
                        rr[i] = base + __popc(lw & ((1u << (vv[i] & 31)) - 1u));
                    }
                    if (vv[i] == 0xFFFFFFFFu) {
                        rec[i] = make_uint2(0xFFFFFFFFu, 0u);
                    } else if (s.prec && live) {
                        rec[i] = ld_nc_v2(s.live_prec + rr[i]);
                    } else if (s.prec) {
                        rec[i] = ld_nc_v2(s.prec + vv[i]);
                    } else {
                        // level without records: the head row, in-degree and
                        // out-degree issued together, folded into a record
                        // (a miss re-reads the row from L1)
                        const uint32_t h0 = __ldg(s.head + (size_t)kPullHead * vv[i]);
                        const uint32_t n = __ldg(&s.indeg[vv[i]]), d = __ldg(&s.degree[vv[i]]);
                        rec[i] = make_uint2(h0, pull_meta(n, d));
                    }
                }
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    slow[i] = false;
                    dg[i] = rec[i].y & kPrecDegMax;
                    if (vv[i] == 0xFFFFFFFFu) continue;
                    const uint32_t h0 = rec[i].x, nin = rec[i].y >> 28;
                    if (h0 < s.V && test_bit(s.front, h0)) {
                        t.inspected += 1;
                        found_w(vv[i], h0, dg[i] == kPrecDegMax ? __ldg(&s.degree[vv[i]]) : dg[i]);
                    } else if (nin <= 1) {
                        t.inspected += nin;
                    } else {
                        slow[i] = true;
                    }
                }
                // the rest: in-degree, ranked head row, then (rarely) the
                // whole in-list, scanned by the warp
#pragma unroll
                for (int i = 0; i < kPPT; i++) {
                    uint32_t need = 0, len = 0;
                    unsigned long long st = 0;
                    if (slow[i]) {
                        const uint32_t v = vv[i];
                        len = live ? __ldg(&s.live_indeg[rr[i]]) : __ldg(&s.indeg[v]);
                        const uint4 h = live ? ld_nc_v4(reinterpret_cast<const uint32_t *>(s.live_head + rr[i]))
                                             : ld_nc_v4(s.head + (size_t)kPullHead * v);
                        if (dg[i] == kPrecDegMax) dg[i] = __ldg(&s.degree[v]);
                        uint32_t par = kNoParent, j = 0;
                        if (h.y < s.V && test_bit(s.front, h.y)) par = h.y, j = 2;
                        else if (h.z < s.V && test_bit(s.front, h.z)) par = h.z, j = 3;
                        else if (h.w < s.V && test_bit(s.front, h.w)) par = h.w, j = 4;
                        if (par != kNoParent) {
                            t.inspected += j;
                            found_w(v, par, dg[i]);
                        } else {
                            t.inspected += min(len, kPullSerial);
                            int pg = -1;
                            need = len > kPullSerial && list_start_w(v, pg, st) ? 1u : 0u;
                        }
                    }
                    uint32_t todo = __ballot_sync(0xFFFFFFFFu, need);
                    while (todo) {
                        const int src_lane = __ffs(todo) - 1;
                        todo &= todo - 1;
                        const uint32_t v = __shfl_sync(0xFFFFFFFFu, vv[i], src_lane);
                        const uint32_t n = __shfl_sync(0xFFFFFFFFu, len, src_lane);
                        const unsigned long long a = __shfl_sync(0xFFFFFFFFu, st, src_lane);
                        const uint32_t dv = __shfl_sync(0xFFFFFFFFu, dg[i], src_lane);
                        const unsigned long long b = a + n, qa = a >> 2, qb = (b + 3) >> 2;
                        uint32_t hit_par = kNoParent;
                        unsigned long long hit_word = b;
                        for (unsigned long long q0 = qa; q0 < qb; q0 += 32) {
                            const unsigned long long qd = q0 + lane;
                            uint32_t myhit = 0;
                            uint4 val = make_uint4(0, 0, 0, 0);
                            if (qd < qb) {
                                val = ld_nc_v4(g.pool + qd * 4);
                                const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
#pragma unroll
                                for (int j = 0; j < 4; j++) {
                                    const unsigned long long word = qd * 4 + j;
                                    if (word >= a && word < b && vals[j] < s.V && test_bit(s.front, vals[j]))
                                        myhit |= 1u << j;
                                }
                            }
                            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, myhit != 0);
                            if (bal) {
                                const int first = __ffs(bal) - 1;
                                const uint32_t fh = __shfl_sync(0xFFFFFFFFu, myhit, first);
                                const int j = __ffs(fh) - 1;
                                const uint32_t pick = j == 0 ? val.x : j == 1 ? val.y : j == 2 ? val.z : val.w;
                                hit_par = __shfl_sync(0xFFFFFFFFu, pick, first);
                                hit_word = (q0 + first) * 4 + j;
                                break;
                            }
                        }
                        if (lane == src_lane) {
                            t.inspected += (uint32_t)(hit_word - a) + (hit_par != kNoParent ? 1u : 0u);
                            if (hit_par != kNoParent) found_w(v, hit_par, dv);
                        }
                    }
                }
            }
            __syncwarp();
            if (lane < (int)kChunkWords && w < rwhi) {
                const uint32_t f = fw[lane];
                if (f) {
                    atomicOr(&s.visited[w], f);
                    atomicOr(&s.next[w], f);
                }
            }
            __syncwarp();
        }
        level_epilogue<BLOCK>(sm, s, t);
        return;
    }

    // Sparse levels (few unvisited vertices, a handful per tile): the
    // vertices of several tiles are gathered into one queue before phases A
    // and B run, so that every thread has a vertex in each round.
    const bool gather = s.pull_gather != 0;
    uint32_t qn = 0;  // gathered vertices (uniform across the CTA)
    if (gather && rl.n == 0 && s.pull_gather == 2) {
        // whole-graph range: the CTA owns one contiguous run of visited
        // words and reads it 4*BLOCK words per round (each thread four
        // coalesced words), instead of one 128-word tile after another
        constexpr uint32_t kCap = kPullTileWords * 32;  // q's capacity
        const uint32_t wlo = vlo >> 5, whi = (uint32_t)(((unsigned long long)vhi + 31) >> 5);
        const uint32_t per = (whi - wlo + gridDim.x - 1) / gridDim.x;
        const uint32_t w0 = wlo + blockIdx.x * per, w1 = min(whi, w0 + per);
        for (uint32_t cw = w0; cw < w1; cw += 4 * BLOCK) {
            uint32_t u[4], n = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t w = cw + k * BLOCK + threadIdx.x;
                u[k] = w < w1 ? ~s.visited[w] & range_mask(w, vlo, vhi) : 0u;
                n += __popc(u[k]);
            }
            if (!__syncthreads_or(n != 0)) continue;
            uint32_t total;
            const uint32_t off = block_exclusive_scan<BLOCK>(n, wsum, total);
            if (qn + total > kCap) {
                if (qn) run_queue(qn, 0, true);
                qn = 0;
            }
            // windows of kCap when one run holds more than q (a dense run)
            for (uint32_t lo = 0; lo < total; lo += kCap) {
                uint32_t at = off;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    uint32_t m = u[k];
                    const uint32_t base = (cw + k * BLOCK + threadIdx.x) << 5;
                    while (m) {
                        if (at >= lo && at < lo + kCap) q[qn + at - lo] = base + (__ffs(m) - 1);
                        at++;
                        m &= m - 1;
                    }
                }
                __syncthreads();
                const uint32_t nwin = min(kCap, total - lo);
                if (total > kCap) {
                    run_queue(nwin, 0, true);
                } else {
                    qn += nwin;
                    if (qn >= (uint32_t)kPPT * BLOCK) {
                        run_queue(qn, 0, true);
                        qn = 0;
                    }
                }
            }
        }
        if (qn) run_queue(qn, 0, true);
        level_epilogue<BLOCK>(sm, s, t);
        return;
    }
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint32_t rlo = vlo, rhi = vhi, local;
        range_of_tile(rl, tile, rlo, rhi, local);
        const uint32_t rwhi = (uint32_t)(((unsigned long long)rhi + 31) >> 5);
        const uint32_t tbase = (rlo >> 5) + local * kPullTileWords;  // first word of the tile
        const uint32_t w = tbase + threadIdx.x;
        uint32_t unv = 0;
        if (threadIdx.x < kPullTileWords) {
            if (!gather) fnd[threadIdx.x] = 0;
            if (w < rwhi) unv = ~s.visited[w] & range_mask(w, rlo, rhi);
            if (!gather && s.live_rank) {
                t_rank[threadIdx.x] = w < rwhi ? s.live_rank[w] : 0u;
                t_live[threadIdx.x] = w < rwhi ? ~s.dead[w] : 0u;
            }
        }
        if (!__syncthreads_or(unv != 0)) continue;
        uint32_t total;
        uint32_t off = block_exclusive_scan<BLOCK>(__popc(unv), wsum, total);
        if (total == 0) continue;
        if (gather) {
            if (qn + total > (uint32_t)kPullTileWords * 32) {
                run_queue(qn, 0, true);
                qn = 0;
            }
            uint32_t m = unv, at = qn + off;
            while (m) {
                q[at++] = (w << 5) + (__ffs(m) - 1);
                m &= m - 1;
            }
            qn += total;
            __syncthreads();
            if (qn >= (uint32_t)kPPT * BLOCK) {
                run_queue(qn, 0, true);
                qn = 0;
            }
            continue;
        }
        {
            uint32_t m = unv;
            while (m) {
                q[off++] = (w << 5) + (__ffs(m) - 1);
                m &= m - 1;
            }
        }
        __syncthreads();
        run_queue(total, tbase, false);
        // ---- the tile's visited / next words, written once (atomically:
        // a word at a range boundary may belong to two tiles)
        if (threadIdx.x < kPullTileWords && w < rwhi) {
            const uint32_t f = fnd[threadIdx.x];
            if (f) {
                atomicOr(&s.visited[w], f);
                atomicOr(&s.next[w], f);
            }
        }
        __syncthreads();
    }
    if (gather && qn) run_queue(qn, 0, true);
    level_epilogue<BLOCK>(sm, s, t);
}

// Deferred-claim push levels: the next frontier holds every unvisited
// vertex some frontier vertex reached; each is claimed here, word by word
// (depth written for 32 consecutive vertices at a time, visited updated
// with a plain store: one thread owns each word), with the level's counters
// and page histograms.
template <int BLOCK>
__device__ __forceinline__ void finalize_body(const BfsDev &s)
{
    __shared__ LevelSmem sm;
    level_prologue<BLOCK>(sm, s);
    const PageLut lut = stage_lut<BLOCK>(s.hg, sm);
    if (blockIdx.x == 0 && threadIdx.x == 0) s.ctr->deferred = 1u;
    __syncthreads();
    ThreadAcc t;
    for (uint32_t w = blockIdx.x * BLOCK + threadIdx.x; w < s.nwords; w += gridDim.x * BLOCK) {
        const uint32_t nx = s.next[w];
        if (!nx) continue;
        const uint32_t vis = s.visited[w];
        uint32_t n = nx & ~vis;
        if (n != nx) s.next[w] = n;
        if (!n) continue;
        s.visited[w] = vis | n;
        while (n) {
            const uint32_t v = (w << 5) + (__ffs(n) - 1);
            n &= n - 1;
            s.depth[v] = s.level + 1;
            const uint32_t dv = __ldg(&s.degree[v]);
            t.next++;
            t.next_edges += dv;
            if (s.page_nodes) hist_add(sm, s, lut.of(v), dv + 3);
            hist_in_add(sm, s, v);
        }
    }
    level_epilogue<BLOCK>(sm, s, t);
}

// graph mode: the level's state from the device control block
__device__ __forceinline__ BfsDev level_state(const BfsGraphArgs &a)
{
    BfsDev s = a.base;
    const BfsCtl *c = a.ctl;
    const uint32_t L = c->level;
    s.level = L;
    s.depth = c->depth;
    s.parent = c->parent;
    s.front = a.bm3 + (size_t)(L % 3) * s.nwords;
    s.next = a.bm3 + (size_t)((L + 1) % 3) * s.nwords;
    s.ctr = a.ctr0 + L;
    s.pull_gather = c->pull_gather;
    s.push_defer = c->push_defer;
    s.push_sparse = c->push_sparse;
    if (!c->pull_rec) s.prec = nullptr;
    if (a.hist0 && L < a.hist_levels) {
        s.page_nodes = a.hist0 + (size_t)L * 2 * a.npages_h;
        s.page_datas = s.page_nodes + a.npages_h;
    } else {
        s.page_nodes = s.page_datas = nullptr;
    }
    return s;
}

// clears the bitmap the NEXT level will write (it held level L-1's frontier)
__device__ __forceinline__ void clear_third(const BfsGraphArgs &a, uint32_t L)
{
    uint32_t *b = a.bm3 + (size_t)((L + 2) % 3) * a.base.nwords;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.base.nwords; i += gridDim.x * blockDim.x) b[i] = 0;
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace

// ---------------------------------------------------------------------------
// kernels: host-argument versions
// ---------------------------------------------------------------------------
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kPushMinThreads / BLOCK) k_push(GraphDev g, BfsDev s, uint32_t vlo, uint32_t vhi, RangeList rl)
{
    push_body<BLOCK>(g, s, vlo, vhi, rl);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_giant(GraphDev g, BfsDev s)
{
    __shared__ LevelSmem sm;
    giant_body<BLOCK>(g, s, sm);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kPullMinThreads / BLOCK) k_pull(GraphDev g, BfsDev s, uint32_t vlo, uint32_t vhi,
                                                            RangeList rl)
{
    __shared__ LevelSmem sm;
    pull_body<BLOCK>(g, s, vlo, vhi, rl, sm);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_finalize(BfsDev s)
{
    finalize_body<BLOCK>(s);
}

// ---------------------------------------------------------------------------
// kernels: graph mode
// ---------------------------------------------------------------------------
// The three level kernels of a graph-mode level run back to back; the one
// the level's direction (decided on the device) does not select leaves at
// once, which costs less than a conditional node per direction.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kPushMinThreads / BLOCK) k_push_g(GraphDev g, BfsGraphArgs a)
{
    if (a.ctl->dir != 0) return;
    const BfsDev s = level_state(a);
    clear_third(a, s.level);
    push_body<BLOCK>(g, s, 0, s.V, RangeList{nullptr, nullptr, nullptr, 0});
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_giant_g(GraphDev g, BfsGraphArgs a)
{
    if (a.ctl->dir != 0) return;
    __shared__ LevelSmem sm;
    giant_body<BLOCK>(g, level_state(a), sm);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_finalize_g(BfsGraphArgs a)
{
    if (a.ctl->dir != 0 || !a.ctl->push_defer) return;
    finalize_body<BLOCK>(level_state(a));
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kPullMinThreads / BLOCK) k_pull_g(GraphDev g, BfsGraphArgs a)
{
    if (a.ctl->dir != 1) return;
    const BfsDev s = level_state(a);
    clear_third(a, s.level);
    __shared__ LevelSmem sm;
    pull_body<BLOCK>(g, s, 0, s.V, RangeList{nullptr, nullptr, nullptr, 0}, sm);
}

// The giant chunks of a push level and the pull of a pull level in one
// kernel node (a level runs one of them), so that each level launches one
// node fewer; one LevelSmem serves either body.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kPullMinThreads / BLOCK) k_giant_pull_g(GraphDev gout, GraphDev gin,
                                                                             BfsGraphArgs a)
{
    __shared__ LevelSmem sm;
    const BfsDev s = level_state(a);
    if (a.ctl->dir == 0) {
        giant_body<BLOCK>(gout, s, sm);
    } else {
        clear_third(a, s.level);
        pull_body<BLOCK>(gin, s, 0, s.V, RangeList{nullptr, nullptr, nullptr, 0}, sm);
    }
}

// First node of a BFS graph: run inputs into the control block, state reset
// (bfs_init, app/bfs.cu:20-30: depth = unreached, nothing active).
__global__ void k_graph_init(BfsGraphArgs a, uint32_t *depth, uint32_t *parent, uint32_t src, uint32_t unreached,
                             const uint32_t *dead, uint32_t nlevels_clear)
{
    const BfsDev &b = a.base;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        BfsCtl *c = a.ctl;
        c->depth = depth;
        c->parent = parent;
        c->src = src;
        c->level = 0;
        c->dir = 0;
        c->done = 0;
        c->pull_gather = 0;
        c->push_defer = 0;
        c->pull_rec = 0;
        c->push_sparse = b.push_sparse;  // level 0: one frontier vertex
        // the source (setsrc, app/bfs.cu:32-37): its depth, parent and bits
        // are written by the fills below, each element by one thread
        const unsigned long long d = b.degree[src];
        c->nf = 1;
        c->prev_nf = 0;
        c->mf = d;
        c->vis_n = 1;
        c->vis_e = d;
        c->t_start = globaltimer();
    }
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    // 16-byte stores where the array allows (the depth fill is most of this
    // kernel: 4 bytes per vertex)
    // value everywhere except element at, which gets at_value
    auto fill = [&](uint32_t *p, uint32_t value, size_t n, size_t at, uint32_t at_value) {
        size_t done = 0;
        if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
            const uint4 v4 = make_uint4(value, value, value, value);
            const size_t n4 = n / 4;
            for (size_t i = i0; i < n4; i += stride) {
                uint4 x = v4;
                if (i == at / 4) {
                    const size_t k = at % 4;
                    x.x = k == 0 ? at_value : value;
                    x.y = k == 1 ? at_value : value;
                    x.z = k == 2 ? at_value : value;
                    x.w = k == 3 ? at_value : value;
                }
                reinterpret_cast<uint4 *>(p)[i] = x;
            }
            done = n4 * 4;
        }
        for (size_t i = done + i0; i < n; i += stride) p[i] = i == at ? at_value : value;
    };
    const uint32_t sbit = 1u << (src & 31);
    fill(depth, unreached, b.V, src, 0u);
    if (parent) fill(parent, kNoParent, b.V, src, src);
    for (size_t i = i0; i < b.nwords; i += stride) b.visited[i] = (dead ? dead[i] : 0u) | (i == (src >> 5) ? sbit : 0u);
    fill(a.bm3, 0u, 3ull * b.nwords, src >> 5, sbit);  // level 0's frontier: the source
    uint32_t *cw = reinterpret_cast<uint32_t *>(a.ctr0);
    const size_t nc = (size_t)nlevels_clear * sizeof(LevelCounters) / 4;
    for (size_t i = i0; i < nc; i += stride) cw[i] = 0u;
    if (a.hist0) {
        const size_t nh = (size_t)a.hist_levels * 2 * a.npages_h;
        for (size_t i = i0; i < nh; i += stride) a.hist0[i] = 0u;
    }
}

// Last node of each level: counters -> next direction (Beamer alpha/beta, or
// the forced direction) and the conditionals of the next iteration.
// The level's decision, run by one thread (k_decide).  Counters are read
// through a volatile pointer, so the body also holds where other CTAs of the
// same launch update them (a last-CTA decision was measured slower:
// 585 vs 603 GTEPS on RMAT-24).
__device__ __forceinline__ void decide_body(const BfsGraphArgs &a, const DecideArgs &d,
                                            cudaGraphConditionalHandle h_loop)
{
    BfsCtl *c = a.ctl;
    const uint32_t L = c->level;
    LevelCounters *lc = a.ctr0 + L;
    const volatile LevelCounters *vlc = lc;
    lc->dir = c->dir;
    lc->t_end = globaltimer();
    c->prev_nf = c->nf;
    c->nf = vlc->next;
    c->mf = vlc->next_edges;
    c->vis_n += c->nf;
    c->vis_e += c->mf;
    const bool stop = c->nf == 0 || vlc->error != 0 || (int)L + 1 >= d.max_levels ||
                      (unsigned long long)L + 2 >= d.unreached;
    if (stop) {
        c->done = 1;
        cudaGraphSetConditional(h_loop, 0);
        return;
    }
    const unsigned long long used = c->vis_e + d.dead_edges;
    const unsigned long long mu = d.E > used ? d.E - used : 0;
    int nd;
    if (d.mode == 1) nd = 0;
    else if (d.mode == 2) nd = 1;
    else nd = alpha_beta_next(c->dir, c->nf, c->prev_nf, c->mf, mu, d.V, d.alpha, d.beta);
    c->dir = nd;
    c->push_defer = nd == 0 && d.defer_edges && c->mf >= d.defer_edges && !c->parent ? 1u : 0u;
    c->push_sparse = nd == 0 && push_use_sparse(d.push_sparse_ratio, c->nf, d.V) ? 1u : 0u;
    {
        const uint32_t src = c->src;
        const unsigned long long src_dead = (d.dead_bm[src >> 5] >> (src & 31)) & 1u;
        const unsigned long long unv = (unsigned long long)d.V - d.dead - c->vis_n + src_dead;
        c->pull_gather = unv * d.gather_ratio < d.V ? d.pull_gather_mode : 0u;
        c->pull_rec = pull_use_records(d.pull_records, c->nf, unv) ? 1u : 0u;
    }
    c->level = L + 1;
    cudaGraphSetConditional(h_loop, 1);
}

__global__ void k_decide(BfsGraphArgs a, DecideArgs d, cudaGraphConditionalHandle h_loop)
{
    decide_body(a, d, h_loop);
}

// Learned variant of k_decide (64 threads): the scheduler's feature row of
// the coming level - the same 16 globals the host loop computes (scaph.h),
// page residency 1 (graph resident), then the new frontier's share of every
// out-page - through the network's three layers; output 0 > 0 means pull.
// Where alpha/beta is far from its switch point its choice stands and the
// network is not run (the host loop does the same).
__global__ void __launch_bounds__(64) k_decide_learned(BfsGraphArgs a, DecideArgs d, MlpDev net,
                                                       cudaGraphConditionalHandle h_loop)
{
    constexpr int kG = 16;
    __shared__ float f[kG + kHistCap];
    __shared__ float h1[64], h2[64];
    __shared__ int s_stop, s_ab, s_guard;
    __shared__ unsigned long long s_unv;
    BfsCtl *c = a.ctl;
    const uint32_t L = c->level;
    const int t = threadIdx.x;
    if (t == 0) {
        LevelCounters *lc = a.ctr0 + L;
        lc->dir = c->dir;
        lc->t_end = globaltimer();
        c->prev_nf = c->nf;
        c->nf = lc->next;
        c->mf = lc->next_edges;
        c->vis_n += c->nf;
        c->vis_e += c->mf;
        s_stop = c->nf == 0 || lc->error != 0 || (int)L + 1 >= d.max_levels ||
                 (unsigned long long)L + 2 >= d.unreached;
        const unsigned long long used = c->vis_e + d.dead_edges;
        const unsigned long long mu = d.E > used ? d.E - used : 0;
        const uint32_t src = c->src;
        const unsigned long long src_dead = (d.dead_bm[src >> 5] >> (src & 31)) & 1u;
        const unsigned long long unv = (unsigned long long)d.V - d.dead - c->vis_n + src_dead;
        s_unv = unv;
        s_ab = alpha_beta_next(c->dir, c->nf, c->prev_nf, c->mf, mu, d.V, d.alpha, d.beta);
        s_guard = alpha_beta_confident(c->dir, c->nf, c->mf, mu, d.V, d.alpha, d.beta);
        f[0] = log2f(1.f + (float)c->nf) / 32.f;
        f[1] = log2f(1.f + (float)c->mf) / 40.f;
        f[2] = log2f(1.f + (float)unv) / 32.f;
        f[3] = log2f(1.f + (float)mu) / 40.f;
        f[4] = (float)c->nf / (float)d.V;
        f[5] = fminf(1.f, (float)c->mf / (float)(d.E ? d.E : 1));
        f[6] = (float)unv / (float)d.V;
        f[7] = fminf(1.f, (float)mu / (float)(d.E ? d.E : 1));
        f[8] = (float)(L + 1) / 32.f;
        f[9] = (float)c->dir;
        f[10] = f[11] = f[12] = f[13] = 1.f;
        f[14] = (float)s_ab;
        f[15] = 1.f;
    }
    __syncthreads();
    if (s_stop) {
        if (t == 0) {
            c->done = 1;
            cudaGraphSetConditional(h_loop, 0);
        }
        return;
    }
    auto finish = [&](int nd) {
        c->dir = nd;
        c->pull_gather = s_unv * d.gather_ratio < d.V ? d.pull_gather_mode : 0u;
        c->pull_rec = pull_use_records(d.pull_records, c->nf, s_unv) ? 1u : 0u;
        c->push_defer = nd == 0 && d.defer_edges && c->mf >= d.defer_edges && !c->parent ? 1u : 0u;
        c->push_sparse = nd == 0 && push_use_sparse(d.push_sparse_ratio, c->nf, d.V) ? 1u : 0u;
        c->level = L + 1;
        cudaGraphSetConditional(h_loop, 1);
    };
    if (d.mode == 1 || d.mode == 2 || s_guard >= 0) {
        // far from the alpha/beta threshold (or a fixed direction) the rule
        // decides, and the network is not run
        if (t == 0) finish(d.mode == 1 ? 0 : d.mode == 2 ? 1 : s_guard);
        return;
    }
    // frontier of level L+1 = vertices discovered by level L (histogram slot L)
    const int np = net.in - kG;
    const PageDev *pg = a.base.hg.pages;
    for (int p = t; p < np; p += 64) {
        const uint32_t hn = (a.hist0 && L < a.hist_levels) ? a.hist0[(size_t)L * 2 * a.npages_h + p] : 0u;
        f[kG + p] = (float)hn / (float)max(1u, pg[p].nodenum);
    }
    __syncthreads();
    // weights (and GEMM operands) rounded to bf16, FP32 accumulation, as in
    // the training kernels
    auto bf = [](float x) { return __bfloat162float(__float2bfloat16_rn(x)); };
    const float *W1 = net.w + net.off_w1, *W2 = net.w + net.off_w2, *W3 = net.w + net.off_w3;
    float acc = net.w[net.off_b1 + t];
    for (int i = 0; i < net.in; i++) acc += bf(f[i]) * bf(W1[(size_t)i * 64 + t]);
    h1[t] = fmaxf(acc, 0.f);
    __syncthreads();
    acc = net.w[net.off_b2 + t];
    for (int i = 0; i < 64; i++) acc += bf(h1[i]) * bf(W2[i * 64 + t]);
    h2[t] = fmaxf(acc, 0.f);
    __syncthreads();
    if (t == 0) {
        float y = net.w[net.off_b3];
        for (int j = 0; j < 64; j++) y += bf(h2[j]) * bf(W3[(size_t)j * net.out]);
        finish(y > 0.f ? 1 : 0);
    }
}

// ---------------------------------------------------------------------------
// state init helpers (host loop)
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
template <int BLOCK>
static cudaError_t launch_level(int dir, int grid, const GraphDev &g, const BfsDev &s, uint32_t vlo, uint32_t vhi,
                                cudaStream_t st)
{
    const RangeList one{nullptr, nullptr, nullptr, 0};
    if (dir == 0) {
        k_push<BLOCK><<<grid, BLOCK, 0, st>>>(g, s, vlo, vhi, one);
        k_push_giant<BLOCK><<<grid, BLOCK, 0, st>>>(g, s);
    } else {
        k_pull<BLOCK><<<grid, BLOCK, 0, st>>>(g, s, vlo, vhi, one);
    }
    return cudaGetLastError();
}

template <int BLOCK>
static cudaError_t launch_ranges(int dir, int grid, const GraphDev &g, const BfsDev &s, const RangeList &rl,
                                 cudaStream_t st)
{
    if (dir == 0) k_push<BLOCK><<<grid, BLOCK, 0, st>>>(g, s, 0, 0, rl);
    else k_pull<BLOCK><<<grid, BLOCK, 0, st>>>(g, s, 0, 0, rl);
    return cudaGetLastError();
}

cudaError_t run_ranges(int dir, int block, int grid, const GraphDev &g, const BfsDev &s, const RangeList &rl,
                       cudaStream_t st)
{
    switch (block) {
    case 128: return launch_ranges<128>(dir, grid, g, s, rl, st);
    case 512: return launch_ranges<512>(dir, grid, g, s, rl, st);
    default: return launch_ranges<256>(dir, grid, g, s, rl, st);
    }
}

cudaError_t run_push_finalize(int block, int grid, const BfsDev &s, cudaStream_t st)
{
    switch (block) {
    case 128: k_push_finalize<128><<<grid, 128, 0, st>>>(s); break;
    case 512: k_push_finalize<512><<<grid, 512, 0, st>>>(s); break;
    default: k_push_finalize<256><<<grid, 256, 0, st>>>(s); break;
    }
    return cudaGetLastError();
}

const void *push_finalize_graph_kernel(int block)
{
    switch (block) {
    case 128: return (const void *)k_push_finalize_g<128>;
    case 512: return (const void *)k_push_finalize_g<512>;
    default: return (const void *)k_push_finalize_g<256>;
    }
}

cudaError_t run_giant(int block, int grid, const GraphDev &g, const BfsDev &s, cudaStream_t st)
{
    switch (block) {
    case 128: k_push_giant<128><<<grid, 128, 0, st>>>(g, s); break;
    case 512: k_push_giant<512><<<grid, 512, 0, st>>>(g, s); break;
    default: k_push_giant<256><<<grid, 256, 0, st>>>(g, s); break;
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

void level_graph_kernels(int block, const void **push, const void **giant, const void **pull,
                         const void **giant_pull)
{
    switch (block) {
    case 128:
        *push = (const void *)k_push_g<128>;
        *giant = (const void *)k_push_giant_g<128>;
        *pull = (const void *)k_pull_g<128>;
        *giant_pull = (const void *)k_giant_pull_g<128>;
        break;
    case 512:
        *push = (const void *)k_push_g<512>;
        *giant = (const void *)k_push_giant_g<512>;
        *pull = (const void *)k_pull_g<512>;
        *giant_pull = (const void *)k_giant_pull_g<512>;
        break;
    default:
        *push = (const void *)k_push_g<256>;
        *giant = (const void *)k_push_giant_g<256>;
        *pull = (const void *)k_pull_g<256>;
        *giant_pull = (const void *)k_giant_pull_g<256>;
        break;
    }
}

const void *graph_init_kernel() { return (const void *)k_graph_init; }
const void *decide_kernel() { return (const void *)k_decide; }
const void *decide_learned_kernel() { return (const void *)k_decide_learned; }

int level_occupancy(int dir, int block)
{
    int n = 0;
    const void *f = nullptr;
    switch (block) {
    case 128: f = dir ? (const void *)k_pull<128> : (const void *)k_push<128>; break;
    case 512: f = dir ? (const void *)k_pull<512> : (const void *)k_push<512>; break;
    default: f = dir ? (const void *)k_pull<256> : (const void *)k_push<256>; break;
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, block, 0);
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
