// Device side of the multi-source BFS (bit-parallel BFS in the manner of
// Then et al., "The More the Merrier", VLDB 2014): per-vertex source masks,
// the push / finalize / pull level bodies (templated on the CTA size so that
// the batch autotuner can pick it), sources and depth unpacking.  Shared by
// msbfs.cu (scaph_msbfs, one launch per phase and level) and batch.cu
// (mixed query batches, the whole traversal in one CUDA-graph launch).
//
// Per vertex u (NW = 1 or 2 64-bit words, bit i = source i):
//   seen[u]    sources that have reached u (stored next to acc[u], the push
//              accumulator, so one 16-byte load returns both)
//   visit[u]   sources whose frontier holds u this level (valid where the
//              `act` bitmap has u's bit)
// push level: every active v sends visit[v] & ~seen[u] to its out-neighbours
//   u with a fire-and-forget red.or into acc[u] (and marks u in `touched`);
//   a finalize pass turns acc into the next frontier.
// pull level: every incomplete u (seen[u] != all sources) ORs visit[v] over
//   its in-neighbours v whose act bit is set, stopping as soon as every
//   missing source has been found.
// Depths are kept as bit planes (plane k, bit i = bit k of depth(i,u)).
#pragma once
#include <cuda_runtime.h>

#include "engine.h"
#include "kernel_common.cuh"

// multi-source pull phase B skips the in-edges of vertices that found
// every source they missed
#ifndef SCAPH_MS_EARLY_EXIT
#define SCAPH_MS_EARLY_EXIT 1
#endif
// ... and, resident, hands its tiles out from a counter
#ifndef SCAPH_MS_DYN_TILES
#define SCAPH_MS_DYN_TILES 1
#endif
// ... and skips the frontier-bit lookups on levels whose frontier holds
// every vertex (MsDev::all_active)
#ifndef SCAPH_MS_ALL_ACTIVE
#define SCAPH_MS_ALL_ACTIVE 1
#endif

namespace scaph {

constexpr int kMsPlanes = 12;  // depths below 4096 = kMaxLevels
constexpr int kMsBlock = 256;
constexpr int kMsTileWords = 128;

template <int NW>
struct Mask {
    unsigned long long w[NW];
};

template <int NW>
__device__ __forceinline__ Mask<NW> ld_mask(const unsigned long long *a, uint32_t u)
{
    Mask<NW> m;
    if constexpr (NW == 2) {
        const ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(a + 2ull * u);
        m.w[0] = x.x;
        m.w[1] = x.y;
    } else {
        m.w[0] = a[u];
    }
    return m;
}

template <int NW>
__device__ __forceinline__ void st_mask(unsigned long long *a, uint32_t u, const Mask<NW> &m)
{
    if constexpr (NW == 2) {
        *reinterpret_cast<ulonglong2 *>(a + 2ull * u) = make_ulonglong2(m.w[0], m.w[1]);
    } else {
        a[u] = m.w[0];
    }
}

// seen and acc of vertex u are interleaved: sa[u] = {seen[NW], acc[NW]}
template <int NW>
__device__ __forceinline__ void ld_seen_acc(const unsigned long long *sa, uint32_t u, Mask<NW> &seen, Mask<NW> &acc)
{
    const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(sa + 2ull * NW * u);
    if constexpr (NW == 1) {
        const ulonglong2 x = *p;
        seen.w[0] = x.x;
        acc.w[0] = x.y;
    } else {
        const ulonglong2 x = p[0], y = p[1];
        seen.w[0] = x.x;
        seen.w[1] = x.y;
        acc.w[0] = y.x;
        acc.w[1] = y.y;
    }
}

template <int NW>
__device__ __forceinline__ Mask<NW> ld_seen(const unsigned long long *sa, uint32_t u)
{
    Mask<NW> m;
    if constexpr (NW == 2) {
        const ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(sa + 4ull * u);
        m.w[0] = x.x;
        m.w[1] = x.y;
    } else {
        m.w[0] = sa[2ull * u];
    }
    return m;
}

template <int NW>
__device__ __forceinline__ void st_seen(unsigned long long *sa, uint32_t u, const Mask<NW> &m)
{
    if constexpr (NW == 2) {
        *reinterpret_cast<ulonglong2 *>(sa + 4ull * u) = make_ulonglong2(m.w[0], m.w[1]);
    } else {
        sa[2ull * u] = m.w[0];
    }
}

template <int NW>
__device__ __forceinline__ bool any(const Mask<NW> &m)
{
    bool r = false;
#pragma unroll
    for (int i = 0; i < NW; i++) r |= m.w[i] != 0;
    return r;
}

template <int NW>
__device__ __forceinline__ uint32_t popc(const Mask<NW> &m)
{
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) r += __popcll(m.w[i]);
    return r;
}

struct MsCounters {
    unsigned long long active;        // vertices in the next frontier
    unsigned long long active_edges;  // their out-degree sum
    unsigned long long pairs;         // (source, vertex) pairs reached this level
    unsigned long long inspected;     // adjacency entries examined
    unsigned long long completed_edges;  // out-degree of vertices that became complete
    unsigned int giant;
    unsigned int error;
    unsigned int tiles;  // pull tiles handed out so far (MsDev::dyn_tiles)
};

struct MsDev {
    unsigned long long *sa;  // {seen, acc} per vertex
    unsigned long long *visit_cur, *visit_nxt;
    unsigned long long *planes[kMsPlanes];
    uint32_t *act_cur, *act_nxt, *touched, *inc;
    const uint32_t *degree;
    MsCounters *ctr;
    GiantChunk *giant;
    uint32_t giant_cap;
    uint32_t V, nwords, level;
    unsigned long long all[2];  // source bits in use
    // pull phase A: dense rows of four in-neighbours per vertex (the first
    // ones, or - head_ranked - the ones of largest out-degree) and the
    // in-degrees; null: read from the pages
    const uint32_t *head;
    const uint32_t *indeg;
    uint32_t head_ranked;
    // pull levels: the frontier masks compacted (fmask[r] = visit_cur[v]
    // for the r-th frontier vertex v) and, per bitmap word w, {act_cur[w],
    // frontier vertices before word w}; one 8-byte load then gives a
    // neighbour's frontier bit and its rank, and the compacted masks stay in
    // L2 where the vertex-indexed array does not.  Null: read visit_cur.
    const uint2 *actrank;
    const unsigned long long *fmask;
    // pull over the whole range in one launch per level: CTAs take tiles
    // from ctr->tiles instead of a fixed stride, so that one holding a
    // hub's long in-list does not leave the others idle at the end
    uint32_t dyn_tiles;
    // every vertex is in this level's frontier (the frontier count equals
    // V): every frontier bit is set and every frontier mask was written
    // last level, so neighbours' masks are read without their bit
    uint32_t all_active;
};

// Frontier bit of v and, when set, its frontier mask (compacted or
// vertex-indexed): the act word (with rank) load, then the mask load.
// ALL: the caller's kernel handles all-active levels (the multi-source
// engine's pull; the mixed-batch kernels, which never have them, compile
// without the test: with it their pull ran 9.8 -> 13.0 ms on config 4b)
template <int NW, bool ALL = false>
__device__ __forceinline__ uint2 ld_actrank(const MsDev &s, uint32_t v)
{
#if SCAPH_MS_ALL_ACTIVE
    if (ALL && s.all_active) return make_uint2(0xFFFFFFFFu, 0u);
#endif
    if (s.actrank) return __ldg(&s.actrank[v >> 5]);
    return make_uint2(__ldg(&s.act_cur[v >> 5]), 0u);
}

template <int NW>
__device__ __forceinline__ Mask<NW> ld_frontier_mask(const MsDev &s, uint32_t v, uint2 ar)
{
    if (s.actrank) return ld_mask<NW>(s.fmask, ar.y + __popc(ar.x & ((1u << (v & 31)) - 1u)));
    return ld_mask<NW>(s.visit_cur, v);
}


namespace {

template <int NW>
__device__ __forceinline__ Mask<NW> all_mask(const MsDev &s)
{
    Mask<NW> m;
#pragma unroll
    for (int i = 0; i < NW; i++) m.w[i] = s.all[i];
    return m;
}

// depth planes: OR the newly reached bits into plane k for every bit k of d
template <int NW>
__device__ __forceinline__ void plane_or(const MsDev &s, uint32_t u, const Mask<NW> &nw, uint32_t d)
{
#pragma unroll 1
    for (int k = 0; k < kMsPlanes; k++) {
        if (!((d >> k) & 1u)) continue;
        unsigned long long *p = s.planes[k];
        Mask<NW> o = ld_mask<NW>(p, u);
#pragma unroll
        for (int i = 0; i < NW; i++) o.w[i] |= nw.w[i];
        st_mask<NW>(p, u, o);
    }
}

struct MsAcc {
    unsigned long long active = 0, active_edges = 0, pairs = 0, inspected = 0, completed_edges = 0;
};

__device__ __forceinline__ void ms_flush(MsAcc a, MsCounters *c)
{
    a.active = kc::warp_sum64(a.active);
    a.active_edges = kc::warp_sum64(a.active_edges);
    a.pairs = kc::warp_sum64(a.pairs);
    a.inspected = kc::warp_sum64(a.inspected);
    a.completed_edges = kc::warp_sum64(a.completed_edges);
    if ((threadIdx.x & 31) == 0) {
        if (a.active) atomicAdd(&c->active, a.active);
        if (a.active_edges) atomicAdd(&c->active_edges, a.active_edges);
        if (a.pairs) atomicAdd(&c->pairs, a.pairs);
        if (a.inspected) atomicAdd(&c->inspected, a.inspected);
        if (a.completed_edges) atomicAdd(&c->completed_edges, a.completed_edges);
    }
}

// Sends a frontier mask to up to four out-neighbours (on[j] marks the valid
// ones): their seen masks are loaded first, all four at once, then the new
// bits go out as reductions.
template <int NW>
__device__ __forceinline__ void ms_send4(const MsDev &s, const uint32_t (&u)[4], const bool (&on)[4],
                                         const Mask<NW> &vis)
{
    Mask<NW> sn[4], ac[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (on[j] && u[j] < s.V) ld_seen_acc<NW>(s.sa, u[j], sn[j], ac[j]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (!on[j]) continue;
        if (u[j] >= s.V) {
            atomicOr(&s.ctr->error, 1u);
            continue;
        }
        bool hit = false;
#pragma unroll
        for (int i = 0; i < NW; i++) {
            // bits some other sender already put in acc need not go again
            const unsigned long long n = vis.w[i] & ~(sn[j].w[i] | ac[j].w[i]);
            if (n) {
                kc::red_or(s.sa + 2ull * NW * u[j] + NW + i, n);
                hit = true;
            }
        }
        if (hit) kc::red_or(s.touched + (u[j] >> 5), 1u << (u[j] & 31));
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// push: active vertices send their frontier masks to out-neighbours
// ---------------------------------------------------------------------------
template <int NW, int B>
__device__ __forceinline__ void ms_push_body(const GraphDev &g, const MsDev &s, const RangeList &rl)
{
    __shared__ PageDev lp[kLutPages];
    __shared__ uint32_t lc[kLutCoarse];
    __shared__ uint32_t q[kMsTileWords * 32];
    __shared__ unsigned long long ebase[B];
    __shared__ uint32_t elen[B], qoff[B], wsum[B / 32];
    __shared__ Mask<NW> vis[B];
    const PageLut lut = kc::stage_lut<B>(g, lp, lc);
    __syncthreads();
    MsAcc a;
    const uint32_t ntiles = rl.n ? rl.tile0[rl.n] : (s.nwords + kMsTileWords - 1) / kMsTileWords;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint32_t rlo = 0, rhi = s.V, local;
        range_of_tile(rl, tile, rlo, rhi, local);
        const uint32_t rwhi = (uint32_t)(((unsigned long long)rhi + 31) >> 5);
        const uint32_t w = (rlo >> 5) + local * kMsTileWords + threadIdx.x;
        uint32_t f = (threadIdx.x < kMsTileWords && w < rwhi) ? s.act_cur[w] & range_mask(w, rlo, rhi) : 0u;
        if (!__syncthreads_or(f != 0)) continue;
        uint32_t total;
        uint32_t off = kc::block_exclusive_scan<B>(__popc(f), wsum, total);
        while (f) {
            q[off++] = (w << 5) + (__ffs(f) - 1);
            f &= f - 1;
        }
        __syncthreads();
        for (uint32_t c0 = 0; c0 < total; c0 += B) {
            const uint32_t k = c0 + threadIdx.x;
            uint32_t nq = 0;
            if (k < total) {
                const uint32_t v = q[k];
                const int p = lut.of(v);
                const PageDev pd = lut.pages[p];
                const uint32_t *node = g.pool + pd.base + 3ull * (v - pd.left);
                uint32_t len = node[2];
                const unsigned long long st = pd.base + 3ull * pd.nodenum + node[1];
                const Mask<NW> m = ld_mask<NW>(s.visit_cur, v);
                vis[threadIdx.x] = m;
                a.inspected += len;
                if (len > kGiantEdges) {
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
                        atomicOr(&s.ctr->error, 2u);
                    }
                }
                ebase[threadIdx.x] = st;
                elen[threadIdx.x] = len;
                nq = len ? (uint32_t)(((st + len + 3) >> 2) - (st >> 2)) : 0u;
            }
            uint32_t tq;
            const uint32_t qo = kc::block_exclusive_scan<B>(nq, wsum, tq);
            qoff[threadIdx.x] = qo;
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < tq; i += B) {
                int lo = 0, hi = B - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (qoff[mid] <= i) lo = mid; else hi = mid - 1;
                }
                const unsigned long long st = ebase[lo], en = st + elen[lo];
                const unsigned long long quad = (st >> 2) + (i - qoff[lo]);
                const uint4 val = ld_nc_v4(g.pool + quad * 4);
                const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
                bool on[4];
#pragma unroll
                for (int j = 0; j < 4; j++) on[j] = quad * 4 + j >= st && quad * 4 + j < en;
                ms_send4<NW>(s, vals, on, vis[lo]);
            }
            __syncthreads();
        }
    }
    ms_flush(a, s.ctr);
}

template <int NW, int B>
__device__ __forceinline__ void ms_push_giant_body(const GraphDev &g, const MsDev &s)
{
    const uint32_t n = min(*((volatile uint32_t *)&s.ctr->giant), s.giant_cap);
    for (uint32_t c = blockIdx.x; c < n; c += gridDim.x) {
        const GiantChunk gc = s.giant[c];
        if (gc.len > kGiantEdges || gc.start + gc.len > g.pool_words || gc.src >= s.V) {
            if (threadIdx.x == 0) atomicOr(&s.ctr->error, 8u);
            continue;
        }
        const Mask<NW> m = ld_mask<NW>(s.visit_cur, gc.src);
        const unsigned long long st = gc.start, en = gc.start + gc.len;
        for (unsigned long long qd = (st >> 2) + threadIdx.x; qd < ((en + 3) >> 2); qd += B) {
            const uint4 val = ld_nc_v4(g.pool + qd * 4);
            const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
            bool on[4];
#pragma unroll
            for (int j = 0; j < 4; j++) on[j] = qd * 4 + j >= st && qd * 4 + j < en;
            ms_send4<NW>(s, vals, on, m);
        }
    }
}

// acc -> next frontier, seen, depth planes; one warp per touched word
template <int NW, int B>
__device__ __forceinline__ void ms_finalize_body(const MsDev &s)
{
    const int lane = threadIdx.x & 31;
    const uint32_t wstride = (gridDim.x * B) >> 5;
    const Mask<NW> all = all_mask<NW>(s);
    MsAcc a;
    for (uint32_t w = (blockIdx.x * B + threadIdx.x) >> 5; w < s.nwords; w += wstride) {
        const uint32_t t = s.touched[w];
        if (!t) continue;
        const uint32_t u = (w << 5) + lane;
        bool act = false, done = false;
        if ((t >> lane) & 1u) {
            Mask<NW> sn, ac, nw, ns;
            ld_seen_acc<NW>(s.sa, u, sn, ac);
            bool complete = true;
#pragma unroll
            for (int i = 0; i < NW; i++) {
                nw.w[i] = ac.w[i] & ~sn.w[i] & all.w[i];
                ns.w[i] = sn.w[i] | nw.w[i];
                complete &= (ns.w[i] & all.w[i]) == all.w[i];
            }
            // seen |= new bits and acc = 0, in one store
            ulonglong2 *p = reinterpret_cast<ulonglong2 *>(s.sa + 2ull * NW * u);
            if constexpr (NW == 1) {
                p[0] = make_ulonglong2(ns.w[0], 0ull);
            } else {
                p[0] = make_ulonglong2(ns.w[0], ns.w[1]);
                p[1] = make_ulonglong2(0ull, 0ull);
            }
            if (any(nw)) {
                st_mask<NW>(s.visit_nxt, u, nw);
                plane_or<NW>(s, u, nw, s.level + 1);
                const uint32_t d = __ldg(&s.degree[u]);
                a.active++;
                a.active_edges += d;
                a.pairs += popc(nw);
                act = true;
                if (complete) {
                    done = true;
                    a.completed_edges += d;
                }
            }
        }
        const uint32_t am = __ballot_sync(0xFFFFFFFFu, act), dm = __ballot_sync(0xFFFFFFFFu, done);
        if (lane == 0) {
            s.touched[w] = 0;
            if (am) s.act_nxt[w] = am;
            if (dm) s.inc[w] &= ~dm;
        }
    }
    ms_flush(a, s.ctr);
}

// ---------------------------------------------------------------------------
// pull: incomplete vertices OR the frontier masks of their in-neighbours
// ---------------------------------------------------------------------------
// ENGINE: the multi-source engine's pull (per-level tile counter and
// all-active levels); the mixed-batch kernels use neither
template <int NW, int B, bool ENGINE = false>
__device__ __forceinline__ void ms_pull_body(const GraphDev &g, const MsDev &s, const RangeList &rl)
{
    __shared__ PageDev lp[kLutPages];
    __shared__ uint32_t lc[kLutCoarse];
    __shared__ uint32_t q[kMsTileWords * 32];
    __shared__ uint32_t fnd[kMsTileWords], dne[kMsTileWords];
    __shared__ uint32_t bq_u[B], bq_len[B];
    __shared__ unsigned long long bq_st[B];
    // phase-B accumulators, seeded with the bits the vertex does not miss:
    // all ones = every missing source found
    __shared__ Mask<NW> bq_acc[B];
    __shared__ uint32_t bq_qoff[B];
    __shared__ uint32_t wsum[B / 32];
    const PageLut lut = kc::stage_lut<B>(g, lp, lc);
    const Mask<NW> all = all_mask<NW>(s);
    __syncthreads();
    MsAcc a;
    const uint32_t ntiles = rl.n ? rl.tile0[rl.n] : (s.nwords + kMsTileWords - 1) / kMsTileWords;
    const bool dyn = ENGINE && SCAPH_MS_DYN_TILES && s.dyn_tiles && rl.n == 0;
    __shared__ uint32_t s_tile;
    // the CTA's next tile: from the level's counter, or a fixed stride
    auto next_tile = [&](uint32_t cur) -> uint32_t {
        if (!dyn) return cur + gridDim.x;
        __syncthreads();  // every thread has read s_tile
        if (threadIdx.x == 0) s_tile = atomicAdd(&s.ctr->tiles, 1u);
        __syncthreads();
        return s_tile;
    };
    for (uint32_t tile = dyn ? next_tile(0) : blockIdx.x; tile < ntiles; tile = next_tile(tile)) {
        uint32_t rlo = 0, rhi = s.V, local;
        range_of_tile(rl, tile, rlo, rhi, local);
        const uint32_t rwhi = (uint32_t)(((unsigned long long)rhi + 31) >> 5);
        const uint32_t wbase = (rlo >> 5) + local * kMsTileWords;
        const uint32_t w = wbase + threadIdx.x;
        uint32_t f = 0;
        if (threadIdx.x < kMsTileWords) {
            fnd[threadIdx.x] = 0;
            dne[threadIdx.x] = 0;
            if (w < rwhi) f = s.inc[w] & range_mask(w, rlo, rhi);
        }
        if (!__syncthreads_or(f != 0)) continue;
        uint32_t total;
        uint32_t off = kc::block_exclusive_scan<B>(__popc(f), wsum, total);
        while (f) {
            q[off++] = (w << 5) + (__ffs(f) - 1);
            f &= f - 1;
        }
        __syncthreads();
        for (uint32_t c0 = 0; c0 < total; c0 += B) {
            const uint32_t k = c0 + threadIdx.x;
            uint32_t u = 0, len = 0, need = 0;
            unsigned long long st = 0;
            Mask<NW> miss, acc;
#pragma unroll
            for (int i = 0; i < NW; i++) miss.w[i] = acc.w[i] = 0;
            if (k < total) {
                u = q[k];
                const Mask<NW> sn = ld_seen<NW>(s.sa, u);
#pragma unroll
                for (int i = 0; i < NW; i++) miss.w[i] = all.w[i] & ~sn.w[i];
                // four in-edges: independent loads, act probes, masks
                uint32_t v[4];
                if (s.head) {
                    len = __ldg(&s.indeg[u]);
                    const uint4 h = ld_nc_v4(s.head + 4ull * u);
                    v[0] = h.x;
                    v[1] = h.y;
                    v[2] = h.z;
                    v[3] = h.w;
                } else {
                    const int p = lut.of(u);
                    const PageDev pd = lut.pages[p];
                    const uint32_t *node = g.pool + pd.base + 3ull * (u - pd.left);
                    len = node[2];
                    st = pd.base + 3ull * pd.nodenum + node[1];
#pragma unroll
                    for (int j = 0; j < 4; j++) v[j] = (uint32_t)j < len ? __ldg(&g.pool[st + j]) : 0xFFFFFFFFu;
                }
                bool on[4];
                uint2 ar[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    ar[j] = v[j] < s.V ? ld_actrank<NW, ENGINE>(s, v[j]) : make_uint2(0u, 0u);
                    on[j] = (ar[j].x >> (v[j] & 31)) & 1u;
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (on[j]) {
                        const Mask<NW> m = ld_frontier_mask<NW>(s, v[j], ar[j]);
#pragma unroll
                        for (int i = 0; i < NW; i++) acc.w[i] |= m.w[i];
                    }
                }
                a.inspected += min(len, 4u);
                bool full = true;
#pragma unroll
                for (int i = 0; i < NW; i++) full &= (acc.w[i] & miss.w[i]) == miss.w[i];
                need = (!full && len > 4) ? 1u : 0u;
                if (need && s.head) {
                    // phase B needs where the list lives
                    const int p = lut.of(u);
                    const PageDev pd = lut.pages[p];
                    const uint32_t *node = g.pool + pd.base + 3ull * (u - pd.left);
                    st = pd.base + 3ull * pd.nodenum + node[1];
                }
            }
            uint32_t nb;
            const uint32_t bo = kc::block_exclusive_scan<B>(need, wsum, nb);
            if (need) {
                bq_u[bo] = u;
                bq_st[bo] = st;
                bq_len[bo] = len;
#pragma unroll
                for (int i = 0; i < NW; i++) bq_acc[bo].w[i] = acc.w[i] | ~miss.w[i];
            }
            __syncthreads();
            // phase B: the remaining in-edges of the unresolved vertices,
            // edge-balanced over the CTA by a scan over 16-byte quads; each
            // quad's frontier masks are OR-ed into the vertex's shared
            // accumulator (an OR-semiring SpMV over those rows)
            uint32_t nq = 0;
            if (threadIdx.x < nb) {
                const unsigned long long a0 = bq_st[threadIdx.x] + (s.head_ranked ? 0u : 4u),
                                         b0 = bq_st[threadIdx.x] + bq_len[threadIdx.x];
                nq = (uint32_t)(((b0 + 3) >> 2) - (a0 >> 2));
            }
            uint32_t tq;
            const uint32_t qo = kc::block_exclusive_scan<B>(nq, wsum, tq);
            bq_qoff[threadIdx.x] = qo;
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < tq; i += B) {
                int lo = 0, hi = (int)nb - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (bq_qoff[mid] <= i) lo = mid; else hi = mid - 1;
                }
                const unsigned long long aa = bq_st[lo] + (s.head_ranked ? 0u : 4u), bb = bq_st[lo] + bq_len[lo];
                const unsigned long long quad = (aa >> 2) + (i - bq_qoff[lo]);
                // a vertex whose accumulated masks already hold every source
                // it misses needs no more of its in-edges: its later quads
                // are skipped (the accumulator only gains bits, so a stale
                // read only skips less); the lane stays active for the
                // segmented OR below
                bool done_lo = SCAPH_MS_EARLY_EXIT != 0;
#pragma unroll
                for (int w2 = 0; w2 < NW; w2++)
                    done_lo &= *reinterpret_cast<volatile const unsigned long long *>(&bq_acc[lo].w[w2]) == ~0ull;
                const uint4 val = done_lo ? make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu)
                                          : ld_nc_v4(g.pool + quad * 4);
                const uint32_t vals[4] = {val.x, val.y, val.z, val.w};
                bool in[4], on[4];
                uint2 ar[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    in[j] = !done_lo && quad * 4 + j >= aa && quad * 4 + j < bb;
                    ar[j] = in[j] && vals[j] < s.V ? ld_actrank<NW, ENGINE>(s, vals[j]) : make_uint2(0u, 0u);
                    on[j] = (ar[j].x >> (vals[j] & 31)) & 1u;
                    a.inspected += in[j] ? 1 : 0;
                }
                Mask<NW> part;
#pragma unroll
                for (int w2 = 0; w2 < NW; w2++) part.w[w2] = 0;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (on[j]) {
                        const Mask<NW> m = ld_frontier_mask<NW>(s, vals[j], ar[j]);
#pragma unroll
                        for (int w2 = 0; w2 < NW; w2++) part.w[w2] |= m.w[w2];
                    }
                }
                // the active lanes of a warp are a prefix and cover consecutive
                // quads, so equal `lo` values are contiguous: a segmented OR by
                // doubling leaves each segment's total in its first lane, which
                // alone issues the shared atomic
                const unsigned int am = __activemask();
                const int lane = threadIdx.x & 31, nact = 32 - __clz(am);
                const int lo_prev = __shfl_up_sync(am, lo, 1);
                const bool head = lane == 0 || lo_prev != lo;
#pragma unroll
                for (int w2 = 0; w2 < NW; w2++) {
                    unsigned long long v = part.w[w2];
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const unsigned long long x = __shfl_down_sync(am, v, o);
                        const int lo2 = __shfl_down_sync(am, lo, o);
                        if (lane + o < nact && lo2 == lo) v |= x;
                    }
                    if (head && v) atomicOr(&bq_acc[lo].w[w2], v);
                }
            }
            __syncthreads();
            // merge phase-B results back into the owning thread
            if (need) acc = bq_acc[bo];
            if (k < total) {
                Mask<NW> nw;
#pragma unroll
                for (int i = 0; i < NW; i++) nw.w[i] = acc.w[i] & miss.w[i];
                if (any(nw)) {
                    const Mask<NW> sn = ld_seen<NW>(s.sa, u);
                    Mask<NW> ns;
                    bool complete = true;
#pragma unroll
                    for (int i = 0; i < NW; i++) {
                        ns.w[i] = sn.w[i] | nw.w[i];
                        complete &= (ns.w[i] & all.w[i]) == all.w[i];
                    }
                    st_seen<NW>(s.sa, u, ns);
                    st_mask<NW>(s.visit_nxt, u, nw);
                    plane_or<NW>(s, u, nw, s.level + 1);
                    const uint32_t d = __ldg(&s.degree[u]);
                    a.active++;
                    a.active_edges += d;
                    a.pairs += popc(nw);
                    atomicOr(&fnd[(u >> 5) - wbase], 1u << (u & 31));
                    if (complete) {
                        a.completed_edges += d;
                        atomicOr(&dne[(u >> 5) - wbase], 1u << (u & 31));
                    }
                }
            }
            __syncthreads();
        }
        if (threadIdx.x < kMsTileWords && w < rwhi) {
            // OR / AND-NOT: the word may be shared with a range of another
            // page batch of this level
            if (fnd[threadIdx.x]) atomicOr(&s.act_nxt[w], fnd[threadIdx.x]);
            if (dne[threadIdx.x]) atomicAnd(&s.inc[w], ~dne[threadIdx.x]);
        }
        __syncthreads();
    }
    ms_flush(a, s.ctr);
}

// host-loop kernels (MsDev by value, one launch per phase and level)
template <int NW>
__global__ void __launch_bounds__(kMsBlock) k_ms_push(GraphDev g, MsDev s, RangeList rl)
{
    ms_push_body<NW, kMsBlock>(g, s, rl);
}

template <int NW>
__global__ void __launch_bounds__(kMsBlock) k_ms_push_giant(GraphDev g, MsDev s)
{
    ms_push_giant_body<NW, kMsBlock>(g, s);
}

template <int NW>
__global__ void __launch_bounds__(kMsBlock) k_ms_finalize(MsDev s)
{
    ms_finalize_body<NW, kMsBlock>(s);
}

template <int NW>
__global__ void __launch_bounds__(kMsBlock) k_ms_pull(GraphDev g, MsDev s, RangeList rl)
{
    ms_pull_body<NW, kMsBlock, true>(g, s, rl);
}

// clears the frontier masks of the source vertices (left over from an
// earlier batch) before k_ms_sources sets their bits
template <int NW>
__global__ void k_ms_clear_sources(MsDev s, const uint32_t *srcs, int nsrc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsrc || srcs[i] >= s.V) return;
#pragma unroll
    for (int j = 0; j < NW; j++) s.visit_cur[(size_t)srcs[i] * NW + j] = 0ull;
}

// sources into the state (setsrc of app/bfs.cu:32-37, one bit per source)
template <int NW>
__global__ void k_ms_sources(MsDev s, const uint32_t *srcs, int nsrc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsrc) return;
    const uint32_t v = srcs[i];
    if (v >= s.V) {
        atomicOr(&s.ctr->error, 32u);
        return;
    }
    const int word = i >> 6;
    const unsigned long long bit = 1ull << (i & 63);
    atomicOr(s.sa + 2ull * NW * v + word, bit);
    atomicOr(s.visit_cur + (size_t)v * NW + word, bit);
    atomicOr(&s.act_cur[v >> 5], 1u << (v & 31));
}

// depth[i][u] from the bit planes; unreached where seen lacks bit i
// ---------------------------------------------------------------------------
// frontier compaction for pull levels (MsDev::actrank / fmask)
// ---------------------------------------------------------------------------
constexpr int kRankWordsPerCta = 4 * kMsBlock;  // bitmap words a CTA ranks

// Frontier vertices in each CTA's run of kRankWordsPerCta words.
static __global__ void __launch_bounds__(kMsBlock) k_ms_rank_sums(const uint32_t *act, uint32_t nwords, uint32_t *bsum)
{
    __shared__ uint32_t wsum[kMsBlock / 32];
    const size_t w0 = (size_t)blockIdx.x * kRankWordsPerCta;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const size_t w = w0 + (size_t)j * kMsBlock + threadIdx.x;
        if (w < nwords) c += __popc(act[w]);
    }
    uint32_t total;
    kc::block_exclusive_scan<kMsBlock>(c, wsum, total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// Exclusive scan of the nb run totals, in place (one CTA).
static __global__ void __launch_bounds__(kMsBlock) k_ms_rank_scan(uint32_t *bsum, uint32_t nb)
{
    __shared__ uint32_t wsum[kMsBlock / 32];
    uint32_t carry = 0;
    for (uint32_t i0 = 0; i0 < nb; i0 += kMsBlock) {
        const uint32_t i = i0 + threadIdx.x;
        const uint32_t x = i < nb ? bsum[i] : 0u;
        uint32_t total;
        const uint32_t ex = kc::block_exclusive_scan<kMsBlock>(x, wsum, total);
        if (i < nb) bsum[i] = carry + ex;
        carry += total;
    }
}

// actrank[w] = {act[w], frontier vertices before word w}, and the frontier
// masks gathered in vertex order into fmask.
template <int NW>
__global__ void __launch_bounds__(kMsBlock) k_ms_rank_gather(const uint32_t *act, uint32_t nwords, const uint32_t *bsum,
                                                             const unsigned long long *visit, uint2 *actrank,
                                                             unsigned long long *fmask)
{
    __shared__ uint32_t wsum[kMsBlock / 32];
    // this thread takes 4 consecutive words of the CTA's run
    const size_t w0 = (size_t)blockIdx.x * kRankWordsPerCta + 4ull * threadIdx.x;
    uint32_t a[4], c = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        a[j] = w0 + j < nwords ? act[w0 + j] : 0u;
        c += __popc(a[j]);
    }
    uint32_t total;
    uint32_t r = bsum[blockIdx.x] + kc::block_exclusive_scan<kMsBlock>(c, wsum, total);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (w0 + j >= nwords) break;
        actrank[w0 + j] = make_uint2(a[j], r);
        uint32_t m = a[j];
        while (m) {
            const uint32_t v = (uint32_t)((w0 + j) << 5) + (__ffs(m) - 1);
            st_mask<NW>(fmask, r++, ld_mask<NW>(visit, v));
            m &= m - 1;
        }
    }
}

// Depth rows out[i][u] from the seen masks and the NP depth bit planes.  NP
// is a template argument so that the planes stay in registers (a run-time
// plane loop put them in local memory and made this pass 4x slower than its
// writes).  When the rows are 16-byte aligned and the planes of four
// vertices fit in registers, a thread takes four consecutive vertices and
// writes each row's four depths with one 16-byte store.
// Word `hi` (0 or 1) of a mask, selected without indexing the array by a
// run-time value (which would put the masks in local memory).
template <int NW>
__device__ __forceinline__ unsigned long long mask_word(const Mask<NW> &m, bool hi)
{
    if constexpr (NW == 1) return m.w[0];
    else return hi ? m.w[NW - 1] : m.w[0];
}

template <int NW, int NP>
__device__ __forceinline__ uint32_t unpack_depth(const Mask<NW> &sn, const Mask<NW> (&pl)[NP > 0 ? NP : 1], int i,
                                                 uint32_t unreached)
{
    const bool hi = i >= 64;
    const int b = i & 63;
    if (!((mask_word<NW>(sn, hi) >> b) & 1ull)) return unreached;
    uint32_t d = 0;
#pragma unroll
    for (int k = 0; k < NP; k++) d |= (uint32_t)((mask_word<NW>(pl[k], hi) >> b) & 1ull) << k;
    return d;
}

template <int NW, int NP>
__global__ void __launch_bounds__(kMsBlock) k_ms_unpack(MsDev s, uint32_t *out, int nsrc, uint32_t unreached)
{
    constexpr bool kVec = NW * NP <= 8;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (kVec && (s.V & 3u) == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0) {
        for (size_t q = t0; q < (s.V >> 2); q += stride) {
            const uint32_t u0 = (uint32_t)q << 2;
            Mask<NW> sn[4], pl[4][NP > 0 ? NP : 1];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                sn[r] = ld_seen<NW>(s.sa, u0 + r);
#pragma unroll
                for (int k = 0; k < NP; k++) pl[r][k] = ld_mask<NW>(s.planes[k], u0 + r);
            }
            for (int i = 0; i < nsrc; i++) {
                uint4 d;
                d.x = unpack_depth<NW, NP>(sn[0], pl[0], i, unreached);
                d.y = unpack_depth<NW, NP>(sn[1], pl[1], i, unreached);
                d.z = unpack_depth<NW, NP>(sn[2], pl[2], i, unreached);
                d.w = unpack_depth<NW, NP>(sn[3], pl[3], i, unreached);
                *reinterpret_cast<uint4 *>(out + (size_t)i * s.V + u0) = d;
            }
        }
        return;
    }
    for (size_t u = t0; u < s.V; u += stride) {
        const Mask<NW> sn = ld_seen<NW>(s.sa, (uint32_t)u);
        Mask<NW> pl[NP > 0 ? NP : 1];
#pragma unroll
        for (int k = 0; k < NP; k++) pl[k] = ld_mask<NW>(s.planes[k], (uint32_t)u);
        for (int i = 0; i < nsrc; i++) out[(size_t)i * s.V + u] = unpack_depth<NW, NP>(sn, pl, i, unreached);
    }
}

// The k_ms_unpack instantiation for nplanes (0..kMsPlanes).
template <int NW>
const void *ms_unpack_kernel(int nplanes)
{
    switch (nplanes) {
    case 0: return (const void *)k_ms_unpack<NW, 0>;
    case 1: return (const void *)k_ms_unpack<NW, 1>;
    case 2: return (const void *)k_ms_unpack<NW, 2>;
    case 3: return (const void *)k_ms_unpack<NW, 3>;
    case 4: return (const void *)k_ms_unpack<NW, 4>;
    case 5: return (const void *)k_ms_unpack<NW, 5>;
    case 6: return (const void *)k_ms_unpack<NW, 6>;
    case 7: return (const void *)k_ms_unpack<NW, 7>;
    case 8: return (const void *)k_ms_unpack<NW, 8>;
    case 9: return (const void *)k_ms_unpack<NW, 9>;
    case 10: return (const void *)k_ms_unpack<NW, 10>;
    case 11: return (const void *)k_ms_unpack<NW, 11>;
    default: return (const void *)k_ms_unpack<NW, 12>;
    }
}
static_assert(kMsPlanes == 12, "ms_unpack_kernel covers 0..12 planes");

}  // namespace scaph
