// Seeded synthetic graph generators and CSR utilities (host, OpenMP).
//
// Every random draw is a hash of (seed, stream, index), so a graph depends
// only on its parameters, never on the thread count.  Adjacency lists come
// out sorted and duplicate-free, without self loops.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "common.h"

using namespace scaph;

namespace {

// Exclusive prefix sum of cnt[0..n) into off[0..n], off[n] = total.
void prefix_sum(const uint32_t *cnt, uint64_t *off, size_t n)
{
    int nt = omp_get_max_threads();
    std::vector<uint64_t> part((size_t)nt + 1, 0);
    #pragma omp parallel num_threads(nt)
    {
        int t = omp_get_thread_num();
        size_t lo = n * t / nt, hi = n * (t + 1) / nt;
        uint64_t s = 0;
        for (size_t i = lo; i < hi; i++) s += cnt[i];
        part[t + 1] = s;
        #pragma omp barrier
        #pragma omp single
        for (int k = 0; k < nt; k++) part[k + 1] += part[k];
        uint64_t run = part[t];
        for (size_t i = lo; i < hi; i++) { off[i] = run; run += cnt[i]; }
    }
    off[n] = part[nt];
}

// Sorts each adjacency list, drops duplicates and self loops, and compacts
// (idx, ngh) in place into a fresh CSR.
int finalize_csr(uint32_t V, std::vector<uint64_t> &idx, uint32_t *ngh, scaph_csr *out)
{
    std::vector<uint32_t> deg(V);
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t v = 0; v < (int64_t)V; v++) {
        uint32_t *b = ngh + idx[v], *e = ngh + idx[v + 1];
        std::sort(b, e);
        uint32_t *w = b;
        for (uint32_t *r = b; r < e; r++) {
            if (*r == (uint32_t)v) continue;
            if (w > b && w[-1] == *r) continue;
            *w++ = *r;
        }
        deg[v] = (uint32_t)(w - b);
    }
    memset(out, 0, sizeof(*out));
    out->V = V;
    out->idx = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    if (!out->idx) return set_error(SCAPH_ENOMEM, "csr idx");
    prefix_sum(deg.data(), out->idx, V);
    out->E = out->idx[V];
    out->ngh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, out->E));
    if (!out->ngh) { scaph_csr_free(out); return set_error(SCAPH_ENOMEM, "csr ngh"); }
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t v = 0; v < (int64_t)V; v++)
        memcpy(out->ngh + out->idx[v], ngh + idx[v], (size_t)deg[v] * 4);
    return SCAPH_OK;
}

// Bijection on [0, 2^bits): odd multiply, xor-shift, odd multiply, keyed.
uint64_t scramble_bits(uint64_t x, int bits, uint64_t key)
{
    const uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    x = (x * 0x9E3779B97F4A7C15ull + (key & mask)) & mask;
    x ^= x >> ((bits + 1) / 2);
    x = (x * (0xD6E8FEB86659FD93ull | 1)) & mask;
    x ^= x >> ((bits + 2) / 3 + 1);
    x = (x * (mix64(key) | 1)) & mask;
    return x;
}

// Keyed bijection on [0, n) by cycle walking a 4-round Feistel network over
// the next even power of two.
struct RangePerm {
    uint64_t n;
    int half;
    uint64_t key;
    uint64_t round(uint64_t r, int i) const { return mix64(r ^ (key + 0x51ull * (uint64_t)(i + 1))) & ((1ull << half) - 1); }
    uint64_t enc1(uint64_t x) const
    {
        uint64_t m = (1ull << half) - 1, L = x >> half, R = x & m;
        for (int i = 0; i < 4; i++) { uint64_t t = R; R = L ^ round(R, i); L = t; }
        return (L << half) | R;
    }
    uint64_t dec1(uint64_t y) const
    {
        uint64_t m = (1ull << half) - 1, L = y >> half, R = y & m;
        for (int i = 3; i >= 0; i--) { uint64_t t = L; L = R ^ round(L, i); R = t; }
        return (L << half) | R;
    }
    RangePerm(uint64_t n_, uint64_t key_) : n(n_), key(key_)
    {
        int bits = 2;
        while ((1ull << bits) < n) bits++;
        half = (bits + 1) / 2;
    }
    uint64_t fwd(uint64_t x) const { do { x = enc1(x); } while (x >= n); return x; }
    uint64_t inv(uint64_t y) const { do { y = dec1(y); } while (y >= n); return y; }
};

// Out-degrees d_v = min(cap, floor(xm * y_v)) with y_v = U^(-1/(s-1)) (a
// Pareto tail with density ~ k^-s), xm chosen by bisection so that the sum
// is as close as possible to E.  Degrees are at least 1.
void powerlaw_degrees(uint32_t V, uint64_t E, double s, uint32_t cap, uint64_t seed,
                      std::vector<uint32_t> &deg)
{
    std::vector<float> y(V);
    const double ex = -1.0 / std::max(1e-3, s - 1.0);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) {
        double u = unit_double(mix64(seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(v + 1))));
        u = std::max(u, 1e-12);
        y[v] = (float)std::min(1e12, std::pow(u, ex));
    }
    auto total = [&](double xm) {
        uint64_t t = 0;
        #pragma omp parallel for reduction(+ : t) schedule(static)
        for (int64_t v = 0; v < (int64_t)V; v++) {
            double d = std::floor(xm * y[v]);
            t += (uint64_t)std::max(1.0, std::min((double)cap, d));
        }
        return t;
    };
    double lo = 1e-6, hi = 1.0;
    while (total(hi) < E && hi < 1e9) hi *= 2;
    for (int it = 0; it < 60; it++) {
        double mid = 0.5 * (lo + hi);
        if (total(mid) < E) lo = mid; else hi = mid;
    }
    deg.resize(V);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) {
        double d = std::floor(hi * y[v]);
        deg[v] = (uint32_t)std::max(1.0, std::min((double)cap, d));
    }
}

}  // namespace

extern "C" {

int scaph_gen_rmat(int scale, double edgefactor, double a, double b, double c, uint64_t seed,
                   int scramble, scaph_csr *out)
{
    clear_error();
    if (!out || scale < 1 || scale > 31 || edgefactor <= 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1)
        return set_error(SCAPH_EINVAL, "bad rmat parameters");
    const uint32_t V = 1u << scale;
    const uint64_t M = (uint64_t)std::llround(edgefactor * (double)V / 2.0);
    // 21-bit probability thresholds; three levels per 64-bit hash.
    const uint32_t ta = (uint32_t)std::lround(a * (1 << 21));
    const uint32_t tab = (uint32_t)std::lround((a + b) * (1 << 21));
    const uint32_t tabc = (uint32_t)std::lround((a + b + c) * (1 << 21));
    std::unique_ptr<uint32_t[]> src(new (std::nothrow) uint32_t[M]), dst(new (std::nothrow) uint32_t[M]);
    if (!src || !dst) return set_error(SCAPH_ENOMEM, "rmat edge buffer");
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)M; i++) {
        uint32_t u = 0, v = 0;
        uint64_t h = 0;
        for (int l = 0; l < scale; l++) {
            if (l % 3 == 0) h = mix64(seed * 0x632BE59BD9B4E019ull + (uint64_t)i * 11 + (uint64_t)(l / 3));
            uint32_t r = (uint32_t)(h & ((1u << 21) - 1));
            h >>= 21;
            uint32_t bu = r >= tab ? 1u : 0u;
            uint32_t bv = (r >= ta && r < tab) || r >= tabc ? 1u : 0u;
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        if (scramble) {
            u = (uint32_t)scramble_bits(u, scale, seed);
            v = (uint32_t)scramble_bits(v, scale, seed);
        }
        src[i] = u;
        dst[i] = v;
    }
    // symmetrise: count both directions, scatter, then dedup per list.
    std::vector<std::atomic<uint32_t>> cnt(V);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) cnt[v].store(0, std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)M; i++) {
        if (src[i] == dst[i]) continue;
        cnt[src[i]].fetch_add(1, std::memory_order_relaxed);
        cnt[dst[i]].fetch_add(1, std::memory_order_relaxed);
    }
    std::vector<uint32_t> deg(V);
    for (uint32_t v = 0; v < V; v++) deg[v] = cnt[v].load(std::memory_order_relaxed);
    std::vector<uint64_t> idx((size_t)V + 1);
    prefix_sum(deg.data(), idx.data(), V);
    std::unique_ptr<uint32_t[]> ngh(new (std::nothrow) uint32_t[std::max<uint64_t>(1, idx[V])]);
    if (!ngh) return set_error(SCAPH_ENOMEM, "rmat adjacency buffer");
    std::vector<std::atomic<uint64_t>> pos(V);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) pos[v].store(idx[v], std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)M; i++) {
        uint32_t u = src[i], v = dst[i];
        if (u == v) continue;
        ngh[pos[u].fetch_add(1, std::memory_order_relaxed)] = v;
        ngh[pos[v].fetch_add(1, std::memory_order_relaxed)] = u;
    }
    src.reset();
    dst.reset();
    return finalize_csr(V, idx, ngh.get(), out);
}

int scaph_gen_powerlaw(uint32_t V, uint64_t E, double zipf_s, uint32_t max_degree, uint64_t seed,
                       scaph_csr *out)
{
    clear_error();
    if (!out || V < 2 || E == 0 || zipf_s <= 1.0) return set_error(SCAPH_EINVAL, "bad power-law parameters");
    if (max_degree == 0 || max_degree > V - 1) max_degree = V - 1;
    std::vector<uint32_t> deg;
    powerlaw_degrees(V, E, zipf_s, max_degree, seed, deg);
    std::vector<uint64_t> idx((size_t)V + 1);
    prefix_sum(deg.data(), idx.data(), V);
    const uint64_t M = idx[V];
    std::unique_ptr<uint32_t[]> ngh(new (std::nothrow) uint32_t[std::max<uint64_t>(1, M)]);
    if (!ngh) return set_error(SCAPH_ENOMEM, "power-law adjacency buffer");
    // Copy-model preferential attachment.  Edge slots are visited in a keyed
    // random "arrival" order; the first V arrivals pick uniform destinations,
    // later ones (in doubling rounds) copy the destination of a uniformly
    // chosen earlier arrival with probability 1/2, else pick uniformly.  So
    // P(dst = v) grows with v's in-degree so far.
    RangePerm perm(M, mix64(seed ^ 0xA5A5A5A5ull));
    uint64_t done = std::min<uint64_t>(M, V);
    #pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)done; t++) {
        uint64_t slot = perm.inv((uint64_t)t);
        ngh[slot] = (uint32_t)(mix64(seed * 31 + (uint64_t)t * 0x9E37ull + 7) % V);
    }
    while (done < M) {
        uint64_t hi = std::min<uint64_t>(M, done * 2);
        #pragma omp parallel for schedule(static)
        for (int64_t t = (int64_t)done; t < (int64_t)hi; t++) {
            uint64_t h = mix64(seed * 131 + (uint64_t)t * 0x2545F491ull + 3);
            uint64_t slot = perm.inv((uint64_t)t);
            if (h & 1) {
                ngh[slot] = (uint32_t)((h >> 1) % V);
            } else {
                uint64_t earlier = mix64(h) % done;
                ngh[slot] = ngh[perm.inv(earlier)];
            }
        }
        done = hi;
    }
    return finalize_csr(V, idx, ngh.get(), out);
}

int scaph_gen_web(uint32_t V, uint64_t E, double s, uint32_t max_degree, uint32_t block,
                  double local_frac, uint64_t seed, scaph_csr *out)
{
    clear_error();
    if (!out || V < 2 || E == 0 || s <= 1.0 || block == 0 || local_frac < 0 || local_frac > 1)
        return set_error(SCAPH_EINVAL, "bad web-graph parameters");
    if (max_degree == 0 || max_degree > V - 1) max_degree = V - 1;
    std::vector<uint32_t> deg;
    powerlaw_degrees(V, E, s, max_degree, seed, deg);
    std::vector<uint64_t> idx((size_t)V + 1);
    prefix_sum(deg.data(), idx.data(), V);
    const uint64_t M = idx[V];
    std::unique_ptr<uint32_t[]> ngh(new (std::nothrow) uint32_t[std::max<uint64_t>(1, M)]);
    if (!ngh) return set_error(SCAPH_ENOMEM, "web adjacency buffer");
    // Per vertex, round(local_frac * deg) DISTINCT neighbours inside its
    // block (a walk with a random odd stride over the block's ids, skipping
    // the vertex itself: a full cycle when the block size is a power of
    // two, otherwise until the block is exhausted), the rest uniform over
    // all vertices; local edges that do not fit the block become uniform
    // ones.  So the deduplicated edge count stays close to E.
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)V; v++) {
        const uint64_t base = ((uint64_t)v / block) * block;
        const uint64_t span = std::min<uint64_t>(block, V - base);
        const uint64_t d = idx[v + 1] - idx[v];
        uint64_t k = (uint64_t)(local_frac * (double)d + 0.5);
        if (k > span - 1) k = span - 1;
        const uint64_t h0 = mix64(seed * 0xD6E8FEB86659FD93ull + (uint64_t)v);
        const uint64_t off = (h0 >> 32) % span;
        uint64_t stride = (h0 & 0xFFFFFFFFull) % span;
        stride |= 1;  // odd: coprime with a power-of-two block
        uint64_t e = idx[v], pos = off, steps = 0;
        while (e < idx[v] + k && steps < span) {
            const uint64_t u = base + pos;
            pos = (pos + stride) % span;
            steps++;
            if (u == (uint64_t)v) continue;
            ngh[e++] = (uint32_t)u;
        }
        for (; e < idx[v + 1]; e++) {
            const uint64_t h = mix64(seed * 0x94D049BBull + e);
            ngh[e] = (uint32_t)((h >> 32) % V);
        }
    }
    return finalize_csr(V, idx, ngh.get(), out);
}

int scaph_csr_transpose(const scaph_csr *in, scaph_csr *out)
{
    clear_error();
    if (!in || !out || !in->idx) return set_error(SCAPH_EINVAL, "null argument");
    const uint32_t V = in->V;
    std::vector<std::atomic<uint32_t>> cnt(V);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) cnt[v].store(0, std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)in->E; e++) cnt[in->ngh[e]].fetch_add(1, std::memory_order_relaxed);
    std::vector<uint32_t> deg(V);
    for (uint32_t v = 0; v < V; v++) deg[v] = cnt[v].load(std::memory_order_relaxed);
    memset(out, 0, sizeof(*out));
    out->V = V;
    out->E = in->E;
    out->idx = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    out->ngh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, in->E));
    if (in->wgh) out->wgh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, in->E));
    if (!out->idx || !out->ngh || (in->wgh && !out->wgh)) { scaph_csr_free(out); return set_error(SCAPH_ENOMEM, "transpose"); }
    prefix_sum(deg.data(), out->idx, V);
    std::vector<std::atomic<uint64_t>> pos(V);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) pos[v].store(out->idx[v], std::memory_order_relaxed);
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < (int64_t)V; u++) {
        for (uint64_t e = in->idx[u]; e < in->idx[u + 1]; e++) {
            uint64_t at = pos[in->ngh[e]].fetch_add(1, std::memory_order_relaxed);
            out->ngh[at] = (uint32_t)u;
            if (in->wgh) out->wgh[at] = in->wgh[e];
        }
    }
    // deterministic order: sort each in-list (weights follow their edge)
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t v = 0; v < (int64_t)V; v++) {
        uint64_t b = out->idx[v], e = out->idx[v + 1];
        if (!out->wgh) {
            std::sort(out->ngh + b, out->ngh + e);
        } else {
            std::vector<std::pair<uint32_t, uint32_t>> tmp(e - b);
            for (uint64_t k = b; k < e; k++) tmp[k - b] = {out->ngh[k], out->wgh[k]};
            std::sort(tmp.begin(), tmp.end());
            for (uint64_t k = b; k < e; k++) { out->ngh[k] = tmp[k - b].first; out->wgh[k] = tmp[k - b].second; }
        }
    }
    return SCAPH_OK;
}

}  // extern "C"
