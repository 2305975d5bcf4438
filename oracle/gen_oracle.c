/* Seeded RMAT generator for the CPU side of the benchmark (TEST
 * INFRASTRUCTURE ONLY).
 *
 * bench.py's reference arm times the reference's CPU BFS on the same graph
 * as the GPU arm, but must not load the product library to build it.  This
 * file states the same generator as scaph_gen_rmat on its own: every edge i
 * of M = round(edgefactor * 2^scale / 2) draws its quadrant bits from
 * splitmix64 hashes of (seed, i, level/3), 21 bits per level against the
 * thresholds round(a * 2^21), round((a+b) * 2^21), round((a+b+c) * 2^21);
 * optional keyed bit scrambling of both endpoints; self loops dropped; both
 * directions kept; each list sorted and deduplicated.  A CPU test checks
 * that the two produce identical CSR arrays.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t sm64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* keyed bijection of [0, 2^bits) */
static uint32_t scramble(uint64_t x, int bits, uint64_t key)
{
    const uint64_t m = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    x = (x * 0x9E3779B97F4A7C15ull + (key & m)) & m;
    x ^= x >> ((bits + 1) / 2);
    x = (x * 0xD6E8FEB86659FD93ull) & m; /* already odd */
    x ^= x >> ((bits + 2) / 3 + 1);
    x = (x * (sm64(key) | 1)) & m;
    return (uint32_t)x;
}

static int cmp_u32(const void *a, const void *b)
{
    const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

/* Fills idx[0..2^scale] and returns the adjacency in *ngh_out (malloc'd,
 * free with oracle_free); *E_out = its length.  Returns 0, or -1 on bad
 * parameters / allocation failure. */
int oracle_gen_rmat(int scale, double edgefactor, double a, double b, double c, uint64_t seed, int do_scramble,
                    uint64_t *idx, uint32_t **ngh_out, uint64_t *E_out)
{
    if (scale < 1 || scale > 31 || edgefactor <= 0 || !idx || !ngh_out || !E_out) return -1;
    const uint32_t V = 1u << scale;
    const int64_t M = (int64_t)llround(edgefactor * (double)V / 2.0);
    const uint32_t t1 = (uint32_t)lround(a * (1 << 21));
    const uint32_t t2 = (uint32_t)lround((a + b) * (1 << 21));
    const uint32_t t3 = (uint32_t)lround((a + b + c) * (1 << 21));
    uint64_t *pair = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(M > 0 ? M : 1));
    uint32_t *cnt = (uint32_t *)calloc(V, sizeof(uint32_t));
    if (!pair || !cnt) {
        free(pair);
        free(cnt);
        return -1;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < M; i++) {
        uint32_t u = 0, v = 0;
        uint64_t h = 0;
        for (int l = 0; l < scale; l++) {
            if (l % 3 == 0) h = sm64(seed * 0x632BE59BD9B4E019ull + (uint64_t)i * 11 + (uint64_t)(l / 3));
            const uint32_t r = (uint32_t)(h & ((1u << 21) - 1));
            h >>= 21;
            u = (u << 1) | (r >= t2);
            v = (v << 1) | ((r >= t1 && r < t2) || r >= t3);
        }
        if (do_scramble) {
            u = scramble(u, scale, seed);
            v = scramble(v, scale, seed);
        }
        pair[i] = ((uint64_t)u << 32) | v;
        if (u != v) {
#pragma omp atomic
            cnt[u]++;
#pragma omp atomic
            cnt[v]++;
        }
    }
    uint64_t *start = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    if (!start) {
        free(pair);
        free(cnt);
        return -1;
    }
    start[0] = 0;
    for (uint32_t v = 0; v < V; v++) start[v + 1] = start[v] + cnt[v];
    uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(start[V] ? start[V] : 1));
    uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)V);
    if (!buf || !fill) {
        free(pair);
        free(cnt);
        free(start);
        free(buf);
        free(fill);
        return -1;
    }
    memcpy(fill, start, sizeof(uint64_t) * V);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < M; i++) {
        const uint32_t u = (uint32_t)(pair[i] >> 32), v = (uint32_t)pair[i];
        if (u == v) continue;
        uint64_t pu, pv;
#pragma omp atomic capture
        pu = fill[u]++;
#pragma omp atomic capture
        pv = fill[v]++;
        buf[pu] = v;
        buf[pv] = u;
    }
    free(pair);
    free(fill);
    /* sort and deduplicate every list in place; cnt becomes the kept length */
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)V; v++) {
        uint32_t *l = buf + start[v];
        const uint32_t n = (uint32_t)(start[v + 1] - start[v]);
        qsort(l, n, sizeof(uint32_t), cmp_u32);
        uint32_t k = 0;
        for (uint32_t j = 0; j < n; j++)
            if (k == 0 || l[k - 1] != l[j]) l[k++] = l[j];
        cnt[v] = k;
    }
    idx[0] = 0;
    for (uint32_t v = 0; v < V; v++) idx[v + 1] = idx[v] + cnt[v];
    const uint64_t E = idx[V];
    uint32_t *ngh = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(E ? E : 1));
    if (!ngh) {
        free(buf);
        free(cnt);
        free(start);
        return -1;
    }
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; v++) memcpy(ngh + idx[v], buf + start[v], sizeof(uint32_t) * cnt[v]);
    free(buf);
    free(cnt);
    free(start);
    *ngh_out = ngh;
    *E_out = E;
    return 0;
}

void oracle_free(void *p) { free(p); }
