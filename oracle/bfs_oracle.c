/*
 * CPU oracle for the Scaph BFS hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs load liboracle.so.  The engine in scaph_b200/ never
 * links or calls it, and has no CPU fallback.
 *
 * Every function restates the reference's algorithm in plain C and cites the
 * reference file:line (paths relative to the N-E-E/Scaph source tree) that it
 * follows.  The single-threaded BFS is pinned against the reference's own
 * bfs::check compiled from source (oracle/ref_harness.cu -> oracle/_ref) and
 * against the committed golden vectors in tests/golden/.
 *
 * Conventions: flat CSR with 64-bit row offsets `idx[V+1]` and 32-bit
 * neighbour ids `ngh[E]`; depths are uint32 with a caller-chosen "unreached"
 * sentinel (63 in the reference convention, app/bfs.cu:18; 0xFFFFFFFF natively).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define ORACLE_NOPARENT 0xFFFFFFFFu

/* ------------------------------------------------------------------------ */
/* Level-synchronous BFS, restated from bfs::check, app/bfs.cu:70-101.       */
/* `cur`/`next` frontier vectors walk the flat CSR; a neighbour is relaxed   */
/* (and pushed) when depth[v]+1 < depth[u] (app/bfs.cu:93-96).  With the     */
/* reference sentinel 63 this caps depths at 63 exactly like the reference.  */
/* Returns the number of levels (frontiers processed), or -1 on bad input.   */
/* ------------------------------------------------------------------------ */
int64_t oracle_bfs(uint32_t V, const uint64_t *idx, const uint32_t *ngh,
                   uint32_t src, uint32_t unreached, uint32_t *depth)
{
    if (src >= V) return -1;
    for (uint32_t i = 0; i < V; i++) depth[i] = unreached;       /* :77-79 */
    uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)V);
    uint32_t *next = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)V);
    if (!cur || !next) { free(cur); free(next); return -1; }
    size_t ncur = 0, nnext = 0;
    cur[ncur++] = src;                                              /* :81 */
    depth[src] = 0;                                                 /* :82 */
    int64_t levels = 0;
    while (ncur) {                                                  /* :86 */
        for (size_t i = 0; i < ncur; i++) {                         /* :87 */
            uint32_t v = cur[i];
            uint32_t dv1 = depth[v] + 1;
            for (uint64_t e = idx[v]; e < idx[v + 1]; e++) {        /* :91 */
                uint32_t u = ngh[e];
                if (dv1 < depth[u]) {                               /* :93 */
                    depth[u] = dv1;
                    next[nnext++] = u;                              /* :95 */
                }
            }
        }
        uint32_t *t = cur; cur = next; next = t;                    /* :99 */
        ncur = nnext; nnext = 0;                                    /* :100 */
        levels++;
    }
    free(cur); free(next);
    return levels;
}

/* ------------------------------------------------------------------------ */
/* The same level-synchronous BFS with the frontier expanded by all host     */
/* threads.  Relaxation is a CAS min as in the reference's CPU writeMin      */
/* (src/tools.h:102-108); because every relaxation inside a level writes the */
/* same value depth+1, the result equals oracle_bfs bit for bit.             */
/* ------------------------------------------------------------------------ */
int64_t oracle_bfs_omp(uint32_t V, const uint64_t *idx, const uint32_t *ngh,
                       uint32_t src, uint32_t unreached, uint32_t *depth,
                       int nthreads)
{
    if (src >= V) return -1;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    #pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t i = 0; i < (int64_t)V; i++) depth[i] = unreached;
    uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)V);
    uint32_t *next = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)V);
    if (!cur || !next) { free(cur); free(next); return -1; }
    size_t ncur = 1, nnext = 0;
    cur[0] = src;
    depth[src] = 0;
    int64_t levels = 0;
    while (ncur) {
        uint32_t dnew = depth[cur[0]] + 1;
        #pragma omp parallel num_threads(nthreads)
        {
            uint32_t lbuf[1024];
            size_t nl = 0;
            #pragma omp for schedule(dynamic, 64)
            for (int64_t i = 0; i < (int64_t)ncur; i++) {
                uint32_t v = cur[i];
                for (uint64_t e = idx[v]; e < idx[v + 1]; e++) {
                    uint32_t u = ngh[e];
                    uint32_t du = __atomic_load_n(&depth[u], __ATOMIC_RELAXED);
                    while (dnew < du) {
                        if (__atomic_compare_exchange_n(&depth[u], &du, dnew, 0,
                                                        __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
                            lbuf[nl++] = u;
                            if (nl == 1024) {
                                size_t at = __atomic_fetch_add(&nnext, nl, __ATOMIC_RELAXED);
                                memcpy(next + at, lbuf, nl * sizeof(uint32_t));
                                nl = 0;
                            }
                            break;
                        }
                    }
                }
            }
            if (nl) {
                size_t at = __atomic_fetch_add(&nnext, nl, __ATOMIC_RELAXED);
                memcpy(next + at, lbuf, nl * sizeof(uint32_t));
            }
        }
        uint32_t *t = cur; cur = next; next = t;
        ncur = nnext; nnext = 0;
        levels++;
    }
    free(cur); free(next);
    return levels;
}

/* ------------------------------------------------------------------------ */
/* Paged-CSR walk.  Page layout restated from tools/pagegencsr.cpp:221-242   */
/* and src/page.h:30-52: a page holds Node{vtx, idx, len}[nodenum] (3 words  */
/* each) followed by the edge words; Node.idx is the edge index relative to  */
/* the page's first edge; weighted pages hold {ngr, wgh} pairs.              */
/* `pinfo` is Page{left,right,nodenum,edgenum}[npages] (src/page.h:22-28).   */
/* ------------------------------------------------------------------------ */
static int64_t page_of(uint32_t v, const uint32_t *pinfo, int64_t npages)
{
    int64_t lo = 0, hi = npages - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) / 2;
        if (pinfo[4 * mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* BFS of app/bfs.cu:70-101 driven from the pages instead of the flat CSR.  */
int64_t oracle_bfs_paged(uint32_t V, int64_t npages, const uint32_t *pinfo,
                         const uint32_t *const *pages, int weighted,
                         uint32_t src, uint32_t unreached, uint32_t *depth)
{
    if (src >= V || npages <= 0) return -1;
    for (uint32_t i = 0; i < V; i++) depth[i] = unreached;
    uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)V);
    uint32_t *next = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)V);
    if (!cur || !next) { free(cur); free(next); return -1; }
    size_t ncur = 0, nnext = 0;
    cur[ncur++] = src;
    depth[src] = 0;
    int64_t levels = 0;
    const int ew = weighted ? 2 : 1;
    while (ncur) {
        for (size_t i = 0; i < ncur; i++) {
            uint32_t v = cur[i];
            int64_t p = page_of(v, pinfo, npages);
            uint32_t left = pinfo[4 * p], nodenum = pinfo[4 * p + 2];
            const uint32_t *pg = pages[p];
            const uint32_t *node = pg + 3 * (size_t)(v - left);
            const uint32_t *edges = pg + 3 * (size_t)nodenum;
            uint32_t pos = node[1], len = node[2];
            uint32_t dv1 = depth[v] + 1;
            for (uint32_t k = 0; k < len; k++) {
                uint32_t u = edges[(size_t)(pos + k) * ew];
                if (dv1 < depth[u]) {
                    depth[u] = dv1;
                    next[nnext++] = u;
                }
            }
        }
        uint32_t *t = cur; cur = next; next = t;
        ncur = nnext; nnext = 0;
        levels++;
    }
    free(cur); free(next);
    return levels;
}

/* ------------------------------------------------------------------------ */
/* Graph500-style BFS-tree validator (no reference counterpart: the          */
/* reference keeps no parents).  For a directed graph pass the out-edge CSR; */
/* the edge parent->v is looked up there.  Returns 0 when valid, otherwise a */
/* negative code and the first offending vertex in *bad.                     */
/*   -1 source wrong, -2 parent out of range, -3 parent depth != depth-1,    */
/*   -4 no edge parent->v, -5 unreached vertex has a parent,                 */
/*   -6 reached vertex has no parent.                                        */
/* ------------------------------------------------------------------------ */
static int has_edge(const uint64_t *idx, const uint32_t *ngh, uint32_t p, uint32_t v)
{
    uint64_t lo = idx[p], hi = idx[p + 1];
    /* adjacency lists from the generators are sorted; fall back to a scan */
    int sorted = 1;
    if (hi - lo > 16) {
        for (uint64_t e = lo + 1; e < lo + 16; e++) if (ngh[e - 1] > ngh[e]) { sorted = 0; break; }
    } else {
        sorted = 0;
    }
    if (sorted) {
        while (lo < hi) {
            uint64_t mid = lo + (hi - lo) / 2;
            if (ngh[mid] < v) lo = mid + 1; else hi = mid;
        }
        if (lo < idx[p + 1] && ngh[lo] == v) return 1;
        /* not found by bisection: the list may be unsorted further on */
    }
    for (uint64_t e = idx[p]; e < idx[p + 1]; e++) if (ngh[e] == v) return 1;
    return 0;
}

int oracle_validate_tree(uint32_t V, const uint64_t *idx, const uint32_t *ngh,
                         uint32_t src, uint32_t unreached, const uint32_t *depth,
                         const uint32_t *parent, uint32_t *bad)
{
    *bad = 0;
    if (src >= V || depth[src] != 0 || parent[src] != src) { *bad = src; return -1; }
    for (uint32_t v = 0; v < V; v++) {
        if (v == src) continue;
        if (depth[v] == unreached) {
            if (parent[v] != ORACLE_NOPARENT) { *bad = v; return -5; }
            continue;
        }
        uint32_t p = parent[v];
        if (p == ORACLE_NOPARENT) { *bad = v; return -6; }
        if (p >= V) { *bad = v; return -2; }
        if (depth[p] + 1 != depth[v]) { *bad = v; return -3; }
        if (!has_edge(idx, ngh, p, v)) { *bad = v; return -4; }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Per-page frontier statistics, restated from get_page_info,               */
/* src/gpu_engine.cuh:397-441: nodes[p] = sum of stat over [left,right],    */
/* datas[p] = sum of stat*(deg+3) (stat*(2*deg+3) for weighted pages), and  */
/* the grand totals of get_total_info (src/gpu_engine.cuh:443-456).         */
/* ------------------------------------------------------------------------ */
void oracle_page_stats(int64_t npages, const uint32_t *pinfo, const uint8_t *stat,
                       const uint32_t *degree, int weighted,
                       uint32_t *nodes, uint32_t *datas,
                       int64_t *total_nodes, int64_t *total_datas)
{
    int64_t tn = 0, td = 0;
    for (int64_t p = 0; p < npages; p++) {
        uint32_t cn = 0, cd = 0;
        for (uint32_t v = pinfo[4 * p]; v <= pinfo[4 * p + 1]; v++) {
            cn += stat[v];
            cd += stat[v] * (weighted ? degree[v] * 2 + 3 : degree[v] + 3);
        }
        nodes[p] = cn; datas[p] = cd;
        tn += cn; td += cd;
    }
    *total_nodes = tn; *total_datas = td;
}

/* ------------------------------------------------------------------------ */
/* Active-vertex page compaction, restated from compress_stat,             */
/* src/compress.h:18-40: copy the Node entries of the active vertices of a  */
/* page (idx re-based to the packed edge offset) and their edge lists into  */
/* a packed page whose edge area starts after dstnodenum Nodes.             */
/* Returns the number of active vertices written.                           */
/* ------------------------------------------------------------------------ */
uint32_t oracle_compact_page(const uint32_t *page_src, uint32_t *page_dst,
                             const uint8_t *stat, uint32_t left,
                             uint32_t srcnodenum, uint32_t dstnodenum, int weighted)
{
    const int ew = weighted ? 2 : 1;
    const uint32_t *esrc = page_src + 3 * (size_t)srcnodenum;
    uint32_t *edst = page_dst + 3 * (size_t)dstnodenum;
    uint32_t offset = 0, counter = 0;
    for (uint32_t i = 0; i < srcnodenum; i++) {
        uint32_t node = i + left;
        if (stat[node]) {
            uint32_t pos = page_src[3 * (size_t)i + 1], len = page_src[3 * (size_t)i + 2];
            page_dst[3 * (size_t)counter + 0] = node;
            page_dst[3 * (size_t)counter + 1] = offset;
            page_dst[3 * (size_t)counter + 2] = len;
            memcpy(edst + (size_t)offset * ew, esrc + (size_t)pos * ew,
                   (size_t)len * ew * sizeof(uint32_t));
            offset += len;
            counter++;
        }
    }
    return counter;
}

/* ------------------------------------------------------------------------ */
/* 32-chunk occupancy-mask helpers, restated from src/tools.h:11-85.        */
/* Bit i of `mark` set = chunk i of a device page slot is occupied.         */
/* ------------------------------------------------------------------------ */
int oracle_max_zero_run(uint32_t mark)                        /* tools.h:11-27 */
{
    int local = 0, best = 0;
    for (int i = 0; i < 32; i++) {
        if (!(mark & 1u)) local++;
        else { if (local > best) best = local; local = 0; }
        mark >>= 1;
    }
    return local > best ? local : best;
}

/* Best fit: the start of the smallest zero run of length >= required; the  */
/* scan stops at the first run of exactly `required` (tools.h:30-64).       */
int oracle_fit_zero_run(uint32_t mark, int required)
{
    int local = 0, localoff = 0, fitoff = -1;
    int fit = oracle_max_zero_run(mark);
    if (fit < required) return -1;
    for (int i = 0; i < 32; i++) {
        if (!(mark & 1u)) {
            local++;
        } else {
            if (local >= required && local <= fit) { fit = local; fitoff = localoff; }
            if (local == required) break;
            local = 0;
            localoff = i + 1;
        }
        mark >>= 1;
    }
    if (local >= required && local <= fit) { fit = local; fitoff = localoff; }
    return fitoff;
}

uint32_t oracle_set_run(uint32_t mark, int off, int n, int value) /* tools.h:67-85 */
{
    for (int i = 0; i < n && off + i < 32; i++) {
        uint32_t bit = 1u << (off + i);
        mark = value ? (mark | bit) : (mark & ~bit);
    }
    return mark;
}

/* ------------------------------------------------------------------------ */
/* App-hook vertex programs (the reference's apps).                          */
/*                                                                           */
/* oracle_hook_fixpoint restates what App::run computes for an app's hooks   */
/* (src/app.cuh:220-265 driving gpu_push_csr, src/gpu_engine.cuh:95-160):    */
/* every active vertex v pushes value[v] along its edges; an edge to u fires */
/* when cond(value[v], value[u][, w]) holds and then update() lowers         */
/* value[u] and makes u active; the run ends when no vertex is active.  The  */
/* hooks, in 32-bit unsigned arithmetic as on the GPU:                       */
/*   app 0 BFS  cond d > s + 1,  update d = s + 1   (app/bfs_kernel.cuh:6-16)  */
/*   app 1 SSSP cond d > s + w,  update d = s + w   (app/sssp_kernel.cuh:6-16) */
/*   app 2 WCC  cond d > s,      update d = s       (app/wcc_kernel.cuh:5-15)  */
/* Active vertices are processed first-in first-out; for these min-updates   */
/* the fixed point does not depend on the order.  `active` (V bytes) is the  */
/* initial stat[] of gpu_init.  Returns the vertices processed, -1 on error. */
/* ------------------------------------------------------------------------ */
int64_t oracle_hook_fixpoint(uint32_t V, const uint64_t *idx, const uint32_t *ngh,
                             const uint32_t *wgh, int app, uint32_t *value,
                             const uint8_t *active)
{
    if (app < 0 || app > 2 || (app == 1 && !wgh)) return -1;
    uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    uint8_t *inq = (uint8_t *)calloc((size_t)V + 1, 1);
    if (!q || !inq) { free(q); free(inq); return -1; }
    size_t head = 0, n = 0;                     /* ring of V+1 slots */
    const size_t cap = (size_t)V + 1;
    for (uint32_t v = 0; v < V; v++)
        if (active[v]) { q[n++] = v; inq[v] = 1; }
    int64_t processed = 0;
    while (n) {
        const uint32_t v = q[head];
        head = (head + 1) % cap;
        n--;
        inq[v] = 0;
        processed++;
        const uint32_t s = value[v];
        for (uint64_t e = idx[v]; e < idx[v + 1]; e++) {
            const uint32_t u = ngh[e];
            const uint32_t cand = app == 0 ? s + 1u : app == 1 ? s + wgh[e] : s;
            if (value[u] > cand) {
                value[u] = cand;
                if (!inq[u]) {
                    q[(head + n) % cap] = u;
                    n++;
                    inq[u] = 1;
                }
            }
        }
    }
    free(q);
    free(inq);
    return processed;
}

/* Independent checks of oracle_hook_fixpoint (not restatements of the      */
/* reference; textbook algorithms that must agree with it):                  */
/* Dijkstra from src with a binary heap over 64-bit distances, then values   */
/* at or above `far` reported as `far` (what the SSSP hooks leave there when */
/* every vertex starts at far, weights < 2^31).                              */
int oracle_sssp_dijkstra(uint32_t V, const uint64_t *idx, const uint32_t *ngh,
                         const uint32_t *wgh, uint32_t src, uint32_t far, uint32_t *value)
{
    if (src >= V) return -1;
    uint64_t *dist = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)V);
    uint64_t *hk = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)idx[V] + 1));
    uint32_t *hv = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)idx[V] + 1));
    if (!dist || !hk || !hv) { free(dist); free(hk); free(hv); return -1; }
    for (uint32_t v = 0; v < V; v++) dist[v] = UINT64_MAX;
    size_t hn = 0;
    dist[src] = 0;
    hk[0] = 0; hv[0] = src; hn = 1;
    while (hn) {
        const uint64_t d = hk[0];
        const uint32_t v = hv[0];
        /* pop */
        hn--;
        if (hn) {
            uint64_t k = hk[hn]; uint32_t x = hv[hn];
            size_t i = 0;
            for (;;) {
                size_t c = 2 * i + 1;
                if (c >= hn) break;
                if (c + 1 < hn && hk[c + 1] < hk[c]) c++;
                if (hk[c] >= k) break;
                hk[i] = hk[c]; hv[i] = hv[c]; i = c;
            }
            hk[i] = k; hv[i] = x;
        }
        if (d != dist[v]) continue;
        for (uint64_t e = idx[v]; e < idx[v + 1]; e++) {
            const uint32_t u = ngh[e];
            const uint64_t nd = d + wgh[e];
            if (nd < dist[u]) {
                dist[u] = nd;
                size_t i = hn++;
                while (i) {
                    size_t p = (i - 1) / 2;
                    if (hk[p] <= nd) break;
                    hk[i] = hk[p]; hv[i] = hv[p]; i = p;
                }
                hk[i] = nd; hv[i] = u;
            }
        }
    }
    for (uint32_t v = 0; v < V; v++) value[v] = dist[v] >= far ? far : (uint32_t)dist[v];
    value[src] = 0;
    free(dist); free(hk); free(hv);
    return 0;
}

/* Smallest id that reaches each vertex along directed edges (itself         */
/* included): what the WCC hooks leave when every vertex starts labelled by  */
/* its id and active.  Sources in increasing order; a search stops at        */
/* vertices already labelled (everything they reach is labelled already).    */
int oracle_min_reaching_id(uint32_t V, const uint64_t *idx, const uint32_t *ngh, uint32_t *label)
{
    uint32_t *stack = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    if (!stack) return -1;
    for (uint32_t v = 0; v < V; v++) label[v] = UINT32_MAX;
    for (uint32_t s = 0; s < V; s++) {
        if (label[s] != UINT32_MAX) continue;
        size_t n = 0;
        label[s] = s;
        stack[n++] = s;
        while (n) {
            const uint32_t v = stack[--n];
            for (uint64_t e = idx[v]; e < idx[v + 1]; e++) {
                const uint32_t u = ngh[e];
                if (label[u] == UINT32_MAX) { label[u] = s; stack[n++] = u; }
            }
        }
    }
    free(stack);
    return 0;
}
