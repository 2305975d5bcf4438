// Flat-CSR and paged-CSR file formats of Scaph, plus in-memory paging.
//
// The paged format is the one tools/pagegencsr.cpp writes and src/graph.h
// reads; the layout (Node{vtx,idx,len} triples, then edges, zero padded to
// pagesize words) is fixed by those files and kept byte-for-byte.
#include <cuda_runtime_api.h>
#include <omp.h>
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "common.h"

namespace scaph {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

namespace {
struct FaultArm {
    std::atomic<int> skip{0}, count{0};
};
FaultArm g_faults[kFaultSites];
const char *const kFaultNames[kFaultSites] = {"pinned_alloc", "host_register", "page_copy", "device_alloc"};
const int kFaultErrors[kFaultSites] = {(int)cudaErrorMemoryAllocation, (int)cudaErrorHostMemoryAlreadyRegistered,
                                       (int)cudaErrorUnknown, (int)cudaErrorMemoryAllocation};
}  // namespace

int injected_fault(FaultSite site)
{
    FaultArm &f = g_faults[site];
    if (f.count.load(std::memory_order_relaxed) <= 0) return (int)cudaSuccess;
    if (f.skip.load(std::memory_order_relaxed) > 0 && f.skip.fetch_sub(1) > 0) return (int)cudaSuccess;
    if (f.count.fetch_sub(1) <= 0) return (int)cudaSuccess;
    return kFaultErrors[site];
}

uint32_t *alloc_words(size_t words)
{
    size_t bytes = std::max<size_t>(4096, (words * 4 + 4095) & ~size_t(4095));
    void *p = nullptr;
    if (posix_memalign(&p, 4096, bytes) != 0) return nullptr;
    memset(p, 0, bytes);
    return (uint32_t *)p;
}

void free_words(uint32_t *p) { free(p); }

Graph::~Graph()
{
    if (pinned && data) cudaHostUnregister(data);
    free_words(data);
}

// tools/pagegencsr.cpp:106-163 (bsearch) finds, for a page starting at
// `left`, the largest right with cost(right) < pagesize where
// cost(r) = (r-left+1)*3 + (idx[r+1]-idx[left]) * (weighted ? 2 : 1).
// The search there starts from right = left + pagesize clamped to V-1
// (:206-207; its clamp misses right == V, which this version clamps too).
bool page_cut(const uint64_t *idx, uint32_t V, uint32_t left, uint32_t pagesize,
              int weighted, uint32_t *right)
{
    const uint64_t ew = weighted ? 2 : 1;
    auto cost = [&](uint64_t r) { return (r - left + 1) * 3 + (idx[r + 1] - idx[left]) * ew; };
    if (cost(left) >= pagesize) return false;
    uint64_t hi = std::min<uint64_t>((uint64_t)left + pagesize, (uint64_t)V - 1);
    if (cost(hi) < pagesize) { *right = (uint32_t)hi; return true; }
    uint64_t lo = left;  // cost(lo) < pagesize <= cost(hi)
    while (hi - lo > 1) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (cost(mid) < pagesize) lo = mid; else hi = mid;
    }
    *right = (uint32_t)lo;
    return true;
}

}  // namespace scaph

using namespace scaph;

// ---------------------------------------------------------------------------
// file helpers
// ---------------------------------------------------------------------------
static long long file_size(const std::string &path)
{
    struct stat st;
    if (stat(path.c_str(), &st) != 0) return -1;
    return (long long)st.st_size;
}

static int read_file(const std::string &path, void *dst, size_t bytes)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return set_error(SCAPH_EIO, "cannot open %s", path.c_str());
    size_t got = fread(dst, 1, bytes, f);
    fclose(f);
    if (got != bytes) return set_error(SCAPH_EIO, "%s: read %zu of %zu bytes", path.c_str(), got, bytes);
    return SCAPH_OK;
}

static int write_file(const std::string &path, const void *src, size_t bytes)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return set_error(SCAPH_EIO, "cannot create %s", path.c_str());
    size_t put = bytes ? fwrite(src, 1, bytes, f) : 0;
    int rc = fclose(f);
    if (put != bytes || rc != 0) return set_error(SCAPH_EIO, "%s: short write", path.c_str());
    return SCAPH_OK;
}

// Builds page p's words (Node triples then edges) into `dst` (pagesize words,
// already zeroed).  Mirrors the copy in tools/pagegencsr.cpp:221-242.
static void fill_page(const scaph_csr *csr, const scaph_page_info &pi, int weighted, uint32_t *dst)
{
    const uint64_t base = csr->idx[pi.left];
    uint32_t *node = dst;
    for (uint32_t v = pi.left; v <= pi.right; v++) {
        size_t k = (size_t)(v - pi.left) * 3;
        node[k + 0] = v;
        node[k + 1] = (uint32_t)(csr->idx[v] - base);
        node[k + 2] = (uint32_t)(csr->idx[v + 1] - csr->idx[v]);
    }
    uint32_t *edges = dst + (size_t)pi.nodenum * 3;
    if (weighted) {
        for (uint32_t e = 0; e < pi.edgenum; e++) {
            edges[2 * (size_t)e] = csr->ngh[base + e];
            edges[2 * (size_t)e + 1] = csr->wgh ? csr->wgh[base + e] : 0;
        }
    } else {
        memcpy(edges, csr->ngh + base, (size_t)pi.edgenum * sizeof(uint32_t));
    }
}

static int cut_pages(const scaph_csr *csr, uint32_t pagesize, int weighted,
                     std::vector<scaph_page_info> &pages)
{
    pages.clear();
    if (csr->V == 0) return set_error(SCAPH_EINVAL, "empty graph");
    if (pagesize < 8) return set_error(SCAPH_EINVAL, "pagesize %u too small", pagesize);
    uint32_t left = 0;
    while (left < csr->V) {
        uint32_t right;
        if (!page_cut(csr->idx, csr->V, left, pagesize, weighted, &right))
            return set_error(SCAPH_EUNSUPPORTED,
                             "vertex %u (degree %llu) does not fit a page of %u words", left,
                             (unsigned long long)(csr->idx[left + 1] - csr->idx[left]), pagesize);
        scaph_page_info pi;
        pi.left = left;
        pi.right = right;
        pi.nodenum = right - left + 1;
        pi.edgenum = (uint32_t)(csr->idx[right + 1] - csr->idx[left]);
        pages.push_back(pi);
        if (right == csr->V - 1) break;
        left = right + 1;
    }
    return SCAPH_OK;
}

namespace scaph {

void adjacency_heads(const Graph &g, uint32_t width, uint32_t *out, const uint32_t *rank)
{
    const uint32_t ew = g.weighted ? 2 : 1;
    const int np = (int)g.pages.size();
    #pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < np; p++) {
        const scaph_page_info &pi = g.pages[p];
        const uint32_t *pg = g.page(p);
        const uint32_t *edges = pg + 3ull * pi.nodenum;
        std::vector<std::pair<uint32_t, uint32_t>> top;  // (rank, neighbour)
        for (uint32_t i = 0; i < pi.nodenum; i++) {
            const uint32_t v = pi.left + i, idx = pg[3 * i + 1], len = pg[3 * i + 2];
            uint32_t *row = out + (size_t)v * width;
            if (!rank || len <= width) {
                for (uint32_t j = 0; j < width; j++) row[j] = j < len ? edges[(uint64_t)(idx + j) * ew] : 0xFFFFFFFFu;
                continue;
            }
            // the `width` neighbours of largest rank, largest first
            top.clear();
            for (uint32_t k = 0; k < len; k++) {
                const uint32_t u = edges[(uint64_t)(idx + k) * ew];
                const uint32_t r = rank[u];
                if (top.size() < width) {
                    top.emplace_back(r, u);
                    std::push_heap(top.begin(), top.end(), std::greater<>());
                } else if (r > top.front().first) {
                    std::pop_heap(top.begin(), top.end(), std::greater<>());
                    top.back() = {r, u};
                    std::push_heap(top.begin(), top.end(), std::greater<>());
                }
            }
            std::sort(top.begin(), top.end(), std::greater<>());
            for (uint32_t j = 0; j < width; j++) row[j] = top[j].second;
        }
    }
}

}  // namespace scaph

extern "C" {

const char *scaph_last_error(void) { return g_last_error.c_str(); }
const char *scaph_version(void) { return "scaph-b200 0.1 (sm_100a)"; }

int scaph_fault_inject(const char *site, int skip, int count)
{
    if (!site) {
        for (auto &f : g_faults) {
            f.count.store(0);
            f.skip.store(0);
        }
        return SCAPH_OK;
    }
    for (int i = 0; i < kFaultSites; i++) {
        if (strcmp(site, kFaultNames[i]) != 0) continue;
        g_faults[i].skip.store(skip > 0 ? skip : 0);
        g_faults[i].count.store(count > 0 ? count : 0);
        return SCAPH_OK;
    }
    return set_error(SCAPH_EINVAL, "unknown fault site '%s'", site);
}

int scaph_csr_from_arrays(uint32_t V, uint64_t E, const uint64_t *idx, const uint32_t *ngh,
                          const uint32_t *wgh, scaph_csr *out)
{
    if (!out || !idx || (!ngh && E)) return set_error(SCAPH_EINVAL, "null argument");
    if (idx[0] != 0 || idx[V] != E) return set_error(SCAPH_EINVAL, "idx[0]/idx[V] inconsistent with E");
    memset(out, 0, sizeof(*out));
    out->V = V;
    out->E = E;
    out->idx = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    out->ngh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<size_t>(1, E));
    if (wgh) out->wgh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<size_t>(1, E));
    if (!out->idx || !out->ngh || (wgh && !out->wgh)) {
        scaph_csr_free(out);
        return set_error(SCAPH_ENOMEM, "csr allocation");
    }
    memcpy(out->idx, idx, sizeof(uint64_t) * ((size_t)V + 1));
    if (E) memcpy(out->ngh, ngh, sizeof(uint32_t) * E);
    if (wgh && E) memcpy(out->wgh, wgh, sizeof(uint32_t) * E);
    for (uint32_t v = 0; v < V; v++)
        if (idx[v + 1] < idx[v]) { scaph_csr_free(out); return set_error(SCAPH_EINVAL, "idx not monotone at %u", v); }
    for (uint64_t e = 0; e < E; e++)
        if (ngh[e] >= V) { scaph_csr_free(out); return set_error(SCAPH_EINVAL, "neighbour %u out of range", ngh[e]); }
    return SCAPH_OK;
}

void scaph_csr_free(scaph_csr *csr)
{
    if (!csr) return;
    free(csr->idx);
    free(csr->ngh);
    free(csr->wgh);
    memset(csr, 0, sizeof(*csr));
}

int scaph_csr_write(const char *prefix, const scaph_csr *csr)
{
    clear_error();
    if (!prefix || !csr || !csr->idx) return set_error(SCAPH_EINVAL, "null argument");
    if (csr->E >= (1ull << 32)) return set_error(SCAPH_EUNSUPPORTED, "E >= 2^32 needs 64-bit index files");
    std::string p(prefix);
    const uint32_t V = csr->V;
    std::vector<uint32_t> idx32((size_t)V + 1), deg(V);
    for (uint32_t v = 0; v <= V; v++) idx32[v] = (uint32_t)csr->idx[v];
    for (uint32_t v = 0; v < V; v++) deg[v] = (uint32_t)(csr->idx[v + 1] - csr->idx[v]);
    int rc;
    if ((rc = write_file(p + "_csr.idx", idx32.data(), idx32.size() * 4))) return rc;
    if ((rc = write_file(p + "_csr.ngh", csr->ngh, csr->E * 4))) return rc;
    if ((rc = write_file(p + "_csr.deg", deg.data(), deg.size() * 4))) return rc;
    if (csr->wgh) {
        rc = write_file(p + "_csr.wgh", csr->wgh, csr->E * 4);
    } else {
        std::vector<uint32_t> zeros(csr->E, 0);
        rc = write_file(p + "_csr.wgh", zeros.data(), csr->E * 4);
    }
    return rc;
}

int scaph_csr_read(const char *prefix, int with_weights, scaph_csr *out)
{
    clear_error();
    if (!prefix || !out) return set_error(SCAPH_EINVAL, "null argument");
    memset(out, 0, sizeof(*out));
    std::string p(prefix);
    long long idx_bytes = file_size(p + "_csr.idx"), ngh_bytes = file_size(p + "_csr.ngh");
    if (idx_bytes < 8 || ngh_bytes < 0 || idx_bytes % 4 || ngh_bytes % 4)
        return set_error(SCAPH_EIO, "missing or malformed %s_csr.idx/.ngh", prefix);
    uint32_t V = (uint32_t)(idx_bytes / 4 - 1);
    uint64_t E = (uint64_t)ngh_bytes / 4;
    std::vector<uint32_t> idx32((size_t)V + 1);
    int rc;
    if ((rc = read_file(p + "_csr.idx", idx32.data(), idx32.size() * 4))) return rc;
    out->V = V;
    out->E = E;
    out->idx = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    out->ngh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, E));
    if (!out->idx || !out->ngh) { scaph_csr_free(out); return set_error(SCAPH_ENOMEM, "csr allocation"); }
    for (size_t v = 0; v <= V; v++) out->idx[v] = idx32[v];
    if (out->idx[V] != E) { scaph_csr_free(out); return set_error(SCAPH_EFORMAT, "idx[V] != edge count"); }
    if ((rc = read_file(p + "_csr.ngh", out->ngh, E * 4))) { scaph_csr_free(out); return rc; }
    if (with_weights) {
        out->wgh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, E));
        if (!out->wgh) { scaph_csr_free(out); return set_error(SCAPH_ENOMEM, "csr allocation"); }
        if ((rc = read_file(p + "_csr.wgh", out->wgh, E * 4))) { scaph_csr_free(out); return rc; }
    }
    return SCAPH_OK;
}

int scaph_pages_write(const char *prefix, const scaph_csr *csr, uint32_t pagesize, int weighted)
{
    clear_error();
    if (!prefix || !csr || !csr->idx) return set_error(SCAPH_EINVAL, "null argument");
    std::vector<scaph_page_info> pages;
    int rc = cut_pages(csr, pagesize, weighted, pages);
    if (rc) return rc;
    std::string p(prefix);
    std::unique_ptr<uint32_t[]> buf(new (std::nothrow) uint32_t[pagesize]);
    if (!buf) return set_error(SCAPH_ENOMEM, "page buffer");
    for (size_t i = 0; i < pages.size(); i++) {
        memset(buf.get(), 0, (size_t)pagesize * 4);
        fill_page(csr, pages[i], weighted, buf.get());
        if ((rc = write_file(p + "page" + std::to_string(i), buf.get(), (size_t)pagesize * 4))) return rc;
    }
    if ((rc = write_file(p + "page.info", pages.data(), pages.size() * sizeof(scaph_page_info)))) return rc;
    struct { uint32_t pagesize, nodenum; uint64_t edgenum; } gi = {pagesize, csr->V, csr->E};
    return write_file(p + "graph.info", &gi, sizeof(gi));
}

// Streaming writer: the flat CSR files are read page by page (the offsets
// whole, the edges one page's range at a time with pread), so the edge
// arrays are never held in memory; the page cut and page contents are the
// ones scaph_pages_write (and tools/pagegencsr.cpp:197-252) produce.
int scaph_pages_write_stream(const char *csr_prefix, const char *out_prefix, uint32_t pagesize, int weighted,
                             int flags, uint32_t *pagesize_out)
{
    clear_error();
    if (!csr_prefix || !out_prefix) return set_error(SCAPH_EINVAL, "null argument");
    if (flags & ~SCAPH_PAGES_GROW) return set_error(SCAPH_EINVAL, "unknown flags 0x%x", flags);
    const std::string in(csr_prefix), outp(out_prefix);
    const long long isz = file_size(in + "_csr.idx"), nsz = file_size(in + "_csr.ngh");
    if (isz < 8 || isz % 4 || nsz < 0 || nsz % 4) return set_error(SCAPH_EIO, "%s_csr.idx/.ngh missing or malformed", csr_prefix);
    const uint64_t V = (uint64_t)isz / 4 - 1;
    if (V == 0 || V > 0xFFFFFFFEull) return set_error(SCAPH_EFORMAT, "%s_csr.idx: bad vertex count", csr_prefix);
    std::vector<uint64_t> idx(V + 1);
    {
        std::vector<uint32_t> i32(V + 1);
        int rc = read_file(in + "_csr.idx", i32.data(), (size_t)isz);
        if (rc) return rc;
        for (uint64_t v = 0; v <= V; v++) idx[v] = i32[v];
    }
    const uint64_t E = (uint64_t)nsz / 4;
    for (uint64_t v = 0; v < V; v++)
        if (idx[v + 1] < idx[v]) return set_error(SCAPH_EFORMAT, "%s_csr.idx not monotone at %llu", csr_prefix,
                                                  (unsigned long long)v);
    if (idx[0] != 0 || idx[V] != E) return set_error(SCAPH_EFORMAT, "%s_csr.idx does not span _csr.ngh", csr_prefix);
    const uint64_t ew = weighted ? 2 : 1;
    if (weighted && file_size(in + "_csr.wgh") != (long long)(4 * E))
        return set_error(SCAPH_EIO, "%s_csr.wgh missing or short", csr_prefix);
    if (flags & SCAPH_PAGES_GROW) {
        // the page grows to hold the longest list: 3 + deg*ew < pagesize
        uint64_t maxdeg = 0;
        for (uint64_t v = 0; v < V; v++) maxdeg = std::max<uint64_t>(maxdeg, idx[v + 1] - idx[v]);
        const uint64_t need = (3 + maxdeg * ew + 1 + 3) & ~3ull;
        if (need > 0xFFFFFFF0ull) return set_error(SCAPH_EUNSUPPORTED, "a list of %llu edges", (unsigned long long)maxdeg);
        if (need > pagesize) pagesize = (uint32_t)need;
    }
    scaph_csr view{};
    view.V = (uint32_t)V;
    view.E = E;
    view.idx = idx.data();
    std::vector<scaph_page_info> pages;
    int rc = cut_pages(&view, pagesize, weighted, pages);
    if (rc) return rc;
    FILE *fn = fopen((in + "_csr.ngh").c_str(), "rb");
    FILE *fw = weighted ? fopen((in + "_csr.wgh").c_str(), "rb") : nullptr;
    if (!fn || (weighted && !fw)) {
        if (fn) fclose(fn);
        if (fw) fclose(fw);
        return set_error(SCAPH_EIO, "cannot open %s_csr.ngh/.wgh", csr_prefix);
    }
    std::unique_ptr<uint32_t[]> buf(new (std::nothrow) uint32_t[pagesize]), eb(new (std::nothrow) uint32_t[pagesize]),
        wb(new (std::nothrow) uint32_t[weighted ? pagesize : 1]);
    if (!buf || !eb || !wb) rc = set_error(SCAPH_ENOMEM, "page buffers");
    for (size_t i = 0; !rc && i < pages.size(); i++) {
        const scaph_page_info &pi = pages[i];
        const uint64_t base = idx[pi.left];
        memset(buf.get(), 0, (size_t)pagesize * 4);
        for (uint32_t v = pi.left; v <= pi.right; v++) {
            const size_t k = (size_t)(v - pi.left) * 3;
            buf[k + 0] = v;
            buf[k + 1] = (uint32_t)(idx[v] - base);
            buf[k + 2] = (uint32_t)(idx[v + 1] - idx[v]);
        }
        const size_t n = pi.edgenum;
        if (n && (fseeko(fn, (off_t)(base * 4), SEEK_SET) != 0 || fread(eb.get(), 4, n, fn) != n)) {
            rc = set_error(SCAPH_EIO, "%s_csr.ngh: short read", csr_prefix);
            break;
        }
        if (n && weighted && (fseeko(fw, (off_t)(base * 4), SEEK_SET) != 0 || fread(wb.get(), 4, n, fw) != n)) {
            rc = set_error(SCAPH_EIO, "%s_csr.wgh: short read", csr_prefix);
            break;
        }
        uint32_t *edges = buf.get() + (size_t)pi.nodenum * 3;
        for (size_t e = 0; e < n; e++) {
            if (eb[e] >= V) {
                rc = set_error(SCAPH_EFORMAT, "%s_csr.ngh: neighbour %u out of range", csr_prefix, eb[e]);
                break;
            }
            edges[e * ew] = eb[e];
            if (weighted) edges[e * ew + 1] = wb[e];
        }
        if (!rc) rc = write_file(outp + "page" + std::to_string(i), buf.get(), (size_t)pagesize * 4);
    }
    fclose(fn);
    if (fw) fclose(fw);
    if (rc) return rc;
    if ((rc = write_file(outp + "page.info", pages.data(), pages.size() * sizeof(scaph_page_info)))) return rc;
    struct { uint32_t pagesize, nodenum; uint64_t edgenum; } gi = {pagesize, (uint32_t)V, E};
    if ((rc = write_file(outp + "graph.info", &gi, sizeof(gi)))) return rc;
    if (pagesize_out) *pagesize_out = pagesize;
    return SCAPH_OK;
}

// Validates page records against the Node triples (the reference trusts
// them blindly; a corrupt file here is an error, not undefined behaviour).
static int check_pages(Graph &g)
{
    uint32_t expect_left = 0;
    uint64_t edges = 0;
    const uint64_t ew = g.weighted ? 2 : 1;
    g.degree.assign(g.V, 0);
    for (size_t p = 0; p < g.pages.size(); p++) {
        const scaph_page_info &pi = g.pages[p];
        if (pi.left != expect_left || pi.right < pi.left || pi.right >= g.V ||
            pi.nodenum != pi.right - pi.left + 1 ||
            3ull * pi.nodenum + ew * pi.edgenum > g.pagesize)
            return set_error(SCAPH_EFORMAT, "page %zu: bad descriptor", p);
        const uint32_t *node = g.page((int)p);
        uint64_t pos = 0;
        for (uint32_t k = 0; k < pi.nodenum; k++) {
            if (node[3 * k] != pi.left + k || node[3 * k + 1] != pos)
                return set_error(SCAPH_EFORMAT, "page %zu node %u: bad record", p, k);
            pos += node[3 * k + 2];
            g.degree[pi.left + k] = node[3 * k + 2];
        }
        if (pos != pi.edgenum) return set_error(SCAPH_EFORMAT, "page %zu: edge count mismatch", p);
        const uint32_t *e = node + 3 * (size_t)pi.nodenum;
        for (uint64_t k = 0; k < pi.edgenum; k++)
            if (e[k * ew] >= g.V) return set_error(SCAPH_EFORMAT, "page %zu: neighbour out of range", p);
        edges += pi.edgenum;
        expect_left = pi.right + 1;
    }
    if (expect_left != g.V) return set_error(SCAPH_EFORMAT, "pages do not cover all vertices");
    if (edges != g.E) return set_error(SCAPH_EFORMAT, "page edges %llu != E %llu",
                                       (unsigned long long)edges, (unsigned long long)g.E);
    return SCAPH_OK;
}

int scaph_graph_open(const char *prefix, int weighted, scaph_graph **out)
{
    clear_error();
    if (!prefix || !out) return set_error(SCAPH_EINVAL, "null argument");
    *out = nullptr;
    std::string p(prefix);
    struct { uint32_t pagesize, nodenum; uint64_t edgenum; } gi;
    long long gsz = file_size(p + "graph.info");
    if (gsz != 16) return set_error(SCAPH_EIO, "%sgraph.info missing or not 16 bytes", prefix);
    int rc;
    if ((rc = read_file(p + "graph.info", &gi, 16))) return rc;
    long long psz = file_size(p + "page.info");
    if (psz <= 0 || psz % 16) return set_error(SCAPH_EIO, "%spage.info missing or malformed", prefix);
    std::unique_ptr<scaph_graph> g(new scaph_graph());
    g->pagesize = gi.pagesize;
    g->V = gi.nodenum;
    g->E = gi.edgenum;
    g->weighted = weighted ? 1 : 0;
    g->pages.resize((size_t)(psz / 16));
    if ((rc = read_file(p + "page.info", g->pages.data(), (size_t)psz))) return rc;
    if (g->pagesize < 8 || g->pagesize % 4) return set_error(SCAPH_EFORMAT, "pagesize %u not a multiple of 4", g->pagesize);
    g->data_words = g->pages.size() * (size_t)g->pagesize;
    g->data = alloc_words(g->data_words);
    if (!g->data) return set_error(SCAPH_ENOMEM, "host pages (%zu MiB)", g->data_words >> 18);
    for (size_t i = 0; i < g->pages.size(); i++) {
        std::string f = p + "page" + std::to_string(i);
        if (file_size(f) != (long long)g->pagesize * 4) return set_error(SCAPH_EIO, "%s: wrong size", f.c_str());
        if ((rc = read_file(f, g->page((int)i), (size_t)g->pagesize * 4))) return rc;
    }
    if ((rc = check_pages(*g))) return rc;
    *out = g.release();
    return SCAPH_OK;
}

int scaph_graph_from_csr(const scaph_csr *csr, uint32_t pagesize, int weighted, scaph_graph **out)
{
    clear_error();
    if (!csr || !out || !csr->idx) return set_error(SCAPH_EINVAL, "null argument");
    *out = nullptr;
    if (pagesize % 4) return set_error(SCAPH_EINVAL, "pagesize must be a multiple of 4 words");
    std::unique_ptr<scaph_graph> g(new scaph_graph());
    int rc = cut_pages(csr, pagesize, weighted, g->pages);
    if (rc) return rc;
    g->pagesize = pagesize;
    g->V = csr->V;
    g->E = csr->E;
    g->weighted = weighted ? 1 : 0;
    g->data_words = g->pages.size() * (size_t)pagesize;
    g->data = alloc_words(g->data_words);
    if (!g->data) return set_error(SCAPH_ENOMEM, "host pages (%zu MiB)", g->data_words >> 18);
    const int np = (int)g->pages.size();
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < np; i++) fill_page(csr, g->pages[i], weighted, g->page(i));
    g->degree.resize(csr->V);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)csr->V; v++) g->degree[v] = (uint32_t)(csr->idx[v + 1] - csr->idx[v]);
    *out = g.release();
    return SCAPH_OK;
}

int scaph_graph_get_info(const scaph_graph *g, scaph_graph_info *info)
{
    if (!g || !info) return set_error(SCAPH_EINVAL, "null argument");
    info->pagesize = g->pagesize;
    info->V = g->V;
    info->E = g->E;
    info->npages = (int32_t)g->pages.size();
    info->weighted = g->weighted;
    return SCAPH_OK;
}

const uint32_t *scaph_graph_page(const scaph_graph *g, int p)
{
    if (!g || p < 0 || p >= (int)g->pages.size()) return nullptr;
    return g->page(p);
}

const scaph_page_info *scaph_graph_page_list(const scaph_graph *g) { return g ? g->pages.data() : nullptr; }
const uint32_t *scaph_graph_degree(const scaph_graph *g) { return g ? g->degree.data() : nullptr; }
void scaph_graph_close(scaph_graph *g) { delete g; }

int scaph_graph_to_csr(const scaph_graph *g, scaph_csr *out)
{
    clear_error();
    if (!g || !out) return set_error(SCAPH_EINVAL, "null argument");
    memset(out, 0, sizeof(*out));
    const uint32_t V = g->V;
    const uint64_t E = g->E;
    out->V = V;
    out->E = E;
    out->idx = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    out->ngh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, E));
    if (g->weighted) out->wgh = (uint32_t *)malloc(sizeof(uint32_t) * std::max<uint64_t>(1, E));
    if (!out->idx || !out->ngh || (g->weighted && !out->wgh)) {
        scaph_csr_free(out);
        return set_error(SCAPH_ENOMEM, "csr allocation");
    }
    out->idx[0] = 0;
    for (uint32_t v = 0; v < V; v++) out->idx[v + 1] = out->idx[v] + g->degree[v];
    if (out->idx[V] != E) {
        scaph_csr_free(out);
        return set_error(SCAPH_EFORMAT, "page degrees sum to %llu, graph.info says %llu",
                         (unsigned long long)out->idx[V], (unsigned long long)E);
    }
    const uint32_t ew = g->weighted ? 2 : 1;
    const int np = (int)g->pages.size();
    #pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < np; p++) {
        const scaph_page_info &pi = g->pages[p];
        const uint32_t *pg = g->page(p);
        const uint32_t *edges = pg + 3ull * pi.nodenum;
        for (uint32_t i = 0; i < pi.nodenum; i++) {
            const uint32_t v = pg[3 * i], idx = pg[3 * i + 1], len = pg[3 * i + 2];
            const uint64_t at = out->idx[v];
            for (uint32_t k = 0; k < len; k++) {
                out->ngh[at + k] = edges[(uint64_t)(idx + k) * ew];
                if (ew == 2) out->wgh[at + k] = edges[(uint64_t)(idx + k) * 2 + 1];
            }
        }
    }
    return SCAPH_OK;
}

int scaph_csr_symmetric(const scaph_csr *csr)
{
    clear_error();
    if (!csr || !csr->idx) return set_error(SCAPH_EINVAL, "null argument");
    scaph_csr t;
    int rc = scaph_csr_transpose(csr, &t);
    if (rc) return rc;
    int sym = 1;
    for (uint32_t v = 0; v <= csr->V && sym; v++)
        if (t.idx[v] != csr->idx[v]) sym = 0;
    if (sym) {
        // in-lists come out sorted: compare with each out-list sorted
        #pragma omp parallel for schedule(dynamic, 1024) reduction(& : sym)
        for (int64_t v = 0; v < (int64_t)csr->V; v++) {
            const uint64_t b = csr->idx[v], e = csr->idx[v + 1];
            std::vector<uint32_t> a(csr->ngh + b, csr->ngh + e);
            std::sort(a.begin(), a.end());
            if (!std::equal(a.begin(), a.end(), t.ngh + b)) sym = 0;
        }
    }
    scaph_csr_free(&t);
    return sym;
}

}  // extern "C""
