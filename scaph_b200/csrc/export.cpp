// Text exports of a flat CSR for cross-framework checks, byte-identical to
// the reference's converters:
//   Ligra adjacency      <p>.ligra          tools/bin2ligra.cpp:66-108
//   Ligra weighted       <p>.ligra.weight   tools/bin2ligraweight.cpp:66-120
//   Totem edge list      <p>.totem          tools/bin2totem.cpp:66-110
//   Totem weighted       <p>weight.totem    tools/bin2totemweight.cpp:66-117
// The inputs are read as those tools read them: V from the size of
// <p>_csr.deg, E from the size of <p>_csr.ngh, V+1 offsets of <p>_csr.idx,
// and E weights of <p>_csr.wgh for the weighted kinds (32-bit words, the
// tools' default build).  The tools append one std::to_string per number to
// a single string; here the threads format disjoint ranges of vertices or
// edges into their own buffers with a direct integer formatter, and the
// buffers are written in order.
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"
#include "scaph/scaph.h"

using scaph::clear_error;
using scaph::set_error;

namespace {

// Appends the decimal digits of x and one terminator byte.
inline void put_u64(std::string &b, unsigned long long x, char term)
{
    char tmp[24];
    int n = 0;
    do {
        tmp[n++] = (char)('0' + x % 10);
        x /= 10;
    } while (x);
    while (n) b.push_back(tmp[--n]);
    b.push_back(term);
}

long long fsize(const std::string &path)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    const long long n = ftell(f);
    fclose(f);
    return n;
}

int read_words(const std::string &path, std::vector<uint32_t> &out, size_t n)
{
    out.resize(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return set_error(SCAPH_EIO, "cannot open %s", path.c_str());
    const size_t got = n ? fread(out.data(), 4, n, f) : 0;
    fclose(f);
    if (got != n) return set_error(SCAPH_EIO, "%s: %zu of %zu words", path.c_str(), got, n);
    return SCAPH_OK;
}

// Formats items [0, n) with fmt(i, buf) in nthreads contiguous ranges whose
// boundaries `bound(t)` the caller picks, and writes the buffers in order.
template <class Bound, class Fmt>
int write_parallel(FILE *f, int nthreads, Bound bound, Fmt fmt)
{
    std::vector<std::string> bufs(nthreads);
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
    for (int t = 0; t < nthreads; t++) {
        const uint64_t lo = bound(t), hi = bound(t + 1);
        std::string &b = bufs[t];
        b.reserve((size_t)(hi - lo) * 8);
        for (uint64_t i = lo; i < hi; i++) fmt(i, b);
    }
    for (const auto &b : bufs)
        if (!b.empty() && fwrite(b.data(), 1, b.size(), f) != b.size()) return set_error(SCAPH_EIO, "short write");
    return SCAPH_OK;
}

}  // namespace

extern "C" int scaph_csr_export(const char *prefix, int kind)
{
    clear_error();
    if (!prefix) return set_error(SCAPH_EINVAL, "null prefix");
    if (kind < SCAPH_EXPORT_LIGRA || kind > SCAPH_EXPORT_TOTEM_WEIGHT)
        return set_error(SCAPH_EINVAL, "unknown export kind %d", kind);
    const bool weighted = kind == SCAPH_EXPORT_LIGRA_WEIGHT || kind == SCAPH_EXPORT_TOTEM_WEIGHT;
    const bool ligra = kind == SCAPH_EXPORT_LIGRA || kind == SCAPH_EXPORT_LIGRA_WEIGHT;
    const std::string p(prefix);
    const long long ngh_bytes = fsize(p + "_csr.ngh"), deg_bytes = fsize(p + "_csr.deg");
    if (ngh_bytes < 0 || deg_bytes < 0 || ngh_bytes % 4 || deg_bytes % 4)
        return set_error(SCAPH_EIO, "missing or malformed %s_csr.ngh/.deg", prefix);
    const uint64_t E = (uint64_t)ngh_bytes / 4, V = (uint64_t)deg_bytes / 4;
    if (V >= (1ull << 31)) return set_error(SCAPH_EUNSUPPORTED, "V >= 2^31");
    std::vector<uint32_t> idx, ngh, wgh;
    int rc;
    if ((rc = read_words(p + "_csr.idx", idx, V + 1))) return rc;
    if ((rc = read_words(p + "_csr.ngh", ngh, E))) return rc;
    if (weighted && (rc = read_words(p + "_csr.wgh", wgh, E))) return rc;
    for (uint64_t v = 0; v < V; v++)
        if (idx[v + 1] < idx[v] || idx[v + 1] > E)
            return set_error(SCAPH_EFORMAT, "%s_csr.idx not monotone within E at %llu", prefix,
                             (unsigned long long)v);

    const std::string out = p + (kind == SCAPH_EXPORT_LIGRA          ? ".ligra"
                                 : kind == SCAPH_EXPORT_LIGRA_WEIGHT ? ".ligra.weight"
                                 : kind == SCAPH_EXPORT_TOTEM        ? ".totem"
                                                                     : "weight.totem");
    FILE *f = fopen(out.c_str(), "wb");
    if (!f) return set_error(SCAPH_EIO, "cannot create %s", out.c_str());
    const int nt = std::max(1, omp_get_max_threads());
    std::string head;
    if (ligra) {
        head = weighted ? "WeightedAdjacencyGraph\n" : "AdjacencyGraph\n";
        put_u64(head, V, '\n');
        put_u64(head, E, '\n');
    } else {
        head = "#Nodes: ";
        put_u64(head, V, '\n');
        head += "#Edges: ";
        put_u64(head, E, '\n');
        head += "#Undirected\n";
    }
    rc = fwrite(head.data(), 1, head.size(), f) == head.size() ? SCAPH_OK : set_error(SCAPH_EIO, "short write");
    auto even = [nt](uint64_t n) { return [n, nt](int t) { return n * (uint64_t)t / (uint64_t)nt; }; };
    if (!rc && ligra) {
        // offsets of vertices 0..V-1, then the neighbours, then the weights
        rc = write_parallel(f, nt, even(V), [&](uint64_t i, std::string &b) { put_u64(b, idx[i], '\n'); });
        if (!rc) rc = write_parallel(f, nt, even(E), [&](uint64_t i, std::string &b) { put_u64(b, ngh[i], '\n'); });
        if (!rc && weighted)
            rc = write_parallel(f, nt, even(E), [&](uint64_t i, std::string &b) { put_u64(b, wgh[i], '\n'); });
    } else if (!rc) {
        // one line per edge, "src\tdst[\tweight]"; vertex ranges cut at equal edge counts
        std::vector<uint64_t> cut(nt + 1);
        for (int t = 0; t <= nt; t++) {
            const uint64_t target = (uint64_t)idx[V] * (uint64_t)t / (uint64_t)nt;
            cut[t] = (uint64_t)(std::lower_bound(idx.begin(), idx.begin() + V, (uint32_t)target) - idx.begin());
        }
        cut[0] = 0;
        cut[nt] = V;
        for (int t = 1; t <= nt; t++) cut[t] = std::max(cut[t], cut[t - 1]);
        rc = write_parallel(f, nt, [&](int t) { return cut[t]; }, [&](uint64_t v, std::string &b) {
            for (uint32_t e = idx[v]; e < idx[v + 1]; e++) {
                put_u64(b, v, '\t');
                if (weighted) {
                    put_u64(b, ngh[e], '\t');
                    put_u64(b, wgh[e], '\n');
                } else {
                    put_u64(b, ngh[e], '\n');
                }
            }
        });
    }
    if (fclose(f) != 0 && !rc) rc = set_error(SCAPH_EIO, "closing %s", out.c_str());
    return rc;
}
