// Internal helpers shared by the host sources of libscaph.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "scaph/scaph.h"

namespace scaph {

// Records the message returned by scaph_last_error() and returns `code`.
int set_error(int code, const char *fmt, ...);
void clear_error();

// Host-side fault injection (scaph_fault_inject): the call sites below ask
// injected_fault() before their CUDA call; while an injection is armed for
// the site, the call is not made and the site's CUDA error is returned
// instead, as if the runtime had failed.
enum FaultSite { kFaultPinnedAlloc = 0, kFaultHostRegister, kFaultPageCopy, kFaultDeviceAlloc, kFaultSites };
// cudaSuccess (no injection) or the error to report for this call.
int injected_fault(FaultSite site);

// Splitmix64 finaliser: a counter-based hash, so that generated graphs do not
// depend on the number of threads used.
static inline uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
static inline double unit_double(uint64_t h) { return (h >> 11) * (1.0 / 9007199254740992.0); }

// Host side of a paged graph: pages are kept as one contiguous,
// 4 KiB-aligned buffer of npages * pagesize words so that it can be pinned
// with one cudaHostRegister call.
struct Graph {
    uint32_t pagesize = 0;      // words per page
    uint32_t V = 0;
    uint64_t E = 0;
    int weighted = 0;
    std::vector<scaph_page_info> pages;
    std::vector<uint32_t> degree;  // from Node.len
    uint32_t *data = nullptr;      // npages * pagesize words
    size_t data_words = 0;
    bool pinned = false;           // registered with cudaHostRegister
    ~Graph();
    const uint32_t *page(int p) const { return data + (size_t)p * pagesize; }
    uint32_t *page(int p) { return data + (size_t)p * pagesize; }
};

// Page cut of tools/pagegencsr.cpp:106-163,204-247: from `left`, the largest
// `right` such that 3*(right-left+1) + edges*(weighted?2:1) < pagesize.
// Returns false if the single vertex `left` does not fit.
bool page_cut(const uint64_t *idx, uint32_t V, uint32_t left, uint32_t pagesize,
              int weighted, uint32_t *right);

// Rows of `width` adjacency entries of every vertex of a paged graph
// (out[v*width + j], 0xFFFFFFFF past the vertex's degree): the first ones,
// or, with rank != null, the ones with the largest rank[] (ties: list order).
void adjacency_heads(const Graph &g, uint32_t width, uint32_t *out, const uint32_t *rank = nullptr);

uint32_t *alloc_words(size_t words);  // zeroed, 4 KiB aligned
void free_words(uint32_t *p);

}  // namespace scaph

// The opaque handle of the C ABI is the host graph itself.
struct scaph_graph : public scaph::Graph {};
