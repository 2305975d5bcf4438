// Device-side layout of the paged graph and of the BFS state, shared by the
// level kernels (bfs_kernels.cu) and the engine (engine.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace scaph {

constexpr uint32_t kPullHead = 4;  // dense in-edge row per vertex read by pull phase A
constexpr unsigned long long kNotResident = ~0ull;
constexpr uint32_t kNoParent = 0xFFFFFFFFu;
constexpr int kHistCap = 512;           // pages histogrammed in shared memory
constexpr int kLutPages = 512;          // page-table entries staged in shared memory
constexpr int kLutCoarse = 1024;        // coarse-index entries staged in shared memory
constexpr uint32_t kGiantEdges = 1024;  // push: adjacency longer than this is split (default)
constexpr int kMaxLevels = 4096;        // hard cap on BFS levels per run

// One page of the device page table.  `base` is the word offset of the page's
// Node array inside the page pool (kNotResident when the page is on the host);
// edges start at base + 3*nodenum (page layout of tools/pagegencsr.cpp:221-242).
struct __align__(16) PageDev {
    unsigned long long base;
    uint32_t left;
    uint32_t nodenum;
};

// Device view of one paged graph (out-edges, or in-edges for pull).
struct GraphDev {
    const uint32_t *pool;           // page pool, 16-byte aligned, slots of pagesize words
    const PageDev *pages;           // npages + 1 entries; pages[npages].left == V
    const uint32_t *coarse;         // coarse[i] = page holding vertex i << cshift
    const uint32_t *zc_pool;        // host pages mapped for zero-copy reads (or null)
    unsigned long long pool_words;  // words addressable through `pool`
    uint32_t cshift;
    uint32_t npages;
    uint32_t V;
    uint32_t pagesize;
};

// Counters of one level, written by that level's kernels.
struct LevelCounters {
    unsigned long long next;        // vertices discovered
    unsigned long long next_edges;  // their out-degree sum
    unsigned long long inspected;   // adjacency entries examined (first-hit for pull)
    unsigned long long headers;     // Node records read
    unsigned int giant;             // giant chunks queued (push)
    unsigned int error;             // nonzero: a kernel saw a bad index / overflow
    unsigned long long zc_words;    // words read zero-copy from host pages
    int dir;                        // direction the level ran (graph mode)
    unsigned int deferred;          // 1: a deferred-claim push (k_push_finalize ran)
    unsigned long long t_end;       // %globaltimer when the level was decided (graph mode)
};

struct GiantChunk {
    unsigned long long start;  // first edge word (pool offset)
    uint32_t len;
    uint32_t src;
};

struct BfsDev {
    uint32_t *depth;
    uint32_t *parent;          // may be null
    uint32_t *visited;         // bitmap, V bits
    const uint32_t *front;     // frontier bitmap of this level
    uint32_t *next;            // frontier bitmap of the next level (pre-cleared)
    const uint32_t *degree;    // out-degree per vertex
    LevelCounters *ctr;        // counters of this level
    uint32_t *page_nodes;      // histogram of the next frontier by page (or null)
    uint32_t *page_datas;
    GiantChunk *giant;
    uint32_t giant_cap;
    uint32_t level;            // discovered vertices get depth level+1
    uint32_t V;
    uint32_t nwords;           // (V + 31) / 32
    GraphDev hg;               // out-edge graph whose pages the histogram counts
    // pull: kPullHead in-edges of every vertex (the first ones, or the ones
    // of largest out-degree), kPullHead words per vertex (16-byte aligned
    // rows, 0xFFFFFFFF past the in-degree), and the in-degrees; null when
    // the caller keeps no such copy
    const uint32_t *head;
    const uint32_t *indeg;
    uint32_t head_ranked;      // head rows are not the list's first edges:
                               // phase B scans the whole list
    // pull: one 8-byte record per vertex read first by phase A (null: phase
    // A reads the in-degree and head row directly): x = the top-ranked
    // in-neighbour (head row entry 0), y = pull_meta(in-degree, out-degree)
    const uint2 *prec;
    // pull: one 16-byte row per vertex read by phase A on levels without the
    // 8-byte records (null: the in-degree, head row and out-degree arrays):
    // x, y, z = the three top-ranked in-neighbours (0xFFFFFFFF past the
    // in-degree), w = pull_meta(in-degree, out-degree)
    const uint4 *prow;
    // pull, CTA tiles on levels without records: the in-degree, out-degree
    // and head row of the live vertices (in-degree > 0) only, in vertex
    // order, so that a 32-byte sector holds no vertex without edges;
    // live_rank[w] = live vertices in the words before w, dead = the bitmap
    // of the others (null: phase A reads the V-entry arrays)
    const uint32_t *live_rank;
    const uint32_t *dead;
    const uint4 *live_head;
    const uint32_t *live_indeg;
    const uint32_t *live_deg;
    const uint2 *live_prec;    // the 8-byte records of the live vertices (read where prec is set)
    // histogram of the discovered vertices over the IN-edge graph's pages
    // (count, sum(indeg+3)): keeps the pull-side page counts current without
    // a pass over all vertices (directed graphs; null when not wanted)
    uint32_t *page_nodes_in;
    uint32_t *page_datas_in;
    GraphDev hgi;
    uint32_t pull_gather;      // sparse pull level: 1 gather several tiles per queue, 2 one run of words per CTA
    uint32_t giant_edges;      // push: adjacency longer than this becomes chunks (0: kGiantEdges)
    // push: 1 = the level defers its claims: the neighbours' bits are OR-ed
    // into `next` (no per-edge atomic round trip, no scattered depth write)
    // and k_push_finalize then writes depths and counters word by word
    uint32_t push_defer;
    uint32_t pull_warp;        // pull: 1 warp-centric chunks, 2 vertex-parallel words (needs prec)
    // push: 1 = sparse level: each CTA reads one contiguous run of frontier
    // words at once and expands all its vertices together, instead of one
    // 128-word tile after another (whole-graph ranges only)
    uint32_t push_sparse;
    uint32_t _pad;
};

// Defaults of scaph_config.alpha and beta (Beamer's switch: push -> pull
// when the frontier's out-edges exceed the unvisited edges / alpha, pull ->
// push when the frontier shrinks below V / beta).  beta = 96 rather than
// Beamer's 24: on RMAT-24 the level after the big pull level then pulls too
// (31 us instead of 45 us pushed) and the tail push levels start smaller
// (alternating A/B on one box: 611 -> 624 GTEPS).
constexpr float kAlphaDefault = 14.0f;
constexpr float kBetaDefault = 96.0f;

// Default of scaph_config.push_defer_edges: push levels whose frontier has
// at least 2^20 out-edges defer their claims (RMAT-24, 8 sources, graph
// mode: 508 -> 521 GTEPS alone, 537 with the warp-centric pull).
constexpr long long kDeferEdgesDefault = 1ll << 20;

// Second word of a pull record: the in-degree capped at 15 in the top four
// bits (phase A needs to know only whether it exceeds the probes already
// made), the out-degree below them; an out-degree of kPrecDegMax or more is
// stored as kPrecDegMax and read from the degree array instead.
constexpr uint32_t kPrecDegMax = (1u << 28) - 1;
__host__ __device__ inline uint32_t pull_meta(uint32_t indeg, uint32_t outdeg)
{
    return ((indeg < 15u ? indeg : 15u) << 28) | (outdeg < kPrecDegMax ? outdeg : kPrecDegMax);
}

// A pull level gathers the vertices of several tiles into one queue when the
// unvisited vertices are this sparse (fewer than one per kPullGatherRatio;
// scaph_config.pull_gather_ratio overrides it).
constexpr unsigned long long kPullGatherRatio = 64;

// A push level reads its frontier words as one contiguous run per CTA when
// the frontier has fewer than one vertex per kPushSparseRatio
// (scaph_config.push_sparse_ratio overrides it; negative: never).
constexpr unsigned long long kPushSparseRatio = 16;
__host__ __device__ inline bool push_use_sparse(long long ratio, unsigned long long nf, unsigned long long V)
{
    return ratio > 0 && nf * (unsigned long long)ratio < V;
}

// Graph mode: state of one traversal kept on the device, so a whole BFS runs
// as one CUDA-graph launch with the level loop in a conditional WHILE node.
struct BfsCtl {
    uint32_t *depth;
    uint32_t *parent;
    uint32_t src;
    uint32_t level;            // level being run
    int32_t dir;               // 0 push, 1 pull
    int32_t done;
    uint32_t pull_gather;      // the level is a sparse pull (BfsDev::pull_gather)
    uint32_t push_defer;       // the level is a deferred-claim push (BfsDev::push_defer)
    uint32_t pull_rec;         // the level's pull reads the 8-byte records (BfsDev::prec)
    uint32_t push_sparse;      // the level is a sparse push (BfsDev::push_sparse)
    unsigned long long nf, prev_nf, mf, vis_n, vis_e;
    unsigned long long t_start;
};

// Static inputs of the graph-mode level kernels.
struct BfsGraphArgs {
    BfsDev base;               // depth/parent/front/next/ctr/level filled per level
    uint32_t *bm3;             // three rotating frontier bitmaps, nwords each
    LevelCounters *ctr0;       // counters of level 0 (level L at ctr0 + L)
    uint32_t *hist0;           // histograms: level L at hist0 + L*2*npages_h (or null)
    uint32_t hist_levels;
    uint32_t npages_h;
    BfsCtl *ctl;
};

// The scheduler network as the decide kernel reads it (weights already
// rounded to bf16): W1[in][64] b1[64] W2[64][64] b2[64] W3[64][out] b3[out].
struct MlpDev {
    const float *w;
    int in, out;
    unsigned long long off_w1, off_b1, off_w2, off_b2, off_w3, off_b3;
};

struct DecideArgs {
    unsigned long long E;           // out-edges (for m_u)
    unsigned long long dead_edges;  // out-edges of vertices no edge reaches
    unsigned long long dead;        // vertices no edge reaches
    const uint32_t *dead_bm;        // their bitmap
    uint32_t V;
    uint32_t unreached;
    int32_t mode;                   // SCAPH_DIR_*
    float alpha, beta;
    int32_t max_levels;
    uint32_t gather_ratio;          // pull levels gather tiles below 1 unvisited per this many
    unsigned long long defer_edges; // push levels with this many frontier edges defer claims (0 never)
    int32_t pull_records;           // scaph_config.pull_records
    int32_t push_sparse_ratio;      // push levels below 1 frontier vertex per this many are sparse (<= 0 never)
    uint32_t pull_gather_mode;      // BfsDev::pull_gather of a sparse pull level (1 tiles, 2 runs)
};

// Whether a pull level reads the 8-byte records (scaph_config.pull_records):
// where the frontier is small next to the unvisited set, the top-ranked
// in-neighbour misses often and the record's second round trip (head row)
// costs more than reading everything at once.
__host__ __device__ inline bool pull_use_records(int mode, unsigned long long nf, unsigned long long unvisited)
{
    return mode == 1 || (mode == 0 && 4 * nf >= unvisited);
}

// Beamer's direction-optimizing rule (SC'12): leave top-down when the
// frontier's out-edges exceed the unexplored edges / alpha; leave bottom-up
// when the frontier is below V / beta and shrinking.  0 = push, 1 = pull.
__host__ __device__ inline int alpha_beta_next(int cur_dir, unsigned long long nf, unsigned long long prev_nf,
                                               unsigned long long mf, unsigned long long mu, unsigned long long V,
                                               float alpha, float beta)
{
    if (cur_dir == 0) return (double)mf > (double)mu / alpha ? 1 : 0;
    return ((double)nf < (double)V / beta && nf < prev_nf) ? 0 : 1;
}

// The learned direction is taken only near the alpha/beta switch point:
// where the rule's own ratio is more than kLearnedBand times past (or short
// of) its threshold, the rule decides.  From push (cur_dir 0) the ratio is
// mf / (mu / alpha), from pull it is nf / (V / beta).  Returns the rule's
// direction when it is that clear, -1 when the network decides.
constexpr float kLearnedBand = 4.f;
__host__ __device__ inline int alpha_beta_confident(int cur_dir, unsigned long long nf, unsigned long long mf,
                                                    unsigned long long mu, unsigned long long V, float alpha,
                                                    float beta)
{
    if (cur_dir == 0) {
        const double r = (double)mf * alpha / (double)(mu ? mu : 1);
        if (r > kLearnedBand) return 1;
        if (r * kLearnedBand < 1.0) return 0;
        return -1;
    }
    const double r = (double)nf * beta / (double)(V ? V : 1);
    if (r > kLearnedBand) return 1;
    if (r * kLearnedBand < 1.0) return 0;
    return -1;
}

// Page lookup (page table + coarse index), in global or shared memory.
struct PageLut {
    const PageDev *pages;
    const uint32_t *coarse;
    uint32_t cshift;
    __device__ __forceinline__ int of(uint32_t v) const
    {
        int p = (int)coarse[v >> cshift];
        while (pages[p + 1].left <= v) ++p;
        return p;
    }
};

__device__ __forceinline__ int page_of(const GraphDev &g, uint32_t v)
{
    int p = (int)__ldg(&g.coarse[v >> g.cshift]);
    while (__ldg(&g.pages[p + 1].left) <= v) ++p;
    return p;
}

__device__ __forceinline__ uint4 ld_nc_v4(const uint32_t *p)
{
    return __ldg(reinterpret_cast<const uint4 *>(p));
}

__device__ __forceinline__ uint2 ld_nc_v2(const uint2 *p) { return __ldg(p); }

__device__ __forceinline__ uint32_t test_bit(const uint32_t *bm, uint32_t v)
{
    return (__ldg(&bm[v >> 5]) >> (v & 31)) & 1u;
}

// Several vertex ranges processed by one launch (out-of-core page batches).
// Tiles of 128 bitmap words are numbered across the ranges: range i owns
// tiles [tile0[i], tile0[i+1]).  n == 0 means the single range (vlo, vhi)
// passed to the kernel directly.
struct RangeList {
    const uint32_t *lo;
    const uint32_t *hi;
    const uint32_t *tile0;  // n + 1 entries
    uint32_t n;
};

// Maps a global tile number to its range and local tile number.
__device__ __forceinline__ void range_of_tile(const RangeList &rl, uint32_t tile, uint32_t &rlo, uint32_t &rhi,
                                              uint32_t &local)
{
    if (rl.n == 0) {
        local = tile;
        return;  // rlo/rhi already hold the single range
    }
    uint32_t lo = 0, hi = rl.n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (rl.tile0[mid] <= tile) lo = mid; else hi = mid - 1;
    }
    rlo = rl.lo[lo];
    rhi = rl.hi[lo];
    local = tile - rl.tile0[lo];
}

// Mask of the vertices of word w that lie in [vlo, vhi).
__device__ __forceinline__ uint32_t range_mask(uint32_t w, uint32_t vlo, uint32_t vhi)
{
    unsigned long long b0 = (unsigned long long)w << 5;
    unsigned long long lo = vlo > b0 ? vlo - b0 : 0;
    unsigned long long hi = vhi < b0 + 32 ? vhi - b0 : 32;
    if (hi <= lo) return 0u;
    uint32_t m = hi >= 32 ? 0xFFFFFFFFu : ((1u << hi) - 1u);
    return m & (0xFFFFFFFFu << lo);
}

}  // namespace scaph
