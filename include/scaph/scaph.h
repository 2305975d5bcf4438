/*
 * scaph.h - C ABI of the B200 (sm_100a) Scaph BFS engine.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (0 = ok, negative = error, message in scaph_last_error()).  Nothing here
 * exits the process or prints.  The reference engine reports errors with
 * H_ERR -> printf + exit (src/gpu_engine.cuh:28-39) and assert; every entry
 * point below returns a status instead.
 *
 * Each declaration names the reference interface (file:line in the
 * N-E-E/Scaph tree) whose job it takes over.
 */
#ifndef SCAPH_H
#define SCAPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SCAPH_OK           0
#define SCAPH_EINVAL      -1   /* bad argument                                */
#define SCAPH_EIO         -2   /* file missing, short or unwritable           */
#define SCAPH_ENOMEM      -3   /* host or device allocation failed            */
#define SCAPH_ECUDA       -4   /* CUDA runtime error                          */
#define SCAPH_EFORMAT     -5   /* paged-CSR files inconsistent                */
#define SCAPH_ETIMEOUT    -6   /* a bounded device wait gave up               */
#define SCAPH_EUNSUPPORTED -7  /* feature not available for this graph/config */
#define SCAPH_EDEVICE     -8   /* a kernel reported a bad index / overflow    */

/* Message of the last failing call on this thread ("" if none). */
const char *scaph_last_error(void);
/* Test hook with no counterpart in the reference, where a failing CUDA call
 * ends the process (H_ERR -> exit, src/gpu_engine.cuh:28-39).  Arms a host
 * side fault: after `skip` further calls at `site` succeed, the next `count`
 * calls there fail as the CUDA runtime would report it, without calling it,
 * so that tests can check that every entry point returns a status (and
 * leaves nothing half-built) instead of aborting.  Sites:
 *   "pinned_alloc"   cudaMallocHost (scaph_host_alloc, engine staging)
 *   "host_register"  cudaHostRegister of a graph's pages (out-of-core pool)
 *   "page_copy"      a host-to-HBM page copy of the out-of-core pool
 *   "device_alloc"   cudaMalloc of scaph_engine_create's per-vertex state
 * site NULL disarms every site.  SCAPH_EINVAL for an unknown site. */
int scaph_fault_inject(const char *site, int skip, int count);
/* Library version string. */
const char *scaph_version(void);

/* ---- on-disk / in-memory records (byte layouts of the reference) ------- */

/* One page descriptor of <p>page.info.  Same 16-byte layout as
 * `struct Page` (tools/pagegencsr.cpp:74-80, src/page.h:22-28). */
typedef struct scaph_page_info {
    uint32_t left;      /* first vertex of the page                          */
    uint32_t right;     /* last vertex of the page (inclusive)               */
    uint32_t nodenum;   /* right - left + 1                                  */
    uint32_t edgenum;   /* edges stored in the page                          */
} scaph_page_info;

/* <p>graph.info: 16 bytes {u32 pagesize_words, u32 V, u64 E}, as written by
 * save_graph_info (tools/pagegencsr.cpp:82-87,181-195).  (The reference
 * loader reads only the first 12 bytes, src/graph.h:79-86; this one reads
 * all 16.) */
typedef struct scaph_graph_info {
    uint32_t pagesize;  /* words per page file                               */
    uint32_t V;
    uint64_t E;
    int32_t  npages;
    int32_t  weighted;  /* pages hold {ngr,wgh} pairs (src/page.h:39-46)     */
} scaph_graph_info;

/* Flat CSR held by the library (generators, readers).  idx has V+1 64-bit
 * offsets, ngh has E neighbour ids, wgh is NULL or E weights. */
typedef struct scaph_csr {
    uint32_t  V;
    uint64_t  E;
    uint64_t *idx;
    uint32_t *ngh;
    uint32_t *wgh;
} scaph_csr;

/* ---- synthetic graph generators (seeded, deterministic for any thread
 *      count).  Output adjacency lists are sorted and duplicate-free. ----- */

/* RMAT (Chakrabarti et al.) with quadrant probabilities a,b,c (d=1-a-b-c):
 * 2^scale vertices, round(edgefactor*2^scale/2) generated pairs, self-loops
 * and duplicates removed, symmetrised (so E ~ edgefactor*V directed edges).
 * scramble != 0 relabels vertices by a seeded permutation. */
int scaph_gen_rmat(int scale, double edgefactor, double a, double b, double c,
                   uint64_t seed, int scramble, scaph_csr *out);

/* Directed power-law graph: out-degrees Zipf-like with exponent `zipf_s`
 * (capped at max_degree), destinations by preferential attachment
 * (copy model, probability proportional to in-degree + 1).  ~E edges. */
int scaph_gen_powerlaw(uint32_t V, uint64_t E, double zipf_s, uint32_t max_degree,
                       uint64_t seed, scaph_csr *out);

/* Directed web-crawl-like graph: power-law out-degrees (exponent s, capped),
 * a fraction `local_frac` of each vertex's edges inside its block of `block`
 * consecutive ids, the rest uniform over all vertices. */
int scaph_gen_web(uint32_t V, uint64_t E, double s, uint32_t max_degree,
                  uint32_t block, double local_frac, uint64_t seed, scaph_csr *out);

/* Text exports of the flat CSR files <p>_csr.* for cross-framework checks,
 * byte-identical to the reference's converters (inputs read as they read
 * them: V from the size of _csr.deg, E from the size of _csr.ngh):
 *   SCAPH_EXPORT_LIGRA         <p>.ligra         (tools/bin2ligra.cpp:66-108)
 *   SCAPH_EXPORT_LIGRA_WEIGHT  <p>.ligra.weight  (tools/bin2ligraweight.cpp:66-120)
 *   SCAPH_EXPORT_TOTEM         <p>.totem         (tools/bin2totem.cpp:66-110)
 *   SCAPH_EXPORT_TOTEM_WEIGHT  <p>weight.totem   (tools/bin2totemweight.cpp:66-117) */
#define SCAPH_EXPORT_LIGRA         1
#define SCAPH_EXPORT_LIGRA_WEIGHT  2
#define SCAPH_EXPORT_TOTEM         3
#define SCAPH_EXPORT_TOTEM_WEIGHT  4
int scaph_csr_export(const char *prefix, int kind);

/* Reverse every edge (in-edge CSR for pull on directed graphs). */
int scaph_csr_transpose(const scaph_csr *in, scaph_csr *out);
/* Copies caller arrays into a library-owned CSR. */
int scaph_csr_from_arrays(uint32_t V, uint64_t E, const uint64_t *idx,
                          const uint32_t *ngh, const uint32_t *wgh, scaph_csr *out);
void scaph_csr_free(scaph_csr *csr);

/* Flat CSR files <p>_csr.idx (u32[V+1]), _csr.ngh (u32[E]), _csr.deg (u32[V])
 * and _csr.wgh (u32[E]; written as zeros when csr->wgh is NULL because the
 * reference generator always reads it, tools/pagegencsr.cpp:281-287).
 * Same files that fetch_graph reads (src/graph.h:27-75). */
int scaph_csr_write(const char *prefix, const scaph_csr *csr);
int scaph_csr_read(const char *prefix, int with_weights, scaph_csr *out);

/* ---- paged CSR --------------------------------------------------------- */

/* Writes <p>page<N>, <p>page.info and <p>graph.info byte-identical to
 * tools/pagegencsr.cpp (page_gen, :197-252): greedy cut so that
 * 3*nodes + edges (x2 if weighted) < pagesize_words, Node{vtx,idx,len}
 * triples then the edges, zero-padded to pagesize_words.  A vertex whose
 * adjacency alone does not fit a page is rejected (SCAPH_EUNSUPPORTED). */
int scaph_pages_write(const char *prefix, const scaph_csr *csr,
                      uint32_t pagesize_words, int weighted);

/* The same page files written by streaming the flat CSR files
 * <csr_prefix>_csr.idx/.ngh (and .wgh when weighted) - the edge arrays are
 * read one page's range at a time, never held in memory - to <out_prefix>.
 * With SCAPH_PAGES_GROW a list longer than a page makes the page grow:
 * pagesize becomes the smallest multiple of 4 words that holds the longest
 * list (the reference generator and scaph_pages_write reject such a vertex,
 * tools/pagegencsr.cpp:106-163); *pagesize_out (may be NULL) receives the
 * page size written.  Without growth, or when every list fits, the files
 * are byte-identical to scaph_pages_write's. */
#define SCAPH_PAGES_GROW 1
int scaph_pages_write_stream(const char *csr_prefix, const char *out_prefix,
                             uint32_t pagesize_words, int weighted, int flags,
                             uint32_t *pagesize_out);

typedef struct scaph_graph scaph_graph;

/* Loads a paged CSR written by pagegencsr / scaph_pages_write into host
 * memory (replaces fetch_graph, src/graph.h:24-108).  The flat _csr.* files
 * are not needed; degrees come from the page Node records.  `weighted` says
 * whether the pages hold {ngr,wgh} pairs; the reference decides this at
 * compile time (-DAPPSSSP -> WEIGHT, src/graph.h:7-9). */
int scaph_graph_open(const char *prefix, int weighted, scaph_graph **g);
/* Pages a flat CSR in memory with the same cut rule (no files). */
int scaph_graph_from_csr(const scaph_csr *csr, uint32_t pagesize_words,
                         int weighted, scaph_graph **g);
int scaph_graph_get_info(const scaph_graph *g, scaph_graph_info *info);
/* Host view of page p (pagesize words) and of the page list. */
const uint32_t *scaph_graph_page(const scaph_graph *g, int p);
const scaph_page_info *scaph_graph_page_list(const scaph_graph *g);
/* Per-vertex out-degree (u32[V]), the reference's csr_deg / d_degree. */
const uint32_t *scaph_graph_degree(const scaph_graph *g);
void scaph_graph_close(scaph_graph *g);
/* The flat CSR of a paged graph, read back from its pages (the arrays that
 * fetch_graph reads from <p>_csr.idx/.ngh/.wgh, src/graph.h:27-75; wgh only
 * for weighted pages).  Free with scaph_csr_free. */
int scaph_graph_to_csr(const scaph_graph *g, scaph_csr *out);
/* 1 if every edge u->v has its reverse v->u (same multiset of neighbours),
 * 0 if not, < 0 on error. */
int scaph_csr_symmetric(const scaph_csr *csr);

/* ---- engine ------------------------------------------------------------ */

/* Direction policy (the reference has only push: gpu_push_csr,
 * src/gpu_engine.cuh:41-169; gpu_pull_iteration is a stub, src/app.cuh:365-369). */
#define SCAPH_DIR_ALPHABETA 0   /* Beamer alpha/beta switch (plain engine)    */
#define SCAPH_DIR_PUSH      1   /* top-down every level                       */
#define SCAPH_DIR_PULL      2   /* bottom-up every level after the first      */
#define SCAPH_DIR_LEARNED   3   /* MLP scheduler (falls back to alpha/beta)   */

/* Engine configuration; zero-initialise and set what you need
 * (replaces the FLAGS_* globals, src/app.cuh:38-52). */
typedef struct scaph_config {
    int64_t  pool_bytes;       /* HBM page-pool cap; 0 = every page resident
                                  (FLAGS_max_memory, src/app.cuh:39,152)    */
    uint32_t unreached;        /* depth of unreached vertices; 0 = 0xFFFFFFFF
                                  (reference app uses 63, app/bfs.cu:18)    */
    int32_t  direction;        /* SCAPH_DIR_*                               */
    float    alpha;            /* 0 -> 14                                   */
    float    beta;             /* 0 -> 96                                   */
    int32_t  block_size;       /* threads per CTA of the level kernels; 0=256
                                  (FLAGS_num_thds, src/app.cuh:43)          */
    int32_t  ctas_per_sm;      /* 0 = from occupancy                        */
    int32_t  copy_streams;     /* side streams for page staging; 0 = 2
                                  (FLAGS_num_stream, src/app.cuh:41)        */
    int32_t  prefetch;         /* out-of-core: 1 = prefetch predicted pages */
    int32_t  compact_threshold;/* out-of-core: pages with active data <=
                                  threshold/32 of a page are read zero-copy
                                  instead of copied (FLAGS_threshold,
                                  src/app.cuh:45,151); 0 = 3                */
    int32_t  use_graph;        /* 0/1: each BFS is one CUDA-graph launch whose
                                  level loop runs on the device; 2: host loop
                                  (one launch per level, per-level events)  */
    int32_t  device;           /* CUDA device ordinal                       */
    void    *stream;           /* cudaStream_t to run on; NULL = own stream */
    int32_t  record_features;  /* host loop: keep the scheduler's feature
                                  vector of every level (scaph_bfs_features);
                                  graph mode: record the per-level page
                                  histograms (scaph_bfs_page_hist), which
                                  the learned direction records anyway     */
    int32_t  dual_timing;      /* host loop, graph resident: run every level
                                  both ways from the same state and record
                                  both times (training labels)             */
    float    link_gbs;         /* out-of-core learned scheduler: host->HBM
                                  page bandwidth (GB/s) its transfer-cost
                                  estimate assumes; 0 = measured at create  */
    /* Launch-shape tunables (the reference's are FLAGS_num_blks /
     * FLAGS_num_thds / FLAGS_num_stream, src/app.cuh:38-52, used per page at
     * src/app.cuh:438); 0 = default.  Searched by scaph_b200/autotune.py.  */
    int32_t  giant_edges;      /* push: adjacency longer than this is cut into
                                  chunks of this many edges, one CTA each;
                                  128..65536, 0 = 1024                      */
    int32_t  pull_gather_ratio;/* a pull level gathers several tiles' vertices
                                  into one queue when fewer than one vertex
                                  in this many is unvisited; 0 = 64         */
    int32_t  ms_compact_l2_div;/* multi-source pull: frontier masks are
                                  compacted when they fit L2 / this; 0 = 3  */
    int32_t  ms_compact_min_deg;/* ... and the frontier has at least this
                                  many out-edges per vertex; 0 = 16        */
    int32_t  pull_warp;        /* pull kernel shape on levels that read the
                                  8-byte records (CTA tiles on the others):
                                  1 warp-centric (each warp compacts its own
                                  512-vertex chunks); 2 vertex-parallel (lane
                                  = bit of the bitmap word, coalesced records
                                  and depths, found bits by ballot); 3 CTA
                                  tiles of 4096 vertices; 0 = 1             */
    int64_t  push_defer_edges; /* a push level whose frontier has at least
                                  this many out-edges defers its claims: the
                                  neighbours' bits are OR-ed into the next
                                  frontier and one pass then writes depths
                                  word by word (not with parents); 0 = 2^20,
                                  negative = never                         */
    int32_t  pull_records;     /* pull phase A from the 8-byte per-vertex
                                  records: 0 = on levels whose frontier has
                                  at least a quarter as many vertices as the
                                  unvisited set (the top-ranked probe mostly
                                  hits there), 1 = every level, 2 = never   */
    int32_t  pull_rows;        /* pull phase A on levels without the 8-byte
                                  records: 1 = one 16-byte row per vertex
                                  (three ranked in-neighbours and the
                                  degrees; 16 bytes of HBM per vertex, built
                                  when first asked for); 0 or 2 = the
                                  in-degree, 16-byte head row (four ranked
                                  in-neighbours) and out-degree arrays      */
    int32_t  push_sparse_ratio;/* a push level whose frontier has fewer than
                                  one vertex per this many reads its
                                  frontier words as one contiguous run per
                                  CTA and expands them together (whole-
                                  graph ranges); 0 = 16, negative = never  */
    int32_t  pull_runs;        /* sparse pull levels (pull_gather_ratio) on
                                  whole-graph ranges: 0 or 1 = each CTA
                                  reads one contiguous run of visited words
                                  at once, 2 = 128-word tiles one after
                                  another                                   */
} scaph_config;

typedef struct scaph_engine scaph_engine;

/* Uploads the graph (all pages, or up to pool_bytes of them) and allocates
 * the per-vertex state (replaces App::App + App::load_graph,
 * src/app.cuh:137-156,267-345).  `gt` is the transposed graph used by pull
 * on directed graphs; NULL means the graph is symmetric and pull reads g. */
int scaph_engine_create(const scaph_graph *g, const scaph_graph *gt,
                        const scaph_config *cfg, scaph_engine **e);
int scaph_engine_destroy(scaph_engine *e);

/* Per-run summary. */
typedef struct scaph_bfs_stats {
    int32_t  levels;            /* BFS levels executed                      */
    int32_t  push_levels;
    int32_t  pull_levels;
    int32_t  _pad;
    uint64_t reached;           /* vertices with a finite depth             */
    uint64_t reached_edges;     /* sum of out-degrees of reached vertices   */
    uint64_t edges_inspected;   /* adjacency words read by the kernels      */
    uint64_t alg_bytes;         /* algorithmic HBM bytes: push levels 12 per
                                   frontier vertex + 4 per edge; pull levels
                                   12 per unvisited vertex + 4 per in-edge
                                   inspected; each level V/8 of bitmap and
                                   4 (+4 with parents) per discovered vertex */
    uint64_t h2d_bytes;         /* page bytes copied host->HBM              */
    uint64_t zc_bytes;          /* page bytes read zero-copy over PCIe      */
    uint64_t page_faults;       /* page loads on demand                     */
    uint64_t prefetched;        /* page loads issued ahead by the scheduler */
    uint64_t launches;          /* kernels this library launched            */
    double   ms;                /* device time of the traversal (events)    */
    uint64_t pcie_alg_bytes;    /* out of core: the least the levels had to
                                   bring over the link, 4 * sum(deg+3) of the
                                   active vertices of needed pages that were
                                   not resident (get_page_info's datas,
                                   src/gpu_engine.cuh:413-419)             */
} scaph_bfs_stats;

/* Single-source level-synchronous BFS (replaces App::run, src/app.cuh:220-265,
 * with the bfs app hooks app/bfs.cu:20-37, app/bfs_kernel.cuh:6-16).
 * depths: u32[V] (unreached = cfg.unreached); parents: u32[V] or NULL
 * (parent[src] = src, unreached = 0xFFFFFFFF).  out_on_device != 0 means the
 * pointers are device pointers; otherwise host memory (copied back).
 * stats may be NULL. */
int scaph_bfs(scaph_engine *e, uint32_t src, uint32_t *depths, uint32_t *parents,
              int out_on_device, scaph_bfs_stats *stats);
/* Sets an engine's run-time tunables from cfg: alpha, beta, block_size,
 * ctas_per_sm, giant_edges, pull_gather_ratio, ms_compact_l2_div,
 * ms_compact_min_deg, pull_warp, push_defer_edges, pull_records,
 * pull_rows, push_sparse_ratio and pull_runs (0 = default; the other
 * fields are ignored).  They
 * change the schedule only, never the depths.  Waits for the engine's work
 * and drops its CUDA graph (the next run rebuilds it).  Replaces setting
 * FLAGS_num_blks / FLAGS_num_thds between runs (src/app.cuh:38-52). */
int scaph_engine_tune(scaph_engine *e, const scaph_config *cfg);
/* Out-of-core engines (pool_bytes smaller than the graph's pages): drops
 * every page from the HBM pool, so the next traversal starts cold. */
int scaph_engine_evict_all(scaph_engine *e);
/* With out_on_device != 0 and stats == NULL, scaph_bfs only enqueues the
 * traversal on the engine's stream and returns; scaph_engine_sync waits,
 * and scaph_bfs_trace / scaph_bfs_page_hist wait for the last run. */
int scaph_engine_sync(scaph_engine *e);
/* Pipelined traversals with host output, for serving many sources: enqueues
 * the traversal of `src` and the copy of its depths into `host_depths`
 * (V words; page-locked memory from scaph_host_alloc for the copy to run
 * asynchronously) and returns.  The copy of one run overlaps the next run's
 * traversal (two device buffers, a copy stream); the caller keeps each host
 * buffer untouched until scaph_engine_sync returns.  Resident graphs in graph
 * mode only (SCAPH_EUNSUPPORTED otherwise).  Same depths as scaph_bfs
 * (App::run, src/app.cuh:220-265, with the copy-back of check(),
 * src/app.cuh:262-264). */
int scaph_bfs_enqueue(scaph_engine *e, uint32_t src, uint32_t *host_depths);

/* Per-level trace of the last scaph_bfs (direction, frontier, edges, time,
 * per-page histogram).  Writes up to `cap` records, returns the count. */
typedef struct scaph_level_trace {
    int32_t  level;
    int32_t  direction;         /* 0 push, 1 pull                           */
    uint64_t frontier;          /* vertices in the frontier of this level   */
    uint64_t frontier_edges;    /* their out-degree sum                     */
    uint64_t unvisited;         /* vertices not yet reached                 */
    uint64_t unvisited_edges;   /* their out-degree sum                     */
    uint64_t next;              /* vertices discovered by this level        */
    uint64_t edges_inspected;
    uint64_t alg_bytes;         /* algorithmic HBM bytes of this level      */
    uint64_t h2d_bytes;
    double   ms;                /* device time of this level's kernels      */
    double   push_ms;           /* dual_timing: both directions' times;     */
    double   pull_ms;           /* multi-source rows: push_ms = device time
                                   between the previous level's end and this
                                   level's start, pull_ms = host time of the
                                   level's census and decisions            */
} scaph_level_trace;
int scaph_bfs_trace(scaph_engine *e, scaph_level_trace *out, int cap);
/* Active-vertex histogram of the frontier at `level` of the last run:
 * nodes[p] / datas[p] as get_page_info computes them (src/gpu_engine.cuh:397-441).
 * Recorded by out-of-core runs, and by resident runs only with
 * record_features or the learned direction (SCAPH_EUNSUPPORTED otherwise). */
int scaph_bfs_page_hist(scaph_engine *e, int level, uint32_t *nodes,
                        uint32_t *datas, int npages);

/* ---- learned scheduler ---------------------------------------------------- */

/* No counterpart in the reference.  A 3-layer perceptron (in -> 64 -> 64 ->
 * out, ReLU; BF16 weights, FP32 accumulation) trained on the GPU with the
 * library's own forward / backward / Adam kernels (tensor-core GEMMs).
 * For a scheduler: in = SCAPH_SCHED_GLOBALS + npages, out = 1 + npages
 * (npages = pages of the out-edge graph); output 0 is the push(<0)/pull(>0)
 * logit of the coming level, outputs 1.. the logits "page p holds frontier
 * vertices at the level after". */
#define SCAPH_SCHED_GLOBALS 16
typedef struct scaph_mlp scaph_mlp;
int scaph_mlp_create(int in_dim, int out_dim, uint64_t seed, int device, scaph_mlp **m);
void scaph_mlp_destroy(scaph_mlp *m);
size_t scaph_mlp_num_params(const scaph_mlp *m);
/* parameters, in order W1[in][64] b1[64] W2[64][64] b2[64] W3[64][out] b3[out] */
int scaph_mlp_get_params(const scaph_mlp *m, float *out, size_t n);
int scaph_mlp_set_params(scaph_mlp *m, const float *in, size_t n);
/* X: n rows of `in` floats (host); Y: n rows of `out` logits (host) */
int scaph_mlp_forward(scaph_mlp *m, const float *X, int n, float *Y);
/* sum over rows and outputs of W * BCE-with-logits(Y, T), and its gradient
 * w.r.t. the parameters (grad may be NULL) */
int scaph_mlp_loss_grad(scaph_mlp *m, const float *X, const float *T, const float *W, int n,
                        float *loss, float *grad);
int scaph_mlp_adam_step(scaph_mlp *m, const float *X, const float *T, const float *W, int n,
                        float lr, float *loss);
int scaph_mlp_train(scaph_mlp *m, const float *X, const float *T, const float *W, int n,
                    int epochs, int batch, float lr, uint64_t seed, float *final_loss);
int scaph_mlp_save(const scaph_mlp *m, const char *path);
/* Device time in microseconds (CUDA events, mean over reps) of a forward
 * pass over n rows (out_us[0]), one training step on n rows (out_us[1]:
 * forward, loss, backward, Adam) and the single-row inference kernel
 * (out_us[2], the network part of the graph-mode learned decision), on zero
 * rows already on the device.  Parameters and Adam state are left as
 * they were. */
int scaph_mlp_time(scaph_mlp *m, int n, int reps, float *out_us);
int scaph_mlp_load(scaph_mlp *m, const char *path);

/* Makes SCAPH_DIR_LEARNED engines use `m` (NULL: back to alpha/beta): the
 * network picks each level's direction and, out of core, pages whose
 * logit exceeds 0 are prefetched while the level runs.  The engine keeps
 * the pointer; it never changes depths. */
int scaph_engine_set_scheduler(scaph_engine *e, scaph_mlp *m);
/* Feature rows of the last host-loop scaph_bfs or of the last scaph_msbfs
 * (record_features or learned mode; a multi-source row counts the union of
 * the batch's frontiers): returns the row count, writes min(rows, cap) rows
 * of *dim floats. */
int scaph_bfs_features(scaph_engine *e, float *out, int cap, int *dim);
/* Unvisited vertices per in-edge page at `level` of the last run
 * (record_features): the pages a pull at that level would read, and their
 * active words sum(indeg+3) (datas may be NULL). */
int scaph_bfs_pull_pages(scaph_engine *e, int level, uint32_t *cnt, uint32_t *datas, int npages);

/* ---- multi-source BFS ---------------------------------------------------- */

/* No counterpart in the reference (it runs one source per App::run,
 * src/app.cuh:220-265).  Up to SCAPH_MSBFS_MAX sources share one traversal:
 * per-vertex 64-bit (or 2x64-bit) source masks, the same direction rule,
 * depths bit-exact with nsrc separate scaph_bfs runs.
 * depths: u32[nsrc][V] (row i = source srcs[i]; unreached = cfg.unreached),
 * host or device memory per out_on_device. */
#define SCAPH_MSBFS_MAX 128
int scaph_msbfs(scaph_engine *e, const uint32_t *srcs, int nsrc, uint32_t *depths,
                int out_on_device, scaph_bfs_stats *stats);
/* Per-level trace of the last scaph_msbfs (frontier = vertices with a
 * nonzero mask; next = vertices newly reached by any source). */
int scaph_msbfs_trace(scaph_engine *e, scaph_level_trace *out, int cap);

/* ---- mixed query batches -------------------------------------------------- */

/* No counterpart in the reference (one source of one graph per App::run,
 * src/app.cuh:220-265).  A batch holds several graphs side by side on the
 * device (their disjoint union, paged like any graph) and runs many
 * single-source BFS queries over them in ONE launch of a CUDA graph:
 * queries on the same graph share a bit-parallel traversal (one bit each,
 * at most 128 per graph per launch), all graphs advance in one device-side
 * level loop.  Depths are bit-exact with scaph_bfs on each graph alone.
 * `transposed` (NULL when every graph is symmetric) gives each graph's
 * in-edges for pull levels. */
typedef struct scaph_batch scaph_batch;
typedef struct scaph_query {
    uint32_t graph;   /* index into the batch's graphs                      */
    uint32_t source;  /* vertex id within that graph                        */
} scaph_query;
/* Tunables of the batch kernels (picked by scaph_b200/autotune.py). */
typedef struct scaph_batch_params {
    int32_t block_size;   /* threads per CTA of the level kernels: 256 or 512 */
    int32_t ctas_per_sm;  /* grid = SMs x this                                 */
    float   alpha, beta;  /* direction-switch thresholds                       */
    int32_t _reserved;
} scaph_batch_params;
int scaph_batch_create(const scaph_csr *graphs, int ngraphs, const scaph_csr *transposed,
                       uint32_t pagesize_words, const scaph_config *cfg, scaph_batch **b);
int scaph_batch_destroy(scaph_batch *b);
/* Union vertex ids of graph `graph`: first_vertex .. first_vertex+nvertices-1. */
int scaph_batch_graph_range(const scaph_batch *b, int graph, uint32_t *first_vertex,
                            uint32_t *nvertices);
int scaph_batch_set_params(scaph_batch *b, const scaph_batch_params *p);
int scaph_batch_get_params(const scaph_batch *b, scaph_batch_params *p);
/* Runs nq queries.  depths: query i's row is u32[V of its graph], rows
 * concatenated in query order (unreached = cfg.unreached); host or device
 * memory per out_on_device.  stats->launches is 1: the traversal is one
 * graph launch. */
int scaph_batch_run(scaph_batch *b, const scaph_query *queries, int nq, uint32_t *depths,
                    int out_on_device, scaph_bfs_stats *stats);
/* Per-level trace of the last run (direction, frontier, time); returns the
 * number of levels. */
int scaph_batch_trace(const scaph_batch *b, scaph_level_trace *out, int cap);

/* ---- page store for App-hook engines ------------------------------------ */

/* The reference's apps supply a vertex program as device hooks
 * (cond/update, app/bfs_kernel.cuh:6-16, app/sssp_kernel.cuh:6-16,
 * app/wcc_kernel.cuh:5-15) that App<> runs over the pages of the graph
 * (gpu_push_csr, src/gpu_engine.cuh:41-169, scheduled by App::gpu_push_batch
 * and App::PageCopy, src/app.cuh:371-468).  Here the application compiles
 * its hooks into its own kernels (include/scaph/compat/app.cuh does this for
 * the reference's apps) and the store hands it pages to run them on.
 *
 * A store keeps the graph's pages (weighted {ngr,wgh} pages too) on the
 * device: all of them, or - when pool_bytes is smaller than the pages - a
 * pool of pool_bytes of them managed like the BFS engine's out-of-core pool
 * (zero-copy reads of pages whose active words are at most
 * compact_threshold/32 of a page; demand copies on copy_streams streams). */
typedef struct scaph_store scaph_store;

/* Device page table entry: page p's words start at pool + base; it holds
 * the vertices left .. left+nodenum-1 (Node{vtx,idx,len} triples, then the
 * edges; idx counts edges, an edge being 1 word, or 2 when weighted). */
typedef struct scaph_page_dev {
    uint64_t base;
    uint32_t left;
    uint32_t nodenum;
} scaph_page_dev;

/* What a batch of pages looks like to the application's kernels. */
typedef struct scaph_page_view {
    const uint32_t       *pool;    /* device words                            */
    const scaph_page_dev *pages;   /* device, npages + 1 (pages[npages].left = V) */
    const uint32_t       *coarse;  /* device: coarse[v >> cshift] = a page at
                                      or before the page holding v          */
    uint32_t cshift, npages, V, pagesize, weighted;
} scaph_page_view;

/* The vertices of a batch: n ranges [lo[i], hi[i]) (device arrays).  Range
 * i owns the tiles tile0[i] .. tile0[i+1]-1 (tile0[n] need not exist; tiles
 * = the total): tile t of range i covers the 4096 vertices starting at
 * 32 * (lo[i] / 32 + 128 * (t - tile0[i])). */
typedef struct scaph_ranges {
    const uint32_t *lo, *hi, *tile0;
    uint32_t n, tiles;
} scaph_ranges;

/* Launches the application's kernels for one batch on `stream` (a
 * cudaStream_t); returns 0, or a nonzero code that the level returns. */
typedef int (*scaph_batch_fn)(void *user, const scaph_page_view *view,
                              const scaph_ranges *ranges, void *stream);

int scaph_store_create(const scaph_graph *g, int64_t pool_bytes, int compact_threshold,
                       int copy_streams, int device, scaph_store **s);
int scaph_store_destroy(scaph_store *s);
/* 1 when every page is resident (then scaph_store_view gives the one view). */
int scaph_store_resident(const scaph_store *s);
int scaph_store_view(const scaph_store *s, scaph_page_view *out);
/* Out-degrees on the device, u32[V] (the reference's d_degree). */
const uint32_t *scaph_store_degree(const scaph_store *s);
/* One round over the active vertices (device bitmap, V bits): calls fn for
 * every batch of pages that hold active vertices, on `stream` or, out of
 * core, on streams ordered after `stream`'s prior work and before its later
 * work.  Out of core it synchronises `stream` once to read the page counts. */
int scaph_store_level(scaph_store *s, const uint32_t *d_active, scaph_batch_fn fn,
                      void *user, void *stream);
/* Page bytes copied, read zero-copy, and demand copies, since create. */
int scaph_store_counters(const scaph_store *s, uint64_t *h2d_bytes, uint64_t *zc_bytes,
                         uint64_t *page_faults);

/* ---- BFS without device allocation -------------------------------------- */

/* No counterpart in the reference.  For callers that must not have the
 * library allocate device memory: hosts that pre-reserve the GPU's memory in
 * their own pool, and latency-critical paths where cudaMalloc/cudaFree would
 * synchronise the device.  Runs the same level kernels as scaph_bfs over ONE
 * paged-CSR page that the caller already holds in device memory (the page
 * must hold vertices 0..nodenum-1, i.e. the whole graph; the layout of
 * <p>page0, tools/pagegencsr.cpp:221-242), writing depths (and parents, if
 * d_parent is not NULL) into the caller's device arrays.
 *   d_page   16-byte aligned, at least round_up(3*nodenum + edgenum, 4) words
 *   limits   nodenum <= SCAPH_NOALLOC_MAX_V, edgenum <= SCAPH_NOALLOC_MAX_E,
 *            larger inputs return SCAPH_EINVAL before any GPU work
 *   flags    SCAPH_NOALLOC_SYMMETRIC: every edge of the page has its reverse,
 *            so pull levels may read the page as in-edges and the alpha/beta
 *            switch is used; without it every level pushes (right for
 *            directed pages)
 *   unreached  depth of unreached vertices; 0 = 0xFFFFFFFF, 1 is rejected
 *   stats    NULL, or the run's levels, push/pull level counts, reached
 *            vertices and edges, edges inspected and kernel launches
 * A page whose Node records do not fit nodenum/edgenum returns SCAPH_EFORMAT
 * before any traversal.  There is no level cap: paths up to nodenum deep
 * get their exact depths.  Its scratch state is a fixed ~1.3 MB __device__
 * array inside the library, held on every GPU that loads it until the
 * process exits.  All calls share it and leave their contents in it; each
 * call clears what it needs, but calls whose GPU work overlaps race on it.
 * Each call looks up the array's address (cudaGetSymbolAddress, current
 * device) and synchronises `stream` (a cudaStream_t; NULL = default stream)
 * once per level. */
#define SCAPH_NOALLOC_MAX_V (1u << 18)
#define SCAPH_NOALLOC_MAX_E (1u << 22)
#define SCAPH_NOALLOC_SYMMETRIC 1
int scaph_bfs_page_noalloc(const uint32_t *d_page, uint32_t nodenum, uint32_t edgenum,
                           uint32_t src, uint32_t unreached, int flags, uint32_t *d_depth,
                           uint32_t *d_parent, scaph_bfs_stats *stats, void *stream);

/* ---- host helpers ------------------------------------------------------ */

/* Page-locked host memory for outputs copied back by scaph_bfs (faster
 * device->host copies than pageable memory).  NULL on failure. */
void *scaph_host_alloc(size_t bytes);
void scaph_host_free(void *p);
/* Number of CUDA devices visible (0 when there is no GPU). */
int scaph_device_count(void);

#ifdef __cplusplus
}
#endif
#endif /* SCAPH_H */
