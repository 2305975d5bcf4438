// Harness that compiles the reference's own BFS application source
// (app/bfs.cu, which pulls in src/app.cuh, src/compress.h, src/tools.h, ...)
// into oracle/_ref/libscaphref.so, so that tests can run the reference's CPU
// code paths unchanged:
//   * bfs::check (app/bfs.cu:67-117)  - the reference CPU level-synchronous BFS;
//   * compress_stat (src/compress.h:18-40) - active-vertex page compaction;
//   * the chunk-mask helpers (src/tools.h:11-85).
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed reference CPU arm).
// No reference source is copied: the file is #included from the reference
// tree at build time (oracle/Makefile).  Only host functions are called; none
// of the reference's GPU kernels is ever launched.
#include <chrono>
#include <cstdint>
#include <sstream>
#include <string>

#define main scaph_reference_bfs_app_main
#include "bfs.cu"
#undef main

typedef unsigned int ref_u32;

extern "C" {

// Runs bfs::check for `src` over the flat CSR (idx u32[V+1], ngh u32[E]).
// bfs::check computes the reference depths internally (sentinel 63) and
// counts how many entries of `values` differ from them (app/bfs.cu:102-115).
// It prints "total errors: N"; that line is captured and parsed.
// Returns 0 on success, -1 if the output could not be parsed.
int ref_bfs_check(ref_u32 V, const ref_u32 *idx, const ref_u32 *ngh, ref_u32 src,
                  ref_u32 *values, long long *errors, double *seconds)
{
    char arg0[] = "scaph_ref";
    char *argv[] = {arg0, nullptr};
    bfs<ref_u32, ref_u32, ref_u32> app(1, argv);
    app.vert_count = V;
    app.csr_idx = const_cast<ref_u32 *>(idx);
    app.csr_ngh = const_cast<ref_u32 *>(ngh);
    app.h_value = values;
    FLAGS_src = (int)src;

    std::ostringstream cap;
    std::streambuf *old = std::cout.rdbuf(cap.rdbuf());
    auto t0 = std::chrono::steady_clock::now();
    app.check();
    auto t1 = std::chrono::steady_clock::now();
    std::cout.rdbuf(old);
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();

    const std::string out = cap.str();
    const std::string key = "total errors: ";
    size_t at = out.rfind(key);
    if (at == std::string::npos) return -1;
    *errors = std::stoll(out.substr(at + key.size()));
    return 0;
}

// src/compress.h:18-40, unchanged.
unsigned ref_compress_stat(unsigned *page_src, unsigned *page_dst, unsigned char *stat,
                           unsigned left, unsigned srcnodenum, unsigned dstnodenum)
{
    double endtime = 0;
    int tid = 0;
    return (unsigned)compress_stat(page_src, page_dst, reinterpret_cast<bool *>(stat), left,
                                   srcnodenum, dstnodenum, endtime, tid);
}

// src/tools.h:11-85, unchanged.
int ref_max_zero_run(int mark) { return get_max_continus_zero(mark); }
int ref_fit_zero_run(int mark, int required) { return get_fit_continus_zero(mark, required); }
int ref_set_run(int mark, int off, int n, int value)
{
    return value ? set_continus_one(mark, off, n) : set_continus_zero(mark, off, n);
}

}  // extern "C"
