// Example applications on the App-hook API (scaph/compat/app.cuh): one
// source built three times, -DAPPBFS, -DAPPSSSP or -DAPPWCC, each a subclass
// of App<> that only initialises the vertex values (gpu_init) - the hooks in
// the matching <name>_kernel.cuh do the rest.
//
//   <app> --graphfile=<prefix> [--src=N] [--far=V] [--sources=a,b,..]
//         [--repeat=N] [--out=<file>] [App flags: --max_memory=MB ...]
//
// BFS / SSSP start from --src (or every vertex of --sources) at value 0,
// every other vertex at --far (BFS default 63, the reference app's
// MAXDEPTH; SSSP default 0x7fffffff, its MAXPATH); WCC labels every vertex
// with its id and starts with all of them active.  --out writes the final
// value array (u32[V]) for the tests; the last line printed says which path
// ran ("engine" = the direction-optimising BFS engine, "hooks" = hook
// rounds) and how many rounds.
#include "app.cuh"

#include <cstdio>
#include <sstream>

namespace {

#ifndef APPWCC
__global__ void k_init_far(unsigned int *value, bool *stat, unsigned int n, unsigned int far)
{
    for (unsigned int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        value[v] = far;
        stat[v] = false;
    }
}

__global__ void k_init_sources(unsigned int *value, bool *stat, const unsigned int *src, int nsrc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsrc) {
        value[src[i]] = 0;
        stat[src[i]] = true;
    }
}
#else
__global__ void k_init_labels(unsigned int *value, bool *stat, unsigned int n)
{
    for (unsigned int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        value[v] = v;
        stat[v] = true;
    }
}
#endif

}  // namespace

class HookApp : public App<unsigned int, unsigned int, unsigned int>
{
public:
    using Base = App<unsigned int, unsigned int, unsigned int>;
    HookApp(int argc, char **argv, unsigned int far, std::vector<unsigned int> sources)
        : Base(argc, argv), far_(far), sources_(std::move(sources))
    {
    }
    ~HookApp() override { cudaFree(d_src_); }

    void gpu_init() override
    {
#ifdef APPWCC
        k_init_labels<<<256, 256, 0, copystream>>>(d_value, d_stat, vert_count);
#else
        if (!d_src_) {
            SCAPH_COMPAT_CUDA(cudaMalloc(&d_src_, sizeof(unsigned int) * sources_.size()));
            SCAPH_COMPAT_CUDA(cudaMemcpy(d_src_, sources_.data(), sizeof(unsigned int) * sources_.size(),
                                         cudaMemcpyHostToDevice));
        }
        k_init_far<<<256, 256, 0, copystream>>>(d_value, d_stat, vert_count, far_);
        k_init_sources<<<1, 128, 0, copystream>>>(d_value, d_stat, d_src_, (int)sources_.size());
#endif
        SCAPH_COMPAT_CUDA(cudaGetLastError());
        SCAPH_COMPAT_CUDA(cudaStreamSynchronize(copystream));
    }

private:
    unsigned int far_;
    std::vector<unsigned int> sources_;
    unsigned int *d_src_ = nullptr;
};

int main(int argc, char **argv)
{
    std::string out;
    int repeat = 1;
#if defined(APPSSSP)
    unsigned long long far = 0x7fffffffu;
#else
    unsigned long long far = 63;
#endif
    std::string sources;
    // the example's own flags; the rest go to App
    std::vector<char *> rest{argv[0]};
    for (int i = 1; i < argc; i++) {
        std::string a(argv[i]);
        if (a.rfind("--out=", 0) == 0) out = a.substr(6);
        else if (a.rfind("--repeat=", 0) == 0) repeat = std::max(1, atoi(a.c_str() + 9));
        else if (a.rfind("--far=", 0) == 0) far = strtoull(a.c_str() + 6, nullptr, 0);
        else if (a.rfind("--sources=", 0) == 0) sources = a.substr(10);
        else rest.push_back(argv[i]);
    }
    std::vector<unsigned int> srcs;
    {
        std::stringstream ss(sources);
        std::string tok;
        while (std::getline(ss, tok, ','))
            if (!tok.empty()) srcs.push_back((unsigned int)strtoul(tok.c_str(), nullptr, 0));
    }
    scaph_compat::parse_flags((int)rest.size(), rest.data());  // for --src
    if (srcs.empty()) srcs.push_back((unsigned int)FLAGS_src);
    HookApp app((int)rest.size(), rest.data(), (unsigned int)far, srcs);
    app.load_graph();
    for (unsigned int s : srcs)
        if (s >= app.vert_count) {
            fprintf(stderr, "source %u out of range (V = %u)\n", s, app.vert_count);
            return 2;
        }
    for (int r = 0; r < repeat; r++) app.run();
    if (!out.empty()) {
        SCAPH_COMPAT_CUDA(cudaMemcpy(app.h_value, app.d_value, sizeof(unsigned int) * app.vert_count,
                                     cudaMemcpyDeviceToHost));
        FILE *f = fopen(out.c_str(), "wb");
        if (!f || fwrite(app.h_value, 4, app.vert_count, f) != app.vert_count) {
            fprintf(stderr, "cannot write %s\n", out.c_str());
            return 2;
        }
        fclose(f);
    }
    printf("path=%s rounds=%d seconds=%.6f h2d=%llu zc=%llu faults=%llu pool_pages=%d pages=%d\n",
           app.last_used_bfs_engine ? "engine" : "hooks", app.last_rounds, app.last_seconds,
           (unsigned long long)app.last_h2d_bytes, (unsigned long long)app.last_zc_bytes,
           (unsigned long long)app.last_page_faults, app.pool_size, app.list_size);
    return 0;
}
