// Host-side inference of the scheduler network (the per-level decision of
// the host-driven level loop): k_forward1 of mlp.cu restated with the same
// operand rounding and the same fused multiply-adds in the same order, so
// the logits equal the device's.  Built for hardware FMA where the CPU has
// it (function multiversioning), with the library fma() elsewhere.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cstdint>

#include "mlp_host.h"

namespace scaph {

namespace {

constexpr int kH = 64;

inline float bf16_round(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return x;
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

}  // namespace

__attribute__((target_clones("fma", "default")))
void mlp_forward_host(const MlpHost &h, const float *x, float *y)
{
    std::vector<float> sx(h.in);
    float h1[kH], h2[kH];
    for (int i = 0; i < h.in; i++) sx[i] = bf16_round(x[i]);
    for (int j = 0; j < kH; j++) {
        float a = h.w[h.off_b1 + j];
        for (int i = 0; i < h.in; i++) a = std::fma(sx[i], h.w[h.off_w1 + (size_t)i * kH + j], a);
        h1[j] = bf16_round(std::max(a, 0.f));
    }
    for (int j = 0; j < kH; j++) {
        float a = h.w[h.off_b2 + j];
        for (int i = 0; i < kH; i++) a = std::fma(h1[i], h.w[h.off_w2 + (size_t)i * kH + j], a);
        h2[j] = bf16_round(std::max(a, 0.f));
    }
    for (int o = 0; o < h.out; o++) {
        float a = h.w[h.off_b3 + o];
        for (int j = 0; j < kH; j++) a = std::fma(h2[j], h.w[h.off_w3 + (size_t)j * h.out + o], a);
        y[o] = a;
    }
}

}  // namespace scaph
