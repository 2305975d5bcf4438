// Host copy of the scheduler network for per-level inference without a
// device round trip (weights pre-rounded to bf16 as the device reads them).
#pragma once
#include <cstddef>
#include <vector>

namespace scaph {

struct MlpHost {
    std::vector<float> w;
    int in = 0, out = 0;
    size_t off_w1 = 0, off_b1 = 0, off_w2 = 0, off_b2 = 0, off_w3 = 0, off_b3 = 0;
};

// The logits of one feature row, equal to the device's k_forward1.
void mlp_forward_host(const MlpHost &h, const float *x, float *y);

}  // namespace scaph
