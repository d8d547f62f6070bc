// Legacy cascade networks (model format 1.0, the `_new.bin` family): tanh activations, max or
// average pooling, and a hidden layer that is either two neurons per L3 map or fully connected.
// Reader: SIMD::ConvNeuralNetwork::Init (src/CNNObjectDetector/cnn_simd.cpp:40-336, plain-C++
// branch); forward pass: Run_single_thread (cnn_simd.cpp:551-874) over the CNNPP operations of
// src/CNNObjectDetector/cnnpp_cplusplus.cpp.
#pragma once

#include <cstdint>
#include <string>

namespace ccnn {

constexpr int kLgMaxM0 = 8, kLgMaxM1 = 16, kLgMaxM2 = 32, kLgMaxK3 = 56, kLgMaxHL = 64;

struct LegacyNet {
    int max_pool;          // 1: 2x2 max of the tanh'd convolution, 0: 2x2 sum (average)
    int min_w, min_h;      // smallest input
    int m0, m1, m2;        // maps of the three convolution layers (m1 = 2 m0, m2 = 2 m1)
    int k3w, k3h;          // third-layer kernel (5 x 6 or 7 x 8)
    int full_connect;      // hidden layer: 0 = two neurons per L3 map, 1 = every neuron reads every map
    int hl;                // hidden neurons
    float af;              // output scale of every tanh layer (af_scale)
    float k1[kLgMaxM0][16];
    float k2[kLgMaxM1][9];
    float k3[kLgMaxM2][kLgMaxK3];
    float cb[3][kLgMaxM2], sw[3][kLgMaxM2], sb[3][kLgMaxM2];  // conv bias, pooling weight, pooling bias
    float hw[kLgMaxHL];               // two-per-map hidden weights
    float hwfc[kLgMaxHL][kLgMaxM2];   // fully connected hidden weights
    float hb[kLgMaxHL], ow[kLgMaxHL];
    float ob;
};

// Parses a format-1.0 model file's bytes; false with a message when the file is not one, is
// truncated, or has a shape the reference refuses (cnn_simd.cpp:267-276) or this build does not
// cover (map counts above the limits above, or not doubling from layer to layer).
bool parse_legacy_model(const uint8_t* data, size_t n, LegacyNet* net, std::string* err);
bool load_legacy_model_file(const std::string& path, LegacyNet* net, std::string* err);

// Response-map size of a w x h input (AllocateMemory, cnn_simd.cpp:339-465): the third layer's
// region of interest.
inline void legacy_output_size(const LegacyNet& n, int w, int h, int* ow, int* oh) {
    const int r1c = w - 3, r1r = h - 3;
    const int r2c = (r1c >> 1) - 2, r2r = (r1r >> 1) - 2;
    *ow = (r2c >> 1) - (n.k3w - 1);
    *oh = (r2r >> 1) - (n.k3h - 1);
}

}  // namespace ccnn
