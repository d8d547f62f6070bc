// CNTK-format (version 1.1) cascade model files.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ccnn_common.cuh"

namespace ccnn {

// Contents of a cnn4face*_cntk.bin file, in file order
// (reader: SIMD::ConvNeuralNetwork::Init, src/CNNObjectDetector/cnn_simd_cntk.cpp:42-404).
struct RawModel {
    float version = 0.f;
    bool max_pool = false;
    int min_w = 0, min_h = 0;
    int layers = 0;
    int maps[3] = {0, 0, 0};
    int kw[3] = {0, 0, 0}, kh[3] = {0, 0, 0};
    std::vector<float> kernels[3];  // maps x (kw*kh), row-major
    float af_scale = 0.f;
    std::vector<float> act[3];      // per map: conv_bias, lrelu_w1, lrelu_w2, bn_weight, bn_bias
    bool full_connect = false;
    int hl = 0, conn = 0, hs = 0;
    std::vector<float> hw, hb, htw, hbn;  // hbn: hs x (weight, bias)
    int nout = 0;
    std::vector<float> ow, ob;
    float otw = 0.f;
};

// Parses the bytes of a model file. Returns false with a message on malformed input.
bool parse_model(const uint8_t* data, size_t n, RawModel* m, std::string* err);
bool load_model_file(const std::string& path, RawModel* m, std::string* err);

// Packs a parsed model into the kernel weight layout for the given output neuron
// (Init :396-397: index clamped to the last neuron; output scale negated for index 0).
// Fails if the shapes differ from the compiled prototype.
template <class NW>
bool pack_model(const RawModel& m, int index_output, NW* out, std::string* err);

// Packs the facial-analysis (landmark) model; all 13 outputs are kept (index_output -1).
bool pack_landmarks(const RawModel& m, LandmarkNet* out, std::string* err);

// Directory holding the bundled model files (next to the shared library).
std::string bundled_model_dir();

}  // namespace ccnn
