// Legacy cascade networks (model format 1.0, `_new.bin`) on the device: the reader and the forward
// pass of SIMD::ConvNeuralNetwork in the reference's plain-C++ build (src/CNNObjectDetector/
// cnn_simd.cpp:40-336 and 551-874 with the CNNPP operations of cnnpp_cplusplus.cpp), reproduced
// operation for operation in IEEE single precision (the file is built with -fmad=false):
//   L1  conv 4x4 (conv_4x4 :92), tanh(c + bias) of the four positions of a 2x2 window, their max
//       or sum, tanh(w * pooled + b) * af                      (max_tanh_tanh :473, tanh_avr_tanh :411)
//   sums of neighbouring L1 maps (add :916, add2 :933), conv 3x3 (conv_3x3 :36), the same pooling
//   sums of neighbouring L2 maps, conv 5x6 or 7x8 (conv_6x5 :212, conv_8x7 :292), then either
//     two hidden neurons per L3 map (tanh_tanh_2tanh :692) summed over the maps, or
//     tanh_tanh (:778) and fully connected hidden neurons (mulC24_add_tanh :1003, or
//     mulC2_add / mulC1_add / tanh :968-1002, :868) summed over the neurons,
//   and the output tanh(sum + bias) * af (tanh :868).
// tanh is the reference's rational form sgn(c) (1 - 1 / (1 + |c| + c^2 + 1.41645 c^4)) (USE_FAST_TANH).
// One thread computes one pooled pixel of one map (L1, L2) or one response pixel (L3 onwards);
// neighbouring-map sums are recomputed where they are read, with the reference's additions.
#include <cuda_runtime.h>

#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "../../include/ccnn_inspect.h"
#include "ccnn_common.cuh"
#include "legacy.h"
#include "legacy_dev.cuh"

namespace ccnn {

void set_error(const std::string& msg);

// ---- reader ----

namespace {
struct LgReader {
    const uint8_t* p;
    size_t n, off = 0;
    bool ok = true;
    template <class T>
    T get() {
        T v{};
        if (off + sizeof(T) > n) {
            ok = false;
            return v;
        }
        std::memcpy(&v, p + off, sizeof(T));
        off += sizeof(T);
        return v;
    }
};
}  // namespace

bool parse_legacy_model(const uint8_t* data, size_t n, LegacyNet* net, std::string* err) {
    LgReader r{data, n};
    std::memset(net, 0, sizeof(LegacyNet));
    const float version = r.get<float>();
    if (!r.ok || version != 1.0f) {
        *err = "not a legacy (format 1.0) model file";
        return false;
    }
    net->max_pool = r.get<uint8_t>() != 0 ? 1 : 0;
    net->min_w = r.get<int32_t>();
    net->min_h = r.get<int32_t>();
    const int layers = r.get<int32_t>();
    if (!r.ok || layers != 3) {
        *err = "this configuration of cnn models is not supported (3 convolution layers expected)";
        return false;
    }
    int maps[3];
    for (int& m : maps) m = r.get<int32_t>();
    net->m0 = maps[0];
    net->m1 = maps[1];
    net->m2 = maps[2];
    if (!r.ok || maps[0] < 2 || maps[0] > kLgMaxM0 || maps[1] != 2 * maps[0] || maps[2] != 2 * maps[1]) {
        *err = "legacy model: map counts must double from layer to layer, with at most 8 first-layer maps";
        return false;
    }
    int kw[3], kh[3];
    for (int l = 0; l < 3; ++l) {
        kw[l] = r.get<int32_t>();
        kh[l] = r.get<int32_t>();
        if (!r.ok || kw[l] <= 0 || kh[l] <= 0 || kw[l] * kh[l] > kLgMaxK3) {
            *err = "legacy model: malformed convolution layer";
            return false;
        }
        for (int m = 0; m < maps[l]; ++m)
            for (int k = 0; k < kw[l] * kh[l]; ++k) {
                const float v = r.get<float>();
                if (l == 0 && k < 16) net->k1[m][k] = v;
                if (l == 1 && k < 9) net->k2[m][k] = v;
                if (l == 2) net->k3[m][k] = v;
            }
    }
    net->k3w = kw[2];
    net->k3h = kh[2];
    net->af = r.get<float>();
    for (int l = 0; l < 3; ++l)
        for (int m = 0; m < maps[l]; ++m) {
            net->cb[l][m] = r.get<float>();
            net->sw[l][m] = r.get<float>();
            net->sb[l][m] = r.get<float>();
        }
    net->full_connect = r.get<uint8_t>() != 0 ? 1 : 0;
    net->hl = r.get<int32_t>();
    if (!r.ok) {
        *err = "legacy model: file is truncated";
        return false;
    }
    // the reference's own shape check (cnn_simd.cpp:267-276)
    if (kw[0] * kh[0] != 16 || kw[1] * kh[1] != 9 || (kw[2] * kh[2] != 30 && kw[2] * kh[2] != 56) || kw[0] != 4 || kw[1] != 3) {
        *err = "this configuration of cnn models is not supported (4x4, 3x3 and 5x6 or 7x8 kernels expected)";
        return false;
    }
    if (net->hl <= 0 || net->hl > kLgMaxHL || (!net->full_connect && net->hl != 2 * net->m2)) {
        *err = "legacy model: hidden layer size is not supported";
        return false;
    }
    if (!net->full_connect) {
        for (int i = 0; i < net->hl; ++i) net->hw[i] = r.get<float>();
    } else {
        for (int i = 0; i < net->hl; ++i)
            for (int j = 0; j < net->m2; ++j) net->hwfc[i][j] = r.get<float>();
    }
    for (int i = 0; i < net->hl; ++i) net->hb[i] = r.get<float>();
    for (int i = 0; i < net->hl; ++i) net->ow[i] = r.get<float>();
    net->ob = r.get<float>();
    if (!r.ok) {
        *err = "legacy model: file is truncated";
        return false;
    }
    return true;
}

bool load_legacy_model_file(const std::string& path, LegacyNet* net, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        *err = "cannot open model file " + path;
        return false;
    }
    std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    return parse_legacy_model(bytes.data(), bytes.size(), net, err);
}

// ---- forward pass ----

namespace {

__global__ void legacy_l1_kernel(const LegacyNet* __restrict__ N, const float* __restrict__ img, int pitch, int p1w, int p1h,
                                 float* __restrict__ pool1) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y, m = blockIdx.z;
    if (px >= p1w || py >= p1h) return;
    const float* k = N->k1[m];
    float c[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const float* s = img + (size_t)(2 * py + (d >> 1)) * pitch + 2 * px + (d & 1);
        float acc = fmul(s[0], k[0]);
#pragma unroll
        for (int t = 1; t < 16; ++t) acc = fadd(acc, fmul(s[(t >> 2) * pitch + (t & 3)], k[t]));
        c[d] = acc;
    }
    pool1[((long long)m * p1h + py) * p1w + px] = lg_pool_tanh(c, N->max_pool, N->cb[0][m], N->sw[0][m], N->sb[0][m], N->af);
}

__global__ void legacy_l2_kernel(const LegacyNet* __restrict__ N, const float* __restrict__ pool1, int p1w, int p1h, int p2w, int p2h,
                                 float* __restrict__ pool2) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, m = blockIdx.z;
    if (x >= p2w || y >= p2h) return;
    const int i = m >> 1;
    const long long plane = (long long)p1w * p1h;
    float S[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) S[r][q] = lg_map_sum(pool1, plane, N->m0, i, (long long)(2 * y + r) * p1w + 2 * x + q);
    const float* k = N->k2[m];
    float c[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const int dy = d >> 1, dx = d & 1;
        float acc = fmul(S[dy][dx], k[0]);
#pragma unroll
        for (int t = 1; t < 9; ++t) acc = fadd(acc, fmul(S[dy + t / 3][dx + t % 3], k[t]));
        c[d] = acc;
    }
    pool2[((long long)m * p2h + y) * p2w + x] = lg_pool_tanh(c, N->max_pool, N->cb[1][m], N->sw[1][m], N->sb[1][m], N->af);
}

__global__ void legacy_out_kernel(const LegacyNet* __restrict__ Np, const float* __restrict__ pool2, int p2w, int p2h, int ow, int oh,
                                  float* __restrict__ resp, int* __restrict__ counts, int chunk_base, float thr) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= ow || y >= oh) return;
    const LegacyNet& N = *Np;
    const long long plane = (long long)p2w * p2h;
    const int it2 = N.m2 >> 1, kw = N.k3w;
    float vals[kLgMaxM2];
    float acc = 0.f;
    for (int i = 0; i < it2; ++i) {
        const auto in = [&](int t) { return lg_map_sum(pool2, plane, N.m1, i, (long long)(y + t / kw) * p2w + x + t % kw); };
        const float v0 = lg_l3_value(N, 2 * i, in), v1 = lg_l3_value(N, 2 * i + 1, in);
        if (N.full_connect) {
            vals[2 * i] = v0;
            vals[2 * i + 1] = v1;
        } else {
            const float pair = fadd(v1, v0);
            acc = (i == 0) ? pair : fadd(acc, pair);
        }
    }
    if (N.full_connect)
        for (int n = 0; n < N.hl; ++n) {
            const float h = lg_hidden_fc(N, n, vals);
            acc = (n == 0) ? h : fadd(acc, h);
        }
    const float r = lg_finish(N, acc);
    resp[(long long)y * ow + x] = r;
    // candidates (response > treshold_1) counted per scan chunk, as the CNTK stage-1 back kernel does
    if (counts && r > thr) atomicAdd(&counts[chunk_base + (y * ow + x) / kCandChunk], 1);
}

}  // namespace

cudaError_t launch_legacy_forward(const LegacyNet* d_net, const LegacyNet& h_net, const float* img, int pitch, int w, int h, float* scratch,
                                  float* resp, cudaStream_t st, int* counts, int chunk_base, float thr) {
    const int p1w = (w - 3) >> 1, p1h = (h - 3) >> 1;
    const int p2w = (((w - 3) >> 1) - 2) >> 1, p2h = (((h - 3) >> 1) - 2) >> 1;
    int ow, oh;
    legacy_output_size(h_net, w, h, &ow, &oh);
    float* pool1 = scratch;
    float* pool2 = scratch + (size_t)h_net.m0 * p1w * p1h;
    const dim3 b(32, 8);
    legacy_l1_kernel<<<dim3((p1w + 31) / 32, (p1h + 7) / 8, h_net.m0), b, 0, st>>>(d_net, img, pitch, p1w, p1h, pool1);
    legacy_l2_kernel<<<dim3((p2w + 31) / 32, (p2h + 7) / 8, h_net.m1), b, 0, st>>>(d_net, pool1, p1w, p1h, p2w, p2h, pool2);
    if (ow > 0 && oh > 0) legacy_out_kernel<<<dim3((ow + 31) / 32, (oh + 7) / 8), b, 0, st>>>(d_net, pool2, p2w, p2h, ow, oh, resp, counts, chunk_base, thr);
    return cudaGetLastError();
}

size_t legacy_scratch_floats(const LegacyNet& n, int w, int h) {
    const size_t p1 = (size_t)((w - 3) >> 1) * ((h - 3) >> 1);
    const size_t p2 = (size_t)((((w - 3) >> 1) - 2) >> 1) * ((((h - 3) >> 1) - 2) >> 1);
    return (size_t)n.m0 * p1 + (size_t)n.m1 * p2;
}

}  // namespace ccnn

using namespace ccnn;

extern "C" CCNN_API ccnn_status ccnn_legacy_model_info(const char* model_path, int* info, int n_info) {
    if (!model_path || !info || n_info < 10) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    LegacyNet net;
    std::string err;
    if (!load_legacy_model_file(model_path, &net, &err)) {
        set_error(err);
        return CCNN_ERR_MODEL;
    }
    const int v[10] = {net.max_pool, net.min_w, net.min_h, net.m0, net.m1, net.m2, net.k3w, net.k3h, net.full_connect, net.hl};
    for (int i = 0; i < 10; ++i) info[i] = v[i];
    return CCNN_OK;
}

extern "C" CCNN_API ccnn_status ccnn_legacy_net_forward(const char* model_path, const float* d_img, int cols, int rows, size_t step, float* d_resp,
                                                        int resp_cap, int* ow, int* oh, void* stream) {
    if (!model_path || !d_img || !d_resp || !ow || !oh || step % sizeof(float) || step < sizeof(float) * (size_t)cols) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    LegacyNet net;
    std::string err;
    if (!load_legacy_model_file(model_path, &net, &err)) {
        set_error(err);
        return CCNN_ERR_MODEL;
    }
    if (cols < net.min_w || rows < net.min_h) {
        set_error("image is smaller than the network's input");
        return CCNN_ERR_INVALID_ARG;
    }
    legacy_output_size(net, cols, rows, ow, oh);
    if ((long long)*ow * *oh > resp_cap) {
        set_error("response buffer too small");
        return CCNN_ERR_INVALID_ARG;
    }
    const cudaStream_t st = (cudaStream_t)stream;
    void* buf = nullptr;
    const size_t scratch = legacy_scratch_floats(net, cols, rows);
    cudaError_t e = cudaMallocAsync(&buf, sizeof(LegacyNet) + sizeof(float) * scratch, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf, &net, sizeof(LegacyNet), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_legacy_forward((const LegacyNet*)buf, net, d_img, (int)(step / sizeof(float)), cols, rows,
                                  (float*)((char*)buf + sizeof(LegacyNet)), d_resp, st, nullptr, 0, 0.f);
    if (buf) {
        const cudaError_t f = cudaFreeAsync(buf, st);
        if (e == cudaSuccess) e = f;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // `net` on the host stack was copied from
    if (e != cudaSuccess) {
        set_error(std::string("legacy forward: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}
