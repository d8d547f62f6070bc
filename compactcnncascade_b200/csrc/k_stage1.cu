// Stage-1 fully-convolutional net over every pyramid level, in two launches per frame.
//
// Reference: SIMD::ConvNeuralNetwork::Run (src/CNNObjectDetector/cnn_simd_cntk.cpp:640-963) with
// the plain CNNPP primitives (cnnpp_cplusplus.cpp): conv_4x4 (:92-157), lrelu_bn_max (:593-622),
// add/add2 (:916-950), conv_3x3 (:36-91), conv_5x4 (:158-187), lrelu_bn (:623-645),
// mulCN_add_tanhW (:646-672), mulC/mulC1_add (:952-984), tanhW (:673-690).
//
// front: one CTA per 32x16 tile of pooled L1 pixels of one level. The level image is never
//        materialised: the CTA samples its (67 x 35) input tile straight from the gray frame
//        with the pyramid's fixed-point resampler, runs the 4x4 conv + folded BN/LReLU + 2x2 max
//        for the 4 L1 maps and writes the 4 neighbour-map sums that L2 consumes (S1 arena).
// back:  one CTA per 16x16 tile of response pixels. It stages the S1 tile (4 x 42 x 40) in shared
//        memory, computes the 8 pooled L2 maps and their sums on the 19 x 20 halo tile, then every
//        thread finishes one response pixel: the 16 L3 maps (4w x 5h), the 52 hidden neurons and
//        the output neuron.
// Every tile of every level is one block of the same grid; a block finds its level by binary
// search over the level table, so a frame is two launches whatever its pyramid depth.
#include "kernels.h"
#include "resample.cuh"

namespace ccnn {

__device__ __forceinline__ int find_level(const LevelDesc* __restrict__ lv, int n, int tile, bool front) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        int base = front ? lv[mid].k1_base : lv[mid].k2_base;
        if (base <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

constexpr int kInW = 2 * kK1TileX + 3;  // 67
constexpr int kInH = 2 * kK1TileY + 3;  // 35

__global__ void __launch_bounds__(256) stage1_front_kernel(const __grid_constant__ Stage1W W, const LevelDesc* __restrict__ levels,
                                                           int n_levels, const float* __restrict__ gray, int gpitch, int gw, int gh,
                                                           float* __restrict__ s1) {
    __shared__ float tin[kInH][kInW + 1];
    const int lvl = find_level(levels, n_levels, blockIdx.x, true);
    const LevelDesc L = levels[lvl];
    const int t = blockIdx.x - L.k1_base;
    const int px0 = (t % L.k1_tiles_x) * kK1TileX;
    const int py0 = (t / L.k1_tiles_x) * kK1TileY;
    const int ix0 = 2 * px0, iy0 = 2 * py0;

    for (int i = threadIdx.x; i < kInH * kInW; i += blockDim.x) {
        int r = i / kInW, c = i - r * kInW;
        int lx = ix0 + c, ly = iy0 + r;
        float v = 0.f;
        if (lx < L.w && ly < L.h) v = level_pixel(gray, gpitch, gw, gh, L, lx, ly);
        tin[r][c] = v;
    }
    __syncthreads();

    const int qx = threadIdx.x & (kK1TileX - 1);
    const int qy = (threadIdx.x >> 5) * 2;
    float win[7][5];
#pragma unroll
    for (int r = 0; r < 7; ++r)
#pragma unroll
        for (int c = 0; c < 5; ++c) win[r][c] = tin[2 * qy + r][2 * qx + c];

#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float P[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            float cv[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const int dy = d >> 1, dx = d & 1;
                float acc = fmul(win[2 * q + dy][dx], W.k1[m][0]);
#pragma unroll
                for (int k = 1; k < 16; ++k) acc = fadd(acc, fmul(win[2 * q + dy + (k >> 2)][dx + (k & 3)], W.k1[m][k]));
                cv[d] = lrelu_bn(acc, W.b1[m], W.w1a[m], W.w1b[m], W.bn1[m]);
            }
            P[m] = fmaxf(fmaxf(cv[0], cv[1]), fmaxf(cv[2], cv[3]));
        }
        const int gx = px0 + qx, gy = py0 + qy + q;
        if (gx < L.p1w && gy < L.p1h) {
            float* o = s1 + L.s1_off + (long long)gy * L.s1_pitch + gx;
            o[0] = fadd(P[0], P[1]);
            o[L.s1_plane] = fadd(fadd(P[0], P[1]), P[2]);
            o[2 * L.s1_plane] = fadd(fadd(P[1], P[2]), P[3]);
            o[3 * L.s1_plane] = fadd(P[2], P[3]);
        }
    }
}

constexpr int kP2TW = kK2TileX + 3;  // 19
constexpr int kP2TH = kK2TileY + 4;  // 20
constexpr int kS1TW = 2 * kP2TW + 2; // 40
constexpr int kS1TH = 2 * kP2TH + 2; // 42

__global__ void __launch_bounds__(256) stage1_back_kernel(const __grid_constant__ Stage1W W, const LevelDesc* __restrict__ levels,
                                                          int n_levels, const float* __restrict__ s1, float* __restrict__ resp) {
    __shared__ float ts1[4][kS1TH][kS1TW + 1];
    __shared__ float ts2[8][kP2TH][kP2TW + 1];
    const int lvl = find_level(levels, n_levels, blockIdx.x, false);
    const LevelDesc L = levels[lvl];
    const int t = blockIdx.x - L.k2_base;
    const int ox0 = (t % L.k2_tiles_x) * kK2TileX;
    const int oy0 = (t / L.k2_tiles_x) * kK2TileY;
    const int sx0 = 2 * ox0, sy0 = 2 * oy0;

    for (int i = threadIdx.x; i < 4 * kS1TH * kS1TW; i += blockDim.x) {
        int m = i / (kS1TH * kS1TW);
        int rem = i - m * (kS1TH * kS1TW);
        int r = rem / kS1TW, c = rem - r * kS1TW;
        int x = sx0 + c, y = sy0 + r;
        float v = 0.f;
        if (x < L.p1w && y < L.p1h) v = s1[L.s1_off + m * L.s1_plane + (long long)y * L.s1_pitch + x];
        ts1[m][r][c] = v;
    }
    __syncthreads();

    // pooled L2 maps and their neighbour sums on the (19 x 20) halo tile
    for (int p = threadIdx.x; p < kP2TW * kP2TH; p += blockDim.x) {
        const int x = p % kP2TW, y = p / kP2TW;
        float P[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float q[4][4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) q[r][c] = ts1[i][2 * y + r][2 * x + c];
#pragma unroll
            for (int hm = 0; hm < 2; ++hm) {
                const int m = 2 * i + hm;
                float cv[4];
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    const int dy = d >> 1, dx = d & 1;
                    float acc = fmul(q[dy][dx], W.k2[m][0]);
#pragma unroll
                    for (int k = 1; k < 9; ++k) acc = fadd(acc, fmul(q[dy + k / 3][dx + k % 3], W.k2[m][k]));
                    cv[d] = lrelu_bn(acc, W.b2[m], W.w2a[m], W.w2b[m], W.bn2[m]);
                }
                P[m] = fmaxf(fmaxf(cv[0], cv[1]), fmaxf(cv[2], cv[3]));
            }
        }
        ts2[0][y][x] = fadd(P[0], P[1]);
#pragma unroll
        for (int k = 1; k < 7; ++k) ts2[k][y][x] = fadd(fadd(P[k - 1], P[k]), P[k + 1]);
        ts2[7][y][x] = fadd(P[6], P[7]);
    }
    __syncthreads();

    const int x = threadIdx.x & (kK2TileX - 1), y = threadIdx.x / kK2TileX;
    float A[16];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float q[5][4];
#pragma unroll
        for (int r = 0; r < 5; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) q[r][c] = ts2[i][y + r][x + c];
#pragma unroll
        for (int hm = 0; hm < 2; ++hm) {
            const int m = 2 * i + hm;
            // conv_5x4 keeps one partial sum per kernel row, added in row order
            float acc = 0.f;
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                float rs = fmul(q[r][0], W.k3[m][4 * r]);
#pragma unroll
                for (int c = 1; c < 4; ++c) rs = fadd(rs, fmul(q[r][c], W.k3[m][4 * r + c]));
                acc = (r == 0) ? rs : fadd(acc, rs);
            }
            A[m] = lrelu_bn(acc, W.b3[m], W.w3a[m], W.w3b[m], W.bn3[m]);
        }
    }
    // hidden neurons n = 4*i + t read L3 maps i..i+3; the output sum runs in the same n order
    float out = 0.f;
#pragma unroll
    for (int i = 0; i < Stage1W::kGroups; ++i) {
#pragma unroll
        for (int tt = 0; tt < Stage1W::kHS; ++tt) {
            const int n = Stage1W::kHS * i + tt;
            float s = W.hb[n];
#pragma unroll
            for (int j = 0; j < Stage1W::kConn; ++j) s = fadd(s, fmul(A[i + j], W.hw[n][j]));
            s = fmul(s, W.htw[i]);
            s = tanh_rational(s);
            s = fadd(fmul(0.5f, s), 0.5f);
            const float h = fadd(fmul(W.hbnw[tt], s), W.hbnb[tt]);
            out = (n == 0) ? fmul(h, W.ow[0]) : fadd(fmul(h, W.ow[n]), out);
        }
    }
    float c = fmul(fadd(out, W.ob), W.otw);
    c = tanh_rational(c);
    const float r = (W.af == 0.f) ? fadd(fmul(0.5f, c), 0.5f) : fmul(W.af, c);
    const int gx = ox0 + x, gy = oy0 + y;
    if (gx < L.ow && gy < L.oh) resp[L.resp_off + (long long)gy * L.ow + gx] = r;
}

cudaError_t launch_stage1_front(const Stage1W& W, const LevelDesc* d_levels, int n_levels, int k1_tiles, const float* gray, int gpitch,
                                int gw, int gh, float* s1, cudaStream_t st) {
    if (k1_tiles > 0) stage1_front_kernel<<<k1_tiles, 256, 0, st>>>(W, d_levels, n_levels, gray, gpitch, gw, gh, s1);
    return cudaGetLastError();
}

cudaError_t launch_stage1_back(const Stage1W& W, const LevelDesc* d_levels, int n_levels, int k2_tiles, const float* s1, float* resp,
                               cudaStream_t st) {
    if (k2_tiles > 0) stage1_back_kernel<<<k2_tiles, 256, 0, st>>>(W, d_levels, n_levels, s1, resp);
    return cudaGetLastError();
}

cudaError_t launch_stage1(const Stage1W& W, const LevelDesc* d_levels, int n_levels, int k1_tiles, int k2_tiles, const float* gray,
                          int gpitch, int gw, int gh, float* s1, float* resp, cudaStream_t st) {
    cudaError_t e = launch_stage1_front(W, d_levels, n_levels, k1_tiles, gray, gpitch, gw, gh, s1, st);
    if (e != cudaSuccess) return e;
    return launch_stage1_back(W, d_levels, n_levels, k2_tiles, s1, resp, st);
}

}  // namespace ccnn
