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
constexpr int kInWh = (kInW + 1) / 2;   // 34 columns of each parity

// Tile layout for the front kernel: row r of the input tile is stored next to row r+2 as a packed
// pair (a thread computes two vertically adjacent pooled pixels, whose windows are 2 rows apart),
// and columns are split by parity so that the stride-2 column walk of a warp is conflict-free.
__global__ void __launch_bounds__(256, 4) stage1_front_kernel(const __grid_constant__ Stage1W W, const LevelDesc* __restrict__ levels,
                                                              int n_levels, const float* __restrict__ gray, int gpitch, int gw, int gh,
                                                              float* __restrict__ s1) {
    __shared__ float2 tinp[kInH - 2][2][kInWh];
    __shared__ float tin_tail[2][kInW];        // the last two rows have no partner below
    __shared__ uint32_t col_idx[kInW], row_idx[kInH];
    __shared__ float col_f[kInW], col_c[kInW], row_f[kInH], row_c[kInH];
    const int lvl = find_level(levels, n_levels, blockIdx.x, true);
    const LevelDesc L = levels[lvl];
    const int t = blockIdx.x - L.k1_base;
    const int px0 = (t % L.k1_tiles_x) * kK1TileX;
    const int py0 = (t / L.k1_tiles_x) * kK1TileY;
    const int ix0 = 2 * px0, iy0 = 2 * py0;

    // per-tile sampling table: one column / row of the resampler each
    if (L.mode != 0) {
        if (threadIdx.x < kInW) {
            const AxisSample sx = sample_col(ix0 + threadIdx.x, L.sclx, gw);
            col_idx[threadIdx.x] = sx.idx;
            col_f[threadIdx.x] = sx.f;
            col_c[threadIdx.x] = sx.c;
        } else if (threadIdx.x >= 128 && threadIdx.x < 128 + kInH) {
            const int r = threadIdx.x - 128;
            const AxisSample sy = sample_row(iy0 + r, L.scly, gh);
            uint32_t py = sy.idx;
            if (L.mode == 2 && py + 1 >= (uint32_t)gh) py--;  // bilinear keeps a row below
            row_idx[r] = py;
            row_f[r] = sy.f;
            row_c[r] = sy.c;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kInH * kInW; i += blockDim.x) {
        const int r = i / kInW, c = i - r * kInW;
        const int lx = ix0 + c, ly = iy0 + r;
        float v = 0.f;
        if (lx < L.w && ly < L.h) {
            if (L.mode == 0) {
                v = gray[(size_t)ly * gpitch + lx];
            } else if (L.mode == 1) {
                v = gray[(size_t)row_idx[r] * gpitch + col_idx[c]];
            } else {
                const float* r0 = gray + (size_t)row_idx[r] * gpitch + col_idx[c];
                const float top = fadd(fmul(r0[0], col_c[c]), fmul(r0[1], col_f[c]));
                const float bot = fadd(fmul(r0[gpitch], col_c[c]), fmul(r0[gpitch + 1], col_f[c]));
                v = fadd(fmul(top, row_c[r]), fmul(bot, row_f[r]));
            }
        }
        float* lo = r < kInH - 2 ? &tinp[r][c & 1][c >> 1].x : &tin_tail[r - (kInH - 2)][c];
        *lo = v;
        if (r >= 2) tinp[r - 2][c & 1][c >> 1].y = v;
    }
    __syncthreads();

    const int qx = threadIdx.x & (kK1TileX - 1);
    const int qy = (threadIdx.x >> 5) * 2;
    const f2_t nz = f2_ld(W.negzero);
    // pr[r][c] = (input row 2qy+r, row 2qy+r+2) at column 2qx+c: the windows of both pixels
    f2_t pr[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int c = 0; c < 5; ++c) pr[r][c] = *reinterpret_cast<const f2_t*>(&tinp[2 * qy + r][c & 1][qx + (c >> 1)]);

    float P[2][4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float cv[2][4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int dy = d >> 1, dx = d & 1;
            f2_t acc = f2_mul(pr[dy][dx], f2_ld(W.k1d[m][0]), nz);
#pragma unroll
            for (int k = 1; k < 16; ++k)
                acc = f2_add(acc, f2_mul(pr[dy + (k >> 2)][dx + (k & 3)], f2_ld(W.k1d[m][k]), nz));
            cv[0][d] = lrelu_bn(f2_lo(acc), W.b1[m], W.w1a[m], W.w1b[m], W.bn1[m]);
            cv[1][d] = lrelu_bn(f2_hi(acc), W.b1[m], W.w1a[m], W.w1b[m], W.bn1[m]);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) P[q][m] = fmaxf(fmaxf(cv[q][0], cv[q][1]), fmaxf(cv[q][2], cv[q][3]));
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int gx = px0 + qx, gy = py0 + qy + q;
        if (gx < L.p1w && gy < L.p1h) {
            float* o = s1 + L.s1_off + (long long)gy * L.s1_pitch + gx;
            o[0] = fadd(P[q][0], P[q][1]);
            o[L.s1_plane] = fadd(fadd(P[q][0], P[q][1]), P[q][2]);
            o[2 * L.s1_plane] = fadd(fadd(P[q][1], P[q][2]), P[q][3]);
            o[3 * L.s1_plane] = fadd(P[q][2], P[q][3]);
        }
    }
}

constexpr int kP2TW = kK2TileX + 3;  // 19
constexpr int kP2TH = kK2TileY + 4;  // 20
constexpr int kS1TW = 2 * kP2TW + 2; // 40
constexpr int kS1TH = 2 * kP2TH + 2; // 42
constexpr int kS1TWh = kS1TW / 2 + 1; // 21 columns of each parity (+1 pad)

__global__ void __launch_bounds__(256) stage1_back_kernel(const __grid_constant__ Stage1W W, const LevelDesc* __restrict__ levels,
                                                          int n_levels, const float* __restrict__ s1, float* __restrict__ resp) {
    __shared__ float ts1[4][kS1TH][2 * kS1TWh];  // column c stored at (c & 1) * kS1TWh + (c >> 1)
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
        ts1[m][r][(c & 1) * kS1TWh + (c >> 1)] = v;
    }
    __syncthreads();

    const f2_t nz = f2_ld(W.negzero);
    // pooled L2 maps and their neighbour sums on the (19 x 20) halo tile; maps 2i and 2i+1 read the
    // same sum map i, so they run as one packed pair
    for (int p = threadIdx.x; p < kP2TW * kP2TH; p += blockDim.x) {
        const int x = p % kP2TW, y = p / kP2TW;
        float P[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            f2_t q[4][4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) q[r][c] = f2_dup(ts1[i][2 * y + r][(c & 1) * kS1TWh + x + (c >> 1)]);
            float cv[2][4];
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const int dy = d >> 1, dx = d & 1;
                f2_t acc = f2_mul(q[dy][dx], f2_ld(W.k2p[i][0]), nz);
#pragma unroll
                for (int k = 1; k < 9; ++k) acc = f2_add(acc, f2_mul(q[dy + k / 3][dx + k % 3], f2_ld(W.k2p[i][k]), nz));
                cv[0][d] = lrelu_bn(f2_lo(acc), W.b2[2 * i], W.w2a[2 * i], W.w2b[2 * i], W.bn2[2 * i]);
                cv[1][d] = lrelu_bn(f2_hi(acc), W.b2[2 * i + 1], W.w2a[2 * i + 1], W.w2b[2 * i + 1], W.bn2[2 * i + 1]);
            }
            P[2 * i] = fmaxf(fmaxf(cv[0][0], cv[0][1]), fmaxf(cv[0][2], cv[0][3]));
            P[2 * i + 1] = fmaxf(fmaxf(cv[1][0], cv[1][1]), fmaxf(cv[1][2], cv[1][3]));
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
        f2_t q[5][4];
#pragma unroll
        for (int r = 0; r < 5; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) q[r][c] = f2_dup(ts2[i][y + r][x + c]);
        // conv_5x4 keeps one partial sum per kernel row, added in row order
        f2_t acc = 0ull;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            f2_t rs = f2_mul(q[r][0], f2_ld(W.k3p[i][4 * r]), nz);
#pragma unroll
            for (int c = 1; c < 4; ++c) rs = f2_add(rs, f2_mul(q[r][c], f2_ld(W.k3p[i][4 * r + c]), nz));
            acc = (r == 0) ? rs : f2_add(acc, rs);
        }
        A[2 * i] = lrelu_bn(f2_lo(acc), W.b3[2 * i], W.w3a[2 * i], W.w3b[2 * i], W.bn3[2 * i]);
        A[2 * i + 1] = lrelu_bn(f2_hi(acc), W.b3[2 * i + 1], W.w3a[2 * i + 1], W.w3b[2 * i + 1], W.bn3[2 * i + 1]);
    }
    // hidden neurons n = 4*i + t read L3 maps i..i+3 (neurons 2p, 2p+1 share them: packed); the
    // output sum then runs over n in order
    f2_t Ad[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) Ad[m] = f2_dup(A[m]);
    float out = 0.f;
#pragma unroll
    for (int i = 0; i < Stage1W::kGroups; ++i) {
#pragma unroll
        for (int tp = 0; tp < Stage1W::kHS / 2; ++tp) {
            const int n = Stage1W::kHS * i + 2 * tp;
            f2_t s = f2_pack(W.hb[n], W.hb[n + 1]);
#pragma unroll
            for (int j = 0; j < Stage1W::kConn; ++j) s = f2_add(s, f2_mul(Ad[i + j], f2_ld(W.hwp[n / 2][j]), nz));
            s = f2_mul(s, f2_dup(W.htw[i]), nz);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int tt = 2 * tp + e;
                float v = tanh_rational(e == 0 ? f2_lo(s) : f2_hi(s));
                v = fadd(fmul(0.5f, v), 0.5f);
                const float h = fadd(fmul(W.hbnw[tt], v), W.hbnb[tt]);
                out = (n + e == 0) ? fmul(h, W.ow[0]) : fadd(fmul(h, W.ow[n + e]), out);
            }
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
