// Learned scale/region gate: a small network on a 1/8-resolution gray frame that predicts, per
// pyramid octave and per 16x16 cell of the frame, whether the plain cascade's stage 2/3 will accept
// a window centred there. Stage-1 tiles whose footprint holds no likely cell are skipped.
//
// No reference counterpart: this is an addition to the cascade, evaluated against the plain (full
// scan) cascade by box recall. Network (fp16 storage, fp32 accumulation):
//   f  = (8x8 box average of the gray frame - 128) / 64             (W/8 x H/8, 1 channel)
//   a1 = LReLU_0.1(conv3x3(f; 8 maps) + b1)                          (zero padding)
//   a2 = LReLU_0.1(conv3x3(a1; 8 -> 8 maps) + b2)
//   q  = 2x2 average of a2                                          (W/16 x H/16 cells)
//   p  = sigmoid(W3 q + b3), one output per octave (kGK)
// Training minimises the positive-weighted binary cross-entropy over all cells with Adam; the
// forward, backward and optimiser kernels below are the whole training step.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/ccnn_gate.h"
#include "kernels.h"

namespace ccnn {

void set_error(const std::string& msg);

namespace {

constexpr int kGC = 8;  // channels
constexpr int kW1 = 0, kB1 = kW1 + kGC * 9, kW2 = kB1 + kGC, kB2 = kW2 + kGC * kGC * 9, kW3 = kB2 + kGC, kB3 = kW3 + kGK * kGC;
static_assert(kB3 + kGK == kGateParams, "gate parameter layout");

__device__ __forceinline__ float lrelu(float z) { return z > 0.f ? z : 0.1f * z; }
__device__ __forceinline__ float dlrelu(float a) { return a > 0.f ? 1.f : 0.1f; }  // a has the sign of z

// (8x8 box average of the gray frame - 128) / 64 (rows/columns past the last whole block are not used)
__global__ void gate_features_kernel(const float* __restrict__ gray, int pitch, int w8, int h8, __half* __restrict__ f) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w8 || y >= h8) return;
    float s = 0.f;
    for (int r = 0; r < 8; ++r) {
        const float* row = gray + (size_t)(8 * y + r) * pitch + 8 * x;
#pragma unroll
        for (int c = 0; c < 8; ++c) s += row[c];
    }
    f[(size_t)y * w8 + x] = __float2half((s * (1.f / 64.f) - 128.f) * (1.f / 64.f));
}

// a1 for every frame of the batch: one thread per pixel, 8 channels
__global__ void gate_fwd1_kernel(const float* __restrict__ P, const __half* __restrict__ f, int n, int w8, int h8, __half* __restrict__ a1) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long plane = (long long)w8 * h8;
    if (i >= n * plane) return;
    const int fr = (int)(i / plane), p = (int)(i - fr * plane);
    const int y = p / w8, x = p - y * w8;
    const __half* F = f + fr * plane;
    float v[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int yy = y + k / 3 - 1, xx = x + k % 3 - 1;
        v[k] = (yy >= 0 && yy < h8 && xx >= 0 && xx < w8) ? __half2float(F[yy * w8 + xx]) : 0.f;
    }
#pragma unroll
    for (int c = 0; c < kGC; ++c) {
        float z = P[kB1 + c];
#pragma unroll
        for (int k = 0; k < 9; ++k) z += P[kW1 + c * 9 + k] * v[k];
        a1[((long long)fr * kGC + c) * plane + p] = __float2half(lrelu(z));
    }
}

__global__ void gate_fwd2_kernel(const float* __restrict__ P, const __half* __restrict__ a1, int n, int w8, int h8, __half* __restrict__ a2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long plane = (long long)w8 * h8;
    if (i >= n * plane) return;
    const int fr = (int)(i / plane), p = (int)(i - fr * plane);
    const int y = p / w8, x = p - y * w8;
    float z[kGC];
#pragma unroll
    for (int c = 0; c < kGC; ++c) z[c] = P[kB2 + c];
    for (int ci = 0; ci < kGC; ++ci) {
        const __half* A = a1 + ((long long)fr * kGC + ci) * plane;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const int yy = y + k / 3 - 1, xx = x + k % 3 - 1;
            const float v = (yy >= 0 && yy < h8 && xx >= 0 && xx < w8) ? __half2float(A[yy * w8 + xx]) : 0.f;
#pragma unroll
            for (int c = 0; c < kGC; ++c) z[c] += P[kW2 + (c * kGC + ci) * 9 + k] * v;
        }
    }
#pragma unroll
    for (int c = 0; c < kGC; ++c) a2[((long long)fr * kGC + c) * plane + p] = __float2half(lrelu(z[c]));
}

// pooled cells and the head: probabilities (inference) or loss, logit gradients and the head's
// weight gradients (training). One thread per cell.
__global__ void gate_head_kernel(const float* __restrict__ P, const __half* __restrict__ a2, int n, int w8, int h8,
                                 const uint8_t* __restrict__ labels, float pos_weight, float inv_cells, float* __restrict__ gq,
                                 float* __restrict__ grad, float* __restrict__ loss, float* __restrict__ prob, float amb_lo, float amb_hi,
                                 int* __restrict__ ambiguous) {
    const int w16 = w8 / 2, h16 = h8 / 2;
    const long long cells = (long long)w16 * h16, plane = (long long)w8 * h8;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ float sg[kGK * (kGC + 1)];
    __shared__ float sl;
    if (grad) {
        for (int k = threadIdx.x; k < kGK * (kGC + 1); k += blockDim.x) sg[k] = 0.f;
        if (threadIdx.x == 0) sl = 0.f;
        __syncthreads();
    }
    const bool live = i < n * cells;
    if (live) {
        const int fr = (int)(i / cells), cidx = (int)(i - fr * cells);
        const int Y = cidx / w16, X = cidx - Y * w16;
        float q[kGC];
#pragma unroll
        for (int c = 0; c < kGC; ++c) {
            const __half* A = a2 + ((long long)fr * kGC + c) * plane;
            q[c] = 0.25f * (__half2float(A[(2 * Y) * w8 + 2 * X]) + __half2float(A[(2 * Y) * w8 + 2 * X + 1]) +
                            __half2float(A[(2 * Y + 1) * w8 + 2 * X]) + __half2float(A[(2 * Y + 1) * w8 + 2 * X + 1]));
        }
        float gqc[kGC];
#pragma unroll
        for (int c = 0; c < kGC; ++c) gqc[c] = 0.f;
        int amb = 0;
        for (int k = 0; k < kGK; ++k) {
            float z = P[kB3 + k];
#pragma unroll
            for (int c = 0; c < kGC; ++c) z += P[kW3 + k * kGC + c] * q[c];
            const float p = 1.f / (1.f + expf(-z));
            const long long o = ((long long)fr * kGK + k) * cells + cidx;
            if (prob) prob[o] = p;
            if (p >= amb_lo && p < amb_hi) amb++;
            if (grad) {
                const float yv = labels[o] ? 1.f : 0.f;
                // positive-weighted binary cross-entropy on the logit
                const float lp = fminf(-logf(fmaxf(p, 1e-7f)), 30.f), ln = fminf(-logf(fmaxf(1.f - p, 1e-7f)), 30.f);
                atomicAdd(&sl, (pos_weight * yv * lp + (1.f - yv) * ln) * inv_cells);
                const float g = (p * (pos_weight * yv + 1.f - yv) - pos_weight * yv) * inv_cells;
#pragma unroll
                for (int c = 0; c < kGC; ++c) {
                    atomicAdd(&sg[k * (kGC + 1) + c], g * q[c]);
                    gqc[c] += g * P[kW3 + k * kGC + c];
                }
                atomicAdd(&sg[k * (kGC + 1) + kGC], g);
            }
        }
        if (ambiguous && amb) atomicAdd(ambiguous, amb);
        if (grad)
#pragma unroll
            for (int c = 0; c < kGC; ++c) gq[((long long)fr * kGC + c) * cells + cidx] = gqc[c];
    }
    if (grad) {
        __syncthreads();
        for (int k = threadIdx.x; k < kGK * kGC; k += blockDim.x) atomicAdd(&grad[kW3 + k], sg[(k / kGC) * (kGC + 1) + k % kGC]);
        for (int k = threadIdx.x; k < kGK; k += blockDim.x) atomicAdd(&grad[kB3 + k], sg[k * (kGC + 1) + kGC]);
        if (threadIdx.x == 0) atomicAdd(loss, sl);
    }
}

// gz2 = d loss / d z2 per pixel (the pooled gradient spread over its 2x2 pixels)
__global__ void gate_bwd2a_kernel(const __half* __restrict__ a2, const float* __restrict__ gq, int n, int w8, int h8, float* __restrict__ gz2) {
    const long long plane = (long long)w8 * h8;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kGC * plane) return;
    const long long fc = i / plane;
    const int p = (int)(i - fc * plane);
    const int y = p / w8, x = p - y * w8;
    const int w16 = w8 / 2, h16 = h8 / 2;
    float g = 0.f;
    if (y < 2 * h16 && x < 2 * w16) g = 0.25f * gq[fc * (long long)(w16 * h16) + (y / 2) * w16 + x / 2] * dlrelu(__half2float(a2[i]));
    gz2[i] = g;
}

// ga1 = conv-transpose of gz2 with W2, then gz1 = ga1 * LReLU'(z1)
__global__ void gate_bwd1a_kernel(const float* __restrict__ P, const __half* __restrict__ a1, const float* __restrict__ gz2, int n, int w8, int h8,
                                  float* __restrict__ gz1) {
    const long long plane = (long long)w8 * h8;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * plane) return;
    const int fr = (int)(i / plane), p = (int)(i - fr * plane);
    const int y = p / w8, x = p - y * w8;
    float ga[kGC];
#pragma unroll
    for (int c = 0; c < kGC; ++c) ga[c] = 0.f;
    for (int co = 0; co < kGC; ++co) {
        const float* G = gz2 + ((long long)fr * kGC + co) * plane;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            // z2 at (y - dy, x - dx) read a1 at (y, x) with tap k = (dy + 1, dx + 1)
            const int yy = y - (k / 3 - 1), xx = x - (k % 3 - 1);
            const float g = (yy >= 0 && yy < h8 && xx >= 0 && xx < w8) ? G[yy * w8 + xx] : 0.f;
#pragma unroll
            for (int ci = 0; ci < kGC; ++ci) ga[ci] += P[kW2 + (co * kGC + ci) * 9 + k] * g;
        }
    }
#pragma unroll
    for (int c = 0; c < kGC; ++c) {
        const long long o = ((long long)fr * kGC + c) * plane + p;
        gz1[o] = ga[c] * dlrelu(__half2float(a1[o]));
    }
}

// weight gradient of a 3x3 convolution: grad[W(co, ci, k)] += sum over pixels of
// gz[co](y, x) * in[ci](y + dy, x + dx); one block per (frame, row band), one thread per weight
template <int CIN>
__global__ void gate_wgrad_kernel(const float* __restrict__ gz, const __half* __restrict__ in, int n, int w8, int h8, int rows, float* __restrict__ gw,
                                  float* __restrict__ gb) {
    const long long plane = (long long)w8 * h8;
    const int fr = blockIdx.y, y0 = blockIdx.x * rows;
    const int y1 = min(y0 + rows, h8);
    constexpr int kParams = kGC * CIN * 9;
    for (int t = threadIdx.x; t < kParams + kGC; t += blockDim.x) {
        float s = 0.f;
        if (t < kParams) {
            const int co = t / (CIN * 9), ci = (t / 9) % CIN, k = t % 9;
            const int dy = k / 3 - 1, dx = k % 3 - 1;
            const float* G = gz + ((long long)fr * kGC + co) * plane;
            const __half* I = in + ((long long)fr * CIN + ci) * plane;
            for (int y = y0; y < y1; ++y) {
                const int yy = y + dy;
                if (yy < 0 || yy >= h8) continue;
                for (int x = 0; x < w8; ++x) {
                    const int xx = x + dx;
                    if (xx >= 0 && xx < w8) s += G[y * w8 + x] * __half2float(I[yy * w8 + xx]);
                }
            }
            atomicAdd(&gw[t], s);
        } else {
            const int co = t - kParams;
            const float* G = gz + ((long long)fr * kGC + co) * plane;
            for (int y = y0; y < y1; ++y)
                for (int x = 0; x < w8; ++x) s += G[y * w8 + x];
            atomicAdd(&gb[co], s);
        }
    }
}

__global__ void gate_adam_kernel(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr,
                                 float b1t, float b2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGateParams) return;
    const float gi = g[i];
    m[i] = 0.9f * m[i] + 0.1f * gi;
    v[i] = 0.999f * v[i] + 0.001f * gi * gi;
    const float mh = m[i] / (1.f - b1t), vh = v[i] / (1.f - b2t);
    P[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ---- inference inside the detector ----

namespace {

// One launch for the whole network on a frame: each block computes a tile of kIX x kIY a2 pixels
// (kIX/2 x kIY/2 cells) from the frame's binary16 input features (written by the gray-conversion
// launch, or by gate_features_kernel), with the same fp16 storage points as the training forward
// (f, a1 and a2 rounded to binary16), writes the octave probabilities and sets the cell's bit in the
// per-octave row bitmaps when the probability reaches the threshold.
constexpr int kIX = 16, kIY = 8;
constexpr int kFX = kIX + 4, kFY = kIY + 4, kAX = kIX + 2, kAY = kIY + 2;

__global__ void __launch_bounds__(256) gate_infer_kernel(const __grid_constant__ GateNet P, const __half* __restrict__ feat, int w8, int h8,
                                                         float thr, float amb_lo, uint32_t* __restrict__ bits, int wwords,
                                                         float* __restrict__ prob, int* __restrict__ ambiguous) {
    const float* sp = P.p;  // the parameters travel in the constant bank (warp-uniform reads)
    __shared__ __half sf[kFY][kFX];
    __shared__ __half sa1[kGC][kAY][kAX];
    __shared__ __half sa2[kGC][kIY][kIX];
    __shared__ int samb;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kIX, y0 = blockIdx.y * kIY;
    if (tid == 0) samb = 0;
    if (tid < kFX * kFY) {
        const int fx = x0 - 2 + tid % kFX, fy = y0 - 2 + tid / kFX;
        // zero padding of the first convolution
        sf[tid / kFX][tid % kFX] = (fx >= 0 && fx < w8 && fy >= 0 && fy < h8) ? feat[(size_t)fy * w8 + fx] : __float2half(0.f);
    }
    __syncthreads();
    if (tid < kAX * kAY) {
        const int ax = tid % kAX, ay = tid / kAX;
        const int gx = x0 - 1 + ax, gy = y0 - 1 + ay;
        const bool in = gx >= 0 && gx < w8 && gy >= 0 && gy < h8;  // zero padding of the second convolution
        float v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = __half2float(sf[ay + k / 3][ax + k % 3]);
#pragma unroll
        for (int c = 0; c < kGC; ++c) {
            float z = sp[kB1 + c];
#pragma unroll
            for (int k = 0; k < 9; ++k) z += sp[kW1 + c * 9 + k] * v[k];
            sa1[c][ay][ax] = __float2half(in ? lrelu(z) : 0.f);
        }
    }
    __syncthreads();
    {
        // warp co computes output map co; lane l four a2 pixels of column l % 16 (rows 4 (l / 16) ..
        // + 3), the map's 72 weights held in registers; every output sums its (ci, tap) products in
        // the training forward's order
        static_assert(kIX == 16 && kIY == 8 && kGC == 8, "one warp per map, 16 columns x 2 row groups of 4");
        const int co = tid >> 5, lane = tid & 31;
        const int ix = lane & 15, iy0 = (lane >> 4) * 4;
        float wt[kGC * 9];
#pragma unroll
        for (int k = 0; k < kGC * 9; ++k) wt[k] = sp[kW2 + co * kGC * 9 + k];
        float z[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) z[j] = sp[kB2 + co];
#pragma unroll
        for (int ci = 0; ci < kGC; ++ci) {
            float v[6][3];
#pragma unroll
            for (int r = 0; r < 6; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) v[r][c] = __half2float(sa1[ci][iy0 + r][ix + c]);
#pragma unroll
            for (int k = 0; k < 9; ++k)
#pragma unroll
                for (int j = 0; j < 4; ++j) z[j] += wt[ci * 9 + k] * v[j + k / 3][k % 3];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) sa2[co][iy0 + j][ix] = __float2half(lrelu(z[j]));
    }
    __syncthreads();
    const int w16 = w8 / 2, h16 = h8 / 2;
    constexpr int kCX = kIX / 2, kCY = kIY / 2;
    if (tid < kCX * kCY * kGK) {
        const int cell = tid % (kCX * kCY), k = tid / (kCX * kCY);
        const int cx = cell % kCX, cy = cell / kCX;
        const int X = x0 / 2 + cx, Y = y0 / 2 + cy;
        if (X < w16 && Y < h16) {
            float z = sp[kB3 + k];
#pragma unroll
            for (int c = 0; c < kGC; ++c) {
                const float q = 0.25f * (__half2float(sa2[c][2 * cy][2 * cx]) + __half2float(sa2[c][2 * cy][2 * cx + 1]) +
                                         __half2float(sa2[c][2 * cy + 1][2 * cx]) + __half2float(sa2[c][2 * cy + 1][2 * cx + 1]));
                z += sp[kW3 + k * kGC + c] * q;
            }
            const float p = 1.f / (1.f + expf(-z));
            prob[((long long)k * h16 + Y) * w16 + X] = p;
            if (p >= thr)
                atomicOr(&bits[((long long)k * h16 + Y) * wwords + X / 32], 1u << (X % 32));
            else if (p >= amb_lo)
                atomicAdd(&samb, 1);
        }
    }
    __syncthreads();
    if (tid == 0 && samb) atomicAdd(ambiguous, samb);
}

// cells within `m` pixels of the window centres ((4*o + 11.5) / s, (4*o + 13.5) / s) of the
// response pixels o in [ox0, ox1] x [oy0, oy1] of a level
__device__ __forceinline__ void centre_cells(const LevelDesc& L, int ox0, int ox1, int oy0, int oy1, int w16, int h16, int m, int* r) {
    r[0] = gate_cell_lo((int)((4.f * ox0 + 11.5f) * L.inv_scale), m);
    r[1] = gate_cell_hi((int)((4.f * ox1 + 11.5f) * L.inv_scale), m, w16);
    r[2] = gate_cell_lo((int)((4.f * oy0 + 13.5f) * L.inv_scale), m);
    r[3] = gate_cell_hi((int)((4.f * oy1 + 13.5f) * L.inv_scale), m, h16);
}

// Tile activity for one group of levels: threads [0, nb) decide the back tiles (32x16 response
// pixels: active when a likely cell of the level's octave lies within `margin` pixels of their window centres), the
// rest the front tiles (active when a back tile that reads their S1 pixels can be: the union of
// those back tiles' cell ranges is tested). A frame with too many ambiguous cells runs in full.
// The bitmaps are staged in shared memory first (a query walks up to a few dozen rows, which as
// dependent global loads took longer than the rest of the kernel); frames whose bitmaps exceed
// kMaskSmemWords read them from global memory.
constexpr int kMaskSmemWords = 12288;

__global__ void gate_mask_kernel(const __grid_constant__ LevelTable LT, int nb, const uint32_t* __restrict__ gbits, int n_words, int wwords,
                                 int w16, int h16, int margin, const int* __restrict__ ambiguous, int amb_limit, uint8_t* __restrict__ back_on,
                                 uint8_t* __restrict__ front_on) {
    extern __shared__ uint32_t sbits[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const LevelDesc& last = LT.lv[LT.n - 1];
    const bool full = *ambiguous > amb_limit;
    const bool staged = n_words <= kMaskSmemWords;
    if (staged && !full) {
        for (int k = threadIdx.x; k < n_words; k += blockDim.x) sbits[k] = gbits[k];
        __syncthreads();  // `full` is uniform over the grid
    }
    const uint32_t* bits = staged ? sbits : gbits;
    if (i < nb) {
        const int g = LT.lv[0].k2_base + i;
        if (full) {
            back_on[g] = 1;
            return;
        }
        const LevelDesc& L = LT.lv[find_level<&LevelDesc::k2_base>(LT, g)];
        const int t = g - L.k2_base;
        const int ox0 = (t % L.k2_tiles_x) * kK2TileX, oy0 = (t / L.k2_tiles_x) * kK2TileY;
        int r[4];
        centre_cells(L, ox0, min(ox0 + kK2TileX, L.ow) - 1, oy0, min(oy0 + kK2TileY, L.oh) - 1, w16, h16, margin, r);
        back_on[g] = gate_any_bit(bits + (long long)min(L.octave, kGK - 1) * h16 * wwords, wwords, r[0], r[1], r[2], r[3]) ? 1 : 0;
        return;
    }
    const int g = LT.lv[0].k1_base + (i - nb);
    if (g >= last.k1_base + last.k1_tiles_x * ((last.p1h + kK1TileY - 1) / kK1TileY)) return;
    if (full) {
        front_on[g] = 1;
        return;
    }
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::k1_base>(LT, g)];
    const int t = g - L.k1_base;
    const int px0 = (t % L.k1_tiles_x) * kK1TileX, py0 = (t / L.k1_tiles_x) * kK1TileY;
    // back tile (bx, by) reads S1 columns [64 bx, 64 bx + 72) and rows [32 by, 32 by + 42)
    const int ty = (L.oh + kK2TileY - 1) / kK2TileY;
    const int bx0 = max(0, (px0 - 71 + 2 * kK2TileX - 1) / (2 * kK2TileX)), bx1 = min(L.k2_tiles_x - 1, (px0 + kK1TileX - 1) / (2 * kK2TileX));
    const int by0 = max(0, (py0 - 41 + 2 * kK2TileY - 1) / (2 * kK2TileY)), by1 = min(ty - 1, (py0 + kK1TileY - 1) / (2 * kK2TileY));
    if (bx0 > bx1 || by0 > by1) {
        front_on[g] = 0;
        return;
    }
    int r[4];
    centre_cells(L, bx0 * kK2TileX, min((bx1 + 1) * kK2TileX, L.ow) - 1, by0 * kK2TileY, min((by1 + 1) * kK2TileY, L.oh) - 1, w16, h16, margin,
                 r);
    front_on[g] = gate_any_bit(bits + (long long)min(L.octave, kGK - 1) * h16 * wwords, wwords, r[0], r[1], r[2], r[3]) ? 1 : 0;
}

}  // namespace

GateCells gate_cells(GateScratch sc, int gw, int gh, float amb_frac, int margin) {
    const int w16 = (gw / 8) / 2, h16 = (gh / 8) / 2;
    GateCells c;
    c.margin = margin;
    c.bits = sc.bits;
    c.ambiguous = sc.ambiguous;
    c.amb_limit = (int)(amb_frac * (float)(w16 * h16 * kGK));
    c.wwords = (w16 + 31) / 32;
    c.w16 = w16;
    c.h16 = h16;
    return c;
}

int gate_bitmap_words(int gw, int gh) {
    const int w16 = (gw / 8) / 2, h16 = (gh / 8) / 2;
    return kGK * h16 * ((w16 + 31) / 32);
}

cudaError_t launch_gate(const GateNet& net, const float* gray, int gpitch, int gw, int gh, bool feat_ready, const LevelDesc* levels,
                        int n_levels, GateScratch sc, float thr, float amb_frac, int margin, uint8_t* back_on, uint8_t* front_on,
                        cudaStream_t st) {
    const int w8 = gw / 8, h8 = gh / 8, w16 = w8 / 2, h16 = h8 / 2;
    const int wwords = (w16 + 31) / 32;
    // the ambiguous-cell counter and the bitmaps right behind it are one zeroed range
    cudaError_t e = cudaMemsetAsync(sc.ambiguous, 0, sizeof(uint32_t) * ((size_t)gate_bitmap_words(gw, gh) + 1), st);
    if (e != cudaSuccess) return e;
    if (!feat_ready) gate_features_kernel<<<dim3(blocks(w8, 128), h8), 128, 0, st>>>(gray, gpitch, w8, h8, sc.feat);
    gate_infer_kernel<<<dim3((w8 + kIX - 1) / kIX, (h8 + kIY - 1) / kIY), 256, 0, st>>>(net, sc.feat, w8, h8, thr, 0.25f * thr, sc.bits,
                                                                                       wwords, sc.prob, sc.ambiguous);
    const int amb_limit = gate_cells(sc, gw, gh, amb_frac, margin).amb_limit;
    const int n_words = gate_bitmap_words(gw, gh);
    for (int g0 = 0; g0 < n_levels; g0 += kParamLevels) {
        LevelTable T;
        T.n = n_levels - g0 < kParamLevels ? n_levels - g0 : kParamLevels;
        for (int i = 0; i < T.n; ++i) T.lv[i] = levels[g0 + i];
        const LevelDesc& last = T.lv[T.n - 1];
        T.first = T.lv[0].k2_base;
        const int nb = last.k2_base + last.k2_tiles_x * ((last.oh + kK2TileY - 1) / kK2TileY) - T.lv[0].k2_base;
        const int nf = last.k1_base + last.k1_tiles_x * ((last.p1h + kK1TileY - 1) / kK1TileY) - T.lv[0].k1_base;
        if (nb + nf > 0)
            gate_mask_kernel<<<blocks(nb + nf, 128), 128, n_words <= kMaskSmemWords ? sizeof(uint32_t) * n_words : 0, st>>>(
                T, nb, sc.bits, n_words, wwords, w16, h16, margin, sc.ambiguous, amb_limit, back_on, front_on);
    }
    return cudaGetLastError();
}

namespace {

// Training labels from the plain cascade's own verdicts: the (octave, cell) of the window centre
// of every candidate that stage 3 accepted. Labels must be zeroed first.
__global__ void gate_label_kernel(const Candidate* __restrict__ cands, const CandResult* __restrict__ res, const int* __restrict__ ncand,
                                  int cap, const LevelDesc* __restrict__ levels, int w16, int h16, uint8_t* __restrict__ labels) {
    const int n = min(*ncand, cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!res[i].accepted) continue;
        const Candidate cd = cands[i];
        const LevelDesc& L = levels[cd.level];
        const int cx = (int)(((float)cd.px + 11.5f) * L.inv_scale) / 16, cy = (int)(((float)cd.py + 13.5f) * L.inv_scale) / 16;
        if (cx < 0 || cx >= w16 || cy < 0 || cy >= h16) continue;
        labels[((long long)min(L.octave, kGK - 1) * h16 + cy) * w16 + cx] = 1;
    }
}

}  // namespace

cudaError_t launch_gate_labels(const Candidate* cands, const CandResult* res, const int* ncand, int cap, const LevelDesc* d_levels, int gw, int gh,
                               uint8_t* labels, cudaStream_t st) {
    const int w16 = (gw / 8) / 2, h16 = (gh / 8) / 2;
    cudaError_t e = cudaMemsetAsync(labels, 0, (size_t)kGK * w16 * h16, st);
    if (e != cudaSuccess) return e;
    gate_label_kernel<<<64, 256, 0, st>>>(cands, res, ncand, cap, d_levels, w16, h16, labels);
    return cudaGetLastError();
}

}  // namespace ccnn

// ---- C ABI: features, gradient, training ----

using namespace ccnn;

extern "C" CCNN_API ccnn_status ccnn_gate_features(const float* d_gray, int cols, int rows, size_t step, void* d_feat, void* stream) {
    if (!d_gray || !d_feat || cols < 16 || rows < 16 || step % sizeof(float)) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    const int w8 = cols / 8, h8 = rows / 8;
    gate_features_kernel<<<dim3(blocks(w8, 128), h8), 128, 0, (cudaStream_t)stream>>>(d_gray, (int)(step / sizeof(float)), w8, h8,
                                                                                       (__half*)d_feat);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("gate features: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}

namespace {

struct TrainBuffers {
    __half *a1 = nullptr, *a2 = nullptr;
    float *gq = nullptr, *gz2 = nullptr, *gz1 = nullptr, *grad = nullptr, *loss = nullptr;
    cudaError_t alloc(int n, int w8, int h8) {
        const size_t plane = (size_t)w8 * h8, cells = (size_t)(w8 / 2) * (h8 / 2);
        cudaError_t e = cudaMalloc(&a1, sizeof(__half) * n * kGC * plane);
        if (e == cudaSuccess) e = cudaMalloc(&a2, sizeof(__half) * n * kGC * plane);
        if (e == cudaSuccess) e = cudaMalloc(&gq, sizeof(float) * n * kGC * cells);
        if (e == cudaSuccess) e = cudaMalloc(&gz2, sizeof(float) * n * kGC * plane);
        if (e == cudaSuccess) e = cudaMalloc(&gz1, sizeof(float) * n * kGC * plane);
        if (e == cudaSuccess) e = cudaMalloc(&grad, sizeof(float) * kGateParams);
        if (e == cudaSuccess) e = cudaMalloc(&loss, sizeof(float));
        return e;
    }
    ~TrainBuffers() {
        cudaFree(a1);
        cudaFree(a2);
        cudaFree(gq);
        cudaFree(gz2);
        cudaFree(gz1);
        cudaFree(grad);
        cudaFree(loss);
    }
};

// one forward + backward pass over n frames: grad (and loss) accumulate into B
cudaError_t gate_pass(const float* P, const __half* f, const uint8_t* labels, int n, int w8, int h8, float pos_weight, TrainBuffers& B,
                      cudaStream_t st) {
    const long long plane = (long long)w8 * h8, cells = (long long)(w8 / 2) * (h8 / 2);
    const float inv_cells = 1.f / (float)(n * cells * kGK);
    gate_fwd1_kernel<<<blocks(n * plane, 256), 256, 0, st>>>(P, f, n, w8, h8, B.a1);
    gate_fwd2_kernel<<<blocks(n * plane, 256), 256, 0, st>>>(P, B.a1, n, w8, h8, B.a2);
    gate_head_kernel<<<blocks(n * cells, 256), 256, 0, st>>>(P, B.a2, n, w8, h8, labels, pos_weight, inv_cells, B.gq, B.grad, B.loss, nullptr,
                                                             2.f, 2.f, nullptr);
    gate_bwd2a_kernel<<<blocks(n * kGC * plane, 256), 256, 0, st>>>(B.a2, B.gq, n, w8, h8, B.gz2);
    const int rows = 16;
    gate_wgrad_kernel<kGC><<<dim3((h8 + rows - 1) / rows, n), 256, 0, st>>>(B.gz2, B.a1, n, w8, h8, rows, B.grad + kW2, B.grad + kB2);
    gate_bwd1a_kernel<<<blocks(n * plane, 256), 256, 0, st>>>(P, B.a1, B.gz2, n, w8, h8, B.gz1);
    gate_wgrad_kernel<1><<<dim3((h8 + rows - 1) / rows, n), 96, 0, st>>>(B.gz1, f, n, w8, h8, rows, B.grad + kW1, B.grad + kB1);
    return cudaGetLastError();
}

}  // namespace

extern "C" CCNN_API ccnn_status ccnn_gate_gradient(const float* d_params, const void* d_feat, const unsigned char* d_labels, int n, int w8, int h8,
                                                   float pos_weight, float* grad_out, float* loss_out) {
    if (!d_params || !d_feat || !d_labels || n <= 0 || w8 < 2 || h8 < 2 || !grad_out || !loss_out) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    TrainBuffers B;
    cudaError_t e = B.alloc(n, w8, h8);
    if (e == cudaSuccess) e = cudaMemset(B.grad, 0, sizeof(float) * kGateParams);
    if (e == cudaSuccess) e = cudaMemset(B.loss, 0, sizeof(float));
    if (e == cudaSuccess) e = gate_pass(d_params, (const __half*)d_feat, d_labels, n, w8, h8, pos_weight, B, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(grad_out, B.grad, sizeof(float) * kGateParams, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(loss_out, B.loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_error(std::string("gate gradient: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}

// Adam over mini-batches of `batch` frames taken in order, `epochs` times; params (host, fp32)
// are read as the start point and overwritten with the result; losses[e] = mean loss of epoch e.
extern "C" CCNN_API ccnn_status ccnn_gate_train(float* params, const void* d_feat, const unsigned char* d_labels, int n, int w8, int h8, int batch,
                                                int epochs, float lr, float pos_weight, float* losses) {
    if (!params || !d_feat || !d_labels || n <= 0 || batch <= 0 || epochs <= 0 || w8 < 2 || h8 < 2) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    batch = std::min(batch, n);
    TrainBuffers B;
    float *P = nullptr, *m = nullptr, *v = nullptr;
    cudaError_t e = B.alloc(batch, w8, h8);
    if (e == cudaSuccess) e = cudaMalloc(&P, sizeof(float) * kGateParams);
    if (e == cudaSuccess) e = cudaMalloc(&m, sizeof(float) * kGateParams);
    if (e == cudaSuccess) e = cudaMalloc(&v, sizeof(float) * kGateParams);
    if (e == cudaSuccess) e = cudaMemcpy(P, params, sizeof(float) * kGateParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m, 0, sizeof(float) * kGateParams);
    if (e == cudaSuccess) e = cudaMemset(v, 0, sizeof(float) * kGateParams);
    const size_t fplane = (size_t)w8 * h8, lplane = (size_t)kGK * (w8 / 2) * (h8 / 2);
    int step = 0;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        double ep_loss = 0.0;
        int nb = 0;
        for (int b0 = 0; b0 + batch <= n && e == cudaSuccess; b0 += batch, ++nb) {
            e = cudaMemset(B.grad, 0, sizeof(float) * kGateParams);
            if (e == cudaSuccess) e = cudaMemset(B.loss, 0, sizeof(float));
            if (e == cudaSuccess)
                e = gate_pass(P, (const __half*)d_feat + b0 * fplane, d_labels + b0 * lplane, batch, w8, h8, pos_weight, B, nullptr);
            ++step;
            if (e == cudaSuccess) {
                gate_adam_kernel<<<blocks(kGateParams, 256), 256>>>(P, B.grad, m, v, lr, powf(0.9f, (float)step), powf(0.999f, (float)step));
                e = cudaGetLastError();
            }
            float l = 0.f;
            if (e == cudaSuccess) e = cudaMemcpy(&l, B.loss, sizeof(float), cudaMemcpyDeviceToHost);
            ep_loss += l;
        }
        if (losses) losses[ep] = (float)(ep_loss / std::max(1, nb));
    }
    if (e == cudaSuccess) e = cudaMemcpy(params, P, sizeof(float) * kGateParams, cudaMemcpyDeviceToHost);
    cudaFree(P);
    cudaFree(m);
    cudaFree(v);
    if (e != cudaSuccess) {
        set_error(std::string("gate training: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}
