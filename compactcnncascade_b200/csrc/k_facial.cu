// Facial analysis: the landmark network on every accepted check window.
//
// Reference: CNNDetector::CPUCheckDetect (src/CNNObjectDetector/cnn_detector_v3.cpp:1731-1764). When
// a window is accepted and facial analysis is on, the fourth network (cnn4landmarks_cntk.bin,
// loaded at :792-810) runs on the float nearest-neighbour crop of that window (the 49x51 image
// before byte rounding and equalisation, :1565). Its 13 outputs give five landmarks as fractions
// of the crop size, and gender, smile and glasses as int(v + 0.5). A detection whose five
// landmarks all fall in the upper-left quarter of the crop is dropped (:1740-1750).
//
// One block per accepted candidate (persistent over the candidate list; rejected candidates
// cost one verdict). The network runs in shared memory:
//   L1: 24 maps, 4x4 conv on 49x51 -> 46x48, BN/LReLU, 2x2 max -> 23x24, neighbour sums;
//   L2: 48 maps, 3x3 -> 21x22 -> 10x11, sums;  L3: 96 maps, 10w x 11h -> 1x1, BN/LReLU;
//   a fully connected hidden layer of 384 neurons and 13 outputs (cnn_simd_cntk.cpp:640-963).
// Map pairs (2i, 2i+1) read the same input and neurons (2q, 2q+1) the same L3 values: each
// pair runs as packed f32x2 operations, every value keeping the reference's roundings.
#include "kernels.h"
#include "resample.cuh"
#include "window_common.cuh"

namespace ccnn {

namespace {

using LN = LandmarkNet;
constexpr int kFT = 256;
constexpr int kC1W = LN::kInW - 3, kC1H = LN::kInH - 3;  // 46 x 48 conv positions
constexpr int kQ1W = kC1W / 2, kQ1H = kC1H / 2;          // 23 x 24 pooled
constexpr int kC2W = kQ1W - 2, kC2H = kQ1H - 2;          // 21 x 22
constexpr int kQ2W = kC2W / 2, kQ2H = kC2H / 2;          // 10 x 11

struct FacialSmem {
    float img[LN::kInH][LN::kInW];
    float s1[LN::kM1][kQ1H][kQ1W];
    union {
        float p1[LN::kM1][kQ1H][kQ1W];
        struct {
            float p2[LN::kM2][kQ2H][kQ2W];
            float s2[LN::kM2][kQ2H][kQ2W];
        } b;
    } u;
    float a3[LN::kM3];
    float hid[LN::kHL];
    float res[LN::kOut];
    int geo[4];
    int accepted;
};

// neighbour-map sums of the reference (add / add2, cnnpp_cplusplus.cpp:916-950)
template <int M, int N>
__device__ __forceinline__ void neighbour_sums(const float (*p)[N], float (*s)[N]) {
    for (int it = threadIdx.x; it < M * N; it += kFT) {
        const int k = it / N, e = it - k * N;
        float v;
        if (k == 0) v = fadd(p[0][e], p[1][e]);
        else if (k == M - 1) v = fadd(p[M - 2][e], p[M - 1][e]);
        else v = fadd(fadd(p[k - 1][e], p[k][e]), p[k + 1][e]);
        s[k][e] = v;
    }
}

__device__ void landmark_net(const LN& W, FacialSmem& S) {
    const f2_t nz = f2_ld(W.negzero);
    // L1: (map pair, pooled pixel) units, map pair uniform across a warp's run of pixels
    for (int it = threadIdx.x; it < (LN::kM1 / 2) * kQ1W * kQ1H; it += kFT) {
        const int mp = it / (kQ1W * kQ1H), px = it - mp * (kQ1W * kQ1H);
        const int x = px % kQ1W, y = px / kQ1W;
        f2_t win[5][5];
#pragma unroll
        for (int r = 0; r < 5; ++r)
#pragma unroll
            for (int c = 0; c < 5; ++c) win[r][c] = f2_dup(S.img[2 * y + r][2 * x + c]);
        f2_t cv[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int dy = d >> 1, dx = d & 1;
            f2_t acc = f2_mul(win[dy][dx], f2_ld(W.k1p[mp][0]), nz);
#pragma unroll
            for (int k = 1; k < 16; ++k) acc = f2_add(acc, f2_mul(win[dy + (k >> 2)][dx + (k & 3)], f2_ld(W.k1p[mp][k]), nz));
            cv[d] = lrelu_bn2(acc, W.a1p[mp], nz);
        }
        const f2_t pm = f2_max4(cv[0], cv[1], cv[2], cv[3]);
        S.u.p1[2 * mp][y][x] = f2_lo(pm);
        S.u.p1[2 * mp + 1][y][x] = f2_hi(pm);
    }
    __syncthreads();
    neighbour_sums<LN::kM1, kQ1W * kQ1H>(reinterpret_cast<const float(*)[kQ1W * kQ1H]>(S.u.p1),
                                         reinterpret_cast<float(*)[kQ1W * kQ1H]>(S.s1));
    __syncthreads();
    // L2: maps (2i, 2i+1) on sum map i, 3x3, BN/LReLU, 2x2 max (floor: the last conv row/column
    // has no partner)
    for (int it = threadIdx.x; it < (LN::kM2 / 2) * kQ2W * kQ2H; it += kFT) {
        const int i = it / (kQ2W * kQ2H), px = it - i * (kQ2W * kQ2H);
        const int x = px % kQ2W, y = px / kQ2W;
        f2_t q[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) q[r][c] = f2_dup(S.s1[i][2 * y + r][2 * x + c]);
        f2_t cv[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int dy = d >> 1, dx = d & 1;
            f2_t acc = f2_mul(q[dy][dx], f2_ld(W.k2p[i][0]), nz);
#pragma unroll
            for (int k = 1; k < 9; ++k) acc = f2_add(acc, f2_mul(q[dy + k / 3][dx + k % 3], f2_ld(W.k2p[i][k]), nz));
            cv[d] = lrelu_bn2(acc, W.a2p[i], nz);
        }
        const f2_t pm = f2_max4(cv[0], cv[1], cv[2], cv[3]);
        S.u.b.p2[2 * i][y][x] = f2_lo(pm);
        S.u.b.p2[2 * i + 1][y][x] = f2_hi(pm);
    }
    __syncthreads();
    neighbour_sums<LN::kM2, kQ2W * kQ2H>(reinterpret_cast<const float(*)[kQ2W * kQ2H]>(S.u.b.p2),
                                         reinterpret_cast<float(*)[kQ2W * kQ2H]>(S.u.b.s2));
    __syncthreads();
    // L3: one 110-term chain per map (conv_11x10 starts from 0.f, cnnpp_cplusplus.cpp:352-377)
    if (threadIdx.x < LN::kM3 / 2) {
        const int i = threadIdx.x;
        f2_t acc = 0ull;  // (+0, +0)
        for (int r = 0; r < LN::kK3H; ++r)
#pragma unroll
            for (int c = 0; c < LN::kK3W; ++c)
                acc = f2_add(acc, f2_mul(f2_dup(S.u.b.s2[i][r][c]), f2_ld(W.k3p[i][r * LN::kK3W + c]), nz));
        const f2_t av = lrelu_bn2(acc, W.a3p[i], nz);
        S.a3[2 * i] = f2_lo(av);
        S.a3[2 * i + 1] = f2_hi(av);
    }
    __syncthreads();
    // hidden layer (mulCN_add_tanhW over all 96 L3 values, :646-672), neuron pairs packed
    if (threadIdx.x < LN::kHL / 2) {
        const int q = threadIdx.x;
        f2_t s = f2_ld(W.hbp[q]);
        for (int j = 0; j < LN::kM3; ++j) s = f2_add(s, f2_mul(f2_dup(S.a3[j]), f2_ld(W.hwp[q][j]), nz));
        s = f2_mul(s, f2_dup(W.htw), nz);
        const f2_t half = f2_pack(0.5f, 0.5f);
        const f2_t v = f2_add(f2_mul(half, tanh_rational2(s, nz), nz), half);
        const f2_t h = f2_add(f2_mul(f2_ld(W.hbnwp[q]), v, nz), f2_ld(W.hbnbp[q]));
        S.hid[2 * q] = f2_lo(h);
        S.hid[2 * q + 1] = f2_hi(h);
    }
    __syncthreads();
    // outputs (mulC / mulC1_add in neuron order, then tanhW, :885-900, :673-690)
    if (threadIdx.x < LN::kOut) {
        const int k = threadIdx.x;
        float acc = fmul(S.hid[0], W.ow[k][0]);
        for (int t = 1; t < LN::kHL; ++t) acc = fadd(fmul(S.hid[t], W.ow[k][t]), acc);
        float c = fmul(fadd(acc, W.ob[k]), W.otw);
        c = tanh_rational(c);
        S.res[k] = (W.af == 0.f) ? fadd(fmul(0.5f, c), 0.5f) : fmul(W.af, c);
    }
    __syncthreads();
}

struct FacialArgs {
    const LN* net;
    const float* gray;
    int gpitch, gw, gh;
    const Candidate* cands;
    const int* n_cand;
    const LevelDesc* levels;
    const WinOut* win;
    CascadeConfig cfg;
    int4* attr;  // per candidate: (dropped, gender, smile, glasses)
};

__global__ void __launch_bounds__(kFT, 1) facial_kernel(const FacialArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FacialSmem& S = *reinterpret_cast<FacialSmem*>(smem_raw);
    const int n = *a.n_cand;
    for (int ci = blockIdx.x; ci < n; ci += gridDim.x) {
        if (threadIdx.x == 0) {
            const Candidate cd = a.cands[ci];
            const LevelDesc& L = a.levels[cd.level];
            const CandResult r = verdict(a.win + (size_t)ci * 4, cd, L.scale, a.cfg);
            S.accepted = r.accepted;
            if (r.accepted) window_geometry(cd, L.inv_scale, r.accepted - 1, a.gw, a.gh, a.cfg.pat_w, a.cfg.pat_h, S.geo);
            a.attr[ci] = make_int4(0, -1, -1, -1);
        }
        __syncthreads();
        if (S.accepted) {
            // nearest-neighbour crop of the accepted window (FastImageResize copies equal sizes)
            const int rx = S.geo[0], ry = S.geo[1], rcols = S.geo[2], rrows = S.geo[3];
            const bool copy = (rcols == LN::kInW && rrows == LN::kInH);
            const uint32_t sclx = fp_step(max(rcols, 1), LN::kInW), scly = fp_step(max(rrows, 1), LN::kInH);
            for (int p = threadIdx.x; p < LN::kInW * LN::kInH; p += kFT) {
                const int ix = p % LN::kInW, iy = p / LN::kInW;
                const int sx = copy ? ix : (int)sample_col(ix, sclx, rcols).idx;
                const int sy = copy ? iy : (int)sample_row(iy, scly, rrows).idx;
                const int gx = min(max(rx + sx, 0), a.gw - 1), gy = min(max(ry + sy, 0), a.gh - 1);  // memory guard
                S.img[iy][ix] = a.gray[(size_t)gy * a.gpitch + gx];
            }
            __syncthreads();
            landmark_net(*a.net, S);
            if (threadIdx.x == 0) {
                int zero = 0;
                for (int t = 0; t < 5; ++t) {
                    const int lx = __float2int_rz(fmul(S.res[2 * t], (float)rcols));
                    const int ly = __float2int_rz(fmul(S.res[2 * t + 1], (float)rrows));
                    if (lx < (rcols >> 1) && ly < (rrows >> 1)) zero++;
                }
                a.attr[ci] = make_int4(zero == 5 ? 1 : 0, __float2int_rz(fadd(S.res[10], 0.5f)), __float2int_rz(fadd(S.res[11], 0.5f)),
                                       __float2int_rz(fadd(S.res[12], 0.5f)));
            }
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t facial_setup() {
    return cudaFuncSetAttribute(facial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FacialSmem));
}

cudaError_t launch_facial(const LandmarkNet* d_net, const float* gray, int gpitch, int gw, int gh, const Candidate* cands,
                          const int* n_cand, const LevelDesc* levels, const WinOut* win, const CascadeConfig& cfg, int4* attr, int grid,
                          cudaStream_t st) {
    FacialArgs a;
    a.net = d_net;
    a.gray = gray;
    a.gpitch = gpitch;
    a.gw = gw;
    a.gh = gh;
    a.cands = cands;
    a.n_cand = n_cand;
    a.levels = levels;
    a.win = win;
    a.cfg = cfg;
    a.attr = attr;
    facial_kernel<<<grid, kFT, sizeof(FacialSmem), st>>>(a);
    return cudaGetLastError();
}

}  // namespace ccnn
