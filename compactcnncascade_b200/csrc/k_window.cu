// Stage-2/3 window CNNs on the compacted stage-1 candidates.
//
// Reference: CNNDetector::CPUCheckDetect (src/CNNObjectDetector/cnn_detector_v3.cpp:1485-1818):
//   crop  x = int((px-6)/s), y = int((py-5)/s), w = int(36/s), h = int(38/s)  (:1492-1495)
//   retry window (mod 1) shrunk by 15 % (:1535-1542), clamped to the frame (:1553-1556)
//   nearest-neighbour resize to 49 x 51 (:1565), byte rounding uchar(v + 0.5) (image_proc.cpp:365),
//   histogram equalisation (image_proc.cpp:720-799),
//   stage 2 on columns 2..48 (UCharToFloat offset 2, image_proc.cpp:417-427),
//   stage 3 on the mirror of columns 0..46 (UCharToFloat_inv, image_proc.cpp:478-490),
//   4x4 response maps counted against treshold_2 / treshold_3 with the type_check early exits
//   (:1655-1706) and the accept rule (:1709-1725); score s0 + k1*max(-1.7159, m1) + k2*max(-1.7159, m2).
//
// Every candidate is evaluated speculatively: both nets on both the first and the retry window,
// as independent CTA work items. Which of them the reference would have reached (early exits,
// retry, drop_detect) is decided by the replay kernel, so the verdicts are the same while all
// items run in parallel.
//
// One CTA (256 threads) per work item, persistent over the item list. The networks run
// entirely in shared memory: L1 (6 maps, 44x48 -> pooled 22x24), neighbour sums, L2 (12 maps,
// 20x22 -> pooled 10x11), sums, L3 (24 maps, 7w x 8h -> 4x4), hidden layer and output neuron.
#include "kernels.h"
#include "resample.cuh"
#include "window_common.cuh"
#include "legacy_dev.cuh"

namespace ccnn {

constexpr int kWT = 256;
constexpr int kP1W = 22, kP1H = 24;   // pooled L1 of a 47x51 window
constexpr int kP2W = 10, kP2H = 11;   // pooled L2
constexpr int kOutN = 16;             // 4x4 response map

struct WindowSmem {
    uint8_t crop[kCropH][kCropW + 3];
    int hist[256];
    int lut[256];
    float s1[6][kP1H][kP1W + 1];
    float p2[12][kP2H][kP2W + 1];
    float s2[12][kP2H][kP2W + 1];
    float a3[24][kOutN];
    float hbuf[84][kOutN];
    float out[kOutN];
    float l1rest[32][6];  // pooled L1 maps of the partial pass's pixels
    int geo[4];
};

// mode: 0 = stage-2 view (columns 2..48), 1 = mirrored (46 - x), 2 = plain (columns 0..46)
__device__ __forceinline__ float win_in(const WindowSmem& S, int mode, int x, int y) {
    int c = mode == 0 ? x + kXOff : (mode == 1 ? (kWinW - 1) - x : x);
    return (float)S.crop[y][c];
}

template <class NW>
__device__ void window_net(const NW& W, WindowSmem& S, int mode) {
    static_assert(NW::kM1 % 2 == 0 && NW::kM2 % 2 == 0 && NW::kM3 % 2 == 0 && NW::kHS % 2 == 0, "maps and neurons run in pairs");
    const f2_t nz = f2_ld(W.negzero);
    // L1: conv 4x4 + folded BN/LReLU + 2x2 max, then neighbour sums (add / add2); every map pair
    // reads the same window, so it runs as one packed pair. Whole passes of kWT pixels run every map
    // pair per thread; the pixels of the last, partial pass are split into (pixel, map pair) units,
    // one warp per map pair, so that it takes a third of a pass.
    constexpr int kFull = (kP1W * kP1H / kWT) * kWT;
    constexpr int kRest = kP1W * kP1H - kFull;
    constexpr int kMP = NW::kM1 / 2;
    static_assert(kRest <= 32 && 32 * kMP <= kWT, "partial L1 pass must fit one warp per map pair");
    for (int p = threadIdx.x; p < kFull + 32 * kMP; p += kWT) {
        const bool unit = p >= kFull;  // one map pair (warp-uniform) of a pixel of the partial pass
        if (unit && ((p - kFull) & 31) >= kRest) continue;
        const int px = unit ? kFull + ((p - kFull) & 31) : p;
        const int mp0 = unit ? (p - kFull) >> 5 : 0;
        const int x = px % kP1W, y = px / kP1W;
        f2_t win[5][5];
#pragma unroll
        for (int r = 0; r < 5; ++r)
#pragma unroll
            for (int c = 0; c < 5; ++c) win[r][c] = f2_dup(win_in(S, mode, 2 * x + c, 2 * y + r));
        float P[NW::kM1];
#pragma unroll
        for (int mp = 0; mp < kMP; ++mp) {
            if (unit && mp != mp0) continue;
            f2_t cv[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const int dy = d >> 1, dx = d & 1;
                f2_t acc = f2_mul(win[dy][dx], f2_ld(W.k1p[mp][0]), nz);
#pragma unroll
                for (int k = 1; k < 16; ++k) acc = f2_add(acc, f2_mul(win[dy + (k >> 2)][dx + (k & 3)], f2_ld(W.k1p[mp][k]), nz));
                cv[d] = lrelu_bn2(acc, W.a1p[mp], nz);  // maps (2mp, 2mp+1)
            }
            const f2_t pm = f2_max4(cv[0], cv[1], cv[2], cv[3]);
            P[2 * mp] = f2_lo(pm);
            P[2 * mp + 1] = f2_hi(pm);
            if (unit) {
                S.l1rest[px - kFull][2 * mp] = P[2 * mp];
                S.l1rest[px - kFull][2 * mp + 1] = P[2 * mp + 1];
            }
        }
        if (unit) continue;
        S.s1[0][y][x] = fadd(P[0], P[1]);
#pragma unroll
        for (int k = 1; k < NW::kM1 - 1; ++k) S.s1[k][y][x] = fadd(fadd(P[k - 1], P[k]), P[k + 1]);
        S.s1[NW::kM1 - 1][y][x] = fadd(P[NW::kM1 - 2], P[NW::kM1 - 1]);
    }
    if (kRest > 0) {
        __syncthreads();
        if (threadIdx.x < kRest) {
            const int px = kFull + threadIdx.x;
            const int x = px % kP1W, y = px / kP1W;
            const float* P = S.l1rest[threadIdx.x];
            S.s1[0][y][x] = fadd(P[0], P[1]);
#pragma unroll
            for (int k = 1; k < NW::kM1 - 1; ++k) S.s1[k][y][x] = fadd(fadd(P[k - 1], P[k]), P[k + 1]);
            S.s1[NW::kM1 - 1][y][x] = fadd(P[NW::kM1 - 2], P[NW::kM1 - 1]);
        }
    }
    __syncthreads();
    // L2: map pair (2i, 2i+1) convolves sum map i; 3x3 + BN/LReLU + 2x2 max
    for (int it = threadIdx.x; it < kP2W * kP2H * NW::kM1; it += kWT) {
        const int i = it / (kP2W * kP2H);
        const int p = it - i * (kP2W * kP2H);
        const int x = p % kP2W, y = p / kP2W;
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
        S.p2[2 * i][y][x] = f2_lo(pm);
        S.p2[2 * i + 1][y][x] = f2_hi(pm);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < kP2W * kP2H; p += kWT) {
        const int x = p % kP2W, y = p / kP2W;
        constexpr int M = NW::kM2;
        S.s2[0][y][x] = fadd(S.p2[0][y][x], S.p2[1][y][x]);
        for (int k = 1; k < M - 1; ++k) S.s2[k][y][x] = fadd(fadd(S.p2[k - 1][y][x], S.p2[k][y][x]), S.p2[k + 1][y][x]);
        S.s2[M - 1][y][x] = fadd(S.p2[M - 2][y][x], S.p2[M - 1][y][x]);
    }
    __syncthreads();
    // L3: 7w x 8h conv summed in one left-to-right chain (conv_8x7), BN/LReLU, no pooling;
    // maps (2i, 2i+1) share the input: packed
    for (int it = threadIdx.x; it < (NW::kM3 / 2) * kOutN; it += kWT) {
        const int i = it / kOutN, o = it - i * kOutN;
        const int ox = o & 3, oy = o >> 2;
        f2_t acc = f2_mul(f2_dup(S.s2[i][oy][ox]), f2_ld(W.k3p[i][0]), nz);
#pragma unroll
        for (int k = 1; k < NW::kK3W * NW::kK3H; ++k)
            acc = f2_add(acc, f2_mul(f2_dup(S.s2[i][oy + k / NW::kK3W][ox + k % NW::kK3W]), f2_ld(W.k3p[i][k]), nz));
        const f2_t av = lrelu_bn2(acc, W.a3p[i], nz);
        S.a3[2 * i][o] = f2_lo(av);
        S.a3[2 * i + 1][o] = f2_hi(av);
    }
    __syncthreads();
    // hidden neurons n = HS*i + t read L3 maps i .. i+CONN-1; neurons (2q, 2q+1) share the
    // group, so they run as one packed pair
    for (int it = threadIdx.x; it < (NW::kHL / 2) * kOutN; it += kWT) {
        const int q = it / kOutN, o = it - q * kOutN;
        const int n = 2 * q;
        const int i = n / NW::kHS;
        f2_t s = f2_pack(W.hb[n], W.hb[n + 1]);
#pragma unroll
        for (int j = 0; j < NW::kConn; ++j) s = f2_add(s, f2_mul(f2_dup(S.a3[i + j][o]), f2_ld(W.hwp[q][j]), nz));
        s = f2_mul(s, f2_dup(W.htw[i]), nz);
        const f2_t half = f2_pack(0.5f, 0.5f);
        const f2_t v = f2_add(f2_mul(half, tanh_rational2(s, nz), nz), half);
        const int t = n - i * NW::kHS;  // neurons n, n+1 are slots t, t+1 of group i
        const f2_t h = f2_add(f2_mul(f2_pack(W.hbnw[t], W.hbnw[t + 1]), v, nz), f2_pack(W.hbnb[t], W.hbnb[t + 1]));
        S.hbuf[n][o] = f2_lo(h);
        S.hbuf[n + 1][o] = f2_hi(h);
    }
    __syncthreads();
    if (threadIdx.x < kOutN) {
        const int o = threadIdx.x;
        float acc = fmul(S.hbuf[0][o], W.ow[0]);
        for (int n = 1; n < NW::kHL; ++n) acc = fadd(fmul(S.hbuf[n][o], W.ow[n]), acc);
        float c = fmul(fadd(acc, W.ob), W.otw);
        c = tanh_rational(c);
        S.out[o] = (W.af == 0.f) ? fadd(fmul(0.5f, c), 0.5f) : fmul(W.af, c);
    }
    __syncthreads();
}

// The legacy (format 1.0) stage-2/3 networks on the window in shared memory: L1 (6 maps, 22x24
// pooled) in S.s1, L2 (12 maps, 10x11) in S.p2, the L3 values of the 16 outputs in S.a3, fully
// connected hidden neurons in S.hbuf; the arithmetic of the standalone legacy forward pass
// (legacy_dev.cuh), spread over the block.
__device__ void legacy_window_net(const LegacyNet& W, WindowSmem& S, int mode) {
    constexpr int kP1 = kP1W * kP1H, kP2 = kP2W * kP2H;
    constexpr long long kS1Plane = kP1H * (kP1W + 1), kP2Plane = kP2H * (kP2W + 1);
    for (int it = threadIdx.x; it < W.m0 * kP1; it += kWT) {
        const int m = it / kP1, p = it - m * kP1;
        const int x = p % kP1W, y = p / kP1W;
        const float* k = W.k1[m];
        float c[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int x0 = 2 * x + (d & 1), y0 = 2 * y + (d >> 1);
            float acc = fmul(win_in(S, mode, x0, y0), k[0]);
#pragma unroll
            for (int t = 1; t < 16; ++t) acc = fadd(acc, fmul(win_in(S, mode, x0 + (t & 3), y0 + (t >> 2)), k[t]));
            c[d] = acc;
        }
        S.s1[m][y][x] = lg_pool_tanh(c, W.max_pool, W.cb[0][m], W.sw[0][m], W.sb[0][m], W.af);
    }
    __syncthreads();
    const float* s1 = &S.s1[0][0][0];
    for (int it = threadIdx.x; it < W.m1 * kP2; it += kWT) {
        const int m = it / kP2, p = it - m * kP2;
        const int x = p % kP2W, y = p / kP2W, i = m >> 1;
        float Q[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int q = 0; q < 4; ++q) Q[r][q] = lg_map_sum(s1, kS1Plane, W.m0, i, (2 * y + r) * (kP1W + 1) + 2 * x + q);
        const float* k = W.k2[m];
        float c[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int dy = d >> 1, dx = d & 1;
            float acc = fmul(Q[dy][dx], k[0]);
#pragma unroll
            for (int t = 1; t < 9; ++t) acc = fadd(acc, fmul(Q[dy + t / 3][dx + t % 3], k[t]));
            c[d] = acc;
        }
        S.p2[m][y][x] = lg_pool_tanh(c, W.max_pool, W.cb[1][m], W.sw[1][m], W.sb[1][m], W.af);
    }
    __syncthreads();
    const float* p2 = &S.p2[0][0][0];
    for (int it = threadIdx.x; it < W.m2 * kOutN; it += kWT) {
        const int m = it / kOutN, o = it - m * kOutN;
        const int ox = o & 3, oy = o >> 2, i = m >> 1, kw = W.k3w;
        S.a3[m][o] = lg_l3_value(W, m, [&](int t) { return lg_map_sum(p2, kP2Plane, W.m1, i, (oy + t / kw) * (kP2W + 1) + ox + t % kw); });
    }
    __syncthreads();
    if (W.full_connect) {
        for (int it = threadIdx.x; it < W.hl * kOutN; it += kWT) {
            const int n = it / kOutN, o = it - n * kOutN;
            float vals[kLgMaxM2];
            for (int j = 0; j < W.m2; ++j) vals[j] = S.a3[j][o];
            S.hbuf[n][o] = lg_hidden_fc(W, n, vals);
        }
        __syncthreads();
    }
    if (threadIdx.x < kOutN) {
        const int o = threadIdx.x;
        float acc;
        if (W.full_connect) {
            acc = S.hbuf[0][o];
            for (int n = 1; n < W.hl; ++n) acc = fadd(acc, S.hbuf[n][o]);
        } else {
            acc = fadd(S.a3[1][o], S.a3[0][o]);
            for (int i = 1; i < W.m2 / 2; ++i) acc = fadd(acc, fadd(S.a3[2 * i + 1][o], S.a3[2 * i][o]));
        }
        S.out[o] = lg_finish(W, acc);
    }
    __syncthreads();
}

struct WinArgs {
    const float* gray;
    int gpitch, gw, gh;
    const Candidate* cands;
    const int* n_cand;
    const LevelDesc* levels;
    WinOut* out;
    CascadeConfig cfg;
    const LegacyNet* lg;  // legacy networks ([1] stage 2, [2] stage 3) instead of the CNTK ones, or null
};

// crop + byte rounding + (optional) equalisation of one window into S.crop
__device__ void prepare_window(const WinArgs& a, WindowSmem& S, const Candidate& cd, float inv_scale, int mod) {
    if (threadIdx.x == 0) window_geometry(cd, inv_scale, mod, a.gw, a.gh, a.cfg.pat_w, a.cfg.pat_h, S.geo);
    if (threadIdx.x < 256) S.hist[threadIdx.x] = 0;
    __syncthreads();
    const int rx = S.geo[0], ry = S.geo[1], rcols = S.geo[2], rrows = S.geo[3];
    const bool copy = (rcols == kCropW && rrows == kCropH);  // FastImageResize copies equal sizes
    const uint32_t sclx = fp_step(max(rcols, 1), kCropW), scly = fp_step(max(rrows, 1), kCropH);
    // every load of the thread's pixels is issued before the first is used (the gray frame is read
    // from L2, so the loads overlap instead of queueing one latency each); the byte values stay in
    // registers until the equalisation table is known
    constexpr int kPx = kCropW * kCropH;
    constexpr int kPerThread = (kPx + kWT - 1) / kWT;
    float v[kPerThread];
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int p = threadIdx.x + k * kWT;
        v[k] = 0.f;
        if (p < kPx) {
            const int ix = p % kCropW, iy = p / kCropW;
            int sx, sy;
            if (copy) {
                sx = ix;
                sy = iy;
            } else {
                sx = (int)sample_col(ix, sclx, rcols).idx;
                sy = (int)sample_row(iy, scly, rrows).idx;
            }
            // memory guard only: valid candidates always sample inside the frame
            const int gx = min(max(rx + sx, 0), a.gw - 1), gy = min(max(ry + sy, 0), a.gh - 1);
            v[k] = a.gray[(size_t)gy * a.gpitch + gx];
        }
    }
    const bool eq = a.cfg.equalize != 0;
    uint32_t u[(kPerThread + 3) / 4];  // the bytes, four to a register
#pragma unroll
    for (int k = 0; k < (kPerThread + 3) / 4; ++k) u[k] = 0u;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int p = threadIdx.x + k * kWT;
        const uint32_t b = (uint8_t)__float2int_rz(fadd(v[k], 0.5f));
        u[k >> 2] |= b << (8 * (k & 3));
        if (p < kPx) {
            if (eq)
                atomicAdd(&S.hist[b], 1);
            else
                S.crop[p / kCropW][p % kCropW] = (uint8_t)b;
        }
    }
    __syncthreads();
    if (!eq) return;
    // cumulative histogram (256 bins, one per thread): shuffle scan + warp totals
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int c = S.hist[threadIdx.x];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y2 = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o) c += y2;
        }
        __shared__ int wsum[8];
        if (lane == 31) wsum[wid] = c;
        __syncthreads();
        int add = 0;
        for (int w = 0; w < wid; ++w) add += wsum[w];
        S.lut[threadIdx.x] = c + add;  // cf_hist
        __syncthreads();
    }
    const float bmin = (float)S.lut[0], bmax = (float)S.lut[255];
    if (bmin != bmax) {
        const float delt = fdiv(255.f, fsub(bmax, bmin));
        const int lv = (int)fadd(fmul(fsub((float)S.lut[threadIdx.x], bmin), delt), 0.5f);
        __syncthreads();
        S.lut[threadIdx.x] = lv;
        __syncthreads();
    }
    // the equalised bytes (the reference leaves the window unchanged when every pixel is equal)
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int p = threadIdx.x + k * kWT;
        const uint32_t b = (u[k >> 2] >> (8 * (k & 3))) & 0xffu;
        if (p < kPx) S.crop[p / kCropW][p % kCropW] = (uint8_t)(bmin != bmax ? S.lut[b] : b);
    }
    __syncthreads();
}

// One work item = (candidate, window): window 0 is the first crop, window 1 the shrunken retry
// crop. Both windows of a candidate run in parallel (the retry is speculative: the verdict reads it
// only when window 0 is rejected, cnn_detector_v3.cpp:1806-1811); running it on demand instead
// would save the ~10 % of retries whose first window accepts but put the two windows of a rejected
// candidate one after the other, doubling the kernel's latency. Inside an item, stage 3 runs only
// when stage 2 does not end the check (the reference's early exits, cnn_detector_v3.cpp:1698-1706);
// otherwise its slot keeps (max -10, count 0), exactly what the reference leaves behind.
// One work item: window `mod` of candidate ci, stage 2 then (unless an early exit ends the check)
// stage 3, the (max, count) pair of each written to a.out.
template <bool kLegacy>
__device__ __forceinline__ void window_item(const WindowNets& N, const WinArgs& a, WindowSmem& S, int ci, int mod) {
    const CascadeConfig& C = a.cfg;
    const Candidate cd = a.cands[ci];
    const LevelDesc& L = a.levels[cd.level];
    const int mn = (C.adapt_min_neighbors && L.scale > 0.7f && C.min_neighbors > 1) ? C.min_neighbors - 1 : C.min_neighbors;
    prepare_window(a, S, cd, L.inv_scale, mod);
    WinOut r[2];
    r[1].max = -10.f;
    r[1].knn = 0;
    for (int stage = 0; stage < 2; ++stage) {
        if constexpr (kLegacy)
            legacy_window_net(a.lg[1 + stage], S, stage == 0 ? 0 : (C.reflection ? 1 : 2));
        else if (stage == 0)
            window_net(N.s2, S, 0);
        else
            window_net(N.s3, S, C.reflection ? 1 : 2);
        // every thread reduces the 16 responses itself (no extra barrier needed)
        const float thr = stage == 0 ? C.thr2 : C.thr3;
        float mx = -10.f;
        int kc = 0;
#pragma unroll
        for (int o = 0; o < kOutN; ++o) {
            const float d = S.out[o];
            mx = (mx < d) ? d : mx;  // MAX(max_score, d) (cnn_detector_v3.cpp:1667-1683)
            if (d > thr) kc++;
        }
        r[stage].max = mx;
        r[stage].knn = kc;
        if (stage == 0) {
            const bool stop = (C.type_check == 0 && kc >= mn) || (C.type_check > 0 && kc <= 0) || (C.type_check == 2 && kc < mn);
            if (stop) break;
        }
    }
    if (threadIdx.x == 0) {
        a.out[(size_t)ci * 4 + 2 * mod] = r[0];
        a.out[(size_t)ci * 4 + 2 * mod + 1] = r[1];
    }
    __syncthreads();
}

// kMinBlocks: the register budget (2 resident blocks a SM: up to 128 registers, no spills; 4: 64;
// 5: 48; 6: 40, more spilled), matched to the schedule's resident blocks
template <bool kLegacy, int kMinBlocks>
__global__ void __launch_bounds__(kWT, kMinBlocks) window_kernel(const __grid_constant__ WindowNets N, const WinArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WindowSmem& S = *reinterpret_cast<WindowSmem*>(smem_raw);
    const int n = *a.n_cand;
    const int per_cand = a.cfg.double_check ? 2 : 1;
    const int total = n * per_cand;
    for (int it = blockIdx.x; it < total; it += gridDim.x) {
        const int ci = it / per_cand;
        window_item<kLegacy>(N, a, S, ci, it - ci * per_cand);
    }
}

// The candidates of every frame of a batch as one persistent item list (frame by frame); the
// per-frame gray image, candidates and outputs come from B, the rest from `base`.
template <int kMinBlocks>
__global__ void __launch_bounds__(kWT, kMinBlocks) window_batch_kernel(const __grid_constant__ WindowNets N, const WinArgs base,
                                                              const __grid_constant__ WinBatch B) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WindowSmem& S = *reinterpret_cast<WindowSmem*>(smem_raw);
    __shared__ int s_pre[kMaxBatch + 1];
    if (threadIdx.x == 0) {
        s_pre[0] = 0;
        for (int f = 0; f < B.n_frames; ++f) s_pre[f + 1] = s_pre[f] + *B.ncand[f];
    }
    __syncthreads();
    const int per_cand = base.cfg.double_check ? 2 : 1;
    const int total = s_pre[B.n_frames] * per_cand;
    for (int it = blockIdx.x; it < total; it += gridDim.x) {
        const int c = it / per_cand;
        int f = 0;
        while (s_pre[f + 1] <= c) ++f;
        WinArgs a = base;
        a.gray = B.gray[f];
        a.cands = B.cands[f];
        a.n_cand = B.ncand[f];
        a.out = B.out[f];
        window_item<false>(N, a, S, c - s_pre[f], it - c * per_cand);
    }
}

int window_smem_bytes() { return (int)sizeof(WindowSmem); }

cudaError_t launch_window_batch(const WindowNets& N, const WinBatch& B, int gpitch, int gw, int gh, const LevelDesc* levels,
                                const CascadeConfig& cfg, int grid, cudaStream_t st, int ctas_per_sm) {
    WinArgs a{};
    a.gpitch = gpitch;
    a.gw = gw;
    a.gh = gh;
    a.levels = levels;
    a.cfg = cfg;
    a.lg = nullptr;
    if (ctas_per_sm <= 2)
        window_batch_kernel<2><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a, B);
    else
        window_batch_kernel<4><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a, B);
    return cudaGetLastError();
}

cudaError_t launch_window(const WindowNets& N, const float* gray, int gpitch, int gw, int gh, const Candidate* cands, const int* n_cand,
                          const LevelDesc* levels, WinOut* out, const CascadeConfig& cfg, int grid, cudaStream_t st, const LegacyNet* lg,
                          int ctas_per_sm) {
    static_assert(sizeof(WindowSmem) + 64 <= 48 * 1024, "window kernel shared memory must stay under the default 48 KB");
    WinArgs a;
    a.gray = gray;
    a.gpitch = gpitch;
    a.gw = gw;
    a.gh = gh;
    a.cands = cands;
    a.n_cand = n_cand;
    a.levels = levels;
    a.out = out;
    a.cfg = cfg;
    a.lg = lg;
    if (lg)
        window_kernel<true, 4><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a);
    else if (ctas_per_sm <= 2)
        window_kernel<false, 2><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a);
    else if (ctas_per_sm == 5)
        window_kernel<false, 5><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a);
    else if (ctas_per_sm >= 6)
        window_kernel<false, 6><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a);
    else
        window_kernel<false, 4><<<grid, kWT, sizeof(WindowSmem), st>>>(N, a);
    return cudaGetLastError();
}

// five or six resident window blocks need most of a SM's 228 KB as shared memory
cudaError_t window_setup() {
    cudaError_t e = cudaFuncSetAttribute(window_kernel<false, 5>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(window_kernel<false, 6>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    return e;
}

}  // namespace ccnn
