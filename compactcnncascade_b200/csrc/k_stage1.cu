// Stage-1 fully-convolutional net over every pyramid level, in two launches per frame.
//
// Reference: SIMD::ConvNeuralNetwork::Run (src/CNNObjectDetector/cnn_simd_cntk.cpp:640-963) with
// the plain CNNPP primitives (cnnpp_cplusplus.cpp): conv_4x4 (:92-157), lrelu_bn_max (:593-622),
// add/add2 (:916-950), conv_3x3 (:36-91), conv_5x4 (:158-187), lrelu_bn (:623-645),
// mulCN_add_tanhW (:646-672), mulC/mulC1_add (:952-984), tanhW (:673-690).
//
// front: one CTA per 32x16 tile of pooled L1 pixels of one level. The CTA stages its (67 x 35)
//        input tile of the level image, runs the 4x4 conv + folded BN/LReLU + 2x2 max for the 4
//        L1 maps and writes the 4 neighbour-map sums that L2 consumes (S1 arena).
// back:  one CTA per 32x16 tile of response pixels. It stages the S1 tile (4 x 42 x 72) in shared
//        memory, computes the 8 pooled L2 maps and their sums on the 35 x 20 halo tile, then every
//        thread finishes two vertically adjacent response pixels: the 16 L3 maps (4w x 5h), the
//        52 hidden neurons and the output neuron.
// Packed f32x2 instructions run two identical chains of IEEE operations at once (two pixels, or
// two maps that read the same input), so every value still sees the reference's roundings.
// Every tile of every level is one block of the same grid; a block finds its level by binary
// search over the level descriptors (kernel parameters), so a frame is two launches per group of
// up to kParamLevels levels.
#include "kernels.h"
#include "resample.cuh"

namespace ccnn {

constexpr int kInW = 2 * kK1TileX + 3;  // 67
constexpr int kInH = 2 * kK1TileY + 3;  // 35
constexpr int kInWh = (kInW + 1) / 2;   // 34 columns of each parity

// One input sample of the front tile: row r, column c (tile coordinates) = value v. Row r is
// stored next to row r+2 as a packed pair (a thread computes two vertically adjacent pooled
// pixels, whose windows are 2 rows apart), and columns are split by parity so that the stride-2
// column walk of a warp is conflict-free.
struct FrontTile {
    float2 p[kInH - 2][2][kInWh];
    float tail[2][kInW];  // the last two rows have no partner below
    __device__ __forceinline__ void put(int r, int c, float v) {
        if (r < kInH - 2)
            p[r][c & 1][c >> 1].x = v;
        else
            tail[r - (kInH - 2)][c] = v;
        if (r >= 2) p[r - 2][c & 1][c >> 1].y = v;
    }
};

// Loads the (67 x 35) input tile of a front CTA from its level image. Rows that start 16-byte
// aligned with a pitch of whole float4 groups are read as 17 float4 per row (columns past the
// image width hold zeros or the caller's own padding; no stored pixel depends on them), other
// images one float at a time.
__device__ __forceinline__ void load_front_tile(FrontTile& T, const float* __restrict__ img, const LevelDesc& L, int ix0, int iy0) {
    if (L.img_vec) {
        constexpr int kV = (kInW + 3) / 4;  // 17
        for (int i = threadIdx.x; i < kInH * kV; i += blockDim.x) {
            const int r = i / kV, c4 = i - r * kV;
            const int x = ix0 + 4 * c4, y = iy0 + r;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (y < L.h && x < L.img_pitch) v = __ldg(reinterpret_cast<const float4*>(img + (long long)y * L.img_pitch + x));
            T.put(r, 4 * c4, v.x);
            T.put(r, 4 * c4 + 1, v.y);
            T.put(r, 4 * c4 + 2, v.z);
            if (4 * c4 + 3 < kInW) T.put(r, 4 * c4 + 3, v.w);
        }
    } else {
        for (int i = threadIdx.x; i < kInH * kInW; i += blockDim.x) {
            const int r = i / kInW, c = i - r * kInW;
            const int x = ix0 + c, y = iy0 + r;
            T.put(r, c, (x < L.w && y < L.h) ? __ldg(img + (long long)y * L.img_pitch + x) : 0.f);
        }
    }
}

__global__ void __launch_bounds__(256, 3) stage1_front_kernel(const __grid_constant__ Stage1W W, const __grid_constant__ LevelTable LT,
                                                              const float* __restrict__ limg, float* __restrict__ s1,
                                                              const uint8_t* __restrict__ front_on) {
    __shared__ FrontTile T;
    const int g = LT.first + blockIdx.x;
    if (front_on && !front_on[g]) return;  // gated off: no back tile reads this one
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::k1_base>(LT, g)];
    const int t = g - L.k1_base;
    const int px0 = (t % L.k1_tiles_x) * kK1TileX;
    const int py0 = (t / L.k1_tiles_x) * kK1TileY;
    const int ix0 = 2 * px0, iy0 = 2 * py0;

    load_front_tile(T, limg + L.img_off, L, ix0, iy0);
    __syncthreads();

    const int qx = threadIdx.x & (kK1TileX - 1);
    const int qy = (threadIdx.x >> 5) * 2;
    const f2_t nz = f2_ld(W.negzero);
    // pr[r][c] = (input row 2qy+r, row 2qy+r+2) at column 2qx+c: the windows of both pixels
    f2_t pr[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int c = 0; c < 5; ++c) pr[r][c] = *reinterpret_cast<const f2_t*>(&T.p[2 * qy + r][c & 1][qx + (c >> 1)]);

    // packed over the two pixels (lo = row qy, hi = row qy + 1)
    f2_t P[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        f2_t cv[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int dy = d >> 1, dx = d & 1;
            f2_t acc = f2_mul(pr[dy][dx], f2_ld(W.k1d[m][0]), nz);
#pragma unroll
            for (int k = 1; k < 16; ++k) acc = f2_add(acc, f2_mul(pr[dy + (k >> 2)][dx + (k & 3)], f2_ld(W.k1d[m][k]), nz));
            cv[d] = lrelu_bn2(acc, W.a1d[m], nz);
        }
        P[m] = f2_max4(cv[0], cv[1], cv[2], cv[3]);
    }
    // neighbour-map sums consumed by L2 (add/add2 of the reference)
    const f2_t s01 = f2_add(P[0], P[1]);
    const f2_t o[4] = {s01, f2_add(s01, P[2]), f2_add(f2_add(P[1], P[2]), P[3]), f2_add(P[2], P[3])};
    const int gx = px0 + qx, gy = py0 + qy;
    if (gx < L.p1w) {
        float* out = s1 + L.s1_off + (long long)gy * L.s1_pitch + gx;
        if (gy < L.p1h) {
#pragma unroll
            for (int k = 0; k < 4; ++k) out[k * L.s1_plane] = f2_lo(o[k]);
        }
        if (gy + 1 < L.p1h) {
#pragma unroll
            for (int k = 0; k < 4; ++k) out[k * L.s1_plane + L.s1_pitch] = f2_hi(o[k]);
        }
    }
}

constexpr int kP2TW = kK2TileX + 3;   // 35 pooled L2 columns (halo 3)
constexpr int kP2TH = kK2TileY + 4;   // 20 pooled L2 rows (halo 4)
constexpr int kS1TW = 2 * kP2TW + 2;  // 72
constexpr int kS1TH = 2 * kP2TH + 2;  // 42
constexpr int kS1TWh = kS1TW / 2;     // 36 columns of each parity
constexpr int kS2P = kP2TW + 1;       // 36: ts2 row pitch

struct BackSmem {
    float s1[4][kS1TH][kS1TW];    // column c stored at (c & 1) * kS1TWh + (c >> 1)
    float s2[8][kP2TH][kS2P];     // the 8 neighbour sums of the pooled L2 maps
};
constexpr int kBackSmemBytes = (int)sizeof(BackSmem);

// back: one CTA per 32 x 16 tile of response pixels.
//   A: the S1 tile (4 x 42 x 72) is staged in shared memory with 16-byte loads;
//   B: the 8 pooled L2 maps and their sums on the 35 x 20 halo tile (maps 2i and 2i+1 read the
//      same S1 map i: one packed pair);
//   C: every thread finishes two vertically adjacent response pixels, every operation packed over
//      the pair: the 16 L3 maps (4w x 5h), the 52 hidden neurons and the output neuron.
__global__ void __launch_bounds__(256, 3) stage1_back_kernel(const __grid_constant__ Stage1W W, const __grid_constant__ Stage1Dup D,
                                                             const __grid_constant__ LevelTable LT, const float* __restrict__ s1,
                                                             float* __restrict__ resp, int* __restrict__ counts, float thr,
                                                             const uint8_t* __restrict__ back_on, const GateCells cells) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BackSmem& S = *reinterpret_cast<BackSmem*>(smem_raw);
    const int g = LT.first + blockIdx.x;
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::k2_base>(LT, g)];
    const int t = g - L.k2_base;
    const int ox0 = (t % L.k2_tiles_x) * kK2TileX;
    const int oy0 = (t / L.k2_tiles_x) * kK2TileY;
    if (back_on && !back_on[g]) {  // gated off: responses below any stage-1 threshold
        for (int i = threadIdx.x; i < kK2TileX * kK2TileY; i += blockDim.x) {
            const int gx = ox0 + (i & (kK2TileX - 1)), gy = oy0 + i / kK2TileX;
            if (gx < L.ow && gy < L.oh) resp[L.resp_off + (long long)gy * L.ow + gx] = -1e30f;
        }
        return;
    }
    const int sx0 = 2 * ox0, sy0 = 2 * oy0;

    // A: rows of 18 float4; columns past the plane pitch and rows past p1h read as 0 (no valid
    // response pixel depends on them)
    {
        const float* base = s1 + L.s1_off;
        constexpr int kV = kS1TW / 4;
        for (int i = threadIdx.x; i < 4 * kS1TH * kV; i += blockDim.x) {
            const int row = i / kV, c4 = i - row * kV;
            const int m = row / kS1TH, rr = row - m * kS1TH;
            const int x = sx0 + 4 * c4, y = sy0 + rr;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (y < L.p1h && x < L.s1_pitch)
                v = __ldg(reinterpret_cast<const float4*>(base + m * L.s1_plane + (long long)y * L.s1_pitch + x));
            *reinterpret_cast<float2*>(&S.s1[m][rr][2 * c4]) = make_float2(v.x, v.z);
            *reinterpret_cast<float2*>(&S.s1[m][rr][kS1TWh + 2 * c4]) = make_float2(v.y, v.w);
        }
    }
    __syncthreads();

    const f2_t nz = f2_ld(W.negzero);
    // B
    for (int p = threadIdx.x; p < kP2TW * kP2TH; p += blockDim.x) {
        const int x = p % kP2TW, y = p / kP2TW;
        f2_t P[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            f2_t q[4][4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) q[r][c] = f2_dup(S.s1[i][2 * y + r][(c & 1) * kS1TWh + x + (c >> 1)]);
            f2_t cv[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const int dy = d >> 1, dx = d & 1;
                f2_t acc = f2_mul(q[dy][dx], f2_ld(W.k2p[i][0]), nz);
#pragma unroll
                for (int k = 1; k < 9; ++k) acc = f2_add(acc, f2_mul(q[dy + k / 3][dx + k % 3], f2_ld(W.k2p[i][k]), nz));
                cv[d] = lrelu_bn2(acc, W.a2p[i], nz);
            }
            P[i] = f2_max4(cv[0], cv[1], cv[2], cv[3]);  // (map 2i, map 2i+1)
        }
        float Pm[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Pm[2 * i] = f2_lo(P[i]);
            Pm[2 * i + 1] = f2_hi(P[i]);
        }
        S.s2[0][y][x] = fadd(Pm[0], Pm[1]);
#pragma unroll
        for (int k = 1; k < 7; ++k) S.s2[k][y][x] = fadd(fadd(Pm[k - 1], Pm[k]), Pm[k + 1]);
        S.s2[7][y][x] = fadd(Pm[6], Pm[7]);
    }
    __syncthreads();

    // C: pixels (x, y) and (x, y + 1)
    const int x = threadIdx.x & (kK2TileX - 1), y = (threadIdx.x / kK2TileX) * 2;
    // L3 maps (2k, 2k+1) of the pixel pair, both from neighbour-sum map k; conv_5x4 keeps one
    // partial sum per kernel row, added in row order
    auto l3_pair = [&](int k, f2_t* m0, f2_t* m1) {
        float v[6][4];
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) v[r][c] = S.s2[k][y + r][x + c];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int mm = 2 * k + e;
            f2_t acc = 0ull;
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                f2_t rs = f2_mul(f2_pack(v[r][0], v[r + 1][0]), f2_ld(D.k3d[mm][4 * r]), nz);
#pragma unroll
                for (int c = 1; c < 4; ++c) rs = f2_add(rs, f2_mul(f2_pack(v[r][c], v[r + 1][c]), f2_ld(D.k3d[mm][4 * r + c]), nz));
                acc = (r == 0) ? rs : f2_add(acc, rs);
            }
            *(e == 0 ? m0 : m1) = lrelu_bn2(acc, D.a3d[mm], nz);
        }
    };
    // hidden neuron n = 4*i + t reads L3 maps i..i+3: the groups run as a loop over a sliding window
    // of four maps (a0..a3, with the second map of the last computed pair kept in `spare`), so the
    // code stays small; the output sum runs over n in order
    static_assert(Stage1W::kConn == 4 && Stage1W::kGroups + 3 == Stage1W::kM3, "sliding window of four L3 maps");
    f2_t a0, a1, a2, a3, spare;
    l3_pair(0, &a0, &a1);
    l3_pair(1, &a2, &spare);
    const f2_t half = f2_pack(0.5f, 0.5f);
    f2_t out = 0ull;
#pragma unroll 1
    for (int i = 0; i < Stage1W::kGroups; ++i) {
        const int m = i + 3;  // the group's newest map
        if (m & 1) a3 = spare;
        else l3_pair(m >> 1, &a3, &spare);
#pragma unroll
        for (int tt = 0; tt < Stage1W::kHS; ++tt) {
            const int n = Stage1W::kHS * i + tt;
            f2_t s = f2_ld(D.hbd[n]);
            s = f2_add(s, f2_mul(a0, f2_ld(D.hwd[n][0]), nz));
            s = f2_add(s, f2_mul(a1, f2_ld(D.hwd[n][1]), nz));
            s = f2_add(s, f2_mul(a2, f2_ld(D.hwd[n][2]), nz));
            s = f2_add(s, f2_mul(a3, f2_ld(D.hwd[n][3]), nz));
            s = f2_mul(s, f2_ld(D.htwd[i]), nz);
            f2_t v = tanh_rational2(s, nz);
            v = f2_add(f2_mul(half, v, nz), half);
            const f2_t h = f2_add(f2_mul(f2_ld(D.hbnwd[tt]), v, nz), f2_ld(D.hbnbd[tt]));
            const f2_t hw = f2_mul(h, f2_ld(D.owd[n]), nz);
            out = (n == 0) ? hw : f2_add(hw, out);
        }
        a0 = a1;
        a1 = a2;
        a2 = a3;
    }
    f2_t c = f2_mul(f2_add(out, f2_ld(D.obd)), f2_ld(D.otwd), nz);
    c = tanh_rational2(c, nz);
    const f2_t r = (W.af == 0.f) ? f2_add(f2_mul(half, c, nz), half) : f2_mul(f2_ld(D.afd), c, nz);
    const int gx = ox0 + x, gy = oy0 + y;
    if (gx < L.ow) {
        float rv[2] = {f2_lo(r), f2_hi(r)};
        if (cells.bits && (rv[0] > thr || rv[1] > thr) && *cells.ambiguous <= cells.amb_limit) {
            // learned gate, per candidate: its window centre ((4x + 11.5) / s, (4y + 13.5) / s) needs a
            // likely cell of its octave within one cell
            const uint32_t* B = cells.bits + (long long)min(L.octave, kGK - 1) * cells.h16 * cells.wwords;
            const int cx = (int)((4.f * gx + 11.5f) * L.inv_scale) / 16;
            for (int k = 0; k < 2; ++k) {
                if (!(rv[k] > thr)) continue;
                const int cy = (int)((4.f * (gy + k) + 13.5f) * L.inv_scale) / 16;
                if (!gate_any_bit(B, cells.wwords, max(0, cx - 1), min(cells.w16 - 1, cx + 1), max(0, cy - 1), min(cells.h16 - 1, cy + 1)))
                    rv[k] = -1e30f;
            }
        }
        // candidates (response > treshold_1) are counted per scan chunk for the compaction
        if (gy < L.oh) {
            resp[L.resp_off + (long long)gy * L.ow + gx] = rv[0];
            if (counts && rv[0] > thr) atomicAdd(&counts[L.chunk_base + (gy * L.ow + gx) / kCandChunk], 1);
        }
        if (gy + 1 < L.oh) {
            resp[L.resp_off + (long long)(gy + 1) * L.ow + gx] = rv[1];
            if (counts && rv[1] > thr) atomicAdd(&counts[L.chunk_base + ((gy + 1) * L.ow + gx) / kCandChunk], 1);
        }
    }
}

// Duplicated stage-1 parameters for the back kernel, derived from the packed weight block.
static Stage1Dup make_dup(const Stage1W& W) {
    Stage1Dup D;
    auto dup = [](float v) { return make_float2(v, v); };
    for (int i = 0; i < Stage1W::kM3 / 2; ++i)
        for (int k = 0; k < Stage1W::kK3W * Stage1W::kK3H; ++k) {
            D.k3d[2 * i][k] = dup(W.k3p[i][k].x);
            D.k3d[2 * i + 1][k] = dup(W.k3p[i][k].y);
        }
    for (int mm = 0; mm < Stage1W::kM3; ++mm) {
        D.a3d[mm][0] = dup(W.b3[mm]);
        D.a3d[mm][1] = dup(W.w3a[mm]);
        D.a3d[mm][2] = dup(W.w3b[mm]);
        D.a3d[mm][3] = dup(W.bn3[mm]);
    }
    for (int q = 0; q < Stage1W::kHL / 2; ++q)
        for (int j = 0; j < Stage1W::kConn; ++j) {
            D.hwd[2 * q][j] = dup(W.hwp[q][j].x);
            D.hwd[2 * q + 1][j] = dup(W.hwp[q][j].y);
        }
    for (int n = 0; n < Stage1W::kHL; ++n) {
        D.hbd[n] = dup(W.hb[n]);
        D.owd[n] = dup(W.ow[n]);
    }
    for (int i = 0; i < Stage1W::kGroups; ++i) D.htwd[i] = dup(W.htw[i]);
    for (int tt = 0; tt < Stage1W::kHS; ++tt) {
        D.hbnwd[tt] = dup(W.hbnw[tt]);
        D.hbnbd[tt] = dup(W.hbnb[tt]);
    }
    D.obd = dup(W.ob);
    D.otwd = dup(W.otw);
    D.afd = dup(W.af);
    return D;
}

cudaError_t stage1_setup() {
    return cudaFuncSetAttribute(stage1_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kBackSmemBytes);
}

// Launches KERNEL once per group of at most kParamLevels levels; tiles(L) is a level's block count
// and base(L) its first global block.
template <class Launch, class Tiles>
static cudaError_t launch_grouped(const LevelDesc* levels, int n_levels, int LevelDesc::*base, Tiles tiles, Launch launch) {
    for (int g0 = 0; g0 < n_levels; g0 += kParamLevels) {
        LevelTable T;
        T.n = n_levels - g0 < kParamLevels ? n_levels - g0 : kParamLevels;
        for (int i = 0; i < T.n; ++i) T.lv[i] = levels[g0 + i];
        T.first = T.lv[0].*base;
        const LevelDesc& last = T.lv[T.n - 1];
        const int blocks = last.*base + tiles(last) - T.first;
        if (blocks > 0) launch(T, blocks);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t launch_stage1_front(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* limg, float* s1, cudaStream_t st,
                                const uint8_t* front_on) {
    return launch_grouped(
        levels, n_levels, &LevelDesc::k1_base, [](const LevelDesc& L) { return L.k1_tiles_x * ((L.p1h + kK1TileY - 1) / kK1TileY); },
        [&](const LevelTable& T, int blocks) { stage1_front_kernel<<<blocks, 256, 0, st>>>(W, T, limg, s1, front_on); });
}

cudaError_t launch_stage1_back(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* s1, float* resp, cudaStream_t st,
                               int* counts, float thr, const uint8_t* back_on, GateCells cells) {
    const Stage1Dup D = make_dup(W);
    return launch_grouped(
        levels, n_levels, &LevelDesc::k2_base, [](const LevelDesc& L) { return L.k2_tiles_x * ((L.oh + kK2TileY - 1) / kK2TileY); },
        [&](const LevelTable& T, int blocks) { stage1_back_kernel<<<blocks, 256, kBackSmemBytes, st>>>(W, D, T, s1, resp, counts, thr, back_on, cells); });
}

cudaError_t launch_stage1(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* limg, float* s1, float* resp,
                          cudaStream_t st, int* counts, float thr, const uint8_t* front_on, const uint8_t* back_on, GateCells cells) {
    cudaError_t e = launch_stage1_front(W, levels, n_levels, limg, s1, st, front_on);
    if (e != cudaSuccess) return e;
    return launch_stage1_back(W, levels, n_levels, s1, resp, st, counts, thr, back_on, cells);
}

}  // namespace ccnn
