// Stage-1 fully-convolutional net over every pyramid level, in two launches per frame.
//
// Reference: SIMD::ConvNeuralNetwork::Run (src/CNNObjectDetector/cnn_simd_cntk.cpp:640-963) with
// the plain CNNPP primitives (cnnpp_cplusplus.cpp): conv_4x4 (:92-157), lrelu_bn_max (:593-622),
// add/add2 (:916-950), conv_3x3 (:36-91), conv_5x4 (:158-187), lrelu_bn (:623-645),
// mulCN_add_tanhW (:646-672), mulC/mulC1_add (:952-984), tanhW (:673-690).
//
// front: one CTA per 32x16 tile of pooled L1 pixels of one level. The CTA resamples its (67 x 35)
//        input tile straight from the gray frame (the pyramid is never stored; a stored image is read
//        instead where the caller gives one; with the learned gate each warp resamples only the 7
//        rows of its own two pooled rows and runs on its own), runs the 4x4 conv + folded
//        BN/LReLU + 2x2 max for the 4 L1 maps and writes the 4 neighbour-map sums that L2 consumes
//        (S1 arena).
// back:  one CTA per 32x16 tile of response pixels. It stages the S1 tile (4 x 42 x 72) one map at a
//        time through two shared-memory buffers (asynchronous copies of the next map overlap the
//        current one's compute), computes the 8 pooled L2 maps and their sums on the 35 x 20 halo
//        tile, then every thread finishes two vertically adjacent response pixels: the 16 L3 maps
//        (4w x 5h), the 52 hidden neurons and the output neuron.
// Both kernels come in two register budgets (3 or 4 resident 256-thread blocks per SM), chosen per
// workload by the schedule (Stage1Sched).
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
// images one float at a time. kCoherent: the image was written earlier in the same launch (read
// through L2, never the read-only path).
template <bool kCoherent>
__device__ __forceinline__ void load_front_tile(FrontTile& T, const float* __restrict__ img, const LevelDesc& L, int ix0, int iy0) {
    if (L.img_vec) {
        constexpr int kV = (kInW + 3) / 4;  // 17
        for (int i = threadIdx.x; i < kInH * kV; i += blockDim.x) {
            const int r = i / kV, c4 = i - r * kV;
            const int x = ix0 + 4 * c4, y = iy0 + r;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (y < L.h && x < L.img_pitch) {
                const float4* src = reinterpret_cast<const float4*>(img + (long long)y * L.img_pitch + x);
                v = kCoherent ? __ldcg(src) : __ldg(src);
            }
            T.put(r, 4 * c4, v.x);
            T.put(r, 4 * c4 + 1, v.y);
            T.put(r, 4 * c4 + 2, v.z);
            if (4 * c4 + 3 < kInW) T.put(r, 4 * c4 + 3, v.w);
        }
    } else {
        for (int i = threadIdx.x; i < kInH * kInW; i += blockDim.x) {
            const int r = i / kInW, c = i - r * kInW;
            const int x = ix0 + c, y = iy0 + r;
            const float* src = img + (long long)y * L.img_pitch + x;
            T.put(r, c, (x < L.w && y < L.h) ? (kCoherent ? __ldcg(src) : __ldg(src)) : 0.f);
        }
    }
}

// The input rows of one warp of a gated front tile: warp w computes pooled rows 2w and 2w + 1 from
// tile rows 4w .. 4w + 6, held here as local rows 0..6, row r next to row r + 2 (columns split by
// parity, as in FrontTile). Rows 4w + 4 .. 4w + 6 are also the next warp's first three; each warp
// resamples its own copy, so no block barrier separates resampling and compute.
struct FrontWarpRows {
    float2 p[5][2][kInWh];
    __device__ __forceinline__ void put(int r, int c, float v) {
        if (r <= 4) p[r][c & 1][c >> 1].x = v;
        if (r >= 2) p[r - 2][c & 1][c >> 1].y = v;
    }
};

struct FrontSmem {
    union {
        FrontTile T;                    // the block's whole input tile (full scan, or a stored level image)
        FrontWarpRows w[kK1TileY / 2];  // each warp's own input rows (gated scan from the gray frame)
    };
};

// level pixel (x, y) = tile (c, r) from its column sample sx
__device__ __forceinline__ float resample_px(const GrayRef& G, const LevelDesc& L, const AxisSample& sx, int x, int y) {
    if (x >= L.w || y >= L.h) return 0.f;
    if (L.mode == 0) return __ldg(G.p + (size_t)y * G.pitch + x);
    const AxisSample sy = sample_row(y, L.scly, G.h);
    if (L.mode == 1) return __ldg(G.p + (size_t)sy.idx * G.pitch + sx.idx);
    uint32_t py = sy.idx;
    if (py + 1 >= (uint32_t)G.h) py--;  // bilinear keeps a row below
    const float* r0 = G.p + (size_t)py * G.pitch + sx.idx;
    const float top = fadd(fmul(__ldg(r0), sx.c), fmul(__ldg(r0 + 1), sx.f));
    const float bot = fadd(fmul(__ldg(r0 + G.pitch), sx.c), fmul(__ldg(r0 + G.pitch + 1), sx.f));
    return fadd(fmul(top, sy.c), fmul(bot, sy.f));
}

// Front-tile input straight from the gray frame: every level pixel resampled the way the pyramid
// kernel writes it (copy, nearest neighbour, or bilinear on the 12-bit fixed-point steps;
// RunCPUDetect, cnn_detector_v3.cpp:2090-2104, with ImageResizer, image_resize.cpp:46-122, 393-541),
// so the level image is never stored. Pixels outside the level read as 0, like the zero columns past
// a stored level image's width. The gray frame was written by an earlier launch (read-only path).
//
// The whole (67 x 35) tile by the block (the full scan: every warp computes, so no row is resampled
// twice): thread (g, c) takes tile column c < 64 (its column sample in registers) and rows g, g + 4,
// ... of it, so a warp reads 32 neighbouring columns of the same gray rows; columns 64-66 follow, one
// sample a thread.
__device__ __forceinline__ void resample_front_tile(FrontTile& T, const GrayRef& G, const LevelDesc& L, int ix0, int iy0) {
    static_assert(kInW == 67 && kInH == 35, "64 + 3 columns, 35 rows in 4 row groups");
    {
        const int c = threadIdx.x & 63, g = threadIdx.x >> 6;
        const AxisSample sx = sample_col(ix0 + c, L.sclx, G.w);
#pragma unroll
        for (int k = 0; k < (kInH + 3) / 4; ++k) {
            const int r = g + 4 * k;
            if (r < kInH) T.put(r, c, resample_px(G, L, sx, ix0 + c, iy0 + r));
        }
    }
    if (threadIdx.x < 3 * kInH) {
        const int c = 64 + threadIdx.x % 3, r = threadIdx.x / 3;
        T.put(r, c, resample_px(G, L, sample_col(ix0 + c, L.sclx, G.w), ix0 + c, iy0 + r));
    }
}

// One warp's 7 input rows from tile row y0 on (the gated scan, where warps run on their own): lane l
// takes tile columns l and l + 32 (their column samples in registers); columns 64-66 of the rows
// follow, one sample a lane.
__device__ __forceinline__ void resample_warp_rows(FrontWarpRows& R, const GrayRef& G, const LevelDesc& L, int ix0, int y0, int lane) {
    const AxisSample sa = sample_col(ix0 + lane, L.sclx, G.w), sb = sample_col(ix0 + lane + 32, L.sclx, G.w);
#pragma unroll
    for (int r = 0; r < 7; ++r) {
        const float va = resample_px(G, L, sa, ix0 + lane, y0 + r);
        const float vb = resample_px(G, L, sb, ix0 + lane + 32, y0 + r);
        R.put(r, lane, va);
        R.put(r, lane + 32, vb);
    }
    if (lane < 21) {
        const int c = 64 + lane % 3, r = lane / 3;
        R.put(r, c, resample_px(G, L, sample_col(ix0 + c, L.sclx, G.w), ix0 + c, y0 + r));
    }
}

// The learned gate inside a running stage-1 tile: whether any response pixel of [rx0, rx1] x [ry0, ry1]
// (clamped to the level's response map) has a likely cell of the level's octave within the margin of
// its window centre ((4x + 11.5) / s, (4y + 13.5) / s). The centre moves monotonically with x and y, so
// the rectangle's cells are those of its corners (the same rule as the gate's tile decisions). Only
// live response pixels can become candidates; everything else a gated tile computes is skipped.
__device__ __forceinline__ bool gate_gating(const GateCells& cells) { return cells.bits && *cells.ambiguous <= cells.amb_limit; }

__device__ __forceinline__ bool gate_live(const GateCells& cells, const LevelDesc& L, int rx0, int rx1, int ry0, int ry1) {
    rx0 = max(rx0, 0);
    ry0 = max(ry0, 0);
    rx1 = min(rx1, L.ow - 1);
    ry1 = min(ry1, L.oh - 1);
    if (rx0 > rx1 || ry0 > ry1) return false;
    const int px0 = (int)((4.f * rx0 + 11.5f) * L.inv_scale), px1 = (int)((4.f * rx1 + 11.5f) * L.inv_scale);
    const int py0 = (int)((4.f * ry0 + 13.5f) * L.inv_scale), py1 = (int)((4.f * ry1 + 13.5f) * L.inv_scale);
    const uint32_t* B = cells.bits + (long long)min(L.octave, kGK - 1) * cells.h16 * cells.wwords;
    const int m = cells.margin;
    return gate_any_bit(B, cells.wwords, gate_cell_lo(px0, m), gate_cell_hi(px1, m, cells.w16), gate_cell_lo(py0, m),
                        gate_cell_hi(py1, m, cells.h16));
}

// Front tile t of level L: its (67 x 35) level-image tile in shared memory (resampled from the gray
// frame G when kFromGray, by the block, or with the gate by each warp for its own 7 rows; else read
// from the stored level images limg by the block), then the 4x4 conv + folded
// BN/LReLU + 2x2 max of the 4 L1 maps for 32 x 16 pooled pixels (two vertically adjacent pixels a
// thread) and the 4 neighbour-map sums written to the S1 arena. kCoherent: a stored level image was
// written earlier in the same launch (read through L2, not the read-only path).
// cells (the learned gate, optional): a warp whose S1 strip (2 rows x 32 columns) feeds no live
// response pixel writes nothing. S1 row y feeds pooled-L2 rows ceil((y - 3) / 2) .. y / 2 (a 3x3
// conv at the 2x2 pool positions), and L2 row Y feeds response rows Y - 4 .. Y (the 4-wide, 5-tall L3
// kernel); columns alike with the 4-wide kernel. The back kernel computes exactly the live pixels'
// inputs, so a skipped strip is never read for a value that is kept.
template <bool kFromGray, bool kCoherent>
__device__ __forceinline__ void front_tile(const Stage1W& W, FrontSmem& S, const LevelDesc& L, int t, const float* __restrict__ limg,
                                           const GrayRef& G, float* __restrict__ s1, const GateCells& cells) {
    const int px0 = (t % L.k1_tiles_x) * kK1TileX;
    const int py0 = (t / L.k1_tiles_x) * kK1TileY;
    const int ix0 = 2 * px0, iy0 = 2 * py0;

    const int qx = threadIdx.x & (kK1TileX - 1);
    const int qy = (threadIdx.x >> 5) * 2;
    // with the gate: whether the warp has a live pixel downstream (warp w computes pooled rows 2w, 2w + 1)
    auto warp_live = [&]() {
        const int ya = py0 + qy, yb = ya + 1, xa = px0, xb = px0 + kK1TileX - 1;
        return gate_live(cells, L, ((xa - 3 + 1) >> 1) - 3, xb >> 1, ((ya - 3 + 1) >> 1) - 4, yb >> 1);
    };
    const float2(*In)[2][kInWh];  // In[r] = (input row 2qy + r, row 2qy + r + 2), r = 0..4
    if (kFromGray && gate_gating(cells)) {
        // with the gate every warp runs on its own: its liveness, its 7 input rows, its two pooled rows
        // (the rows a live warp shares with a dead neighbour are not resampled twice over the tile, and
        // no warp waits for the block)
        int lv = 0;
        if ((threadIdx.x & 31) == 0) lv = warp_live() ? 1 : 0;
        if (!__shfl_sync(0xffffffffu, lv, 0)) return;  // no live response pixel downstream of this warp
        FrontWarpRows& R = S.w[threadIdx.x >> 5];
        resample_warp_rows(R, G, L, ix0, iy0 + 2 * qy, threadIdx.x & 31);
        __syncwarp();
        In = R.p;
    } else if (kFromGray) {
        // the full scan: the block resamples the tile once
        resample_front_tile(S.T, G, L, ix0, iy0);
        __syncthreads();
        In = &S.T.p[2 * qy];
    } else {
        uint32_t live = 0xffu;
        if (gate_gating(cells)) {
            __shared__ int s_flive[kK1TileY / 2];
            if ((threadIdx.x & 31) == 0) s_flive[threadIdx.x >> 5] = warp_live() ? 1 : 0;
            __syncthreads();
            live = 0u;
#pragma unroll
            for (int w = 0; w < kK1TileY / 2; ++w)
                if (s_flive[w]) live |= 1u << w;
        }
        load_front_tile<kCoherent>(S.T, limg + L.img_off, L, ix0, iy0);
        __syncthreads();
        if (!((live >> (threadIdx.x >> 5)) & 1u)) return;  // no live response pixel downstream of this warp
        In = &S.T.p[2 * qy];
    }
    const f2_t nz = f2_ld(W.negzero);
    // pr[r][c] = (input row 2qy+r, row 2qy+r+2) at column 2qx+c: the windows of both pixels
    f2_t pr[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int c = 0; c < 5; ++c) pr[r][c] = *reinterpret_cast<const f2_t*>(&In[r][c & 1][qx + (c >> 1)]);

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


// kFromGray: level tiles resampled from the gray frame G (the detection path), else read from the
// stored level images limg (a caller's own level image)
template <bool kFromGray, int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) stage1_front_kernel(const __grid_constant__ Stage1W W, const __grid_constant__ LevelTable LT,
                                                              const float* __restrict__ limg, const GrayRef G, float* __restrict__ s1,
                                                              const uint8_t* __restrict__ front_on, const GateCells cells) {
    __shared__ FrontSmem S;
    const int g = LT.first + blockIdx.x;
    if (front_on && !front_on[g]) return;  // gated off: no back tile reads this one
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::k1_base>(LT, g)];
    front_tile<kFromGray, false>(W, S, L, g - L.k1_base, limg, G, s1, cells);
}

constexpr int kP2TW = kK2TileX + 3;   // 35 pooled L2 columns (halo 3)
constexpr int kP2TH = kK2TileY + 4;   // 20 pooled L2 rows (halo 4)
constexpr int kS1TW = 2 * kP2TW + 2;  // 72
constexpr int kS1TH = 2 * kP2TH + 2;  // 42
constexpr int kS2P = kP2TW + 1;       // 36: ts2 row pitch

struct BackSmem {
    float s1[2][kS1TH][kS1TW];    // two S1 maps of the tile, row-major: map k in s1[k & 1] (double buffer)
    float s2[8][kP2TH][kS2P];     // the 8 neighbour sums of the pooled L2 maps
};
constexpr int kBackSmemBytes = (int)sizeof(BackSmem);  // 47,232 B: four blocks fit a SM
constexpr int kP2Px = kP2TW * kP2TH;                    // 700 pooled L2 pixels of a tile
constexpr int kP2Passes = (kP2Px + 255) / 256;          // 3

// Pooled L2 pixel k of a tile: the 32 x 20 block first (a warp takes 32 consecutive columns of one
// row, so its shared-memory reads and writes are conflict-free), then the 3 x 20 right edge.
__device__ __forceinline__ void p2_pixel(int p, int* x, int* y) {
    if (p < 32 * kP2TH) {
        *x = p & 31;
        *y = p >> 5;
    } else {
        const int q = p - 32 * kP2TH;
        *x = 32 + q % 3;
        *y = q / 3;
    }
}

// S1 map k of a back tile into S.s1[k & 1] by asynchronous 16-byte copies (cp.async through L2, one
// commit group); columns past the plane pitch and rows past p1h are zero-filled (no valid response
// pixel depends on them). The copies land while the block computes on the other buffer.
__device__ __forceinline__ void load_back_map_async(BackSmem& S, const float* __restrict__ s1, const LevelDesc& L, int sx0, int sy0, int k) {
    const float* base = s1 + L.s1_off + (long long)k * L.s1_plane;
    constexpr int kV = kS1TW / 4;
    float* buf = &S.s1[k & 1][0][0];
    for (int i = threadIdx.x; i < kS1TH * kV; i += blockDim.x) {
        const int rr = i / kV, c4 = i - rr * kV;
        const int x = sx0 + 4 * c4, y = sy0 + rr;
        const bool in = y < L.p1h && x < L.s1_pitch;  // x and the pitch are multiples of 4: the whole vector is in the row
        const float* src = in ? base + (long long)y * L.s1_pitch + x : base;
        const unsigned dst = (unsigned)__cvta_generic_to_shared(buf + rr * kS1TW + 4 * c4);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(in ? 16 : 0) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The pooled L2 maps (2i, 2i+1) at tile pixel (x, y), both from S1 map i (the buffer T): 3x3 conv +
// BN/LReLU at the four positions of the 2x2 window, then their max. A warp reads 32 consecutive
// column pairs of a row (8-byte loads, no bank conflicts).
__device__ __forceinline__ f2_t pool_l2_pair(const float (*T)[kS1TW], const Stage1W& W, int i, int x, int y, f2_t nz) {
    f2_t q[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const float2 u = *reinterpret_cast<const float2*>(&T[2 * y + r][2 * x]);
        const float2 v = *reinterpret_cast<const float2*>(&T[2 * y + r][2 * x + 2]);
        q[r][0] = f2_dup(u.x);
        q[r][1] = f2_dup(u.y);
        q[r][2] = f2_dup(v.x);
        q[r][3] = f2_dup(v.y);
    }
    f2_t cv[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const int dy = d >> 1, dx = d & 1;
        f2_t acc = f2_mul(q[dy][dx], f2_ld(W.k2p[i][0]), nz);
#pragma unroll
        for (int k = 1; k < 9; ++k) acc = f2_add(acc, f2_mul(q[dy + k / 3][dx + k % 3], f2_ld(W.k2p[i][k]), nz));
        cv[d] = lrelu_bn2(acc, W.a2p[i], nz);
    }
    return f2_max4(cv[0], cv[1], cv[2], cv[3]);
}

// back: one CTA per 32 x 16 tile of response pixels.
//   A/B map by map: the four S1 maps of the tile (42 x 72 each) pass through two shared-memory
//      buffers, map k + 1 copied asynchronously while the pooled L2 maps (2k, 2k+1) are computed from
//      map k on the 35 x 20 halo tile (one packed pair); the neighbour sums are written as soon as
//      their three maps are known, the two partial sums a pixel still needs kept in registers. Two
//      S1 maps in shared memory is what lets four blocks share a SM.
//   C: every thread finishes two vertically adjacent response pixels, every operation packed over
//      the pair: the 16 L3 maps (4w x 5h), the 52 hidden neurons and the output neuron.
// Back tile t of level L as above; g is its global back-tile index (the gate's tile index).
// kCoherent: the S1 arena was written earlier in the same launch (read through L2).
// With the learned gate (cells), a warp (32 x 2 response pixels) without a live pixel writes the skip
// marker instead of computing, the L2 phase computes only the rows live warps read (warp w reads L2
// rows 2w .. 2w + 5), and every pixel that is not live is written as the skip marker: only live
// pixels can become candidates, and their inputs are exactly what runs (the front kernel skips the
// rest of S1).
template <bool kCoherent>
__device__ __forceinline__ void back_tile(const Stage1W& W, const Stage1Dup& D, BackSmem& S, const LevelDesc& L, int t, int g,
                                          const float* __restrict__ s1, float* __restrict__ resp, int* __restrict__ counts, float thr,
                                          const uint8_t* __restrict__ back_on, const GateCells& cells) {
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
    const f2_t nz = f2_ld(W.negzero);
    const bool gating = gate_gating(cells);
    __shared__ int s_live[kK2TileY / 2];  // per warp: any live response pixel
    if (gating && (threadIdx.x & 31) == 0) {
        const int ry = oy0 + 2 * (threadIdx.x >> 5);
        s_live[threadIdx.x >> 5] = gate_live(cells, L, ox0, ox0 + kK2TileX - 1, ry, ry + 1) ? 1 : 0;
    }

    load_back_map_async(S, s1, L, sx0, sy0, 0);
    load_back_map_async(S, s1, L, sx0, sy0, 1);
    uint32_t live = 0xffu;  // live warps
    // L2 row y is read by warps ceil((y - 5) / 2) .. y / 2
    auto need_row = [&](int y) {
        const int wlo = max(0, (y - 5 + 1) >> 1), whi = min(kK2TileY / 2 - 1, y >> 1);
        return wlo <= whi && ((live >> wlo) & ((1u << (whi - wlo + 1)) - 1u)) != 0u;
    };
    // pooled L2 maps (2k, 2k+1) = (A, B) from S1 map k; the sums in the reference's order:
    // s0 = P0 + P1, s1 = s0 + P2, s(2j) = (P(2j-1) + P(2j)) + P(2j+1), s(2j+1) = (P(2j) + P(2j+1)) + P(2j+2),
    // s7 = P6 + P7; ca and cb carry (P(2k) + P(2k+1)) and P(2k+1) to the next map
    float ca[kP2Passes], cb[kP2Passes];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k == 0)
            cp_async_wait<1>();
        else
            cp_async_wait<0>();
        __syncthreads();  // map k is in shared memory for every thread, and map k - 1's buffer is free
        if (k == 0 && gating) {
            live = 0u;
#pragma unroll
            for (int w = 0; w < kK2TileY / 2; ++w) live |= (s_live[w] ? 1u : 0u) << w;
        }
        if (k == 1 || k == 2) load_back_map_async(S, s1, L, sx0, sy0, k + 1);
        const float(*T)[kS1TW] = S.s1[k & 1];
#pragma unroll
        for (int kk = 0; kk < kP2Passes; ++kk) {
            const int p = threadIdx.x + 256 * kk;
            int x = 0, y = 0;
            if (p < kP2Px) p2_pixel(p, &x, &y);
            if (p < kP2Px && need_row(y)) {
                const f2_t a = pool_l2_pair(T, W, k, x, y, nz);
                const float A = f2_lo(a), B = f2_hi(a);
                if (k == 0) {
                    const float s01 = fadd(A, B);
                    S.s2[0][y][x] = s01;
                    ca[kk] = s01;
                } else {
                    S.s2[2 * k - 1][y][x] = fadd(ca[kk], A);
                    S.s2[2 * k][y][x] = fadd(fadd(cb[kk], A), B);
                    if (k < 3) ca[kk] = fadd(A, B);
                    else S.s2[7][y][x] = fadd(A, B);
                }
                cb[kk] = B;
            }
        }
    }
    __syncthreads();

    // C: pixels (x, y) and (x, y + 1)
    const int x = threadIdx.x & (kK2TileX - 1), y = (threadIdx.x / kK2TileX) * 2;
    if (!((live >> (threadIdx.x >> 5)) & 1u)) {
        // no live pixel in the warp: the skip marker instead of the responses
        const int gx = ox0 + x, gy = oy0 + y;
        if (gx < L.ow) {
            if (gy < L.oh) resp[L.resp_off + (long long)gy * L.ow + gx] = -1e30f;
            if (gy + 1 < L.oh) resp[L.resp_off + (long long)(gy + 1) * L.ow + gx] = -1e30f;
        }
        return;
    }
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
        if (gating) {
            // only live pixels keep their response (a candidate needs a likely cell of its octave within
            // the margin of its window centre); the others may have read skipped inputs
            for (int k = 0; k < 2; ++k)
                if (!gate_live(cells, L, gx, gx, gy + k, gy + k)) rv[k] = -1e30f;
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

template <int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) stage1_back_kernel(const __grid_constant__ Stage1W W, const __grid_constant__ Stage1Dup D,
                                                             const __grid_constant__ LevelTable LT, const float* __restrict__ s1,
                                                             float* __restrict__ resp, int* __restrict__ counts, float thr,
                                                             const uint8_t* __restrict__ back_on, const GateCells cells) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BackSmem& S = *reinterpret_cast<BackSmem*>(smem_raw);
    const int g = LT.first + blockIdx.x;
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::k2_base>(LT, g)];
    const int t = g - L.k2_base;
    back_tile<false>(W, D, S, L, t, g, s1, resp, counts, thr, back_on, cells);
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
                                const uint8_t* front_on, Stage1Sched sched, GrayRef gray, GateCells cells) {
    return launch_grouped(
        levels, n_levels, &LevelDesc::k1_base, [](const LevelDesc& L) { return L.k1_tiles_x * ((L.p1h + kK1TileY - 1) / kK1TileY); },
        [&](const LevelTable& T, int blocks) {
            const bool four = sched.front_blocks_per_sm >= 4;
            if (gray.p)
                (four ? stage1_front_kernel<true, 4> : stage1_front_kernel<true, 3>)<<<blocks, 256, 0, st>>>(W, T, limg, gray, s1, front_on,
                                                                                                              cells);
            else
                (four ? stage1_front_kernel<false, 4> : stage1_front_kernel<false, 3>)<<<blocks, 256, 0, st>>>(W, T, limg, gray, s1, front_on,
                                                                                                                cells);
        });
}

cudaError_t launch_stage1_back(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* s1, float* resp, cudaStream_t st,
                               int* counts, float thr, const uint8_t* back_on, GateCells cells, Stage1Sched sched) {
    const Stage1Dup D = make_dup(W);
    return launch_grouped(
        levels, n_levels, &LevelDesc::k2_base, [](const LevelDesc& L) { return L.k2_tiles_x * ((L.oh + kK2TileY - 1) / kK2TileY); },
        [&](const LevelTable& T, int blocks) {
            if (sched.back_blocks_per_sm >= 4)
                stage1_back_kernel<4><<<blocks, 256, kBackSmemBytes, st>>>(W, D, T, s1, resp, counts, thr, back_on, cells);
            else
                stage1_back_kernel<3><<<blocks, 256, kBackSmemBytes, st>>>(W, D, T, s1, resp, counts, thr, back_on, cells);
        });
}

cudaError_t launch_stage1(const Stage1W& W, const LevelDesc* levels, int n_levels, const float* limg, float* s1, float* resp,
                          cudaStream_t st, int* counts, float thr, const uint8_t* front_on, const uint8_t* back_on, GateCells cells,
                          Stage1Sched sched, GrayRef gray) {
    cudaError_t e = launch_stage1_front(W, levels, n_levels, limg, s1, st, front_on, sched, gray, cells);
    if (e != cudaSuccess) return e;
    return launch_stage1_back(W, levels, n_levels, s1, resp, st, counts, thr, back_on, cells, sched);
}

// ---------------- batched form: one persistent launch over B frames ----------------
//
// Every front tile and back tile of every level of every frame of a batch is one item of a device
// work queue (an atomic counter); a persistent grid takes items in queue order until none are left,
// claiming its next item while it works on the current one. Items of the back stage of frame f wait
// until every front item of frame f has finished (a counter per (frame, stage), polled with acquire
// loads by one thread, a bounded number of times); the diagonal queue order puts about one frame's
// worth of other items between a frame's front tiles and its back tiles, so the polls almost never
// wait. An item only waits on items queued before it, and a block holds at most the item it works on
// and the one it claimed after it, so every wait ends whatever the number of resident blocks. Front
// items resample their level tiles from the gray frames (written by the gray launch before); the S1
// planes are written earlier in the same launch and are read through L2 (ld.global.cg), never the
// read-only path.

void build_batch_queue(BatchQueue* q, int n_frames, int n_levels, int n_chunks, int front_items, int back_items, float thr) {
    q->n_frames = n_frames;
    q->n_levels = n_levels;
    q->n_chunks = n_chunks;
    q->thr = thr;
    q->stage_items[0] = front_items;
    q->stage_items[1] = back_items;
    q->wait_limit = 1 << 22;  // x 256 ns of sleep: about a second before the launch gives up
    int n = 0, first = 0;
    for (int t = 0; t < n_frames + kBatchStages - 1; ++t)
        for (int st = 0; st < kBatchStages; ++st) {
            const int f = t - st;
            if (f < 0 || f >= n_frames || q->stage_items[st] <= 0) continue;
            q->seg_stage[n] = st;
            q->seg_frame[n] = f;
            q->seg_first[n] = first;
            first += q->stage_items[st];
            ++n;
        }
    q->seg_first[n] = first;
    q->n_seg = n;
    q->total = first;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr int kBatchSmem = (int)sizeof(BackSmem) > (int)sizeof(FrontSmem) ? (int)sizeof(BackSmem) : (int)sizeof(FrontSmem);

template <int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) stage1_batch_kernel(const __grid_constant__ Stage1W W, const __grid_constant__ Stage1Dup D,
                                                              const __grid_constant__ BatchFrames F, const __grid_constant__ BatchQueue Q,
                                                              const LevelDesc* __restrict__ levels, int* __restrict__ sync,
                                                              int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ unsigned long long s_ready;  // bit 2f+s: stage s of frame f is known complete
    __shared__ int s_base[kBatchStages][kMaxBatchLevels];  // first front / back item of each level
    const int nl = Q.n_levels < kMaxBatchLevels ? Q.n_levels : kMaxBatchLevels;
    for (int l = threadIdx.x; l < nl; l += blockDim.x) {
        s_base[0][l] = levels[l].k1_base;
        s_base[1][l] = levels[l].k2_base;
    }
    if (threadIdx.x == 0) {
        s_ready = 0ull;
        s_item = atomicAdd(&sync[0], 1);
    }
    __syncthreads();
    int item = s_item;
    while (item < Q.total) {
        int next = 0;
        if (threadIdx.x == 0) next = atomicAdd(&sync[0], 1);  // the next item, claimed while this one runs
        int sg = 0;
        while (sg + 1 < Q.n_seg && Q.seg_first[sg + 1] <= item) ++sg;
        const int stage = Q.seg_stage[sg], f = Q.seg_frame[sg], g = item - Q.seg_first[sg];
        if (stage > 0) {
            const int dep = kBatchStages * f + stage - 1;
            if (!(s_ready & (1ull << dep))) {  // uniform: every thread reads the same word
                if (threadIdx.x == 0) {
                    const int need = Q.stage_items[stage - 1];
                    int polls = 0;
                    while (ld_acquire(&sync[1 + dep]) < need) {
                        if (++polls > Q.wait_limit || ld_acquire(err) != 0) {
                            atomicExch(err, 1);
                            break;
                        }
                        __nanosleep(256);
                    }
                    __threadfence();
                }
                __syncthreads();
                if (threadIdx.x == 0) s_ready |= 1ull << dep;
            }
        }
        // the level of the item: the last level whose first item is <= g
        int lo = 0, hi = nl - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_base[stage][mid] <= g) lo = mid; else hi = mid - 1;
        }
        const LevelDesc& L = levels[lo];
        if (stage == 0) {
            if (!F.front_on[f] || F.front_on[f][g])
                front_tile<true, false>(W, *reinterpret_cast<FrontSmem*>(smem_raw), L, g - L.k1_base, nullptr,
                                        GrayRef{F.gray[f], F.gpitch, F.gw, F.gh}, F.s1[f], F.cells[f]);
        } else {
            back_tile<true>(W, D, *reinterpret_cast<BackSmem*>(smem_raw), L, g - L.k2_base, g, F.s1[f], F.resp[f], F.counts[f], Q.thr,
                            F.back_on[f], F.cells[f]);
        }
        __syncthreads();  // every thread is done with the item (and with the shared memory)
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&sync[1 + kBatchStages * f + stage], 1);
            s_item = next;
        }
        __syncthreads();
        item = s_item;
    }
}

// The candidate counts of every frame of a batch zeroed (blockIdx.x is the frame), before the
// persistent stage-1 launch counts into them.
__global__ void __launch_bounds__(256) counts_zero_batch_kernel(const __grid_constant__ BatchFrames F, int n_chunks) {
    int* c = F.counts[blockIdx.x];
    for (int i = threadIdx.x; i < n_chunks; i += blockDim.x) c[i] = 0;
}

cudaError_t launch_counts_zero_batch(const BatchFrames& F, int n_chunks, int n_frames, cudaStream_t st) {
    if (n_chunks <= 0 || n_frames <= 0) return cudaSuccess;
    counts_zero_batch_kernel<<<n_frames, 256, 0, st>>>(F, n_chunks);
    return cudaGetLastError();
}

// resident blocks per SM of the persistent kernel: the schedule's count (1-4), at most what fits
int stage1_batch_blocks_per_sm(int blocks_per_sm) {
    int n = 0;
    if (blocks_per_sm >= 4)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage1_batch_kernel<4>, 256, kBatchSmem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage1_batch_kernel<3>, 256, kBatchSmem);
    if (blocks_per_sm >= 1 && blocks_per_sm < n) n = blocks_per_sm;
    return n > 0 ? n : 1;
}

cudaError_t launch_stage1_batch(const Stage1W& W, const BatchFrames& F, const BatchQueue& Q, const LevelDesc* d_levels, int* sync, int* err,
                                int grid, cudaStream_t st, int blocks_per_sm) {
    if (Q.total <= 0) return cudaSuccess;
    if (Q.n_levels > kMaxBatchLevels) return cudaErrorInvalidValue;
    const Stage1Dup D = make_dup(W);
    grid = grid < Q.total ? grid : Q.total;
    if (blocks_per_sm >= 4)
        stage1_batch_kernel<4><<<grid, 256, kBatchSmem, st>>>(W, D, F, Q, d_levels, sync, err);
    else
        stage1_batch_kernel<3><<<grid, 256, kBatchSmem, st>>>(W, D, F, Q, d_levels, sync, err);
    return cudaGetLastError();
}

cudaError_t stage1_setup() {
    cudaError_t e = cudaFuncSetAttribute(stage1_back_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBackSmemBytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage1_back_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBackSmemBytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage1_batch_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBatchSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage1_batch_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBatchSmem);
    return e;
}

}  // namespace ccnn
