// Shared device-side definitions of the B200 detection path.
//
// Exactness contract: the detector must reproduce the reference's CPU cascade bit for bit
// (gray image, pyramid levels, response maps, candidate indices, raw detections). The
// reference's plain C++ path evaluates every expression in source order with IEEE single
// precision and no contraction, so every float operation here goes through the _rn
// intrinsics below (never contracted into FMA) in the same order. The library is also built
// with -fmad=false as a second guard.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ccnn {

#if defined(__CUDACC__)
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// Packed pairs of fp32 (sm_100 f32x2 instructions): two independent IEEE round-to-nearest
// operations per lane per instruction. Used where two outputs run the same operation chain, so
// each element still sees exactly the reference's sequence of roundings. (Tested against the
// scalar _rn chain bit for bit by the parity tests.)
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2_pack(float lo, float hi) {
    f2_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float f2_lo(f2_t v) {
    float lo;
    asm("{ .reg .f32 t; mov.b64 {%0, t}, %1; }" : "=f"(lo) : "l"(v));
    return lo;
}
__device__ __forceinline__ float f2_hi(f2_t v) {
    float hi;
    asm("{ .reg .f32 t; mov.b64 {t, %0}, %1; }" : "=f"(hi) : "l"(v));
    return hi;
}
__device__ __forceinline__ f2_t f2_dup(float v) { return f2_pack(v, v); }
__device__ __forceinline__ f2_t f2_ld(const float2& v) { return *reinterpret_cast<const f2_t*>(&v); }
// Packed product. ptxas contracts a packed mul followed by a packed add into one packed FMA
// (a single rounding), even with fmad disabled, which would break the reference's two-rounding
// arithmetic. The product is therefore an FMA whose addend is a (-0, -0) pair the compiler cannot
// see (it comes from the kernel's weight block at run time): fma(a, b, -0) is exactly the rounded
// product a*b, sign of zero included, and an FMA cannot be merged with the following add.
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b, f2_t negzero) {
    f2_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(negzero));
    return r;
}
__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
    f2_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b) {
    f2_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2_t f2_max0(f2_t c) { return f2_pack(fmaxf(0.f, f2_lo(c)), fmaxf(0.f, f2_hi(c))); }
__device__ __forceinline__ f2_t f2_max4(f2_t a, f2_t b, f2_t c, f2_t d) {
    return f2_pack(fmaxf(fmaxf(f2_lo(a), f2_lo(b)), fmaxf(f2_lo(c), f2_lo(d))),
                   fmaxf(fmaxf(f2_hi(a), f2_hi(b)), fmaxf(f2_hi(c), f2_hi(d))));
}

// Rational tanh approximation of the reference (cnnpp_cplusplus.cpp:662-666, 680-683):
//   s = sgn(c) * (1 - 1 / (((1 + |c|) + c*c) + (((a*c)*c)*c)*c)),  a = 1.41645
__device__ __forceinline__ float tanh_rational(float c) {
    const float a = 1.41645f;
    float sgn = c < 0.f ? -1.f : 1.f;
    float ac = fabsf(c);
    float c2 = fmul(c, c);
    float c4 = fmul(fmul(fmul(fmul(a, c), c), c), c);
    float den = fadd(fadd(fadd(1.f, ac), c2), c4);
    return fmul(sgn, fsub(1.f, fdiv(1.f, den)));
}

// Folded BN + LeakyReLU of the reference (cnnpp_cplusplus.cpp:604-605):
//   c = x + b;  y = (w1*c + w2*max(0, c)) + bn_b
__device__ __forceinline__ float lrelu_bn(float x, float b, float w1, float w2, float bnb) {
    float c = fadd(x, b);
    return fadd(fadd(fmul(w1, c), fmul(w2, fmaxf(0.f, c))), bnb);
}

__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
    f2_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Correctly rounded IEEE reciprocals of two values in [1, 2^126): the hardware approximation
// (rcp.approx, within about an ulp) refined by two Newton-Raphson steps with fused residuals,
// e = 1 - d*y, y' = y + y*e (Markstein's FMA iteration). For every float of that range the result
// equals __frcp_rn bit for bit (compared exhaustively on B200, ccnn_check_reciprocal). Outside it
// (subnormal results, infinity, NaN) both lanes take __frcp_rn.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ f2_t f2_rcp(f2_t d) {
    const float d0 = f2_lo(d), d1 = f2_hi(d);
    if (!(d0 >= 1.f && d0 < 0x1p126f && d1 >= 1.f && d1 < 0x1p126f)) return f2_pack(__frcp_rn(d0), __frcp_rn(d1));
    const f2_t one = f2_pack(1.f, 1.f);
    const f2_t nd = f2_pack(-d0, -d1);
    f2_t y = f2_pack(rcp_approx(d0), rcp_approx(d1));
    y = f2_fma(y, f2_fma(nd, y, one), y);
    return f2_fma(y, f2_fma(nd, y, one), y);
}

// Two independent lanes of tanh_rational. The reciprocal 1/den is the correctly rounded IEEE
// value, the same number as the reference's 1.f / den.
__device__ __forceinline__ f2_t tanh_rational2(f2_t c, f2_t nz) {
    const f2_t one = f2_pack(1.f, 1.f), a = f2_pack(1.41645f, 1.41645f);
    const float lo = f2_lo(c), hi = f2_hi(c);
    const f2_t ac = f2_pack(fabsf(lo), fabsf(hi));
    const f2_t c2 = f2_mul(c, c, nz);
    const f2_t c4 = f2_mul(f2_mul(f2_mul(f2_mul(a, c, nz), c, nz), c, nz), c, nz);
    const f2_t den = f2_add(f2_add(f2_add(one, ac), c2), c4);
    const f2_t r = f2_rcp(den);  // den >= 1 (or NaN)
    const f2_t sgn = f2_pack(lo < 0.f ? -1.f : 1.f, hi < 0.f ? -1.f : 1.f);
    return f2_mul(sgn, f2_sub(one, r), nz);
}

// Two lanes of lrelu_bn; p = {b, w1, w2, bn_b}, each a (lane 0, lane 1) pair.
__device__ __forceinline__ f2_t lrelu_bn2(f2_t x, const float2* p, f2_t nz) {
    const f2_t c = f2_add(x, f2_ld(p[0]));
    return f2_add(f2_add(f2_mul(f2_ld(p[1]), c, nz), f2_mul(f2_ld(p[2]), f2_max0(c), nz)), f2_ld(p[3]));
}
#endif  // __CUDACC__

// ---------------------------------------------------------------------------------------
// Network weights, passed to kernels by value (__grid_constant__) so that every tap is a
// constant-bank operand. Shapes are the CNTK prototypes of cntk/stage_{1,2,3}.cntk. Taps are
// stored as the (lo, hi) pairs the packed-pair kernels consume.
// ---------------------------------------------------------------------------------------

template <int M1, int M2, int M3, int K1W, int K1H, int K2W, int K2H, int K3W, int K3H, int HL, int CONN, int HS>
struct NetWeights {
    static constexpr int kM1 = M1, kM2 = M2, kM3 = M3;
    static constexpr int kK1W = K1W, kK1H = K1H, kK2W = K2W, kK2H = K2H, kK3W = K3W, kK3H = K3H;
    static constexpr int kHL = HL, kConn = CONN, kHS = HS, kGroups = HL / HS;
    float2 k1d[M1][K1W * K1H];      // L1 taps duplicated (w, w): two pixels of one map per packed op
    float2 k1p[M1 / 2][K1W * K1H];  // L1 taps of maps (2i, 2i+1), which read the same input
    float b1[M1], w1a[M1], w1b[M1], bn1[M1];
    float2 a1d[M1][4];              // L1 {b, w1a, w1b, bn} of each map duplicated (v, v)
    float2 a1p[M1 / 2][4];          // L1 {b, w1a, w1b, bn} of map pairs (2i, 2i+1)
    float2 k2p[M2 / 2][K2W * K2H];  // L2 taps of maps (2i, 2i+1), which read the same sum map i
    float b2[M2], w2a[M2], w2b[M2], bn2[M2];
    float2 a2p[M2 / 2][4];          // L2 {b, w2a, w2b, bn} of map pairs
    float2 k3p[M3 / 2][K3W * K3H];  // L3 taps of maps (2i, 2i+1)
    float b3[M3], w3a[M3], w3b[M3], bn3[M3];
    float2 a3p[M3 / 2][4];          // L3 {b, w3a, w3b, bn} of map pairs
    float2 hwp[HL / 2][CONN];       // hidden weights of neurons (2q, 2q+1); neuron n = HS*i + t reads
                                    // L3 maps i .. i+CONN-1 (HS even, so a pair shares its group)
    float hb[HL];
    float htw[HL / HS];  // per-group tanh slope
    float hbnw[HS], hbnb[HS];
    float ow[HL];        // selected output neuron's weights, index t*(HL/HS) + i
    float ob, otw, af;   // output bias, output tanh slope, signed output scale
    float2 negzero;      // (-0.f, -0.f): the run-time addend of f2_mul
};

// cnn4face1_cntk.bin: 23x27 window, 4/8/16 maps, 4x4 / 3x3 / 4(w)x5(h), hidden 52 = 13 x 4
using Stage1W = NetWeights<4, 8, 16, 4, 4, 3, 3, 4, 5, 52, 4, 4>;
// cnn4face2_cntk.bin: 36x40 window, 6/12/24 maps, 4x4 / 3x3 / 7(w)x8(h), hidden 84 = 21 x 4
using Stage2W = NetWeights<6, 12, 24, 4, 4, 3, 3, 7, 8, 84, 4, 4>;
// cnn4face3_cntk.bin: 36x40 window, 6/12/24 maps, 4x4 / 3x3 / 7(w)x8(h), hidden 34 = 17 x 2
using Stage3W = NetWeights<6, 12, 24, 4, 4, 3, 3, 7, 8, 34, 8, 2>;

// Stage-1 parameters duplicated (v, v) for the back kernel, which runs every operation of the L3
// maps, the hidden layer and the output neuron on two vertically adjacent response pixels at once.
struct Stage1Dup {
    float2 k3d[Stage1W::kM3][Stage1W::kK3W * Stage1W::kK3H];
    float2 a3d[Stage1W::kM3][4];
    float2 hwd[Stage1W::kHL][Stage1W::kConn];
    float2 hbd[Stage1W::kHL];
    float2 htwd[Stage1W::kGroups];
    float2 hbnwd[Stage1W::kHS], hbnbd[Stage1W::kHS];
    float2 owd[Stage1W::kHL];
    float2 obd, otwd, afd;
};

// cnn4landmarks_cntk.bin (facial analysis): 49x51 window, 24/48/96 maps, 4x4 / 3x3 / 10(w)x11(h),
// a fully connected hidden layer of 384 neurons over the 96 L3 values, 13 outputs (5 landmarks
// (x, y) as fractions of the window, gender, smile, glasses). Too large for kernel parameters: it
// lives in device memory.
struct LandmarkNet {
    static constexpr int kM1 = 24, kM2 = 48, kM3 = 96, kHL = 384, kOut = 13;
    static constexpr int kInW = 49, kInH = 51, kK3W = 10, kK3H = 11;
    float2 k1p[kM1 / 2][16];        // L1 taps of map pairs (2i, 2i+1)
    float2 a1p[kM1 / 2][4];         // L1 {b, w1a, w1b, bn} of map pairs
    float2 k2p[kM2 / 2][9];         // L2 maps (2i, 2i+1) read neighbour sum i
    float2 a2p[kM2 / 2][4];
    float2 k3p[kM3 / 2][kK3W * kK3H];  // L3 maps (2i, 2i+1) read neighbour sum i
    float2 a3p[kM3 / 2][4];
    float2 hwp[kHL / 2][kM3];       // hidden neurons (2q, 2q+1) over every L3 value
    float2 hbp[kHL / 2];            // their biases
    float2 hbnwp[kHL / 2], hbnbp[kHL / 2];
    float htw;                      // tanh slope (one group)
    float ow[kOut][kHL];
    float ob[kOut];
    float otw, af;
    float2 negzero;
};

struct WindowNets {
    Stage2W s2;
    Stage3W s3;
};

// ---------------------------------------------------------------------------------------
// Pyramid level table (one entry per processed level, in the reference's level order
// scl = 0 (largest) .. n-1). All sizes follow cnn_simd_cntk.cpp:997-1012.
// ---------------------------------------------------------------------------------------
struct LevelDesc {
    int w, h;            // level image size: Size(int(W*s), int(H*s)) (type.h:63-66)
    int mode;            // 0 = copy of the gray image (s == 1), 1 = nearest neighbour, 2 = bilinear
    uint32_t sclx, scly; // 12-bit fixed-point steps (image_resize.cpp:57-58)
    float scale, inv_scale;
    int p1w, p1h;        // L1 pooled size: (w-3)>>1, (h-3)>>1
    int p2w, p2h;        // L2 pooled size: (p1w-2)>>1, (p1h-2)>>1
    int ow, oh;          // response map: p2w-3, p2h-4
    int s1_pitch;        // floats per row of each S1 plane
    long long s1_off;    // offset of this level's S1 planes in the S1 arena (floats)
    long long s1_plane;  // floats per S1 plane
    long long resp_off;  // offset of this level's response map (dense, pitch ow)
    int k1_tiles_x, k1_base;  // stage-1 front kernel tiles
    int k2_tiles_x, k2_base;  // stage-1 back kernel tiles
    int order;           // processing position of this level in the candidate scan (0 = first)
    long long img_off;   // offset of this level's image in the level arena (floats)
    int img_pitch;       // floats per level image row
    int img_vec;         // 1: rows start 16-byte aligned and the pitch is a multiple of 4 floats
    int pyr_base;        // first pyramid-kernel block of this level
    int pyr_wq;          // pyramid-kernel column blocks per row band
    int chunk_base;      // first candidate-scan chunk of this level
    int octave;          // floor(log2(largest scale / scale)): the learned gate's output for this level
};

// The learned gate's per-octave cell bitmaps as the stage-1 back kernel reads them: bits == nullptr
// means no gate. Rows of wwords words, one bit per 16x16-pixel cell of the frame. A candidate needs a
// set bit in a cell within `margin` pixels (per axis) of its window centre.
struct GateCells {
    const uint32_t* bits;
    const int* ambiguous;  // frames with more ambiguous cells than amb_limit are scanned in full
    int amb_limit, wwords, w16, h16, margin;
};

// The cells [lo, hi] of one axis within m pixels of the window-centre pixel coordinate p (p >= 0,
// truncated); n16 cells on the axis. m = 16 is the centre's cell and one cell on either side.
__host__ __device__ __forceinline__ int gate_cell_lo(int p, int m) { return (p - m) / 16 > 0 ? (p - m) / 16 : 0; }
__host__ __device__ __forceinline__ int gate_cell_hi(int p, int m, int n16) { return (p + m) / 16 < n16 - 1 ? (p + m) / 16 : n16 - 1; }

// any set bit of octave row bitmaps `B` in cells [cx0, cx1] x [cy0, cy1]
__device__ __forceinline__ bool gate_any_bit(const uint32_t* __restrict__ B, int wwords, int cx0, int cx1, int cy0, int cy1) {
    if (cx0 > cx1 || cy0 > cy1) return false;
    const int w0 = cx0 >> 5, w1 = cx1 >> 5;
    const uint32_t m0 = 0xffffffffu << (cx0 & 31), m1 = 0xffffffffu >> (31 - (cx1 & 31));
    for (int y = cy0; y <= cy1; ++y) {
        const uint32_t* row = B + (long long)y * wwords;
        for (int w = w0; w <= w1; ++w) {
            uint32_t m = 0xffffffffu;
            if (w == w0) m &= m0;
            if (w == w1) m &= m1;
            if (row[w] & m) return true;
        }
    }
    return false;
}

// candidate-scan chunk: response pixels of one level per compaction block, in raster order
constexpr int kCandChunk = 2048;

// Level descriptors passed by value to the kernels that find their level per block (a frame's
// pyramid is launched in groups of at most kParamLevels levels). Every block of a launch maps to
// global block index first + blockIdx.x, whose level is found by binary search over the
// descriptors' base fields, all in the constant bank.
constexpr int kParamLevels = 32;
struct LevelTable {
    int n;      // levels in lv[]
    int first;  // global block index of this launch's block 0
    LevelDesc lv[kParamLevels];
};

#if defined(__CUDACC__)
// Level of global block g: the last level whose first block is <= g (binary search over the
// descriptors in the constant bank; FIELD selects the front or back kernel's tile base).
template <int LevelDesc::*FIELD>
__device__ __forceinline__ int find_level(const LevelTable& T, int g) {
    int lo = 0, hi = T.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (T.lv[mid].*FIELD <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}
#endif

// stage-1 front kernel tile (pooled L1 pixels) and back kernel tile (response pixels)
constexpr int kK1TileX = 32, kK1TileY = 16;
constexpr int kK2TileX = 32, kK2TileY = 16;

// stage-1 window and the stage-2/3 crop geometry (cnn_detector_v3.cpp:54-55, 1489-1501)
constexpr int kPatW = 23, kPatH = 27;           // stage-1 pattern
constexpr int kExtOff = 11, kXOff = 2;          // ext_pattern_offset, x_pattern_offset
constexpr int kWinW = 47, kWinH = 51;           // stage-2/3 input (36+11, 40+11)
constexpr int kCropW = kWinW + kXOff, kCropH = kWinH;  // 49 x 51 resized crop

struct Candidate {
    int level;   // level index scl
    int px, py;  // point in level coordinates (4 * response index)
    float score; // stage-1 response
};

struct CandResult {
    int accepted;  // 0 rejected, 1 accepted by the first window, 2 accepted by the shrunken retry window
    float score;
    int knn;
    int pad;
};

// stage-2/3 output summary of one (candidate, window, stage) work item
struct WinOut {
    float max;  // largest of the 16 responses (starting from -10)
    int knn;    // responses above the stage threshold
};

struct Det {
    int x, y, w, h, x2, y2;
    float score, scale;
    int knn, num_detect;
};

// runtime switches of the cascade (cnn_detector_v3.h:124-175 after Init's precision rules)
struct CascadeConfig {
    float thr1, thr2, thr3;
    int type_check;
    int min_neighbors;
    int adapt_min_neighbors;
    int double_check;
    int drop_detect;
    int equalize;
    int reflection;
    int detect_enabled;   // detect_mode != disable
    int merger_detect;
    int min_num_detect;
    int rescale_output;   // gray_image_only input downscale: rects scaled back
    float rescale;        // min_obj_size.height / pattern height
    int pat_w, pat_h;     // stage-1 pattern (the stage-1 network's smallest input)
};

}  // namespace ccnn
