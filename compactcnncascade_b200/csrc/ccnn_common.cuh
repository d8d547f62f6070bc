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
#endif  // __CUDACC__

// ---------------------------------------------------------------------------------------
// Network weights, passed to kernels by value (__grid_constant__) so that every tap is a
// constant-bank operand. Shapes are the CNTK prototypes of cntk/stage_{1,2,3}.cntk.
// ---------------------------------------------------------------------------------------

template <int M1, int M2, int M3, int K1W, int K1H, int K2W, int K2H, int K3W, int K3H, int HL, int CONN, int HS>
struct NetWeights {
    static constexpr int kM1 = M1, kM2 = M2, kM3 = M3;
    static constexpr int kK1W = K1W, kK1H = K1H, kK2W = K2W, kK2H = K2H, kK3W = K3W, kK3H = K3H;
    static constexpr int kHL = HL, kConn = CONN, kHS = HS, kGroups = HL / HS;
    float k1[M1][K1W * K1H];
    float b1[M1], w1a[M1], w1b[M1], bn1[M1];
    float k2[M2][K2W * K2H];
    float b2[M2], w2a[M2], w2b[M2], bn2[M2];
    float k3[M3][K3W * K3H];
    float b3[M3], w3a[M3], w3b[M3], bn3[M3];
    float hw[HL][CONN];  // hidden weights, neuron n = HS*i + t reads L3 maps i .. i+CONN-1
    float hb[HL];
    float htw[HL / HS];  // per-group tanh slope
    float hbnw[HS], hbnb[HS];
    float ow[HL];        // selected output neuron's weights, index t*(HL/HS) + i
    float ob, otw, af;   // output bias, output tanh slope, signed output scale
};

// cnn4face1_cntk.bin: 23x27 window, 4/8/16 maps, 4x4 / 3x3 / 4(w)x5(h), hidden 52 = 13 x 4
using Stage1W = NetWeights<4, 8, 16, 4, 4, 3, 3, 4, 5, 52, 4, 4>;
// cnn4face2_cntk.bin: 36x40 window, 6/12/24 maps, 4x4 / 3x3 / 7(w)x8(h), hidden 84 = 21 x 4
using Stage2W = NetWeights<6, 12, 24, 4, 4, 3, 3, 7, 8, 84, 4, 4>;
// cnn4face3_cntk.bin: 36x40 window, 6/12/24 maps, 4x4 / 3x3 / 7(w)x8(h), hidden 34 = 17 x 2
using Stage3W = NetWeights<6, 12, 24, 4, 4, 3, 3, 7, 8, 34, 8, 2>;

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
};

// stage-1 front kernel tile (pooled L1 pixels) and back kernel tile (response pixels)
constexpr int kK1TileX = 32, kK1TileY = 16;
constexpr int kK2TileX = 16, kK2TileY = 16;

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
};

}  // namespace ccnn
