// Fixed-point image resampling shared by the pyramid and the stage-2/3 crops.
//
// Follows SIMD::ImageResizer (src/CNNObjectDetector/image_resize.cpp): 12-bit fixed point
// steps `scl = (src << 12) / dst + 1` (:57-58); source row clamped to src_h-1 (:74) and,
// for bilinear, moved up one row at the bottom edge (:409); source column clamped to src_w-2
// (:94); fractional weights taken from the UNclamped position (:69-72, :89-92); vertical
// weights pre-divided by 2^24 (:75-76); bilinear value
//   ((p0*cx + p1*fx)*cy + (p2*cx + p3*fx)*fy)   (:537)
#pragma once

#include "ccnn_common.cuh"

namespace ccnn {

__host__ __device__ __forceinline__ uint32_t fp_step(int src, int dst) { return ((uint32_t)src << 12) / (uint32_t)dst + 1u; }

struct AxisSample {
    uint32_t idx;  // clamped source index
    float f, c;    // fractional weight and its complement (f + c == 4096, or /2^24 for rows)
};

__device__ __forceinline__ AxisSample sample_col(int ix, uint32_t scl, int src_w) {
    uint32_t x = (uint32_t)ix * scl;
    uint32_t p = x >> 12;
    AxisSample s;
    s.f = (float)(x - (p << 12));
    s.c = 4096.f - s.f;
    uint32_t lim = (uint32_t)(src_w - 2);
    s.idx = p > lim ? lim : p;
    return s;
}

__device__ __forceinline__ AxisSample sample_row(int iy, uint32_t scl, int src_h) {
    uint32_t y = (uint32_t)iy * scl;
    uint32_t p = y >> 12;
    float fy = (float)(y - (p << 12));
    float cy = 4096.f - fy;
    AxisSample s;
    s.f = fy / 16777216.f;  // exact: power-of-two scaling of an integer < 4096
    s.c = cy / 16777216.f;
    uint32_t lim = (uint32_t)(src_h - 1);
    s.idx = p > lim ? lim : p;
    return s;
}

// nearest neighbour on float rows
__device__ __forceinline__ float nn_f32(const float* src, int pitch, const AxisSample& sx, const AxisSample& sy) {
    return src[(size_t)sy.idx * pitch + sx.idx];
}

// bilinear on float rows (BilinearInterpolation(Image_32f&...) :393-541)
__device__ __forceinline__ float bilinear_f32(const float* src, int pitch, int src_h, const AxisSample& sx, const AxisSample& sy) {
    uint32_t py = sy.idx;
    if (py + 1 >= (uint32_t)src_h) py--;
    const float* r0 = src + (size_t)py * pitch;
    const float* r1 = r0 + pitch;
    float p0 = r0[sx.idx], p1 = r0[sx.idx + 1], p2 = r1[sx.idx], p3 = r1[sx.idx + 1];
    float top = fadd(fmul(p0, sx.c), fmul(p1, sx.f));
    float bot = fadd(fmul(p2, sx.c), fmul(p3, sx.f));
    return fadd(fmul(top, sy.c), fmul(bot, sy.f));
}

// bilinear on byte rows, truncated back to a byte (BilinearInterpolation(Image_8u&...) :197-326)
__device__ __forceinline__ uint8_t bilinear_u8(const uint8_t* src, int pitch, int src_h, const AxisSample& sx, const AxisSample& sy) {
    uint32_t py = sy.idx;
    if (py + 1 >= (uint32_t)src_h) py--;
    const uint8_t* r0 = src + (size_t)py * pitch;
    const uint8_t* r1 = r0 + pitch;
    float p0 = (float)r0[sx.idx], p1 = (float)r0[sx.idx + 1], p2 = (float)r1[sx.idx], p3 = (float)r1[sx.idx + 1];
    float top = fadd(fmul(p0, sx.c), fmul(p1, sx.f));
    float bot = fadd(fmul(p2, sx.c), fmul(p3, sx.f));
    return (uint8_t)__float2int_rz(fadd(fmul(top, sy.c), fmul(bot, sy.f)));
}

// One pyramid level pixel from the full-resolution gray image (RunCPUDetect,
// cnn_detector_v3.cpp:2090-2104: s == 1 copies, s > 0.7 nearest neighbour, else bilinear).
__device__ __forceinline__ float level_pixel(const float* gray, int gpitch, int gw, int gh, const LevelDesc& L, int lx, int ly) {
    if (L.mode == 0) return gray[(size_t)ly * gpitch + lx];
    AxisSample sx = sample_col(lx, L.sclx, gw);
    AxisSample sy = sample_row(ly, L.scly, gh);
    if (L.mode == 1) return nn_f32(gray, gpitch, sx, sy);
    return bilinear_f32(gray, gpitch, gh, sx, sy);
}

}  // namespace ccnn
