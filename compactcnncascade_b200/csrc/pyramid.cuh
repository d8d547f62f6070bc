// One block of the pyramid resampling (RunCPUDetect, cnn_detector_v3.cpp:2090-2104, with
// ImageResizer::FastImageResize, image_resize.cpp:564-584): block `local` of level L covers kPyrCols
// columns (one a thread) of kPyrRows rows of the level image, computed from the gray frame and
// written to the level arena at L.img_off (columns past the level width up to its pitch get zeros).
// front_on (optional, the learned gate): a block that no running stage-1 front tile reads is left out.
#pragma once

#include "kernels.h"
#include "resample.cuh"

namespace ccnn {

__device__ __forceinline__ void pyramid_block(const LevelDesc& L, int local, const float* __restrict__ gray, int gpitch, int gw, int gh,
                                              float* __restrict__ limg, const uint8_t* __restrict__ front_on) {
    const int rb = local / L.pyr_wq;
    const int cb = local - rb * L.pyr_wq;
    if (front_on) {
        // with the learned gate only the stage-1 front tiles that run read the level image: a block
        // that none of them reads is left out (front tile (tx, ty) reads rows [32 ty, 32 ty + 35)
        // and columns [64 tx, 64 tx + 68))
        const int ty0 = max(0, (kPyrRows * rb - (2 * kK1TileY + 3) + 2 * kK1TileY) / (2 * kK1TileY));
        const int ty1 = min((L.p1h + kK1TileY - 1) / kK1TileY - 1, (kPyrRows * rb + kPyrRows - 1) / (2 * kK1TileY));
        const int tx0 = max(0, (kPyrCols * cb - (2 * kK1TileX + 4) + 2 * kK1TileX) / (2 * kK1TileX));
        const int tx1 = min(L.k1_tiles_x - 1, (kPyrCols * cb + kPyrCols - 1) / (2 * kK1TileX));
        bool need = false;
        for (int ty = ty0; ty <= ty1 && !need; ++ty)
            for (int tx = tx0; tx <= tx1; ++tx)
                if (front_on[L.k1_base + ty * L.k1_tiles_x + tx]) {
                    need = true;
                    break;
                }
        if (!need) return;
    }
    const int x = cb * kPyrCols + threadIdx.x;
    if (x >= L.img_pitch) return;
    float* out = limg + L.img_off + x;
    const int y0 = rb * kPyrRows;
    const int y1 = y0 + kPyrRows < L.h ? y0 + kPyrRows : L.h;
    if (x >= L.w) {
        for (int y = y0; y < y1; ++y) out[(long long)y * L.img_pitch] = 0.f;
        return;
    }
    if (L.mode == 0) {
        for (int y = y0; y < y1; ++y) out[(long long)y * L.img_pitch] = __ldg(gray + (size_t)y * gpitch + x);
        return;
    }
    const AxisSample sx = sample_col(x, L.sclx, gw);
    if (L.mode == 1) {
        for (int y = y0; y < y1; ++y)
            out[(long long)y * L.img_pitch] = __ldg(gray + (size_t)sample_row(y, L.scly, gh).idx * gpitch + sx.idx);
        return;
    }
#pragma unroll 4
    for (int y = y0; y < y1; ++y) {
        const AxisSample sy = sample_row(y, L.scly, gh);
        uint32_t py = sy.idx;
        if (py + 1 >= (uint32_t)gh) py--;  // bilinear keeps a row below
        const float* r0 = gray + (size_t)py * gpitch + sx.idx;
        const float top = fadd(fmul(__ldg(r0), sx.c), fmul(__ldg(r0 + 1), sx.f));
        const float bot = fadd(fmul(__ldg(r0 + gpitch), sx.c), fmul(__ldg(r0 + gpitch + 1), sx.f));
        out[(long long)y * L.img_pitch] = fadd(fmul(top, sy.c), fmul(bot, sy.f));
    }
}

}  // namespace ccnn
