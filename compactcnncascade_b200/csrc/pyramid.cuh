// One block of the pyramid resampling (RunCPUDetect, cnn_detector_v3.cpp:2090-2104, with
// ImageResizer::FastImageResize, image_resize.cpp:564-584): block `local` of level L covers kPyrCols
// columns (one a thread) of kPyrRows rows of the level image, computed from the gray frame and
// written to the level arena at L.img_off (columns past the level width up to its pitch get zeros).
// Only the legacy family stores level images (the CNTK stage-1 front kernel resamples its own tiles).
#pragma once

#include "kernels.h"
#include "resample.cuh"

namespace ccnn {

__device__ __forceinline__ void pyramid_block(const LevelDesc& L, int local, const float* __restrict__ gray, int gpitch, int gw, int gh,
                                              float* __restrict__ limg) {
    const int rb = local / L.pyr_wq;
    const int cb = local - rb * L.pyr_wq;
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
