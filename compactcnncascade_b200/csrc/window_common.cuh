// Pieces of the stage-2/3 window check shared by the window, facial-analysis and replay kernels.
#pragma once

#include "ccnn_common.cuh"
#include "replay.cuh"

namespace ccnn {

// Crop of a candidate's check window in gray-frame coordinates (cnn_detector_v3.cpp:1489-1556):
// the extended pattern around the stage-1 point, for mod 1 the retry window shrunk by 15 %, then
// clamped to the frame. geo = {x, y, cols, rows}.
__device__ __forceinline__ void window_geometry(const Candidate& cd, float inv_scale, int mod, int gw, int gh, int pat_w, int pat_h, int* geo) {
    int x = (int)((float)(cd.px - (kExtOff + kXOff) / 2) * inv_scale);
    int y = (int)((float)(cd.py - kExtOff / 2) * inv_scale);
    int width = (int)((float)(pat_w + kExtOff + kXOff) * inv_scale);
    int height = (int)((float)(pat_h + kExtOff) * inv_scale);
    if (mod == 1) {
        const float k = 0.15f;
        x = (int)(fadd((float)x, fdiv(fmul((float)width, k), 2.f)));
        width = (int)(fsub((float)width, fmul((float)width, k)));
        y = (int)(fadd((float)y, fdiv(fmul((float)height, k), 2.f)));
        height = (int)(fsub((float)height, fmul((float)height, k)));
    }
    const int rx = min(max(x, 0), gw);
    const int ry = min(max(y, 0), gh);
    geo[0] = rx;
    geo[1] = ry;
    geo[2] = min(max(x + width, 0), gw) - rx;
    geo[3] = min(max(y + height, 0), gh) - ry;
}

// the accept rule of one window from its stage-2 and stage-3 counts (cnn_detector_v3.cpp:1709-1725)
__device__ __forceinline__ bool window_accepts(int k1, int k2, int mn, const CascadeConfig& C) {
    switch (C.type_check) {
        case 0: return k1 >= mn || k2 >= mn;
        case 1: return (k1 >= mn && k2 > 0) || (k1 > 0 && k2 >= mn);
        case 2: return k1 >= mn && k2 >= mn;
    }
    return false;
}

// stage-2/3 verdict of one candidate from its (max, count) pairs, applying the
// reference's order: stage 2, early exits (:1698-1706), stage 3, accept rule (:1709-1725), retry
// with the shrunken window when rejected and double_check is on (:1806-1811)
__device__ __forceinline__ CandResult verdict(const WinOut* w, const Candidate& cd, float scale, const CascadeConfig& C) {
    const int mn = (C.adapt_min_neighbors && scale > 0.7f && C.min_neighbors > 1) ? C.min_neighbors - 1 : C.min_neighbors;
    CandResult r;
    r.accepted = 0;
    r.score = 0.f;
    r.knn = 0;
    r.pad = 0;
    const int n_mod = C.double_check ? 2 : 1;
    for (int mod = 0; mod < n_mod; ++mod) {
        const float max1 = w[2 * mod].max;
        const int k1 = w[2 * mod].knn;
        const bool stop = (C.type_check == 0 && k1 >= mn) || (C.type_check > 0 && k1 <= 0) || (C.type_check == 2 && k1 < mn);
        const float max2 = stop ? -10.f : w[2 * mod + 1].max;
        const int k2 = stop ? 0 : w[2 * mod + 1].knn;
        if (window_accepts(k1, k2, mn, C)) {
            const float m1 = (-1.7159f < max1) ? max1 : -1.7159f;
            const float m2 = (-1.7159f < max2) ? max2 : -1.7159f;
            r.accepted = mod + 1;
            r.score = fadd(fadd(cd.score, fmul((float)k1, m1)), fmul((float)k2, m2));
            r.knn = imin(k1, k2);
            return r;
        }
    }
    return r;
}

}  // namespace ccnn
