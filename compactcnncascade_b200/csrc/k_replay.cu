// Sequential cascade bookkeeping, sort and box clustering on the device (one CTA).
//
// Reference order (src/CNNObjectDetector/cnn_detector_v3.cpp):
//   for every level, smallest first (RunCheckDetectAsync :2041-2049):
//     scan candidates in raster order; with drop_detect each one is tested against the
//       detections gathered so far (DropDetection :1820-1840): the first earlier box that
//       overlaps it by > 0.5 appends a copy (this box, that box's score/knn) and drops it, a box
//       that contains its 70 % core drops it (:1928-1941);
//     then for the survivors in order (CPUCheckDetect :1485-1818): a survivor overlapping
//       (> 0.5) a box appended since the scan appends a copy instead of running stages 2/3
//       (:1507-1527); otherwise the stage-2/3 verdict (precomputed by the window kernel)
//       appends the detection.
//   reverse, std::sort by scale (:2746-2750), Merger(0.5), min_num_detect filter,
//   Merger(0.2, del) (:2753-2772), optional rescale for shrunken gray input (:2785-2806).
//
// The scan test of a level against the detections of earlier levels has no order dependence,
// so all 32 warps run it in parallel (one warp per candidate, 32 earlier boxes per ballot).
// What depends on order (copies appended during the level's own scan, the survivors' pass,
// the sort and the clustering) runs in warp 0 with ballots over 32 boxes at a time.
#include "kernels.h"
#include "replay.cuh"

namespace ccnn {

constexpr int kRT = 1024;

__device__ __forceinline__ Det cand_rect(const Candidate& c, float inv_scale, float scale) {
    return make_det((int)((float)c.px * inv_scale), (int)((float)c.py * inv_scale), (int)((float)kPatW * inv_scale),
                    (int)((float)kPatH * inv_scale), 0.f, scale, 0);
}

__device__ __forceinline__ Det shfl_det(const Det& d, int src) {
    Det r;
    r.x = __shfl_sync(0xffffffffu, d.x, src);
    r.y = __shfl_sync(0xffffffffu, d.y, src);
    r.w = __shfl_sync(0xffffffffu, d.w, src);
    r.h = __shfl_sync(0xffffffffu, d.h, src);
    r.x2 = __shfl_sync(0xffffffffu, d.x2, src);
    r.y2 = __shfl_sync(0xffffffffu, d.y2, src);
    r.score = __shfl_sync(0xffffffffu, d.score, src);
    r.scale = __shfl_sync(0xffffffffu, d.scale, src);
    r.knn = __shfl_sync(0xffffffffu, d.knn, src);
    r.num_detect = __shfl_sync(0xffffffffu, d.num_detect, src);
    return r;
}

__device__ __forceinline__ void sort4(int* v) {
    // any correct sort gives the same ascending values
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3 - i; ++j)
            if (v[j] > v[j + 1]) {
                int t = v[j];
                v[j] = v[j + 1];
                v[j + 1] = t;
            }
}

// Merger's pair test (cnn_detector_v3.cpp:2842-2881). Returns ratio > threshold and the data
// needed to apply the merge.
struct MergeTest {
    bool hit;
    bool s1_gt_s2;
    int X[4], Y[4];
};

__device__ __forceinline__ MergeTest merge_test(const Det& a, const Det& b, float threshold) {
    MergeTest t;
    t.hit = false;
    t.s1_gt_s2 = false;
    int X[4] = {a.x, a.x2, b.x, b.x2};
    int Y[4] = {a.y, a.y2, b.y, b.y2};
    if (X[0] >= X[3] || X[1] <= X[2] || Y[0] >= Y[3] || Y[1] <= Y[2]) return t;
    const float S1 = (float)((X[1] - X[0]) * (Y[1] - Y[0]));
    const float S2 = (float)((X[3] - X[2]) * (Y[3] - Y[2]));
    sort4(X);
    sort4(Y);
    const float su = (float)((X[3] - X[0]) * (Y[3] - Y[0]));
    const float si = (float)((X[2] - X[1]) * (Y[2] - Y[1]));
    const float r1 = fdiv(si, S1), r2 = fdiv(si, S2), r3 = fdiv(si, su);
    float ratio = r1 > r2 ? r2 : r1;
    const int CX1 = X[0] + ((X[3] - X[0]) >> 1);
    const int CY1 = Y[0] + ((Y[3] - Y[0]) >> 1);
    const int CX2 = X[1] + ((X[2] - X[1]) >> 1);
    const int CY2 = Y[1] + ((Y[2] - Y[1]) >> 1);
    const int thrC = imin(X[3] - X[0], X[2] - X[1]) >> 1;
    if (r3 > fmul(0.75f, threshold) && (r1 < r2 ? r2 : r1) > 0.7f && abs(CX1 - CX2) < thrC && abs(CY1 - CY2) < thrC) ratio = 1.f;
    t.hit = ratio > threshold;
    t.s1_gt_s2 = S1 > S2;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        t.X[i] = X[i];
        t.Y[i] = Y[i];
    }
    return t;
}

// Merger (cnn_detector_v3.cpp:2814-2936) run by one warp. in[] is read-only; checked[] is scratch.
__device__ int merger_warp(const Det* in, int n, uint8_t* checked, Det* out, float threshold, bool del) {
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < n; k += 32) checked[k] = 0;
    __syncwarp();
    int nout = 0;
    for (int i1 = 0; i1 < n; ++i1) {
        if (checked[i1]) continue;
        Det nmax = in[i1], nmin = in[i1];
        bool dropped = false;
        for (int base = i1 + 1; base < n && !dropped; base += 32) {
            const int j = base + lane;
            bool live = j < n && !checked[j];
            const Det e = live ? in[j] : nmax;
            if (del) {
                const MergeTest mt = merge_test(nmax, e, threshold);
                const bool pred = live && mt.hit;
                const unsigned mb = __ballot_sync(0xffffffffu, pred && !mt.s1_gt_s2);
                const int lim = mb ? __ffs(mb) - 1 : 32;
                if (pred && mt.s1_gt_s2 && lane < lim) checked[j] = 1;
                if (mb) dropped = true;
            } else {
                int start = 0;
                while (true) {
                    const MergeTest mt = merge_test(nmax, e, threshold);
                    const bool pred = live && lane >= start && mt.hit;
                    const unsigned m = __ballot_sync(0xffffffffu, pred);
                    if (!m) break;
                    const int f = __ffs(m) - 1;
                    const Det ef = shfl_det(e, f);
                    int X[4], Y[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        X[i] = __shfl_sync(0xffffffffu, mt.X[i], f);
                        Y[i] = __shfl_sync(0xffffffffu, mt.Y[i], f);
                    }
                    nmax.x = imin(nmax.x, X[0]);
                    nmax.y = imin(nmax.y, Y[0]);
                    nmax.x2 = imax(nmax.x2, X[3]);
                    nmax.y2 = imax(nmax.y2, Y[3]);
                    nmin.x = imax(nmin.x, X[1]);
                    nmin.y = imax(nmin.y, Y[1]);
                    nmin.x2 = imin(nmin.x2, X[2]);
                    nmin.y2 = imin(nmin.y2, Y[2]);
                    nmax.score = (nmax.score < ef.score) ? ef.score : nmax.score;
                    nmax.knn = imax(nmax.knn, ef.knn);
                    nmax.scale = (nmax.scale > ef.scale) ? ef.scale : nmax.scale;
                    nmax.num_detect++;
                    if (lane == f) {
                        checked[j] = 1;
                        live = false;
                    }
                    start = f + 1;
                }
            }
            __syncwarp();
        }
        if (del && dropped) continue;
        Det r = nmax;
        r.x = (nmin.x + nmax.x) >> 1;
        r.y = (nmin.y + nmax.y) >> 1;
        r.x2 = (nmin.x2 + nmax.x2) >> 1;
        r.y2 = (nmin.y2 + nmax.y2) >> 1;
        r.w = r.x2 - r.x;
        r.h = r.y2 - r.y;
        if (lane == 0) out[nout] = r;
        nout++;
        __syncwarp();
    }
    return nout;
}

__global__ void __launch_bounds__(kRT, 1) replay_kernel(const ReplayArgs a) {
    __shared__ int s_e, s_nD, s_nS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const CascadeConfig& C = a.cfg;
    const int n = *a.n_cand;
    int nD = 0;  // kept uniform in every thread through s_nD
    int g = 0;
    while (g < n) {
        const int lev = a.cands[g].level;
        if (tid == 0) s_e = n;
        __syncthreads();
        for (int base = g; base < n; base += kRT) {
            const int i = base + tid;
            if (i < n && a.cands[i].level != lev) atomicMin(&s_e, i);
            __syncthreads();
            if (s_e < n) break;
        }
        const int e = s_e;
        const LevelDesc L = a.levels[lev];
        const float scale = L.scale, inv_scale = L.inv_scale;
        const int n_prefix = nD;

        if (C.drop_detect) {
            // scan test against the detections of earlier levels, one warp per candidate
            for (int c = g + warp; c < e; c += kRT / 32) {
                const Det nr = cand_rect(a.cands[c], inv_scale, scale);
                const Det ex = rect_shrink(nr, 0.7f);
                int code = -1;
                for (int base = 0; base < n_prefix; base += 32) {
                    const int k = base + lane;
                    const int t = k < n_prefix ? drop_test(nr, ex, a.D[k]) : 0;
                    const unsigned m = __ballot_sync(0xffffffffu, t != 0);
                    if (m) {
                        const int f = __ffs(m) - 1;
                        const int tf = __shfl_sync(0xffffffffu, t, f);
                        code = (base + f) * 2 + (tf - 1);
                        break;
                    }
                }
                if (lane == 0) a.first_dec[c] = code;
            }
            __syncthreads();
            if (warp == 0) {
                int nS = 0;
                for (int c = g; c < e; ++c) {
                    const Det nr = cand_rect(a.cands[c], inv_scale, scale);
                    int code = a.first_dec[c];
                    int k0 = -1, type = 0;
                    if (code >= 0) {
                        k0 = code >> 1;
                        type = (code & 1) + 1;
                    } else {
                        const Det ex = rect_shrink(nr, 0.7f);
                        for (int base = n_prefix; base < nD; base += 32) {
                            const int k = base + lane;
                            const int t = k < nD ? drop_test(nr, ex, a.D[k]) : 0;
                            const unsigned m = __ballot_sync(0xffffffffu, t != 0);
                            if (m) {
                                const int f = __ffs(m) - 1;
                                type = __shfl_sync(0xffffffffu, t, f);
                                k0 = base + f;
                                break;
                            }
                        }
                    }
                    if (k0 >= 0) {
                        if (type == 1) {
                            if (lane == 0) {
                                const Det src = a.D[k0];
                                a.D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, src.score, scale, src.knn);
                            }
                            nD++;
                        }
                        __syncwarp();
                        continue;
                    }
                    if (lane == 0) a.survivors[nS] = c;
                    nS++;
                }
                if (lane == 0) {
                    s_nS = nS;
                    s_nD = nD;
                }
            }
            __syncthreads();
            nD = s_nD;
        }

        if (warp == 0) {
            const int nS = C.drop_detect ? s_nS : (e - g);
            const int rect_size = nD;
            for (int si = 0; si < nS; ++si) {
                const int c = C.drop_detect ? a.survivors[si] : g + si;
                const Candidate cd = a.cands[c];
                const Det nr = cand_rect(cd, inv_scale, scale);
                if (C.drop_detect && C.detect_enabled) {
                    int k0 = -1;
                    for (int base = rect_size; base < nD; base += 32) {
                        const int k = base + lane;
                        const bool hit = k < nD && rect_overlap(nr, a.D[k]) > 0.5f;
                        const unsigned m = __ballot_sync(0xffffffffu, hit);
                        if (m) {
                            k0 = base + __ffs(m) - 1;
                            break;
                        }
                    }
                    if (k0 >= 0) {
                        if (lane == 0) {
                            const Det src = a.D[k0];
                            a.D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, src.score, scale, src.knn);
                        }
                        nD++;
                        __syncwarp();
                        continue;
                    }
                }
                if (!C.detect_enabled) {
                    if (lane == 0) a.D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, cd.score, scale, 0);
                    nD++;
                } else {
                    const CandResult r = a.results[c];
                    if (r.accepted) {
                        if (lane == 0) a.D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, r.score, scale, r.knn);
                        nD++;
                    }
                }
                __syncwarp();
            }
            if (lane == 0) s_nD = nD;
        }
        __syncthreads();
        nD = s_nD;
        g = e;
    }

    // post-processing in warp 0
    if (warp != 0) return;
    if (lane == 0) *a.n_raw = nD;
    for (int i = lane; i < nD; i += 32) a.R[i] = a.D[nD - 1 - i];
    __syncwarp();
    if (nD > 16 && lane == 0) introsort_scale_desc(a.R, nD);
    __syncwarp();
    int nF = 0;
    const Det* fin = a.R;
    if (nD > 0) {
        if (C.merger_detect) {
            int nM = merger_warp(a.R, nD, a.checked, a.M, 0.5f, false);
            if (C.min_num_detect > 1) {
                // stable erase of clusters with fewer than min_num_detect merges
                int w = 0;
                for (int base = 0; base < nM; base += 32) {
                    const int k = base + lane;
                    const bool keep = k < nM && a.M[k].num_detect >= C.min_num_detect;
                    const Det v = k < nM ? a.M[k] : a.M[0];
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    const int pos = w + __popc(m & ((1u << lane) - 1u));
                    __syncwarp();
                    if (keep) a.M[pos] = v;
                    __syncwarp();
                    w += __popc(m);
                }
                nM = w;
            }
            if (nM > 0) {
                nF = merger_warp(a.M, nM, a.checked, a.F, 0.2f, true);
                fin = a.F;
            } else {
                nF = 0;
            }
        } else {
            nF = nD;
            fin = a.R;
        }
    }
    for (int i = lane; i < nF && i < a.face_cap; i += 32) {
        Det d = fin[i];
        FaceOut f;
        if (C.rescale_output) {
            f.x = (int)((float)d.x * C.rescale);
            f.y = (int)((float)d.y * C.rescale);
            f.w = (int)((float)d.w * C.rescale);
            f.h = (int)((float)d.h * C.rescale);
        } else {
            f.x = d.x;
            f.y = d.y;
            f.w = d.w;
            f.h = d.h;
        }
        f.score = d.score;
        a.faces[i] = f;
    }
    if (lane == 0) *a.n_faces = nF;
}

cudaError_t launch_replay(const ReplayArgs& a, cudaStream_t st) {
    replay_kernel<<<1, kRT, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ccnn
