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
// Every box a level appends has the geometry of one of that level's candidates, so the tests
// against boxes appended during the level (its own scan, then the survivors' pass) are candidate
// pairs: all warps evaluate them into bit matrices first, and warp 0 then replays the order-
// dependent decisions with one ballot over the bit words per candidate. Levels with more than
// kBitMax candidates take the direct route (warp 0 tests the appended boxes 32 at a time). The sort
// permutes (scale, index) keys. The first clustering pass runs per group of boxes that cannot
// interact (a warp a group), the second on bit matrices of its pair tests; lists too long for the
// shared scratch take one warp through the reference's loop.
#include <climits>
#include <vector>

#include "kernels.h"
#include "replay.cuh"
#include "window_common.cuh"

namespace ccnn {

constexpr int kRT = 1024;

// the candidate's stage-1 pattern rectangle (new_rect, cnn_detector_v3.cpp:1497-1501); the pattern is
// the stage-1 network's smallest input
__device__ __forceinline__ Det cand_rect(const Candidate& c, float inv_scale, float scale, int pat_w, int pat_h) {
    return make_det((int)((float)c.px * inv_scale), (int)((float)c.py * inv_scale), (int)((float)pat_w * inv_scale),
                    (int)((float)pat_h * inv_scale), 0.f, scale, 0);
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

// fl(a / b) > t for a >= 0, b > 0 and t > 0 (normal floats), without the division: the rounded
// quotient exceeds t exactly when the real one lies above the midpoint between t and the next float,
// or on it when the tie rounds to that next float (t's last significand bit is 1). mid * b carries at
// most 25 + 24 significant bits, so the double product and comparison are exact.
__device__ __forceinline__ bool quot_gt(float a, float b, float t) {
    const double mid = 0.5 * ((double)t + (double)nextafterf(t, __int_as_float(0x7f800000)));
    const double prod = mid * (double)b;
    const double aa = (double)a;
    if (aa > prod) return true;
    if (aa < prod) return false;
    return (__float_as_uint(t) & 1u) != 0u;
}

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
    const int CX1 = X[0] + ((X[3] - X[0]) >> 1);
    const int CY1 = Y[0] + ((Y[3] - Y[0]) >> 1);
    const int CX2 = X[1] + ((X[2] - X[1]) >> 1);
    const int CY2 = Y[1] + ((Y[2] - Y[1]) >> 1);
    const int thrC = imin(X[3] - X[0], X[2] - X[1]) >> 1;
    const bool centred = abs(CX1 - CX2) < thrC && abs(CY1 - CY2) < thrC;
    if (S1 > 0.f && S2 > 0.f && su > 0.f && si >= 0.f && threshold > 0.f) {
        // r1 = si / S1, r2 = si / S2, r3 = si / su as the reference rounds them, compared without
        // dividing: min(r1, r2) > threshold is both > threshold, max(r1, r2) > 0.7 is either
        const bool over = centred && quot_gt(si, su, fmul(0.75f, threshold)) && (quot_gt(si, S1, 0.7f) || quot_gt(si, S2, 0.7f));
        t.hit = over ? (1.f > threshold) : (quot_gt(si, S1, threshold) && quot_gt(si, S2, threshold));
    } else {
        const float r1 = fdiv(si, S1), r2 = fdiv(si, S2), r3 = fdiv(si, su);
        float ratio = r1 > r2 ? r2 : r1;
        if (r3 > fmul(0.75f, threshold) && (r1 < r2 ? r2 : r1) > 0.7f && centred) ratio = 1.f;
        t.hit = ratio > threshold;
    }
    t.s1_gt_s2 = S1 > S2;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        t.X[i] = X[i];
        t.Y[i] = Y[i];
    }
    return t;
}

// Merger (cnn_detector_v3.cpp:2814-2936) run by one warp. in[] is read-only; checked[] is scratch.
// clus (optional): cluster (output index) of every input box; src (optional): input index of
// every output box.
__device__ int merger_warp(const Det* in, int n, uint8_t* checked, Det* out, float threshold, bool del, int* clus = nullptr,
                           int* src = nullptr) {
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
                // the first lane (at or after `start`) whose box merges into the running cluster is
                // absorbed; every lane then re-tests against the grown cluster box. The absorbed
                // box is read by all lanes from shared memory (a broadcast), not shuffled.
                int start = 0;
                while (true) {
                    const MergeTest mt = merge_test(nmax, e, threshold);
                    const bool pred = live && lane >= start && mt.hit;
                    const unsigned m = __ballot_sync(0xffffffffu, pred);
                    if (!m) break;
                    const int f = __ffs(m) - 1;
                    const Det ef = in[base + f];
                    int X[4] = {nmax.x, nmax.x2, ef.x, ef.x2};
                    int Y[4] = {nmax.y, nmax.y2, ef.y, ef.y2};
                    sort4(X);
                    sort4(Y);
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
                        if (clus) clus[j] = nout;
                    }
                    start = f + 1;
                }
            }
            __syncwarp();
        }
        if (del && dropped) continue;
        if (lane == 0) {
            if (clus) clus[i1] = nout;
            if (src) src[nout] = i1;
        }
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

// ---- the first merge by independent groups ----
// Merger(0.5, false) grows a cluster box as the bounding box of the boxes it absorbed, and a box
// only merges into a cluster box it overlaps. Split the boxes into groups whose bounding boxes do not
// overlap each other (the overlap relation closed under bounding boxes): no cluster box of one group
// can then overlap a box of another, so each group runs the reference's loop on its own and the
// clusters, listed by their first box, come out in the order of the single loop.

// concurrent union-find in shared memory: parent[x] <= x, roots have parent[x] == x. Linking CASes
// the larger root onto the smaller and retries from the value found (the hooking of Jaiganesh and
// Burtscher's ECL-CC, SC'18); roots only ever move to a smaller index, so a compression write, even
// a late one, still points at an ancestor.
__device__ __forceinline__ int uf_root(volatile int* parent, int x) {
    int cur = parent[x];
    if (cur != x) {
        int prev = x, next;
        while (cur > (next = parent[cur])) {
            parent[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

__device__ __forceinline__ bool uf_hook(volatile int* parent, int a, int b) {
    int ra = uf_root(parent, a), rb = uf_root(parent, b);
    while (ra != rb) {
        if (ra < rb) {
            const int t = ra;
            ra = rb;
            rb = t;
        }
        const int old = atomicCAS(const_cast<int*>(parent + ra), ra, rb);
        if (old == ra) return true;
        ra = old;
    }
    return false;
}

// The reference's loop over the boxes of group r (parent[j] == r) by one warp, as merger_warp does
// for the whole list; seed_box[i1] / seed_of[j]: the merged box of the cluster that box i1 starts,
// the first box of the cluster that absorbed box j.
__device__ void merge_group_warp(const Det* in, int n, const int* parent, int r, uint8_t* checked, Det* seed_box, int* seed_of) {
    const int lane = threadIdx.x & 31;
    for (int cb = r & ~31; cb < n; cb += 32) {
        const int jj = cb + lane;
        unsigned mm = __ballot_sync(0xffffffffu, jj < n && jj >= r && parent[jj] == r);
        while (mm) {
            const int i1 = cb + __ffs(mm) - 1;
            mm &= mm - 1;
            if (checked[i1]) continue;
            Det nmax = in[i1], nmin = in[i1];
            for (int base = i1 + 1; base < n; base += 32) {
                const int j = base + lane;
                bool live = j < n && parent[j] == r && !checked[j];
                if (!__any_sync(0xffffffffu, live)) continue;
                const Det e = live ? in[j] : nmax;
                int start = 0;
                while (true) {
                    const MergeTest mt = merge_test(nmax, e, 0.5f);
                    const unsigned m = __ballot_sync(0xffffffffu, live && lane >= start && mt.hit);
                    if (!m) break;
                    const int f = __ffs(m) - 1;
                    const Det ef = in[base + f];
                    int X[4] = {nmax.x, nmax.x2, ef.x, ef.x2};
                    int Y[4] = {nmax.y, nmax.y2, ef.y, ef.y2};
                    sort4(X);
                    sort4(Y);
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
                        seed_of[j] = i1;
                    }
                    start = f + 1;
                }
                __syncwarp();
            }
            Det rr = nmax;
            rr.x = (nmin.x + nmax.x) >> 1;
            rr.y = (nmin.y + nmax.y) >> 1;
            rr.x2 = (nmin.x2 + nmax.x2) >> 1;
            rr.y2 = (nmin.y2 + nmax.y2) >> 1;
            rr.w = rr.x2 - rr.x;
            rr.h = rr.y2 - rr.y;
            if (lane == 0) {
                seed_of[i1] = i1;
                seed_box[i1] = rr;
            }
            __syncwarp();
        }
    }
}

// Merger(0.5, false) of n <= kGroupMax sorted boxes by the whole block; returns the cluster count
// (every thread). out: the clusters in reference order; seed_box: n Det of scratch; clus (optional):
// cluster of every box; ws_a / ws_b: 4n / 3n ints of shared memory.
constexpr int kGroupMax = 512;
__device__ int first_merge_groups(const Det* in, int n, uint8_t* checked, Det* out, Det* seed_box, int* clus, int* ws_a, int* ws_b) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    volatile int* parent = ws_a;
    int* bx0 = ws_a + n;
    int* by0 = ws_a + 2 * n;
    int* bx1 = ws_a + 3 * n;
    int* by1 = ws_b;
    int* seed_of = ws_b + n;
    int* rank_of = ws_b + 2 * n;
    __shared__ int s_groups;
    for (int j = tid; j < n; j += blockDim.x) {
        parent[j] = j;
        checked[j] = 0;
    }
    __syncthreads();
    // boxes that overlap or touch share a group
    for (int i = warp; i < n; i += nwarps) {
        const Det bi = in[i];
        const int ax0 = imin(bi.x, bi.x2), ax1 = imax(bi.x, bi.x2), ay0 = imin(bi.y, bi.y2), ay1 = imax(bi.y, bi.y2);
        for (int j = i + 1 + lane; j < n; j += 32) {
            const Det bj = in[j];
            if (ax0 <= imax(bj.x, bj.x2) && imin(bj.x, bj.x2) <= ax1 && ay0 <= imax(bj.y, bj.y2) && imin(bj.y, bj.y2) <= ay1)
                uf_hook(parent, i, j);
        }
    }
    __syncthreads();
    // groups whose bounding boxes overlap or touch are joined until none do
    for (;;) {
        for (int j = tid; j < n; j += blockDim.x) {
            int v = parent[j];
            while (v != parent[v]) v = parent[v];
            parent[j] = v;  // only this thread writes parent[j] in this pass
            bx0[j] = by0[j] = INT_MAX;
            bx1[j] = by1[j] = INT_MIN;
        }
        __syncthreads();
        for (int j = tid; j < n; j += blockDim.x) {
            const Det b = in[j];
            const int g = parent[j];
            atomicMin(&bx0[g], imin(b.x, b.x2));
            atomicMin(&by0[g], imin(b.y, b.y2));
            atomicMax(&bx1[g], imax(b.x, b.x2));
            atomicMax(&by1[g], imax(b.y, b.y2));
        }
        __syncthreads();
        bool linked = false;
        for (int i = warp; i < n; i += nwarps) {
            if (parent[i] != i) continue;
            for (int j = i + 1 + lane; j < n; j += 32)
                if (parent[j] == j && bx0[i] <= bx1[j] && bx0[j] <= bx1[i] && by0[i] <= by1[j] && by0[j] <= by1[i])
                    linked |= uf_hook(parent, i, j);
        }
        if (!__syncthreads_or(linked)) break;
    }
    // a pass without links left every parent a root: group g = the root; warp w takes the groups
    // w, w + nwarps, ... in order of their roots
    int ord = 0;
    for (int cb = 0; cb < n; cb += 32) {
        const int j = cb + lane;
        unsigned rm = __ballot_sync(0xffffffffu, j < n && parent[j] == j);
        while (rm) {
            const int g = cb + __ffs(rm) - 1;
            rm &= rm - 1;
            if (ord++ % nwarps == warp) merge_group_warp(in, n, const_cast<const int*>(ws_a), g, checked, seed_box, seed_of);
        }
    }
    __syncthreads();
    // clusters ranked by their first box
    if (warp == 0) {
        int w = 0;
        for (int cb = 0; cb < n; cb += 32) {
            const int j = cb + lane;
            const bool s = j < n && seed_of[j] == j;
            const unsigned m = __ballot_sync(0xffffffffu, s);
            if (s) rank_of[j] = w + __popc(m & ((1u << lane) - 1u));
            w += __popc(m);
        }
        if (lane == 0) s_groups = w;
    }
    __syncthreads();
    const int nM = s_groups;
    for (int j = tid; j < n; j += blockDim.x) {
        const int s = seed_of[j];
        if (s == j) out[rank_of[j]] = seed_box[j];
        if (clus) clus[j] = rank_of[s];
    }
    __syncthreads();
    return nM;
}

// Merger(0.2, true) of n <= 256 boxes by the whole block. With deletion a box never grows, so each
// pair test depends on the two boxes only: bit j of word w of row i (j = 32w + bit > i) is set in
// `take` when box i deletes box j (the test hits and box i is larger), in `drop` when box j deletes
// box i. The reference's loop then runs on bit sets in warp 0: a box not yet deleted deletes its live
// `take` boxes up to its first live `drop` box, and is itself dropped if there is one.
// take / drop: n * ceil(n / 32) words each. Returns the output count (every thread).
__device__ int second_merge_bits(const Det* in, int n, Det* out, int* src, uint32_t* take, uint32_t* drop) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int W = (n + 31) >> 5;
    __shared__ int s_out;
    for (int it = warp; it < n * W; it += nwarps) {
        const int i = it / W, w = it - i * W;
        const int j = 32 * w + lane;
        bool hit = false, gt = false;
        if (j > i && j < n) {
            const MergeTest mt = merge_test(in[i], in[j], 0.2f);
            hit = mt.hit;
            gt = mt.s1_gt_s2;
        }
        const uint32_t bt = __ballot_sync(0xffffffffu, hit && gt), bd = __ballot_sync(0xffffffffu, hit && !gt);
        if (lane == 0) {
            take[it] = bt;
            drop[it] = bd;
        }
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t del = 0u;  // lane w < W: the deleted boxes of word w
        int nout = 0;
        for (int i = 0; i < n; ++i) {
            if ((__shfl_sync(0xffffffffu, del, i >> 5) >> (i & 31)) & 1u) continue;
            const uint32_t t = lane < W ? take[i * W + lane] & ~del : 0u;
            const uint32_t d = lane < W ? drop[i * W + lane] & ~del : 0u;
            const unsigned dm = __ballot_sync(0xffffffffu, d != 0u);
            if (dm) {
                const int wf = __ffs(dm) - 1;
                const uint32_t first = __shfl_sync(0xffffffffu, d, wf);
                if (lane < wf) del |= t;
                else if (lane == wf) del |= t & ((1u << (__ffs(first) - 1)) - 1u);
                continue;
            }
            del |= t;
            if (lane == 0) {
                const Det b = in[i];
                Det rr = b;
                rr.x = (b.x + b.x) >> 1;
                rr.y = (b.y + b.y) >> 1;
                rr.x2 = (b.x2 + b.x2) >> 1;
                rr.y2 = (b.y2 + b.y2) >> 1;
                rr.w = rr.x2 - rr.x;
                rr.h = rr.y2 - rr.y;
                out[nout] = rr;
                if (src) src[nout] = i;
            }
            nout++;
        }
        if (lane == 0) s_out = nout;
    }
    __syncthreads();
    return s_out;
}

constexpr int kMaxLevels = 1024;


constexpr int kBitMax = 256;              // candidates per level handled with bit matrices
constexpr int kBitWords = kBitMax / 32;
constexpr int kOwnVerdict = -kBitMax - 1;  // the candidate's own stage-2/3 verdict
constexpr int kOwnScore = -kBitMax - 2;    // the candidate's stage-1 score (detection disabled)

__device__ __forceinline__ void replay_body(const ReplayArgs& a) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ int s_lvl_start[kMaxLevels + 1];
    __shared__ int s_nD, s_nS;
    // bit j of word w of row i: drop_test(candidate i, box of candidate 32w + j) == 1 (A1) / == 2 (A2)
    __shared__ uint32_t s_a1[kBitMax * kBitWords], s_a2[kBitMax * kBitWords];
    __shared__ int s_didx[kBitMax];  // D index of the box a candidate appended, or -1
    __shared__ int s_src[kBitMax];   // where that box's score/knn come from
    __shared__ uint32_t s_S[kBitWords], s_T[kBitWords];  // candidate sets of the level (see below)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const CascadeConfig& C = a.cfg;
    const int n = *a.n_cand;
    const int nl = a.n_levels;

    // working set in shared memory when it fits (121 bytes per candidate), else global scratch:
    //   region A: candidates, verdicts, scan results, survivors (40 B each); later the first merge
    //   region B: detections in reference order; later the second merge
    //   region C: reversed + sorted detections; region E: merge flags
    const bool fits = (long long)n * 121 + 64 <= kReplaySmemBytes;
    Candidate* cands;
    CandResult* res;
    int* first_dec;
    int* surv;
    Det *D, *R, *M, *F;
    uint8_t* checked;
    if (fits) {
        unsigned char* p = sm;
        cands = reinterpret_cast<Candidate*>(p);
        res = reinterpret_cast<CandResult*>(p + 16LL * n);
        first_dec = reinterpret_cast<int*>(p + 32LL * n);
        surv = reinterpret_cast<int*>(p + 36LL * n);
        M = reinterpret_cast<Det*>(p);
        D = reinterpret_cast<Det*>(p + 40LL * n);
        F = D;
        R = reinterpret_cast<Det*>(p + 80LL * n);
        checked = p + 120LL * n;
        for (int i = tid; i < n; i += kRT) cands[i] = a.cands[i];
    } else {
        cands = const_cast<Candidate*>(a.cands);
        res = a.results;
        first_dec = a.first_dec;
        surv = a.survivors;
        D = a.D;
        R = a.R;
        M = a.M;
        F = a.F;
        checked = a.checked;
    }
    // With drop_detect, the candidate-pair tests of every level (bit j of word w of candidate i's row:
    // drop_test(candidate i, box of candidate 32w + j of the same level) == 1 / == 2) are evaluated
    // for all levels at once before the level loop, where the rows (kBitWords words per candidate)
    // fit in shared memory beside the working set; the loop then only reads them.
    const bool pre_rows = fits && C.drop_detect && ((121LL * n + 15) & ~15LL) + 8LL * kBitWords * n <= kReplaySmemBytes;
    uint32_t* P1 = pre_rows ? reinterpret_cast<uint32_t*>(sm + ((121LL * n + 15) & ~15LL)) : nullptr;
    uint32_t* P2 = pre_rows ? P1 + (size_t)kBitWords * n : nullptr;
    for (int l = tid; l <= nl; l += kRT) s_lvl_start[l] = 0;
    __syncthreads();
    // verdicts and per-level candidate counts (candidates are grouped by level, smallest first)
    for (int i = tid; i < n; i += kRT) {
        const Candidate cd = cands[i];
        if (C.detect_enabled) {
            const CandResult r = verdict(a.win + (size_t)i * 4, cd, a.levels[cd.level].scale, C);
            res[i] = r;
            if (fits) a.results[i] = r;  // kept for inspection
        }
        atomicAdd(&s_lvl_start[nl - 1 - cd.level + 1], 1);
    }
    __syncthreads();
    if (tid == 0) {
        for (int k = 1; k <= nl; ++k) s_lvl_start[k] += s_lvl_start[k - 1];
        s_nD = 0;
    }
    __syncthreads();
    if (pre_rows) {
        // a warp a candidate row, one ballot a word
        for (int c = warp; c < n; c += kRT / 32) {
            const Candidate cd = cands[c];
            const int k = nl - 1 - cd.level;
            const int g = s_lvl_start[k], m = s_lvl_start[k + 1] - g, i = c - g;
            if (m > kBitMax) continue;
            const LevelDesc& Lc = a.levels[cd.level];
            const Det nr = cand_rect(cd, Lc.inv_scale, Lc.scale, C.pat_w, C.pat_h);
            const Det ex = rect_shrink(nr, 0.7f);
            for (int w = 0; w < ((i + 31) >> 5); ++w) {
                const int j = 32 * w + lane;
                int t = 0;
                if (j < i) t = drop_test(nr, ex, cand_rect(cands[g + j], Lc.inv_scale, Lc.scale, C.pat_w, C.pat_h));
                const uint32_t b1 = __ballot_sync(0xffffffffu, t == 1), b2 = __ballot_sync(0xffffffffu, t == 2);
                if (lane == 0) {
                    P1[(size_t)c * kBitWords + w] = b1;
                    P2[(size_t)c * kBitWords + w] = b2;
                }
            }
            // words at and past the candidate's own index stay 0
            if (lane < kBitWords && lane >= ((i + 31) >> 5)) {
                P1[(size_t)c * kBitWords + lane] = 0u;
                P2[(size_t)c * kBitWords + lane] = 0u;
            }
        }
        __syncthreads();
    }

    int nD = 0;
    for (int k = 0; k < nl; ++k) {
        const int g = s_lvl_start[k], e = s_lvl_start[k + 1];
        if (g == e) continue;
        const int lev = nl - 1 - k;
        const LevelDesc& L = a.levels[lev];
        const float scale = L.scale, inv_scale = L.inv_scale;
        const int n_prefix = nD;

        if (C.drop_detect) {
            // scan test against the detections of earlier levels, one warp per candidate
            for (int c = g + warp; c < e; c += kRT / 32) {
                const Det nr = cand_rect(cands[c], inv_scale, scale, C.pat_w, C.pat_h);
                const Det ex = rect_shrink(nr, 0.7f);
                int code = -1;
                for (int base = 0; base < n_prefix; base += 32) {
                    const int kk = base + lane;
                    const int t = kk < n_prefix ? drop_test(nr, ex, D[kk]) : 0;
                    const unsigned m = __ballot_sync(0xffffffffu, t != 0);
                    if (m) {
                        const int f = __ffs(m) - 1;
                        const int tf = __shfl_sync(0xffffffffu, t, f);
                        code = (base + f) * 2 + (tf - 1);
                        break;
                    }
                }
                if (lane == 0) first_dec[c] = code;
            }
            const int m = e - g;
            const int W = (m + 31) >> 5;
            // box of candidate i of the level: its rect, score/knn from the end of its copy chain;
            // facial data travels with a candidate's own accepted box, not with copies
            auto emit_box = [&](int i) {
                int r = i, src = s_src[i];
                while (src < 0 && src > kOwnVerdict) {  // a box of this level: follow it
                    r = -1 - src;
                    src = s_src[r];
                }
                float sc;
                int kn;
                if (src >= 0) {
                    sc = D[src].score;
                    kn = D[src].knn;
                } else if (src == kOwnVerdict) {
                    sc = res[g + r].score;
                    kn = res[g + r].knn;
                } else {
                    sc = cands[g + r].score;
                    kn = 0;
                }
                const Det nr = cand_rect(cands[g + i], inv_scale, scale, C.pat_w, C.pat_h);
                D[s_didx[i]] = make_det(nr.x, nr.y, nr.w, nr.h, sc, scale, kn);
                if (a.fa_scratch) a.fa_scratch[s_didx[i]] = (s_src[i] == kOwnVerdict) ? g + i : -1;
            };
            if (pre_rows) {
                // the level's rows, evaluated before the loop (levels of up to 32 read them in warp 0)
                if (m > 32 && m <= kBitMax)
                    for (int it = tid; it < m * W; it += kRT) {
                        const int i = it / W, w = it - i * W;
                        s_a1[it] = P1[(size_t)(g + i) * kBitWords + w];
                        s_a2[it] = P2[(size_t)(g + i) * kBitWords + w];
                    }
            } else if (m <= kBitMax) {
                // candidate-pair tests of this level, one ballot per (row i, word w)
                for (int it = warp; it < m * W; it += kRT / 32) {
                    const int i = it / W, w = it - i * W;
                    const int j = 32 * w + lane;
                    int t = 0;
                    if (j < i) {
                        const Det nr = cand_rect(cands[g + i], inv_scale, scale, C.pat_w, C.pat_h);
                        t = drop_test(nr, rect_shrink(nr, 0.7f), cand_rect(cands[g + j], inv_scale, scale, C.pat_w, C.pat_h));
                    }
                    const uint32_t b1 = __ballot_sync(0xffffffffu, t == 1), b2 = __ballot_sync(0xffffffffu, t == 2);
                    if (lane == 0) {
                        s_a1[i * W + w] = b1;
                        s_a2[i * W + w] = b2;
                    }
                }
            }
            __syncthreads();
            // The order-dependent decisions of the level as fixed points over candidate sets (bit j of
            // word w = candidate 32w + j). Candidate i's decision depends only on candidates j < i, so
            // after t rounds the first t candidates are final, and a round that changes nothing has
            // reached the unique solution, which is the sequential one.
            //   S: boxes appended during the scan: the first decisive box of candidate i (earlier
            //      levels first, then S in order) has drop type 1;
            //   T: boxes appended by the survivors' pass: survivor i overlaps (> 0.5) a box of T
            //      (a copy), or its stage-2/3 verdict accepts it (or detection is disabled).
            const bool check = C.detect_enabled != 0;
            if (m <= 32) {
                // one word: warp 0 alone, candidate i = lane, its rows and decisions in registers;
                // a round is one ballot
                if (warp == 0) {
                    const int i = lane;
                    const bool valid = i < m;
                    int code = -1, acc = 0;
                    uint32_t r1 = 0u, r2 = 0u;
                    if (valid) {
                        code = first_dec[g + i];
                        acc = C.detect_enabled ? res[g + i].accepted : 1;
                        if (acc && a.attr && a.attr[g + i].x) acc = 0;  // facial analysis dropped it
                        r1 = pre_rows ? P1[(size_t)(g + i) * kBitWords] : s_a1[i];
                        r2 = pre_rows ? P2[(size_t)(g + i) * kBitWords] : s_a2[i];
                    }
                    uint32_t S = 0u;
                    for (int round = 0; round <= m; ++round) {
                        bool in = false;
                        if (valid) {
                            if (code >= 0) {
                                in = (code & 1) == 0;
                            } else {
                                const uint32_t hit = (r1 | r2) & S;
                                if (hit) in = ((r1 >> (__ffs(hit) - 1)) & 1u) != 0u;
                            }
                        }
                        const uint32_t nS = __ballot_sync(0xffffffffu, in);
                        if (nS == S) break;
                        S = nS;
                    }
                    // survivors: not decided by the scan
                    const bool surv_i = valid && code < 0 && ((r1 | r2) & S) == 0u;
                    uint32_t T = 0u;
                    for (int round = 0; round <= m; ++round) {
                        const bool in = surv_i && (acc != 0 || (check && (r1 & T) != 0u));
                        const uint32_t nT = __ballot_sync(0xffffffffu, in);
                        if (nT == T) break;
                        T = nT;
                    }
                    // D index (scan appends in candidate order, then the survivors' appends) and the
                    // source of each box's score/knn
                    const int nScan = __popc(S);
                    const uint32_t below = (1u << i) - 1u;
                    if (valid) {
                        int dst = -1, src = 0;
                        if ((S >> i) & 1u) {
                            dst = nD + __popc(S & below);
                            src = code >= 0 ? (code >> 1) : -1 - (__ffs((r1 | r2) & S) - 1);
                        } else if ((T >> i) & 1u) {
                            dst = nD + nScan + __popc(T & below);
                            src = C.detect_enabled ? kOwnVerdict : kOwnScore;
                            if (check && (r1 & T)) src = -1 - (__ffs(r1 & T) - 1);
                        }
                        s_didx[i] = dst;
                        s_src[i] = src;
                    }
                    __syncwarp();
                    if (valid && s_didx[i] >= 0) emit_box(i);
                    if (lane == 0) s_nD = nD + nScan + __popc(T);
                }
                __syncthreads();
                nD = s_nD;
                continue;
            }
            if (m <= kBitMax) {
                // several words: a thread a candidate (m <= 256: warps 0..7), block-wide rounds
                const bool thread_item = tid < m;
                const int i = tid;
                int code = -1, acc = 0;
                if (thread_item) {
                    code = first_dec[g + i];
                    acc = C.detect_enabled ? res[g + i].accepted : 1;
                    if (acc && a.attr && a.attr[g + i].x) acc = 0;  // facial analysis dropped it
                }
                if (tid < kBitWords) {
                    s_S[tid] = 0u;
                    s_T[tid] = 0u;
                }
                __syncthreads();
                bool inS = false;
                for (int round = 0; round <= m; ++round) {
                    bool in = false;
                    if (thread_item) {
                        if (code >= 0) {
                            in = (code & 1) == 0;
                        } else {
                            for (int w = 0; w < W; ++w) {
                                const uint32_t hit = (s_a1[i * W + w] | s_a2[i * W + w]) & s_S[w];
                                if (hit) {
                                    in = (s_a1[i * W + w] >> (__ffs(hit) - 1)) & 1u;
                                    break;
                                }
                            }
                        }
                    }
                    const uint32_t word = __ballot_sync(0xffffffffu, in);
                    __syncthreads();  // every thread has read the previous round's S
                    const bool changed = (lane == 0 && warp < W && s_S[warp] != word);
                    if (lane == 0 && warp < W) s_S[warp] = word;
                    inS = in;
                    if (!__syncthreads_or(changed)) break;
                }
                // survivors: not decided by the scan
                bool surv_i = false;
                if (thread_item && code < 0) {
                    surv_i = true;
                    for (int w = 0; w < W; ++w)
                        if ((s_a1[i * W + w] | s_a2[i * W + w]) & s_S[w]) {
                            surv_i = false;
                            break;
                        }
                }
                for (int round = 0; round <= m; ++round) {
                    bool in = false;
                    if (surv_i) {
                        in = acc != 0;
                        if (check)
                            for (int w = 0; w < W && !in; ++w) in = (s_a1[i * W + w] & s_T[w]) != 0u;
                    }
                    const uint32_t word = __ballot_sync(0xffffffffu, in);
                    __syncthreads();
                    const bool changed = (lane == 0 && warp < W && s_T[warp] != word);
                    if (lane == 0 && warp < W) s_T[warp] = word;
                    if (!__syncthreads_or(changed)) break;
                }
                int nScan = 0, nSurv = 0;
                for (int w = 0; w < W; ++w) {
                    nScan += __popc(s_S[w]);
                    nSurv += __popc(s_T[w]);
                }
                if (thread_item) {
                    const uint32_t below = (1u << (i & 31)) - 1u;
                    int dst = -1, src = 0;
                    if (inS) {
                        int r = 0;
                        for (int w = 0; w < (i >> 5); ++w) r += __popc(s_S[w]);
                        dst = nD + r + __popc(s_S[i >> 5] & below);
                        if (code >= 0) {
                            src = code >> 1;
                        } else {
                            for (int w = 0; w < W; ++w) {
                                const uint32_t hit = (s_a1[i * W + w] | s_a2[i * W + w]) & s_S[w];
                                if (hit) {
                                    src = -1 - (32 * w + __ffs(hit) - 1);
                                    break;
                                }
                            }
                        }
                    } else if ((s_T[i >> 5] >> (i & 31)) & 1u) {
                        int r = 0;
                        for (int w = 0; w < (i >> 5); ++w) r += __popc(s_T[w]);
                        dst = nD + nScan + r + __popc(s_T[i >> 5] & below);
                        src = C.detect_enabled ? kOwnVerdict : kOwnScore;
                        if (check)
                            for (int w = 0; w < W; ++w) {
                                const uint32_t hit = s_a1[i * W + w] & s_T[w];
                                if (hit) {
                                    src = -1 - (32 * w + __ffs(hit) - 1);
                                    break;
                                }
                            }
                    }
                    s_didx[i] = dst;
                    s_src[i] = src;
                }
                __syncthreads();
                if (thread_item && s_didx[i] >= 0) emit_box(i);
                nD += nScan + nSurv;
                __syncthreads();
                continue;
            }
            if (warp == 0) {
                int nS = 0;
                for (int c = g; c < e; ++c) {
                    const int code = first_dec[c];
                    int k0 = -1, type = 0;
                    Det nr;
                    if (code >= 0) {
                        k0 = code >> 1;
                        type = (code & 1) + 1;
                    } else if (nD > n_prefix) {
                        nr = cand_rect(cands[c], inv_scale, scale, C.pat_w, C.pat_h);
                        const Det ex = rect_shrink(nr, 0.7f);
                        for (int base = n_prefix; base < nD; base += 32) {
                            const int kk = base + lane;
                            const int t = kk < nD ? drop_test(nr, ex, D[kk]) : 0;
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
                                nr = cand_rect(cands[c], inv_scale, scale, C.pat_w, C.pat_h);
                                const Det src = D[k0];
                                D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, src.score, scale, src.knn);
                                if (a.fa_scratch) a.fa_scratch[nD] = -1;
                            }
                            nD++;
                            __syncwarp();
                        }
                        continue;
                    }
                    if (lane == 0) surv[nS] = c;
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
                const int c = C.drop_detect ? surv[si] : g + si;
                const Candidate cd = cands[c];
                const Det nr = cand_rect(cd, inv_scale, scale, C.pat_w, C.pat_h);
                if (C.drop_detect && C.detect_enabled && nD > rect_size) {
                    int k0 = -1;
                    for (int base = rect_size; base < nD; base += 32) {
                        const int kk = base + lane;
                        const bool hit = kk < nD && rect_overlap(nr, D[kk]) > 0.5f;
                        const unsigned m = __ballot_sync(0xffffffffu, hit);
                        if (m) {
                            k0 = base + __ffs(m) - 1;
                            break;
                        }
                    }
                    if (k0 >= 0) {
                        if (lane == 0) {
                            const Det src = D[k0];
                            D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, src.score, scale, src.knn);
                            if (a.fa_scratch) a.fa_scratch[nD] = -1;
                        }
                        nD++;
                        __syncwarp();
                        continue;
                    }
                }
                if (!C.detect_enabled) {
                    if (lane == 0) {
                        D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, cd.score, scale, 0);
                        if (a.fa_scratch) a.fa_scratch[nD] = -1;
                    }
                    nD++;
                } else {
                    const CandResult r = res[c];
                    // facial analysis drops a window whose landmarks collapse (cnn_detector_v3.cpp:1750)
                    if (r.accepted && !(a.attr && a.attr[c].x)) {
                        if (lane == 0) {
                            D[nD] = make_det(nr.x, nr.y, nr.w, nr.h, r.score, scale, r.knn);
                            if (a.fa_scratch) a.fa_scratch[nD] = c;
                        }
                        nD++;
                    }
                }
                __syncwarp();
            }
            if (lane == 0) s_nD = nD;
        }
        __syncthreads();
        nD = s_nD;
    }

    // raw list (reference order) to global memory for inspection; the reversed list is sorted by
    // permuting (scale, index) keys (the first region is free once the levels are done)
    if (fits)
        for (int i = tid; i < nD; i += kRT) a.D[i] = D[i];
    ScaleKey* K = fits ? reinterpret_cast<ScaleKey*>(sm) : reinterpret_cast<ScaleKey*>(a.M);
    for (int i = tid; i < nD; i += kRT) K[i] = ScaleKey{D[nD - 1 - i].scale, i};
    __syncthreads();
    // n <= 16: insertion sort of a sorted list. The block-wide sort keeps its segment lists in the
    // bit-matrix words (free after the level loop) and its partitions' stop lists in the scan and
    // survivor scratch (also free).
    constexpr int kSortSegs = (kBitMax * kBitWords) / 3;
    if (nD > 16 && nD / 17 <= kSortSegs) {
        introsort_scale_desc_block(K, nD, reinterpret_cast<int*>(s_a1), reinterpret_cast<int*>(s_a2), kSortSegs, first_dec, surv);
    } else {
        if (nD > 16 && tid == 0) introsort_scale_desc(K, nD);
        __syncthreads();
    }
    for (int i = tid; i < nD; i += kRT) {
        R[i] = D[nD - 1 - K[i].idx];
        if (a.fa_scratch) a.fa_scratch[a.face_cap + i] = a.fa_scratch[nD - 1 - K[i].idx];
    }
    __syncthreads();

    // post-processing: the two merges by the whole block where their scratch fits in the bit-matrix
    // words (free after the level loop and the sort), else in warp 0
    __shared__ int s_nM;
    if (tid == 0) {
        *a.n_raw = nD;
        if (a.n_m_out) *a.n_m_out = 0;
    }
    int nF = 0;
    const Det* fin = R;
    int* fa = a.fa_scratch;
    const int cap = a.face_cap;
    int* clus = fa ? fa + 2 * cap : nullptr;     // cluster of every sorted box
    int* keepmap = fa ? fa + 3 * cap : nullptr;  // first-merge cluster of every kept box
    int* fsrc = fa ? fa + 4 * cap : nullptr;     // kept box of every final box
    uint32_t* ws_a = reinterpret_cast<uint32_t*>(s_a1);
    uint32_t* ws_b = reinterpret_cast<uint32_t*>(s_a2);
    if (nD > 0 && C.merger_detect) {
        int nM;
        if (nD <= kGroupMax) {
            // F is scratch here (the first box of every cluster's merged box) until the second merge
            nM = first_merge_groups(R, nD, checked, M, F, clus, reinterpret_cast<int*>(ws_a), reinterpret_cast<int*>(ws_b));
        } else {
            if (warp == 0) {
                const int k = merger_warp(R, nD, checked, M, 0.5f, false, clus);
                if (lane == 0) s_nM = k;
            }
            __syncthreads();
            nM = s_nM;
        }
        if (keepmap)
            for (int k = tid; k < nM; k += kRT) keepmap[k] = k;
        __syncthreads();
        if (C.min_num_detect > 1) {
            // stable erase of clusters with fewer than min_num_detect merges
            if (warp == 0) {
                int w = 0;
                for (int base = 0; base < nM; base += 32) {
                    const int kk = base + lane;
                    const bool keep = kk < nM && M[kk].num_detect >= C.min_num_detect;
                    const Det v = kk < nM ? M[kk] : M[0];
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    const int pos = w + __popc(m & ((1u << lane) - 1u));
                    __syncwarp();
                    if (keep) {
                        M[pos] = v;
                        if (keepmap) keepmap[pos] = kk;
                    }
                    __syncwarp();
                    w += __popc(m);
                }
                if (lane == 0) s_nM = w;
            }
            __syncthreads();
            nM = s_nM;
        }
        if (a.m_out) {
            for (int k = tid; k < nM; k += kRT) a.m_out[k] = M[k];
            if (tid == 0) *a.n_m_out = nM;
        }
        if (nM > 0) {
            if (nM <= kBitMax) {
                nF = second_merge_bits(M, nM, F, fsrc, ws_a, ws_b);
            } else {
                __syncthreads();
                if (warp == 0) {
                    const int k = merger_warp(M, nM, checked, F, 0.2f, true, nullptr, fsrc);
                    if (lane == 0) s_nM = k;
                }
                __syncthreads();
                nF = s_nM;
            }
            fin = F;
        }
    } else if (nD > 0) {
        if (fa)
            for (int k = tid; k < nD; k += kRT) {
                clus[k] = k;
                keepmap[k] = k;
                fsrc[k] = k;
            }
        nF = nD;
        fin = R;
    }
    __syncthreads();
    for (int i = tid; i < nF && i < a.face_cap; i += kRT) {
        const Det d = fin[i];
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
        f.scale = d.scale;
        f.knn = d.knn;
        f.num_detect = d.num_detect;
        f.pad = 0;
        f.gender = f.smile = f.glasses = -1;
        if (a.fa_scratch) {
            // CompactCNNLibAPI_v2.cpp:296-319: each attribute is the element at size/2 of the
            // merged box's facial data sorted in descending order
            const int c = a.fa_scratch[3 * a.face_cap + a.fa_scratch[4 * a.face_cap + i]];
            const int* rcand = a.fa_scratch + a.face_cap;
            const int* cl = a.fa_scratch + 2 * a.face_cap;
            int size = 0;
            for (int r = 0; r < nD; ++r)
                if (cl[r] == c && rcand[r] >= 0) size++;
            if (size > 0) {
                const int k = size / 2;
                int outv[3];
                for (int q = 0; q < 3; ++q) {
                    // the k-th largest value (0-based): a value v with #(> v) <= k < #(>= v)
                    outv[q] = -1;
                    for (int r = 0; r < nD && outv[q] == -1; ++r) {
                        if (cl[r] != c || rcand[r] < 0) continue;
                        const int4 at = a.attr[rcand[r]];
                        const int v = q == 0 ? at.y : (q == 1 ? at.z : at.w);
                        int gt = 0, ge = 0;
                        for (int u = 0; u < nD; ++u) {
                            if (cl[u] != c || rcand[u] < 0) continue;
                            const int4 bu = a.attr[rcand[u]];
                            const int w = q == 0 ? bu.y : (q == 1 ? bu.z : bu.w);
                            gt += w > v;
                            ge += w >= v;
                        }
                        if (gt <= k && k < ge) outv[q] = v;
                    }
                }
                f.gender = outv[0];
                f.smile = outv[1];
                f.glasses = outv[2];
            }
        }
        a.faces[i] = f;
    }
    if (tid == 0) *a.n_faces = nF;
}

// Detect with the caller's detections in front (cnn_detector_v3.cpp:2753-2806), one warp: the
// priors pass the stable min_num_detect filter (the new clusters arrive filtered), then the
// whole list goes through Merger(0.2, del) and the optional rescale of a shrunken input frame.
__global__ void __launch_bounds__(32, 1) prior_merge_kernel(const Det* prior, int n_prior, const Det* clusters, const int* n_clusters,
                                                            const CascadeConfig C, Det* list, uint8_t* checked, Det* out, int* n_out) {
    const int lane = threadIdx.x;
    const int nc = *n_clusters;
    int n = 0;
    for (int base = 0; base < n_prior; base += 32) {  // stable erase of priors below min_num_detect
        const int k = base + lane;
        const bool keep = k < n_prior && (C.min_num_detect <= 1 || prior[k].num_detect >= C.min_num_detect);
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) list[n + __popc(m & ((1u << lane) - 1u))] = prior[k];
        n += __popc(m);
    }
    for (int k = lane; k < nc; k += 32) list[n + k] = clusters[k];
    n += nc;
    __syncwarp();
    const int nf = n > 0 ? merger_warp(list, n, checked, list + n, 0.2f, true) : 0;
    for (int i = lane; i < nf; i += 32) {
        Det d = list[n + i];
        if (C.rescale_output) {
            d.x = (int)((float)d.x * C.rescale);
            d.y = (int)((float)d.y * C.rescale);
            d.w = (int)((float)d.w * C.rescale);
            d.h = (int)((float)d.h * C.rescale);
        }
        out[i] = d;
    }
    if (lane == 0) *n_out = nf;
}

// CNNDetector::NMS: Merger(detections, rect, 0.5) of the caller's boxes, one warp
__global__ void __launch_bounds__(32, 1) nms_kernel(const Det* in, int n, uint8_t* checked, Det* out, int* n_out) {
    const int nf = merger_warp(in, n, checked, out, 0.5f, false);
    if (threadIdx.x == 0) *n_out = nf;
}

cudaError_t launch_prior_merge(const Det* prior, int n_prior, const Det* clusters, const int* n_clusters, const CascadeConfig& cfg, Det* scratch,
                               uint8_t* checked, Det* out, int* n_out, cudaStream_t st) {
    prior_merge_kernel<<<1, 32, 0, st>>>(prior, n_prior, clusters, n_clusters, cfg, scratch, checked, out, n_out);
    return cudaGetLastError();
}

cudaError_t launch_nms(const Det* in, int n, uint8_t* checked, Det* out, int* n_out, cudaStream_t st) {
    nms_kernel<<<1, 32, 0, st>>>(in, n, checked, out, n_out);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(kRT, 1) replay_kernel(const ReplayArgs a) { replay_body(a); }

// the frames of a batch: block f replays args[f]
__global__ void __launch_bounds__(kRT, 1) replay_batch_kernel(const ReplayArgs* __restrict__ args) {
    __shared__ ReplayArgs s_args;
    if (threadIdx.x == 0) s_args = args[blockIdx.x];
    __syncthreads();
    replay_body(s_args);
}

// The block-wide sort of n (scale, index) keys (device memory) and its permutation, for tests.
__global__ void __launch_bounds__(kRT, 1) sort_check_kernel(ScaleKey* K, int n, int* scratch, int* perm) {
    constexpr int kSegs = (kBitMax * kBitWords) / 3;
    __shared__ int seg_a[3 * kSegs], seg_b[3 * kSegs];
    if (n > 16 && n / 17 <= kSegs) {
        introsort_scale_desc_block(K, n, seg_a, seg_b, kSegs, scratch, scratch + n);
    } else {
        if (threadIdx.x == 0) {
            if (n > 16) introsort_scale_desc(K, n);
            else insertion_sort(K, 0, n);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = K[i].idx;
}

cudaError_t sort_permutation_device(const float* scales, int n, int* perm) {
    std::vector<ScaleKey> k(n);
    for (int i = 0; i < n; ++i) k[i] = ScaleKey{scales[i], i};
    ScaleKey* d_k = nullptr;
    int *d_leaves = nullptr, *d_perm = nullptr;
    cudaError_t e = cudaMalloc(&d_k, sizeof(ScaleKey) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_leaves, sizeof(int) * (2 * n + 2));
    if (e == cudaSuccess) e = cudaMalloc(&d_perm, sizeof(int) * (n + 1));
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(d_k, k.data(), sizeof(ScaleKey) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        sort_check_kernel<<<1, kRT>>>(d_k, n, d_leaves, d_perm);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(perm, d_perm, sizeof(int) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_k);
    cudaFree(d_leaves);
    cudaFree(d_perm);
    return e;
}

cudaError_t replay_setup() {
    cudaError_t e = cudaFuncSetAttribute(replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kReplaySmemBytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(replay_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kReplaySmemBytes);
    return e;
}

cudaError_t launch_replay(const ReplayArgs& a, cudaStream_t st) {
    replay_kernel<<<1, kRT, kReplaySmemBytes, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_replay_batch(const ReplayArgs* d_args, int n_frames, cudaStream_t st) {
    replay_batch_kernel<<<n_frames, kRT, kReplaySmemBytes, st>>>(d_args);
    return cudaGetLastError();
}

}  // namespace ccnn
