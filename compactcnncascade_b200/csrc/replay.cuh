// Box geometry, the reference's sort order and its box clustering, usable on host and device.
//
// Rect semantics follow src/CNNObjectDetector/type.h:239-328 (Rect, overlap, intersects,
// operator*). The sort reproduces the permutation of the reference's
//   std::sort(v.begin(), v.end(), [](Detection& a, Detection& b){ return b.scale < a.scale; })
// (cnn_detector_v3.cpp:2750). std::sort is not stable, so equal-scale detections come out in
// the order of libstdc++'s introsort (GCC 13): depth limit 2*floor(log2 n), 16-element
// threshold, median-of-three pivot moved to the front, unguarded Hoare partition, heapsort
// fallback, final (unguarded) insertion sort. The same steps are written out here so the GPU
// yields the identical order; tests compare the permutation with std::sort on the host.
#pragma once

#include "ccnn_common.cuh"

#if defined(__CUDACC__)
#define CCNN_HD __host__ __device__ __forceinline__
#else
#define CCNN_HD inline
#endif

namespace ccnn {

CCNN_HD Det make_det(int x, int y, int w, int h, float score, float scale, int knn) {
    Det d;
    d.x = x;
    d.y = y;
    d.w = w;
    d.h = h;
    d.x2 = x + w;
    d.y2 = y + h;
    d.score = score;
    d.scale = scale;
    d.knn = knn;
    d.num_detect = 0;
    return d;
}

CCNN_HD int imin(int a, int b) { return a > b ? b : a; }
CCNN_HD int imax(int a, int b) { return a < b ? b : a; }

// Rect::overlap (type.h:284-305): intersection over the bounding-box "union"
CCNN_HD float rect_overlap(const Det& a, const Det& b) {
    if (a.x > b.x2 || b.x > a.x2 || a.y > b.y2 || b.y > a.y2) return 0.f;
    const int X0 = imin(a.x, b.x), X1 = imax(a.x, b.x), X2 = imin(a.x2, b.x2), X3 = imax(a.x2, b.x2);
    const int Y0 = imin(a.y, b.y), Y1 = imax(a.y, b.y), Y2 = imin(a.y2, b.y2), Y3 = imax(a.y2, b.y2);
    const float su = (float)((X3 - X0) * (Y3 - Y0));
    const float si = (float)((X2 - X1) * (Y2 - Y1));
    return si / su;
}

// Rect::intersects (type.h:269-283)
CCNN_HD int rect_intersects(const Det& a, const Det& b) {
    if (a.x > b.x2 || b.x > a.x2 || a.y > b.y2 || b.y > a.y2) return 0;
    const int X1 = imax(a.x, b.x), X2 = imin(a.x2, b.x2);
    const int Y1 = imax(a.y, b.y), Y2 = imin(a.y2, b.y2);
    return (X2 - X1) * (Y2 - Y1);
}

// Rect::operator*(0.7f) (type.h:320-327)
CCNN_HD Det rect_shrink(const Det& r, float s) {
    s = 1.f - s;
    const int sx = (int)((float)r.w * s);
    const int sy = (int)((float)r.h * s);
    return make_det(r.x + (sx >> 1), r.y + (sy >> 1), r.w - sx, r.h - sy, 0.f, 0.f, 0);
}

// DropDetection's test of one earlier detection (cnn_detector_v3.cpp:1820-1840):
// 0 = not decisive, 1 = overlap > 0.5 (a copy is appended, candidate dropped), 2 = dropped
CCNN_HD int drop_test(const Det& nr, const Det& exp_r, const Det& e) {
    const float ov = rect_overlap(nr, e);
    if (ov == 0.f) return 0;
    if (ov > 0.5f) return 1;
    if (rect_intersects(e, exp_r) == exp_r.w * exp_r.h) return 2;
    return 0;
}

// ---- libstdc++ introsort order for comp(a, b) = b.scale < a.scale ----
// The steps only compare .scale and move whole elements, so they run on any element type with a
// .scale member: sorting (scale, index) pairs gives the permutation that sorting the detections
// themselves would apply.

struct ScaleKey {
    float scale;
    int idx;
};

template <class T>
CCNN_HD bool comp_scale_desc(const T& a, const T& b) { return b.scale < a.scale; }

template <class T>
CCNN_HD void swap_el(T* a, T* b) {
    T t = *a;
    *a = *b;
    *b = t;
}

template <class T>
CCNN_HD void push_heap_el(T* first, int hole, int top, T value) {
    int parent = (hole - 1) / 2;
    while (hole > top && comp_scale_desc(first[parent], value)) {
        first[hole] = first[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    first[hole] = value;
}

template <class T>
CCNN_HD void adjust_heap_el(T* first, int hole, int len, T value) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (comp_scale_desc(first[child], first[child - 1])) child--;
        first[hole] = first[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        first[hole] = first[child - 1];
        hole = child - 1;
    }
    push_heap_el(first, hole, top, value);
}

template <class T>
CCNN_HD void heap_sort_el(T* first, int len) {
    if (len >= 2) {  // make_heap
        int parent = (len - 2) / 2;
        while (true) {
            T v = first[parent];
            adjust_heap_el(first, parent, len, v);
            if (parent == 0) break;
            parent--;
        }
    }
    // (heap_select over an empty tail is a no-op) sort_heap:
    int last = len;
    while (last > 1) {
        --last;
        T v = first[last];
        first[last] = first[0];
        adjust_heap_el(first, 0, last, v);
    }
}

template <class T>
CCNN_HD void median_to_first(T* result, T* a, T* b, T* c) {
    if (comp_scale_desc(*a, *b)) {
        if (comp_scale_desc(*b, *c)) swap_el(result, b);
        else if (comp_scale_desc(*a, *c)) swap_el(result, c);
        else swap_el(result, a);
    } else if (comp_scale_desc(*a, *c)) swap_el(result, a);
    else if (comp_scale_desc(*b, *c)) swap_el(result, c);
    else swap_el(result, b);
}

template <class T>
CCNN_HD int unguarded_partition(T* v, int first, int last, int pivot) {
    while (true) {
        while (comp_scale_desc(v[first], v[pivot])) ++first;
        --last;
        while (comp_scale_desc(v[pivot], v[last])) --last;
        if (!(first < last)) return first;
        swap_el(&v[first], &v[last]);
        ++first;
    }
}

template <class T>
CCNN_HD void unguarded_linear_insert(T* v, int last) {
    T val = v[last];
    int next = last - 1;
    while (comp_scale_desc(val, v[next])) {
        v[last] = v[next];
        last = next;
        --next;
    }
    v[last] = val;
}

template <class T>
CCNN_HD void insertion_sort(T* v, int first, int last) {
    if (first == last) return;
    for (int i = first + 1; i != last; ++i) {
        if (comp_scale_desc(v[i], v[first])) {
            T val = v[i];
            for (int k = i; k > first; --k) v[k] = v[k - 1];
            v[first] = val;
        } else {
            unguarded_linear_insert(v, i);
        }
    }
}

CCNN_HD int floor_log2(int n) {
    int r = 0;
    while (n > 1) {
        n >>= 1;
        ++r;
    }
    return r;
}

// iterative form of the introsort loop: the recursion is on the right part, the loop on the left
template <class T>
CCNN_HD void introsort_scale_desc(T* v, int n) {
    if (n <= 1) return;
    const int kThreshold = 16;
    // explicit stack of (first, last, depth) for the recursive calls
    int st_first[64], st_last[64], st_depth[64];
    int sp = 0;
    st_first[sp] = 0;
    st_last[sp] = n;
    st_depth[sp] = 2 * floor_log2(n);
    sp++;
    while (sp > 0) {
        sp--;
        int first = st_first[sp], last = st_last[sp], depth = st_depth[sp];
        while (last - first > kThreshold) {
            if (depth == 0) {
                heap_sort_el(v + first, last - first);
                break;
            }
            --depth;
            const int mid = first + (last - first) / 2;
            median_to_first(&v[first], &v[first + 1], &v[mid], &v[last - 1]);
            const int cut = unguarded_partition(v, first + 1, last, first);
            // the reference recurses into [cut, last) before continuing with [first, cut);
            // both halves are disjoint, so finishing the left first gives the same result
            st_first[sp] = cut;
            st_last[sp] = last;
            st_depth[sp] = depth;
            sp++;
            last = cut;
        }
    }
    if (n > kThreshold) {
        insertion_sort(v, 0, kThreshold);
        for (int i = kThreshold; i < n; ++i) unguarded_linear_insert(v, i);
    } else {
        insertion_sort(v, 0, n);
    }
}

#if defined(__CUDACC__)
// unguarded_partition(v, piv + 1, hi, piv) by one warp. The left pointer stops at the elements that
// do not compare before the pivot, the right one at those the pivot does not compare before; a
// pointer only ever examines positions the other has not swapped yet, except at the crossing. So with
// L_k / R_k the k-th stop of each pointer on the values as they are now (left ascending from piv + 1,
// right descending from hi - 1), the partition swaps (L_k, R_k) for every k before the first k* with
// L_k* >= R_k* (or no stop left), and returns the left pointer's last stop: L_k*, or R_(k*-1) where
// the left pointer runs into the swapped region first. lbuf / rbuf: scratch of hi - piv ints each.
template <class T>
__device__ int warp_partition(T* v, int piv, int hi, int* lbuf, int* rbuf) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const T p = v[piv];
    int nL = 0, nR = 0;
    for (int base = piv + 1; base < hi; base += 32) {
        const int i = base + lane;
        const bool f = i < hi && !comp_scale_desc(v[i], p);
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (f) lbuf[nL + __popc(m & lt)] = i;
        nL += __popc(m);
    }
    for (int base = hi - 1; base >= piv; base -= 32) {
        const int j = base - lane;
        const bool g = j >= piv && !comp_scale_desc(p, v[j]);
        const unsigned m = __ballot_sync(0xffffffffu, g);
        if (g) rbuf[nR + __popc(m & lt)] = j;
        nR += __popc(m);
    }
    __syncwarp();
    int ks = 0;
    for (int kb = 0;; kb += 32) {
        const int k = kb + lane;
        const bool stop = k >= nL || k >= nR || lbuf[k] >= rbuf[k];
        const unsigned m = __ballot_sync(0xffffffffu, stop);
        if (m) {
            ks = kb + __ffs(m) - 1;
            break;
        }
    }
    // the swapped pairs are disjoint: L_j < R_j for j < k*, both lists strictly monotone
    for (int k = lane; k < ks; k += 32) swap_el(&v[lbuf[k]], &v[rbuf[k]]);
    int cut = ks < nL ? lbuf[ks] : hi;
    if (ks > 0 && rbuf[ks - 1] < cut) cut = rbuf[ks - 1];
    __syncwarp();
    return cut;
}

// insertion_sort(v, lo, hi) by one warp (hi - lo <= 32): the insertion sort never moves an element
// past an equal one, so it is the stable sort, and every element's place is its rank.
template <class T>
__device__ void warp_stable_sort(T* v, int lo, int hi) {
    const int lane = threadIdx.x & 31;
    const int len = hi - lo;
    T val;
    int r = 0;
    if (lane < len) {
        val = v[lo + lane];
        for (int q = 0; q < len; ++q) {
            const T o = v[lo + q];
            if (comp_scale_desc(o, val) || (q < lane && !comp_scale_desc(val, o))) ++r;
        }
    }
    __syncwarp();
    if (lane < len) v[lo + r] = val;
    __syncwarp();
}

// The same introsort by the whole block. The partitions of one recursion depth touch disjoint
// segments, so each round partitions every segment longer than the threshold at once (a warp a
// segment, the partition itself parallel as above; the heapsort fallback by one lane). The final
// insertion sort of the reference never moves an element across a partition cut (everything before a
// cut has a scale >= the pivot >= everything after it, and the insertion stops at the first element
// that is not smaller), so it is the same as an insertion sort of each leaf segment, which the warp
// that splits a leaf off runs at once. seg_a / seg_b: 3 * max_segs ints each (shared memory);
// lbuf / rbuf: n ints each of scratch (any memory); n must be > 16 and n / 17 <= max_segs. Every
// thread of the block calls it.
template <class T>
__device__ void introsort_scale_desc_block(T* v, int n, int* seg_a, int* seg_b, int max_segs, int* lbuf, int* rbuf) {
    const int kThreshold = 16;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    __shared__ int s_cur, s_next;
    if (threadIdx.x == 0) {
        seg_a[0] = 0;
        seg_a[1] = n;
        seg_a[2] = 2 * floor_log2(n);
        s_cur = 1;
    }
    __syncthreads();
    int* cur = seg_a;
    int* nxt = seg_b;
    for (;;) {
        const int ncur = s_cur;
        if (ncur == 0) break;
        __syncthreads();
        if (threadIdx.x == 0) s_next = 0;
        __syncthreads();
        for (int k = warp; k < ncur; k += nwarps) {
            const int first = cur[3 * k], last = cur[3 * k + 1];
            int depth = cur[3 * k + 2];
            if (depth == 0) {
                if (lane == 0) heap_sort_el(v + first, last - first);
                __syncwarp();
                continue;
            }
            --depth;
            const int mid = first + (last - first) / 2;
            if (lane == 0) median_to_first(&v[first], &v[first + 1], &v[mid], &v[last - 1]);
            __syncwarp();
            const int cut = warp_partition(v, first, last, lbuf + first, rbuf + first);
            const int lo[2] = {first, cut}, hi[2] = {cut, last};
            for (int c = 0; c < 2; ++c) {
                const int len = hi[c] - lo[c];
                if (len > kThreshold) {
                    if (lane == 0) {
                        const int slot = atomicAdd(&s_next, 1);
                        if (slot < max_segs) {
                            nxt[3 * slot] = lo[c];
                            nxt[3 * slot + 1] = hi[c];
                            nxt[3 * slot + 2] = depth;
                        }
                    }
                } else if (len > 1) {
                    warp_stable_sort(v, lo[c], hi[c]);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_cur = s_next < max_segs ? s_next : max_segs;
        int* t = cur;
        cur = nxt;
        nxt = t;
        __syncthreads();
    }
}
#endif

}  // namespace ccnn
