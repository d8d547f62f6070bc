// Stage-1 candidate compaction.
//
// Reference: the raster scan of each response map in RunCheckDetect
// (src/CNNObjectDetector/cnn_detector_v3.cpp:1918-1945): a response r > treshold_1 at (i, j)
// becomes the point (4i, 4j); levels are visited from the smallest (scl = n-1) to the largest
// (RunCheckDetectAsync :2041-2049). The output list keeps exactly that order.
//
// The scan space is cut into chunks that never straddle two levels (host-built chunk table,
// chunks in visiting order). The stage-1 back kernel counts each chunk's hits as it writes the
// responses; this kernel gives each chunk its offset (sum of the counts of earlier chunks) and
// writes its hits in order using a ballot/popc prefix inside each warp and a warp-total scan
// across the block.
#include "kernels.h"

namespace ccnn {

constexpr int kChunkThreads = 256;

// Exclusive prefix of a 0/1 predicate across the block: warp ballot + popc inside a warp,
// then a shuffle scan over the (<= 32) warp totals. Returns the rank; *total gets the count.
__device__ __forceinline__ int block_pred_rank(int pred, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    const int rank = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[wid] = __popc(m);
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) warp_tot[lane] = t;  // inclusive
        if (lane == nw - 1) *total = t;
    }
    __syncthreads();
    const int r = (wid ? warp_tot[wid - 1] : 0) + rank;
    __syncthreads();
    return r;
}

__device__ __forceinline__ int block_sum(int v, int* warp_tot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) warp_tot[wid] = v;
    __syncthreads();
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += warp_tot[w];
    __syncthreads();
    return t;
}

// the hits of chunk `c` of a frame's scan, written in raster order after those of earlier chunks
__device__ __forceinline__ void cand_write_chunk(const int4* __restrict__ chunks, int n_chunks, const LevelDesc* __restrict__ levels,
                                                 const float* __restrict__ resp, float thr, const int* __restrict__ counts,
                                                 Candidate* __restrict__ out, int* __restrict__ n_out, int cap, int c) {
    __shared__ int wt[32];
    __shared__ int tot;
    // offset of this chunk = sum of the counts of the chunks visited before it
    int part = 0;
    for (int i = threadIdx.x; i < c; i += blockDim.x) part += counts[i];
    int off = block_sum(part, wt);
    if (c == n_chunks - 1 && threadIdx.x == 0) *n_out = min(off + counts[c], cap);

    const int4 ck = chunks[c];
    const LevelDesc L = levels[ck.x];
    for (int b0 = 0; b0 < ck.z; b0 += blockDim.x) {
        const int i = b0 + threadIdx.x;
        float r = 0.f;
        int hit = 0;
        if (i < ck.z) {
            r = resp[L.resp_off + ck.y + i];
            hit = r > thr ? 1 : 0;
        }
        const int pos = block_pred_rank(hit, wt, &tot);
        if (hit && off + pos < cap) {
            const int e = ck.y + i;
            const int j = e / L.ow, ii = e - j * L.ow;
            Candidate c;
            c.level = ck.x;
            c.px = ii * 4;
            c.py = j * 4;
            c.score = r;
            out[off + pos] = c;
        }
        off += tot;
    }
}

__global__ void __launch_bounds__(kChunkThreads) cand_write_kernel(const int4* __restrict__ chunks, int n_chunks,
                                                                   const LevelDesc* __restrict__ levels, const float* __restrict__ resp,
                                                                   float thr, const int* __restrict__ counts, Candidate* __restrict__ out,
                                                                   int* __restrict__ n_out, int cap) {
    cand_write_chunk(chunks, n_chunks, levels, resp, thr, counts, out, n_out, cap, blockIdx.x);
}

// the frames of a batch: blockIdx.y is the frame
__global__ void __launch_bounds__(kChunkThreads) cand_write_batch_kernel(const int4* __restrict__ chunks, int n_chunks,
                                                                         const LevelDesc* __restrict__ levels,
                                                                         const __grid_constant__ BatchFrames F,
                                                                         const __grid_constant__ BatchCands C, float thr, int cap) {
    const int f = blockIdx.y;
    cand_write_chunk(chunks, n_chunks, levels, F.resp[f], thr, F.counts[f], C.cands[f], C.ncand[f], cap, blockIdx.x);
}

cudaError_t launch_cand_write_batch(const int4* d_chunks, int n_chunks, const LevelDesc* d_levels, const BatchFrames& F, const BatchCands& C,
                                    int n_frames, float thr, int cap, cudaStream_t st) {
    if (n_chunks <= 0) {
        for (int f = 0; f < n_frames; ++f) {
            const cudaError_t e = cudaMemsetAsync(C.ncand[f], 0, sizeof(int), st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    cand_write_batch_kernel<<<dim3(n_chunks, n_frames), kChunkThreads, 0, st>>>(d_chunks, n_chunks, d_levels, F, C, thr, cap);
    return cudaGetLastError();
}

cudaError_t launch_cand_write(const int4* d_chunks, int n_chunks, const LevelDesc* d_levels, const float* resp, float thr,
                              const int* counts, Candidate* out, int* n_out, int cap, cudaStream_t st) {
    if (n_chunks <= 0) return cudaMemsetAsync(n_out, 0, sizeof(int), st);
    cand_write_kernel<<<n_chunks, kChunkThreads, 0, st>>>(d_chunks, n_chunks, d_levels, resp, thr, counts, out, n_out, cap);
    return cudaGetLastError();
}

}  // namespace ccnn
