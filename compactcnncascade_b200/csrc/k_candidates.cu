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
// writes its hits in order, ranked by warp ballots and per-(round, warp) counts.
#include "kernels.h"

namespace ccnn {

constexpr int kChunkThreads = 256;

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

// the hits of chunk `c` of a frame's scan, written in raster order after those of earlier chunks.
// A chunk the stage-1 kernel counted no hit in writes nothing (only the last chunk, which stores the
// frame's total, still sums the counts). The others load all their responses at once (round k of
// thread t holds element 256 k + t), rank every hit by ballots (one count per (round, warp) in
// shared memory, one barrier) and write it at the chunk's offset plus its rank.
constexpr int kChunkRounds = kCandChunk / kChunkThreads;  // 8
static_assert(kChunkRounds * kChunkThreads == kCandChunk, "a chunk is whole rounds of the block");

__device__ __forceinline__ void cand_write_chunk(const int4* __restrict__ chunks, int n_chunks, const LevelDesc* __restrict__ levels,
                                                 const float* __restrict__ resp, float thr, const int* __restrict__ counts,
                                                 Candidate* __restrict__ out, int* __restrict__ n_out, int cap, int c) {
    __shared__ int wt[32];
    __shared__ int rw[kChunkRounds * (kChunkThreads / 32)];
    const int hits = counts[c];  // uniform over the block
    const bool last = c == n_chunks - 1;
    if (hits == 0 && !last) return;
    // offset of this chunk = sum of the counts of the chunks visited before it
    int part = 0;
    for (int i = threadIdx.x; i < c; i += blockDim.x) part += counts[i];
    const int off = block_sum(part, wt);
    if (last && threadIdx.x == 0) *n_out = min(off + hits, cap);
    if (hits == 0) return;

    const int4 ck = chunks[c];
    const LevelDesc& L = levels[ck.x];
    const float* src = resp + L.resp_off + ck.y;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float r[kChunkRounds];
#pragma unroll
    for (int k = 0; k < kChunkRounds; ++k) {
        const int i = k * kChunkThreads + threadIdx.x;
        r[k] = i < ck.z ? src[i] : thr;  // thr itself is never a hit
    }
    unsigned m[kChunkRounds];
#pragma unroll
    for (int k = 0; k < kChunkRounds; ++k) {
        m[k] = __ballot_sync(0xffffffffu, r[k] > thr);
        if (lane == 0) rw[k * (kChunkThreads / 32) + wid] = __popc(m[k]);
    }
    __syncthreads();
    const int ow = L.ow;
#pragma unroll
    for (int k = 0; k < kChunkRounds; ++k) {
        if (!(r[k] > thr)) continue;
        int pos = off + __popc(m[k] & ((1u << lane) - 1u));
        for (int q = 0; q < k * (kChunkThreads / 32) + wid; ++q) pos += rw[q];
        if (pos < cap) {
            const int e = ck.y + k * kChunkThreads + threadIdx.x;
            const int j = e / ow, ii = e - j * ow;
            Candidate cd;
            cd.level = ck.x;
            cd.px = ii * 4;
            cd.py = j * 4;
            cd.score = r[k];
            out[pos] = cd;
        }
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
