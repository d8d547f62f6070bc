// Measured ceiling of the fp32 pipe for the instructions the exact stage-1 and stage-2/3 kernels
// issue: packed add.rn.f32x2 and the packed product fma.rn.f32x2 with a run-time (-0, -0) addend.
// Every thread runs eight independent chains (no dependency stalls at 256 threads a block and
// several blocks a SM), alternating the two instructions; the grid fills every SM several times.
// One packed instruction is two IEEE lane operations per thread, the unit the kernels' work is
// counted in, so the result is directly the denominator of their fp32 roofline.
#include "kernels.h"

#include <vector>

#include "../../include/ccnn_inspect.h"

namespace ccnn {

void set_error(const std::string& msg);

namespace {

constexpr int kPeakThreads = 256, kPeakChains = 8, kPeakUnroll = 16;

__global__ void __launch_bounds__(kPeakThreads) fp32_peak_kernel(const float2* __restrict__ seed, float2* __restrict__ sink, int iters) {
    const f2_t nz = f2_ld(seed[0]);  // (-0, -0): unknown to the compiler
    const f2_t k = f2_ld(seed[1]);   // (1, 1)
    f2_t a[kPeakChains];
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) a[c] = f2_pack((float)(threadIdx.x + c), (float)(blockIdx.x + c));
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kPeakUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kPeakChains; ++c) a[c] = (u & 1) ? f2_add(a[c], k) : f2_mul(a[c], k, nz);
        }
    }
    f2_t acc = a[0];
#pragma unroll
    for (int c = 1; c < kPeakChains; ++c) acc = f2_add(acc, a[c]);
    if (f2_lo(acc) == -1.f) sink[blockIdx.x * blockDim.x + threadIdx.x] = make_float2(f2_lo(acc), f2_hi(acc));  // never true
}

}  // namespace
}  // namespace ccnn

extern "C" CCNN_API ccnn_status ccnn_measure_fp32_peak(int iters, int reps, double* lane_ops_per_s, float* best_ms) {
    using namespace ccnn;
    if (!lane_ops_per_s || iters <= 0 || reps <= 0) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp32_peak_kernel, kPeakThreads, 0);
    float2* buf = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&buf, sizeof(float2) * (2 + (size_t)sms * per_sm * 4 * kPeakThreads));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    float best = 1e30f;
    const int blocks = sms * per_sm * 4;  // four full waves
    if (e == cudaSuccess) {
        const float2 seed[2] = {make_float2(-0.f, -0.f), make_float2(1.f, 1.f)};
        e = cudaMemcpy(buf, seed, sizeof(seed), cudaMemcpyHostToDevice);
    }
    for (int r = 0; r <= reps && e == cudaSuccess; ++r) {  // the first launch is a warm-up
        cudaEventRecord(t0, 0);
        fp32_peak_kernel<<<blocks, kPeakThreads>>>(buf, buf + 2, iters);
        cudaEventRecord(t1, 0);
        e = cudaEventSynchronize(t1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (e == cudaSuccess && r > 0 && ms < best) best = ms;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (buf) cudaFree(buf);
    if (e != cudaSuccess) {
        set_error(std::string("fp32 peak measurement: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    const double lane_ops = (double)blocks * kPeakThreads * (double)iters * kPeakUnroll * kPeakChains * 2.0;
    *lane_ops_per_s = lane_ops / (best * 1e-3);
    if (best_ms) *best_ms = best;
    return CCNN_OK;
}
