// Device renderer of the seeded synthetic frames: the same bytes as the host generator
// (synth_frame.c) for every seed and size. The host half (ccnn_synth_plan) draws the background
// phases, the face patches and the noise stream's start; one thread per pixel then evaluates the
// background from the phase tables, blends every face whose box holds the pixel in drawing order,
// jumps the PCG32 stream to the pixel's two draws and quantises. Built without contraction
// (-fmad=false) so the double arithmetic rounds exactly as the host's.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/ccnn_inspect.h"
// the host half (ccnn_synth_plan), compiled into this library as well
#include "synth_frame.c"

namespace ccnn {
void set_error(const std::string& msg);
}

namespace {

constexpr int kGeomChunk = 64;

__global__ void __launch_bounds__(256) synth_render_kernel(const double* __restrict__ tab, const ccnn_synth_geom* __restrict__ geom, int n_faces,
                                                           int width, int height, int channels, size_t step, int4 jit, uint64_t ns_state,
                                                           uint64_t ns_inc, uint8_t* __restrict__ out) {
    __shared__ ccnn_synth_geom sg[kGeomChunk];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const bool live = x < width;
    float lum = 0.f;
    if (live) {
        const double* ca = tab;
        const double* sa = ca + 4 * (size_t)width;
        const double* cb = sa + 4 * (size_t)width;
        const double* sb = cb + 4 * (size_t)height;
        double bg = 128.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) bg += 15.0 * (ca[k * width + x] * cb[k * height + y] - sa[k * width + x] * sb[k * height + y]);
        lum = (float)bg;
    }
    const int bx0 = blockIdx.x * blockDim.x, bx1 = min(bx0 + (int)blockDim.x, width) - 1;
    for (int c0 = 0; c0 < n_faces; c0 += kGeomChunk) {
        const int nc = min(kGeomChunk, n_faces - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < nc; i += blockDim.x) sg[i] = geom[c0 + i];
        __syncthreads();
        for (int i = 0; i < nc; ++i) {
            const ccnn_synth_geom& g = sg[i];
            if (y < g.y0 || y > g.y1 || bx1 < g.x0 || bx0 > g.x1) continue;  // block-uniform
            if (live && x >= g.x0 && x <= g.x1) lum = synth_draw_face(&g, x, y, lum);
        }
    }
    if (!live) return;
    pcg32_t r;
    r.state = ns_state;
    r.inc = ns_inc;
    r = pcg32_advanced(r, 2ull * ((uint64_t)y * (uint64_t)width + (uint64_t)x));
    const uint32_t r0 = pcg32_next(&r), r1 = pcg32_next(&r);
    const int jitter[4] = {jit.x, jit.y, jit.z, jit.w};
    uint8_t px[4];
    synth_pixel_out(lum, r0, r1, jitter, channels, px);
    uint8_t* o = out + (size_t)y * step + (size_t)x * channels;
    for (int c = 0; c < channels; ++c) o[c] = px[c];
}

}  // namespace

extern "C" CCNN_API ccnn_status ccnn_synth_frame_device(void* d_out, int width, int height, int channels, size_t step, unsigned long long seed,
                                                        int n_faces, int min_face, int max_face, void* faces_out, void* stream) {
    if (!d_out || width <= 0 || height <= 0 || (channels != 1 && channels != 3 && channels != 4) || step < (size_t)width * channels ||
        n_faces < 0 || min_face <= 0 || max_face < min_face) {
        ccnn::set_error("synthetic frame: invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    std::vector<double> tables(8 * ((size_t)width + (size_t)height));
    std::vector<ccnn_synth_geom> geom((size_t)(n_faces > 0 ? n_faces : 1));
    int jitter[4];
    uint64_t ns[2];
    ccnn_synth_plan(width, height, (uint64_t)seed, n_faces, min_face, max_face, tables.data(), geom.data(), jitter, ns,
                    (ccnn_synth_face*)faces_out);
    const cudaStream_t st = (cudaStream_t)stream;
    const size_t tab_bytes = sizeof(double) * tables.size(), geom_bytes = sizeof(ccnn_synth_geom) * geom.size();
    void* buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, tab_bytes + geom_bytes, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf, tables.data(), tab_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((char*)buf + tab_bytes, geom.data(), geom_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        synth_render_kernel<<<dim3((width + 255) / 256, height), 256, 0, st>>>(
            (const double*)buf, (const ccnn_synth_geom*)((char*)buf + tab_bytes), n_faces, width, height, channels, step,
            make_int4(jitter[0], jitter[1], jitter[2], jitter[3]), ns[0], ns[1], (uint8_t*)d_out);
        e = cudaGetLastError();
    }
    if (buf) {
        const cudaError_t f = cudaFreeAsync(buf, st);
        if (e == cudaSuccess) e = f;
    }
    // the host tables are released on return: wait for the copies that read them
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ccnn::set_error(std::string("synthetic frame: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    return CCNN_OK;
}
