// Gray conversion and resampling kernels.
//
// gray_kernel: 8-bit gray / BGR / BGRA -> fp32 gray, bit-exact with
//   ImageConverter::Img8uToImg32fGRAY (src/CNNObjectDetector/image_proc.cpp:299-317), whose
//   plain path computes 0.114f*B + 0.587f*G + 0.299f*R left to right (:195-201, :287-293) and
//   float(v) for one channel (:99-102).
// Each thread converts 16 consecutive pixels of one row with 128-bit loads (1, 3 or 4 x uint4)
// and 128-bit stores; the staging buffer's row pitch is a multiple of 64 bytes so every
// vector access is aligned. Rows whose width is not a multiple of 16 finish with scalar code.
#include "kernels.h"
#include "pyramid.cuh"
#include "resample.cuh"

namespace ccnn {

__device__ __forceinline__ float gray_bgr(uint32_t b, uint32_t g, uint32_t r) {
    return fadd(fadd(fmul(0.114f, (float)b), fmul(0.587f, (float)g)), fmul(0.299f, (float)r));
}

// 16 pixels of a row (item = row x 16-pixel chunk), 128-bit loads and stores
template <int CH>
__device__ __forceinline__ void gray_chunk(const uint8_t* __restrict__ src, int spitch, int w, int h, float* __restrict__ dst, int dpitch,
                                           int item) {
    const int chunks = (w + 15) >> 4;  // 16-pixel chunks per row; one chunk per thread
    const int y = item / chunks;
    const int x0 = (item - y * chunks) * 16;
    if (y >= h) return;
    const uint8_t* row = src + (size_t)y * spitch;
    float* out = dst + (size_t)y * dpitch;
    if (x0 + 16 <= w) {
        uint8_t px[16 * CH];
        const uint4* vsrc = reinterpret_cast<const uint4*>(row + (size_t)x0 * CH);
#pragma unroll
        for (int v = 0; v < CH; ++v) *reinterpret_cast<uint4*>(px + 16 * v) = __ldg(vsrc + v);
        float g[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            if (CH == 1)
                g[i] = (float)px[i];
            else
                g[i] = gray_bgr(px[i * CH + 0], px[i * CH + 1], px[i * CH + 2]);
        }
        float4* vdst = reinterpret_cast<float4*>(out + x0);
#pragma unroll
        for (int v = 0; v < 4; ++v) vdst[v] = make_float4(g[4 * v], g[4 * v + 1], g[4 * v + 2], g[4 * v + 3]);
    } else {
        for (int x = x0; x < w; ++x) {
            const uint8_t* p = row + (size_t)x * CH;
            out[x] = (CH == 1) ? (float)p[0] : gray_bgr(p[0], p[1], p[2]);
        }
    }
}

template <int CH>
__global__ void __launch_bounds__(256) gray_kernel(const uint8_t* __restrict__ src, int spitch, int w, int h,
                                                   float* __restrict__ dst, int dpitch) {
    gray_chunk<CH>(src, spitch, w, h, dst, dpitch, blockIdx.x * blockDim.x + threadIdx.x);
}

// the frames of a batch: blockIdx.y is the frame; sources (64-byte aligned base and pitch) from a
// device table the host fills before every launch
template <int CH>
__global__ void __launch_bounds__(256) gray_batch_kernel(const FrameSrc* __restrict__ src, int w, int h, const __grid_constant__ BatchFrames F,
                                                         int dpitch) {
    const FrameSrc fs = src[blockIdx.y];
    gray_chunk<CH>(fs.data, fs.pitch, w, h, const_cast<float*>(F.gray[blockIdx.y]), dpitch, blockIdx.x * blockDim.x + threadIdx.x);
}

cudaError_t launch_gray_batch(const FrameSrc* d_src, int n_frames, int w, int h, int ch, const BatchFrames& F, int dpitch, cudaStream_t st) {
    const long long items = (long long)h * ((w + 15) / 16);
    dim3 grid((unsigned)((items + 255) / 256), (unsigned)n_frames);
    switch (ch) {
        case 1: gray_batch_kernel<1><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 3: gray_batch_kernel<3><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 4: gray_batch_kernel<4><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

const void* gray_kernel_fn(int ch) {
    switch (ch) {
        case 1: return reinterpret_cast<const void*>(gray_kernel<1>);
        case 3: return reinterpret_cast<const void*>(gray_kernel<3>);
        case 4: return reinterpret_cast<const void*>(gray_kernel<4>);
    }
    return nullptr;
}

cudaError_t launch_gray(const uint8_t* src, int spitch, int w, int h, int ch, float* dst, int dpitch, cudaStream_t st) {
    if ((spitch & 63) || (dpitch & 15) || (reinterpret_cast<uintptr_t>(src) & 63) || (reinterpret_cast<uintptr_t>(dst) & 63))
        return cudaErrorMisalignedAddress;  // the staging buffers are allocated 64-byte aligned
    dim3 block(256);
    const long long items = (long long)h * ((w + 15) / 16);
    dim3 grid((unsigned)((items + 255) / 256));
    switch (ch) {
        case 1: gray_kernel<1><<<grid, block, 0, st>>>(src, spitch, w, h, dst, dpitch); break;
        case 3: gray_kernel<3><<<grid, block, 0, st>>>(src, spitch, w, h, dst, dpitch); break;
        case 4: gray_kernel<4><<<grid, block, 0, st>>>(src, spitch, w, h, dst, dpitch); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// 1-channel frames when the smallest face is larger than the window: the reference first
// shrinks the 8-bit frame bilinearly (cnn_detector_v3.cpp:2531-2538 with InitScales :299-307),
// then converts it (float(v)). Both steps are fused here.
__global__ void __launch_bounds__(256) gray_from_u8_resized(const uint8_t* __restrict__ src, int spitch, int sw, int sh,
                                                            float* __restrict__ dst, int dpitch, int dw, int dh, uint32_t sclx,
                                                            uint32_t scly, int copy) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    float v;
    if (copy) {
        v = (float)src[(size_t)y * spitch + x];
    } else {
        AxisSample sx = sample_col(x, sclx, sw);
        AxisSample sy = sample_row(y, scly, sh);
        v = (float)bilinear_u8(src, spitch, sh, sx, sy);
    }
    dst[(size_t)y * dpitch + x] = v;
}

cudaError_t launch_gray_u8_resized(const uint8_t* src, int spitch, int sw, int sh, float* dst, int dpitch, int dw, int dh,
                                   cudaStream_t st) {
    int copy = (sw == dw && sh == dh);
    dim3 grid((dw + 255) / 256, dh);
    gray_from_u8_resized<<<grid, 256, 0, st>>>(src, spitch, sw, sh, dst, dpitch, dw, dh, fp_step(sw, dw), fp_step(sh, dh), copy);
    return cudaGetLastError();
}

// Pyramid: every processed level image of a frame in one launch (RunCPUDetect,
// cnn_detector_v3.cpp:2090-2104: scale 1 copies the gray image, scale > 0.7 nearest neighbour,
// else bilinear; ImageResizer::FastImageResize, image_resize.cpp:564-584). A block covers 256
// consecutive columns x kPyrRows rows of one level: each thread keeps its column's resampling
// weights for all its rows, and a warp's loads and stores walk consecutive columns. Columns between
// the level width and the row pitch are written as zeros.
__global__ void __launch_bounds__(kPyrCols) pyramid_kernel(const __grid_constant__ LevelTable LT, const float* __restrict__ gray,
                                                           int gpitch, int gw, int gh, float* __restrict__ limg,
                                                           const uint8_t* __restrict__ front_on) {
    const int g = LT.first + blockIdx.x;
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::pyr_base>(LT, g)];
    pyramid_block(L, g - L.pyr_base, gray, gpitch, gw, gh, limg, front_on);
}

cudaError_t launch_pyramid(const LevelDesc* levels, int n_levels, const float* gray, int gpitch, int gw, int gh, float* limg,
                           cudaStream_t st, const uint8_t* front_on) {
    for (int g0 = 0; g0 < n_levels; g0 += kParamLevels) {
        LevelTable T;
        T.n = n_levels - g0 < kParamLevels ? n_levels - g0 : kParamLevels;
        for (int i = 0; i < T.n; ++i) T.lv[i] = levels[g0 + i];
        T.first = T.lv[0].pyr_base;
        const LevelDesc& last = T.lv[T.n - 1];
        const int blocks = last.pyr_base + last.pyr_wq * ((last.h + kPyrRows - 1) / kPyrRows) - T.first;
        if (blocks > 0) pyramid_kernel<<<blocks, kPyrCols, 0, st>>>(T, gray, gpitch, gw, gh, limg, front_on);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Standalone float resize (ImageResizer::FastImageResize(Image_32f&...), image_resize.cpp:564-584).
__global__ void __launch_bounds__(256) resize_f32_kernel(const float* __restrict__ src, int spitch, int sw, int sh,
                                                         float* __restrict__ dst, int dpitch, int dw, int dh, int mode) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    LevelDesc L;
    L.mode = (sw == dw && sh == dh) ? 0 : mode;
    L.sclx = fp_step(sw, dw);
    L.scly = fp_step(sh, dh);
    dst[(size_t)y * dpitch + x] = level_pixel(src, spitch, sw, sh, L, x, y);
}

cudaError_t launch_resize_f32(const float* src, int spitch, int sw, int sh, float* dst, int dpitch, int dw, int dh, int type,
                              cudaStream_t st) {
    dim3 grid((dw + 255) / 256, dh);
    resize_f32_kernel<<<grid, 256, 0, st>>>(src, spitch, sw, sh, dst, dpitch, dw, dh, type == 0 ? 1 : 2);
    return cudaGetLastError();
}

}  // namespace ccnn
