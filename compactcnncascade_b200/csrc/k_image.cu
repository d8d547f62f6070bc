// Gray conversion and resampling kernels.
//
// gray_kernel: 8-bit gray / BGR / BGRA -> fp32 gray, bit-exact with
//   ImageConverter::Img8uToImg32fGRAY (src/CNNObjectDetector/image_proc.cpp:299-317), whose
//   plain path computes 0.114f*B + 0.587f*G + 0.299f*R left to right (:195-201, :287-293) and
//   float(v) for one channel (:99-102).
// Each thread converts 16 consecutive pixels of one row with 128-bit loads (1, 3 or 4 x uint4)
// and 128-bit stores; the staging buffer's row pitch is a multiple of 64 bytes so every
// vector access is aligned. Rows whose width is not a multiple of 16 finish with scalar code.
// With the learned gate on, the same launch also writes the gate's 1/8-resolution input features.
#include "kernels.h"
#include "pyramid.cuh"
#include "resample.cuh"

namespace ccnn {

__device__ __forceinline__ float gray_bgr(uint32_t b, uint32_t g, uint32_t r) {
    return fadd(fadd(fmul(0.114f, (float)b), fmul(0.587f, (float)g)), fmul(0.299f, (float)r));
}

// One block converts 8 rows (a warp each) x 32 chunks of 16 pixels (a lane each): 128-bit loads
// and stores, a warp's accesses walking one row. kFeat (the learned gate is on): the block also keeps
// its rows in shared memory and writes the gate's input features of its 8x8 cells, each the sum of
// the cell's 64 gray values in row-major order from 0 (the order the gate's training forward uses,
// gate.cu), (sum / 64 - 128) / 64 in binary16; only cells wholly inside the frame (W/8 x H/8) get one.
constexpr int kGrayRows = 8, kGrayChunks = 32;
constexpr int kCellPitch = 9;  // floats per 8-pixel cell row in shared memory (padded: conflict-free sums)

template <int CH, bool kFeat>
__device__ __forceinline__ void gray_block(const uint8_t* __restrict__ src, int spitch, int w, int h, float* __restrict__ dst, int dpitch,
                                           __half* __restrict__ feat, int bx, int by) {
    __shared__ float keep[kFeat ? kGrayRows : 1][kFeat ? 2 * kGrayChunks * kCellPitch : 1];
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    const int x0 = (bx * kGrayChunks + lane) * 16;
    const int y = by * kGrayRows + r;
    if (y < h && x0 < w) {
        const uint8_t* row = src + (size_t)y * spitch;
        float* out = dst + (size_t)y * dpitch;
        // pixel k of the chunk: cell 2 * lane + k / 8, position k % 8
        auto keep_px = [&](int k, float v) {
            if constexpr (kFeat) keep[r][(2 * lane + (k >> 3)) * kCellPitch + (k & 7)] = v;
        };
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
                keep_px(i, g[i]);
            }
            float4* vdst = reinterpret_cast<float4*>(out + x0);
#pragma unroll
            for (int v = 0; v < 4; ++v) vdst[v] = make_float4(g[4 * v], g[4 * v + 1], g[4 * v + 2], g[4 * v + 3]);
        } else {
            for (int x = x0; x < w; ++x) {
                const uint8_t* p = row + (size_t)x * CH;
                const float v = (CH == 1) ? (float)p[0] : gray_bgr(p[0], p[1], p[2]);
                out[x] = v;
                keep_px(x - x0, v);
            }
        }
    }
    if constexpr (kFeat) {
        __syncthreads();
        const int w8 = w / 8, h8 = h / 8;
        const int cx = bx * 2 * kGrayChunks + threadIdx.x;
        if (threadIdx.x < 2 * kGrayChunks && cx < w8 && by < h8) {
            float sum = 0.f;
#pragma unroll
            for (int rr = 0; rr < kGrayRows; ++rr)
#pragma unroll
                for (int c = 0; c < 8; ++c) sum = fadd(sum, keep[rr][threadIdx.x * kCellPitch + c]);
            feat[(size_t)by * w8 + cx] = __float2half(fmul(fsub(fmul(sum, 1.f / 64.f), 128.f), 1.f / 64.f));
        }
    }
}

template <int CH, bool kFeat>
__global__ void __launch_bounds__(256) gray_kernel(const uint8_t* __restrict__ src, int spitch, int w, int h,
                                                   float* __restrict__ dst, int dpitch, __half* __restrict__ feat) {
    gray_block<CH, kFeat>(src, spitch, w, h, dst, dpitch, feat, blockIdx.x, blockIdx.y);
}

static dim3 gray_grid(int w, int h, int frames = 1) {
    const int chunks = (w + 15) / 16;
    return dim3((unsigned)((chunks + kGrayChunks - 1) / kGrayChunks), (unsigned)((h + kGrayRows - 1) / kGrayRows), (unsigned)frames);
}

// the frames of a batch: blockIdx.z is the frame; sources (64-byte aligned base and pitch) from a
// device table the host fills before every launch
template <int CH, bool kFeat>
__global__ void __launch_bounds__(256) gray_batch_kernel(const FrameSrc* __restrict__ src, int w, int h, const __grid_constant__ BatchFrames F,
                                                         int dpitch) {
    const FrameSrc fs = src[blockIdx.z];
    gray_block<CH, kFeat>(fs.data, fs.pitch, w, h, const_cast<float*>(F.gray[blockIdx.z]), dpitch, F.feat[blockIdx.z], blockIdx.x, blockIdx.y);
}

cudaError_t launch_gray_batch(const FrameSrc* d_src, int n_frames, int w, int h, int ch, const BatchFrames& F, int dpitch, cudaStream_t st) {
    const dim3 grid = gray_grid(w, h, n_frames);
    const bool feat = F.feat[0] != nullptr;
    switch (ch * 2 + (feat ? 1 : 0)) {
        case 2: gray_batch_kernel<1, false><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 3: gray_batch_kernel<1, true><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 6: gray_batch_kernel<3, false><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 7: gray_batch_kernel<3, true><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 8: gray_batch_kernel<4, false><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        case 9: gray_batch_kernel<4, true><<<grid, 256, 0, st>>>(d_src, w, h, F, dpitch); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int CH>
static const void* gray_fn(bool feat) {
    return feat ? reinterpret_cast<const void*>(gray_kernel<CH, true>) : reinterpret_cast<const void*>(gray_kernel<CH, false>);
}

const void* gray_kernel_fn(int ch, bool feat) {
    switch (ch) {
        case 1: return gray_fn<1>(feat);
        case 3: return gray_fn<3>(feat);
        case 4: return gray_fn<4>(feat);
    }
    return nullptr;
}

cudaError_t launch_gray(const uint8_t* src, int spitch, int w, int h, int ch, float* dst, int dpitch, cudaStream_t st, __half* feat) {
    if ((spitch & 63) || (dpitch & 15) || (reinterpret_cast<uintptr_t>(src) & 63) || (reinterpret_cast<uintptr_t>(dst) & 63))
        return cudaErrorMisalignedAddress;  // the staging buffers are allocated 64-byte aligned
    const dim3 grid = gray_grid(w, h);
    switch (ch * 2 + (feat ? 1 : 0)) {
        case 2: gray_kernel<1, false><<<grid, 256, 0, st>>>(src, spitch, w, h, dst, dpitch, feat); break;
        case 3: gray_kernel<1, true><<<grid, 256, 0, st>>>(src, spitch, w, h, dst, dpitch, feat); break;
        case 6: gray_kernel<3, false><<<grid, 256, 0, st>>>(src, spitch, w, h, dst, dpitch, feat); break;
        case 7: gray_kernel<3, true><<<grid, 256, 0, st>>>(src, spitch, w, h, dst, dpitch, feat); break;
        case 8: gray_kernel<4, false><<<grid, 256, 0, st>>>(src, spitch, w, h, dst, dpitch, feat); break;
        case 9: gray_kernel<4, true><<<grid, 256, 0, st>>>(src, spitch, w, h, dst, dpitch, feat); break;
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
                                                           int gpitch, int gw, int gh, float* __restrict__ limg) {
    const int g = LT.first + blockIdx.x;
    const LevelDesc& L = LT.lv[find_level<&LevelDesc::pyr_base>(LT, g)];
    pyramid_block(L, g - L.pyr_base, gray, gpitch, gw, gh, limg);
}

cudaError_t launch_pyramid(const LevelDesc* levels, int n_levels, const float* gray, int gpitch, int gw, int gh, float* limg,
                           cudaStream_t st) {
    for (int g0 = 0; g0 < n_levels; g0 += kParamLevels) {
        LevelTable T;
        T.n = n_levels - g0 < kParamLevels ? n_levels - g0 : kParamLevels;
        for (int i = 0; i < T.n; ++i) T.lv[i] = levels[g0 + i];
        T.first = T.lv[0].pyr_base;
        const LevelDesc& last = T.lv[T.n - 1];
        const int blocks = last.pyr_base + last.pyr_wq * ((last.h + kPyrRows - 1) / kPyrRows) - T.first;
        if (blocks > 0) pyramid_kernel<<<blocks, kPyrCols, 0, st>>>(T, gray, gpitch, gw, gh, limg);
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
