// extern "C" boundary: include/ccnn.h and include/ccnn_inspect.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "detector.h"
#include "replay.cuh"

namespace ccnn {
const char* last_error_cstr();
}

struct ccnn_detector {
    ccnn::Detector det;
};

using ccnn::set_error;

extern "C" {

CCNN_API const char* ccnn_version(void) { return "compactcnncascade_b200 0.1 (sm_100a)"; }

CCNN_API const char* ccnn_last_error(void) { return ccnn::last_error_cstr(); }

CCNN_API void ccnn_default_params(ccnn_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->max_image_width = 1920;
    p->max_image_height = 1080;
    p->min_face_height = 80;
    p->max_face_height = 0;
    p->scale_factor = 1.15f;
    p->min_neighbors = 2;
    p->detect_precision = CCNN_PRECISION_HIGH;
    p->treshold[0] = -1.5f;
    p->treshold[1] = -1.25f;
    p->treshold[2] = -1.0f;
    p->drop_detect = 1;
    p->equalize = 1;
    p->reflection = 1;
    p->pipeline = CCNN_PIPELINE_GPU;
    p->detect_mode = CCNN_DETECT_ASYNC;
    p->num_threads = 2;
    p->index_output[0] = 1;
    p->index_output[1] = 0;
    p->index_output[2] = 0;
    p->device_info = 1;
    p->cuda_device_id = 0;
    p->cl_platform_id = -1;
    p->cl_device_id = -1;
    p->facial_analysis = 0;
}

CCNN_API ccnn_status ccnn_create(const ccnn_params* params, const char* const* model_paths, ccnn_handle* out) {
    if (!params || !out) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    *out = nullptr;
    ccnn_detector* h = new (std::nothrow) ccnn_detector();
    if (!h) {
        set_error("out of host memory");
        return CCNN_ERR_OOM;
    }
    ccnn_status st = h->det.create(*params, model_paths);
    if (st != CCNN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_destroy(ccnn_handle h) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    delete h;
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_detect(ccnn_handle h, const ccnn_image* img, ccnn_face* faces, int capacity, int* n_faces) {
    if (!h || !img) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    return h->det.detect(*img, false, nullptr, faces, capacity, n_faces);
}

CCNN_API ccnn_status ccnn_detect_device(ccnn_handle h, const ccnn_image* img, void* stream, ccnn_face* faces, int capacity, int* n_faces) {
    if (!h || !img) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    return h->det.detect(*img, true, (cudaStream_t)stream, faces, capacity, n_faces);
}

CCNN_API ccnn_status ccnn_detect_batch(ccnn_handle h, const ccnn_image* imgs, int n_images, ccnn_face* faces, int capacity_per_image,
                                       int* n_faces) {
    if (!h) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    return h->det.detect_batch(imgs, n_images, false, faces, capacity_per_image, n_faces, nullptr);
}

CCNN_API ccnn_status ccnn_detect_device_batch(ccnn_handle h, const ccnn_image* imgs, int n_images, ccnn_face* faces,
                                              int capacity_per_image, int* n_faces, float* gpu_ms) {
    if (!h) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    return h->det.detect_batch(imgs, n_images, true, faces, capacity_per_image, n_faces, gpu_ms);
}

CCNN_API ccnn_status ccnn_profile_last_frame(ccnn_handle h, int iters, float* kernel_ms, int n_kernels) {
    if (!h || !kernel_ms || n_kernels <= 0) return CCNN_ERR_INVALID_ARG;
    return h->det.profile(iters, kernel_ms, n_kernels);
}

// ---- the internal CNNDetector class: include/ccnn_cnn.h ----

CCNN_API void ccnn_cnn_default_params(ccnn_cnn_param* p, ccnn_cnn_advanced_param* ap) {
    // member defaults of CNNDetector::Param / AdvancedParam (cnn_detector_v3.h:114-175)
    if (p) {
        std::memset(p, 0, sizeof(*p));
        p->pipeline = CCNN_PIPELINE_CPU;
        p->max_image_width = 1280;
        p->max_image_height = 720;
        p->min_obj_width = 48;
        p->min_obj_height = 48;
        p->max_obj_width = 0;
        p->max_obj_height = 0;
        p->scale_factor = 1.2f;
        p->min_neighbors = 2;
        p->num_threads = 0;
    }
    if (ap) {
        std::memset(ap, 0, sizeof(*ap));
        ap->detect_mode = CCNN_DETECT_SYNC;
        ap->detect_precision = CCNN_PRECISION_NORMAL;
        ap->packet_detection = 0;
        ap->gray_image_only = 0;
        ap->facial_analysis = 0;
        ap->equalize = 1;
        ap->reflection = 1;
        ap->type_check = 1;
        ap->treshold_1 = ap->treshold_2 = ap->treshold_3 = 0.f;
        ap->adapt_min_neighbors = 0;
        ap->double_check = 1;
        ap->drop_detect = 1;
        ap->min_num_detect = 1;
        ap->device_info = 0;
        ap->cuda_device_id = 0;
        ap->cl_platform_id = -1;
        ap->cl_device_id = -1;
        ap->concurrent_kernels = 3;
        ap->num_cnn_copy = 1;
        ap->blur = 0;
        ap->img_resize = 0;  // ImgResize::NearestNeighbor
        ap->uniform_noise = 0;
        ap->merger_detect = 1;
        ap->index_output[0] = 1;
        ap->index_output[1] = 0;
        ap->index_output[2] = 0;
        ap->index_output[3] = -1;
    }
}

CCNN_API ccnn_status ccnn_cnn_create(const ccnn_cnn_param* p, const ccnn_cnn_advanced_param* ap, const char* const* model_paths,
                                     ccnn_handle* out) {
    if (!out) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    *out = nullptr;
    ccnn_cnn_param dp;
    ccnn_cnn_advanced_param dap;
    ccnn_cnn_default_params(&dp, &dap);  // CNNDetector(Param* = 0, AdvancedParam* = 0): the defaults
    ccnn_detector* h = new (std::nothrow) ccnn_detector();
    if (!h) {
        set_error("out of host memory");
        return CCNN_ERR_OOM;
    }
    ccnn_status st = h->det.create_cnn(p ? *p : dp, ap ? *ap : dap, model_paths);
    if (st != CCNN_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_cnn_detect(ccnn_handle h, const ccnn_image* img, const ccnn_detection* prior, int n_prior, ccnn_detection* out,
                                     int capacity, int* n) {
    if (!h || !img) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    return h->det.detect_cnn(*img, prior, n_prior, out, capacity, n);
}

CCNN_API ccnn_status ccnn_cnn_nms(ccnn_handle h, const ccnn_detection* rect, int n_rect, ccnn_detection* out, int capacity, int* n_out) {
    if (!h) {
        set_error("null argument");
        return CCNN_ERR_INVALID_ARG;
    }
    return h->det.nms(rect, n_rect, out, capacity, n_out);
}

CCNN_API ccnn_status ccnn_cnn_get_params(ccnn_handle h, ccnn_cnn_param* p, ccnn_cnn_advanced_param* ap) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.get_cnn_params(p, ap);
}

CCNN_API ccnn_status ccnn_cnn_set_params(ccnn_handle h, const ccnn_cnn_param* p, const ccnn_cnn_advanced_param* ap) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.set_cnn_params(p, ap);
}

CCNN_API ccnn_status ccnn_set_schedule(ccnn_handle h, int frame_slots, int window_ctas_per_sm) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.set_schedule(frame_slots, window_ctas_per_sm);
}

CCNN_API ccnn_status ccnn_get_schedule(ccnn_handle h, int* frame_slots, int* window_ctas_per_sm) {
    if (!h || !frame_slots || !window_ctas_per_sm) return CCNN_ERR_INVALID_ARG;
    h->det.get_schedule(frame_slots, window_ctas_per_sm);
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_set_schedule_ex(ccnn_handle h, const ccnn_schedule* s) {
    if (!h || !s) return CCNN_ERR_INVALID_ARG;
    return h->det.set_schedule(s->frame_slots, s->window_ctas_per_sm, s->front_blocks_per_sm, s->back_blocks_per_sm, s->batch_frames,
                               s->batch_blocks_per_sm);
}

CCNN_API ccnn_status ccnn_get_schedule_ex(ccnn_handle h, ccnn_schedule* s) {
    if (!h || !s) return CCNN_ERR_INVALID_ARG;
    h->det.get_schedule(&s->frame_slots, &s->window_ctas_per_sm, &s->front_blocks_per_sm, &s->back_blocks_per_sm, &s->batch_frames,
                        &s->batch_blocks_per_sm);
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_gate_set(ccnn_handle h, const float* params, int n_params, float threshold, float fallback_fraction) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.gate_set(params, n_params, threshold, fallback_fraction);
}

CCNN_API ccnn_status ccnn_gate_disable(ccnn_handle h) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.gate_disable();
}

CCNN_API ccnn_status ccnn_gate_stats(ccnn_handle h, int* front_run, int* front_total, int* back_run, int* back_total, int* fallback) {
    if (!h || !front_run || !front_total || !back_run || !back_total || !fallback) return CCNN_ERR_INVALID_ARG;
    return h->det.gate_stats(front_run, front_total, back_run, back_total, fallback);
}

CCNN_API ccnn_status ccnn_gate_set_margin(ccnn_handle h, int pixels) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.gate_set_margin(pixels);
}

CCNN_API ccnn_status ccnn_gate_probabilities(ccnn_handle h, float* out, int capacity, int* n) {
    if (!h || !n || capacity < 0) return CCNN_ERR_INVALID_ARG;
    return h->det.gate_probabilities(out, capacity, n);
}

CCNN_API ccnn_status ccnn_gate_labels(ccnn_handle h, unsigned char* d_labels, void* stream) {
    if (!h || !d_labels) return CCNN_ERR_INVALID_ARG;
    return h->det.gate_labels(d_labels, (cudaStream_t)stream);
}

CCNN_API ccnn_status ccnn_get_gray_device(ccnn_handle h, const float** data, int* cols, int* rows, size_t* step) {
    if (!h || !data || !cols || !rows || !step) return CCNN_ERR_INVALID_ARG;
    return h->det.get_gray_device(data, cols, rows, step);
}

CCNN_API ccnn_status ccnn_get_gray_host(ccnn_handle h, float* out, int capacity, int* cols, int* rows) {
    if (!h || !out || !cols || !rows) return CCNN_ERR_INVALID_ARG;
    return h->det.get_gray_host(out, capacity, cols, rows);
}

CCNN_API ccnn_status ccnn_get_params(ccnn_handle h, ccnn_params* out) {
    if (!h || !out) return CCNN_ERR_INVALID_ARG;
    return h->det.get_params(out);
}
CCNN_API ccnn_status ccnn_set_params(ccnn_handle h, const ccnn_params* p) {
    if (!h || !p) return CCNN_ERR_INVALID_ARG;
    return h->det.set_params(*p);
}
CCNN_API ccnn_status ccnn_set_max_image_size(ccnn_handle h, int width, int height) {
    if (!h || width <= 0 || height <= 0) return CCNN_ERR_INVALID_ARG;
    return h->det.set_max_image_size(width, height);
}
CCNN_API ccnn_status ccnn_set_min_object_height(ccnn_handle h, int v) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.set_min_object_height(v);
}
CCNN_API ccnn_status ccnn_set_max_object_height(ccnn_handle h, int v) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.set_max_object_height(v);
}
CCNN_API ccnn_status ccnn_set_num_threads(ccnn_handle h, int v) {
    if (!h) return CCNN_ERR_INVALID_ARG;
    return h->det.set_num_threads(v);
}

// ---- inspection ----

CCNN_API ccnn_status ccnn_gray_u8_to_f32(const unsigned char* d_src, int cols, int rows, int channels, size_t src_step, float* d_dst,
                                         size_t dst_step, void* stream) {
    if (!d_src || !d_dst || cols <= 0 || rows <= 0 || (dst_step % 64) != 0) {
        set_error("invalid arguments (dst_step must be a multiple of 64 bytes)");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaError_t e = ccnn::launch_gray(d_src, (int)src_step, cols, rows, channels, d_dst, (int)(dst_step / sizeof(float)), (cudaStream_t)stream);
    if (e == cudaErrorInvalidValue) {
        set_error("unsupported channel count");
        return CCNN_ERR_UNSUPPORTED;
    }
    if (e == cudaErrorMisalignedAddress) {
        set_error("buffers must be 64-byte aligned with a source step that is a multiple of 64");
        return CCNN_ERR_INVALID_ARG;
    }
    ccnn_status st = ccnn::cuda_status(e, "gray kernel");
    if (st != CCNN_OK) return st;
    return ccnn::cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "gray kernel");
}

CCNN_API ccnn_status ccnn_resize_f32(const float* d_src, int src_cols, int src_rows, size_t src_step, float* d_dst, int dst_cols,
                                     int dst_rows, size_t dst_step, int type, void* stream) {
    if (!d_src || !d_dst || src_cols < 2 || src_rows < 2 || dst_cols <= 0 || dst_rows <= 0 || (src_step % 4) || (dst_step % 4)) {
        set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    cudaError_t e = ccnn::launch_resize_f32(d_src, (int)(src_step / 4), src_cols, src_rows, d_dst, (int)(dst_step / 4), dst_cols, dst_rows,
                                            type, (cudaStream_t)stream);
    ccnn_status st = ccnn::cuda_status(e, "resize kernel");
    if (st != CCNN_OK) return st;
    return ccnn::cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "resize kernel");
}

CCNN_API ccnn_status ccnn_stage1_forward(ccnn_handle h, const float* d_img, int cols, int rows, size_t step, float* d_resp, int resp_cap,
                                         int* resp_cols, int* resp_rows, void* stream) {
    if (!h || !d_img || !d_resp || !resp_cols || !resp_rows) return CCNN_ERR_INVALID_ARG;
    return h->det.stage1_forward(d_img, cols, rows, step, d_resp, resp_cap, resp_cols, resp_rows, (cudaStream_t)stream);
}

CCNN_API ccnn_status ccnn_inspect_levels(ccnn_handle h, ccnn_level_info* out, int capacity, int* n_levels) {
    if (!h || !n_levels || (capacity > 0 && !out)) return CCNN_ERR_INVALID_ARG;
    return h->det.inspect_levels(out, capacity, n_levels);
}
CCNN_API ccnn_status ccnn_inspect_response(ccnn_handle h, int level, float* out, int capacity) {
    if (!h || !out) return CCNN_ERR_INVALID_ARG;
    return h->det.inspect_response(level, out, capacity);
}
CCNN_API ccnn_status ccnn_inspect_candidates(ccnn_handle h, ccnn_candidate* out, int capacity, int* n) {
    if (!h || !n || (capacity > 0 && !out)) return CCNN_ERR_INVALID_ARG;
    return h->det.inspect_candidates(out, capacity, n);
}
CCNN_API ccnn_status ccnn_inspect_raw_detections(ccnn_handle h, ccnn_detection* out, int capacity, int* n) {
    if (!h || !n || (capacity > 0 && !out)) return CCNN_ERR_INVALID_ARG;
    return h->det.inspect_raw(out, capacity, n);
}

CCNN_API ccnn_status ccnn_plan_levels(const ccnn_params* p, int cols, int rows, int channels, ccnn_level_info* out, int capacity,
                                      int* n_levels) {
    if (!p || !n_levels || cols <= 0 || rows <= 0 || (capacity > 0 && !out)) return CCNN_ERR_INVALID_ARG;
    // a fresh handle: a frame above max_image_size raises it; a colour frame turns gray_image_only off
    int max_h = p->max_image_height;
    if (cols > p->max_image_width || rows > p->max_image_height) max_h = rows;  // Detect :2499-2513 takes the frame size
    const bool detect = p->detect_mode != CCNN_DETECT_DISABLE;
    const int ext_w = detect ? 36 + ccnn::kExtOff : ccnn::kPatW, ext_h = detect ? 40 + ccnn::kExtOff : ccnn::kPatH;
    std::vector<float> scales;
    bool down = false;
    float in_scale = 0.f;
    bool gray_only = channels == 1 || p->detect_precision == CCNN_PRECISION_DEF;
    if (!ccnn::compute_scales(*p, gray_only, ccnn::kPatH, max_h, &scales, &down, &in_scale)) {
        set_error("invalid configuration: empty scale list");
        return CCNN_ERR_CONFIG;
    }
    int gw = cols, gh = rows;
    if (down && channels == 1) {
        gw = (int)((float)cols * in_scale);
        gh = (int)((float)rows * in_scale);
    } else if (down) {
        set_error("precision 'def' with a colour frame needs min_face_height < 34 (the reference recurses forever)");
        return CCNN_ERR_CONFIG;
    }
    int n = 0;
    if (cols >= ext_w && rows >= ext_h) {
        for (size_t i = 0; i < scales.size(); ++i) {
            const int w = (int)((float)gw * scales[i]), h = (int)((float)gh * scales[i]);
            if (w < ext_w || h < ext_h) break;
            if (n < capacity) {
                out[n].width = w;
                out[n].height = h;
                out[n].scale = scales[i];
                const int p1w = (w - 3) >> 1, p1h = (h - 3) >> 1;
                out[n].resp_width = ((p1w - 2) >> 1) - 3;
                out[n].resp_height = ((p1h - 2) >> 1) - 4;
            }
            ++n;
        }
    }
    *n_levels = n;
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_sort_permutation(const float* scales, int n, int* perm) {
    if (n < 0 || (n > 0 && (!scales || !perm))) return CCNN_ERR_INVALID_ARG;
    std::vector<ccnn::Det> v(n);
    for (int i = 0; i < n; ++i) {
        v[i] = ccnn::make_det(i, 0, 1, 1, 0.f, scales[i], 0);
    }
    if (n > 16) ccnn::introsort_scale_desc(v.data(), n);  // n <= 16: insertion sort of a sorted list
    else ccnn::insertion_sort(v.data(), 0, n);
    for (int i = 0; i < n; ++i) perm[i] = v[i].x;
    return CCNN_OK;
}

CCNN_API ccnn_status ccnn_sort_permutation_device(const float* scales, int n, int* perm) {
    if (n < 0 || (n > 0 && (!scales || !perm))) return CCNN_ERR_INVALID_ARG;
    return ccnn::cuda_status(ccnn::sort_permutation_device(scales, n, perm), "block-wide sort");
}

}  // extern "C"

// Exhaustive check of the packed reciprocal used by the rational tanh against the IEEE reciprocal.
namespace ccnn {
__global__ void rcp_check_kernel(uint32_t start, uint32_t pairs, unsigned long long* bad) {
    unsigned long long local = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += gridDim.x * blockDim.x) {
        const float d0 = __uint_as_float(start + 2 * i), d1 = __uint_as_float(start + 2 * i + 1);
        const f2_t r = f2_rcp(f2_pack(d0, d1));
        local += (__float_as_uint(f2_lo(r)) != __float_as_uint(__frcp_rn(d0))) + (__float_as_uint(f2_hi(r)) != __float_as_uint(__frcp_rn(d1)));
    }
    if (local) atomicAdd(bad, local);
}
}  // namespace ccnn

extern "C" CCNN_API ccnn_status ccnn_check_reciprocal(long long* mismatches, long long* checked) {
    if (!mismatches || !checked) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(unsigned long long));
    const uint32_t lo = 0x3F800000u, hi = 0x7F800000u + 2u;  // 1.0 up to +inf and the first NaN
    if (e == cudaSuccess) {
        ccnn::rcp_check_kernel<<<148 * 8, 256>>>(lo, (hi - lo) / 2, d);
        e = cudaDeviceSynchronize();
    }
    unsigned long long nb = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&nb, d, sizeof(nb), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        ccnn::set_error(std::string("reciprocal check: ") + cudaGetErrorString(e));
        return CCNN_ERR_CUDA;
    }
    *mismatches = (long long)nb;
    *checked = (long long)(hi - lo);
    return CCNN_OK;
}
