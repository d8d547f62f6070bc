// Test infrastructure only: a C-ABI harness around the UNMODIFIED reference sources
// (Bkmz21/CompactCNNCascade, src/CNNObjectDetector/), compiled by oracle/Makefile into
// oracle/_ref/libccnn_ref*.so. Only tests/, the smoke check and bench.py's reference arm load it.
// It never ships in the product path.
//
// Every function drives the reference's own classes; nothing here re-implements the
// reference arithmetic except `ref_detect_steps`, which replays the body of
// CNNDetector::Detect (src/CNNObjectDetector/cnn_detector_v3.cpp:2483-2813, CPU pipeline)
// so that the raw detection list can be captured before Merger; the tests check that its
// final boxes equal those of the genuine FaceDetector::Detect.

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <list>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

// The harness reads private members of CNNDetector (scales, level buffers, raw detections) and
// calls its `inline` members (Merger, RunCPUDetect ...), whose bodies live only in
// cnn_detector_v3.cpp. That translation unit is therefore compiled here, unmodified, as part of
// the harness (the Makefile does not compile it separately).
#define private public
#include "cnn_detector_v3.cpp"
#include "CompactCNNLibAPI_v2.h"
#undef private

using namespace NeuralNetworksLib;

namespace CompactCNNLib {
std::pair<CNNDetector::Param, CNNDetector::AdvancedParam> paramConverter(FaceDetector::Param param);
}

extern "C" {

typedef struct {
    int max_image_w, max_image_h;
    int min_face_height, max_face_height;
    float scale_factor;
    int min_neighbors;
    int detect_precision;  // 0 def, 1 low, 2 normal, 3 high, 4 ultra
    float treshold[3];
    int drop_detect, equalize, reflection;
    int detect_mode;       // 0 disable, 1 sync, 2 async
} ref_params;

typedef struct {
    int x, y, w, h;
    float score;
    float scale;
    int knn;
    int num_detect;
} ref_det;

static CompactCNNLib::FaceDetector::Param to_api_param(const ref_params* p) {
    CompactCNNLib::FaceDetector::Param q;
    q.max_image_size = CompactCNNLib::FaceDetector::Size(p->max_image_w, p->max_image_h);
    q.min_face_height = p->min_face_height;
    q.max_face_height = p->max_face_height;
    q.scale_factor = p->scale_factor;
    q.min_neighbors = p->min_neighbors;
    q.detect_precision = static_cast<CompactCNNLib::FaceDetector::DetectPrecision>(p->detect_precision);
    for (int i = 0; i < 3; ++i) q.treshold[i] = p->treshold[i];
    q.drop_detect = p->drop_detect != 0;
    q.equalize = p->equalize != 0;
    q.reflection = p->reflection != 0;
    q.pipeline = CompactCNNLib::FaceDetector::Pipeline::CPU;
    q.detect_mode = static_cast<CompactCNNLib::FaceDetector::DetectMode>(p->detect_mode);
    q.num_threads = 1;
    q.device_info = false;
    q.facial_analysis = false;
    return q;
}

// ---- image ops (src/CNNObjectDetector/image_proc.cpp:299-317, image_resize.cpp:564-584) ----

int ref_gray(const uint8_t* img, int w, int h, int ch, int step, float* out) {
    SIMD::Image_8u src(w, h, ch, const_cast<uint8_t*>(img), step);
    SIMD::Image_32f dst(w, h, 1, out, w);
    return SIMD::ImageConverter::Img8uToImg32fGRAY(dst, src, 1);
}

int ref_resize_f32(const float* src, int sw, int sh, int sstride, float* dst, int dw, int dh, int type) {
    SIMD::Image_32f s(sw, sh, 1, const_cast<float*>(src), sstride);
    SIMD::Image_32f d(dw, dh, 1, dst, dw);
    SIMD::ImageResizer rz(Size(dw, dh), Size(sw, sh));
    rz.FastImageResize(d, s, type, 1);
    return 0;
}

int ref_resize_u8(const uint8_t* src, int sw, int sh, int sstride, uint8_t* dst, int dw, int dh, int type) {
    SIMD::Image_8u s(sw, sh, 1, const_cast<uint8_t*>(src), sstride);
    SIMD::Image_8u d(dw, dh, 1, dst, dw);
    SIMD::ImageResizer rz(Size(dw, dh), Size(sw, sh));
    rz.FastImageResize(d, s, type, 1);
    return 0;
}

int ref_equalize(uint8_t* img, int w, int h) {
    SIMD::Image_8u im(w, h, 1, img, w);
    SIMD::equalizeImage(im);
    return 0;
}

// ---- one network on one f32 image (cnn_simd_cntk.cpp:42-404, 405-539, 964-995) ----

int ref_net_forward(const char* model_path, int index_output, const float* img, int w, int h, int stride,
                    float* out, int out_cap, int* ow, int* oh) {
    SIMD::ConvNeuralNetwork net;
    net.Init(std::string(model_path), index_output, nullptr);
    if (net.isEmpty()) return -1;
    Size mn = net.getMinInputImgSize();
    if (w < mn.width || h < mn.height) return -2;
    net.AllocateMemory(Size(w, h));
    SIMD::Image_32f in(w, h, 1, const_cast<float*>(img), stride);
    SIMD::Image_32f resp;
    net.Forward(resp, in);
    *ow = resp.width;
    *oh = resp.height;
    if (resp.width * resp.height > out_cap) return -3;
    for (int y = 0; y < resp.height; ++y)
        for (int x = 0; x < resp.width; ++x) out[y * resp.width + x] = resp.data[y * resp.widthStep + x];
    return 0;
}

// The same with the model given as its bytes. The legacy loader (format 1.0,
// src/CNNObjectDetector/cnn_simd.cpp:40-60) reads a path into a stream that shadows the one it parses,
// so only the in-memory form (a string of 255 bytes or more, as the detector passes its embedded
// models) loads.
int ref_net_forward_bytes(const char* model, int model_bytes, const float* img, int w, int h, int stride, float* out, int out_cap, int* ow,
                          int* oh) {
    SIMD::ConvNeuralNetwork net;
    net.Init(std::string(model, (size_t)model_bytes), 0, nullptr);
    if (net.isEmpty()) return -1;
    Size mn = net.getMinInputImgSize();
    if (w < mn.width || h < mn.height) return -2;
    net.AllocateMemory(Size(w, h));
    SIMD::Image_32f in(w, h, 1, const_cast<float*>(img), stride);
    SIMD::Image_32f resp;
    net.Forward(resp, in);
    *ow = resp.width;
    *oh = resp.height;
    if (resp.width * resp.height > out_cap) return -3;
    for (int y = 0; y < resp.height; ++y)
        for (int x = 0; x < resp.width; ++x) out[y * resp.width + x] = resp.data[y * resp.widthStep + x];
    return 0;
}

int ref_net_min_size(const char* model_path, int* w, int* h) {
    SIMD::ConvNeuralNetwork net;
    net.Init(std::string(model_path), 0, nullptr);
    if (net.isEmpty()) return -1;
    *w = net.getMinInputImgSize().width;
    *h = net.getMinInputImgSize().height;
    return 0;
}

// ---- genuine public API (CompactCNNLibAPI_v2.cpp:373-544) ----

static std::mutex g_api_mutex;

int ref_face_detect(const ref_params* p, const uint8_t* img, int w, int h, int ch, int step,
                    ref_det* out, int cap) {
    std::lock_guard<std::mutex> lk(g_api_mutex);
    CompactCNNLib::FaceDetector fd;
    CompactCNNLib::FaceDetector::Param q = to_api_param(p);
    if (fd.Init(q) < 0) return -1;
    std::vector<CompactCNNLib::FaceDetector::Face> faces(4096);
    CompactCNNLib::FaceDetector::ImageData im(w, h, ch, const_cast<uint8_t*>(img), (size_t)step);
    int n = fd.Detect(faces.data(), im);
    if (n < 0) return n;
    for (int i = 0; i < n && i < cap; ++i) {
        out[i].x = faces[i].x;
        out[i].y = faces[i].y;
        out[i].w = faces[i].width;
        out[i].h = faces[i].height;
        out[i].score = faces[i].score;
        out[i].scale = 0.f;
        out[i].knn = 0;
        out[i].num_detect = 0;
    }
    fd.Clear();
    return n;
}

// The same with facial analysis on (landmark network, CompactCNNLibAPI_v2.cpp:296-319): faces
// carry gender / smile / glasses.
typedef struct {
    int x, y, w, h;
    float score;
    int gender, smile, glasses;
} ref_face;

int ref_face_detect_fa(const ref_params* p, const uint8_t* img, int w, int h, int ch, int step, ref_face* out, int cap) {
    std::lock_guard<std::mutex> lk(g_api_mutex);
    CompactCNNLib::FaceDetector fd;
    CompactCNNLib::FaceDetector::Param q = to_api_param(p);
    q.facial_analysis = true;
    if (fd.Init(q) < 0) return -1;
    std::vector<CompactCNNLib::FaceDetector::Face> faces(4096);
    CompactCNNLib::FaceDetector::ImageData im(w, h, ch, const_cast<uint8_t*>(img), (size_t)step);
    int n = fd.Detect(faces.data(), im);
    if (n < 0) return n;
    for (int i = 0; i < n && i < cap; ++i) {
        out[i].x = faces[i].x;
        out[i].y = faces[i].y;
        out[i].w = faces[i].width;
        out[i].h = faces[i].height;
        out[i].score = faces[i].score;
        out[i].gender = faces[i].gender;
        out[i].smile = faces[i].smile;
        out[i].glasses = faces[i].glasses;
    }
    fd.Clear();
    return n;
}

// CNTK dump -> binary model (CompactCNNLibAPI_v2.cpp:509-519)
int ref_cntk_dump2binary(const char* binary_file, const char* dump_file) {
    CompactCNNLib::FaceDetector::CNTKDump2Binary(binary_file, dump_file);
    return 0;
}

// Persistent detector for repeated timing of the reference (bench reference arm).
static CompactCNNLib::FaceDetector* g_fd = nullptr;

int ref_api_init(const ref_params* p) {
    std::lock_guard<std::mutex> lk(g_api_mutex);
    if (!g_fd) g_fd = new CompactCNNLib::FaceDetector();
    CompactCNNLib::FaceDetector::Param q = to_api_param(p);
    return g_fd->Init(q);
}

int ref_api_detect(const uint8_t* img, int w, int h, int ch, int step, ref_det* out, int cap) {
    std::lock_guard<std::mutex> lk(g_api_mutex);
    if (!g_fd) return -1;
    static std::vector<CompactCNNLib::FaceDetector::Face> faces(65536);
    CompactCNNLib::FaceDetector::ImageData im(w, h, ch, const_cast<uint8_t*>(img), (size_t)step);
    int n = g_fd->Detect(faces.data(), im);
    for (int i = 0; i < n && i < cap; ++i) {
        out[i].x = faces[i].x;
        out[i].y = faces[i].y;
        out[i].w = faces[i].width;
        out[i].h = faces[i].height;
        out[i].score = faces[i].score;
        out[i].scale = 0.f;
        out[i].knn = 0;
        out[i].num_detect = 0;
    }
    return n;
}

// ---- step-wise replay of CNNDetector::Detect (CPU pipeline), capturing intermediates ----
//
// level_* arrays have room for `level_cap` levels; `levels_out` gets the concatenated level
// images (row-major, width-contiguous) when non-null; `resp_out` likewise the response maps.
// Returns the number of final detections, or a negative error.

static void copy_det(ref_det* o, CNNDetector::Detection& d) {
    o->x = d.rect.x;
    o->y = d.rect.y;
    o->w = d.rect.width;
    o->h = d.rect.height;
    o->score = d.score;
    o->scale = d.scale;
    o->knn = d.knn;
    o->num_detect = d.num_detect;
}

int ref_detect_steps(const ref_params* p, const uint8_t* img, int w, int h, int ch, int step,
                     float* gray_out, int* gray_w, int* gray_h,
                     int level_cap, int* n_levels, float* scales_out, int* level_w, int* level_h,
                     float* levels_out, long levels_cap,
                     int* resp_w, int* resp_h, float* resp_out, long resp_cap,
                     ref_det* raw_out, int raw_cap, int* n_raw,
                     ref_det* final_out, int final_cap) {
    CompactCNNLib::FaceDetector::Param q = to_api_param(p);
    if (q.max_image_size.width < w) q.max_image_size.width = w;
    if (q.max_image_size.height < h) q.max_image_size.height = h;
    auto cp = CompactCNNLib::paramConverter(q);
    // A multi-channel frame makes the genuine Detect clear gray_image_only and re-Init
    // (cnn_detector_v3.cpp:2531-2546); start from that state directly.
    if (ch != 1) cp.second.gray_image_only = false;
    CNNDetector det(&cp.first, &cp.second);
    if (det.isEmpty()) return -1;

    SIMD::Image_8u image(w, h, ch, const_cast<uint8_t*>(img), step);
    if (image.width < det.ext_pattern_size_cd.width || image.height < det.ext_pattern_size_cd.height) {
        *n_levels = 0;
        *n_raw = 0;
        return 0;
    }
    if (image.width != det.param.max_image_size.width || image.height != det.param.max_image_size.height)
        det.num_scales = (int)det.scales.size();

    if (det.advanced_param.gray_image_only && det.cpu_input_img_resizer != nullptr) {
        det.cpu_input_img.setSize(image.getSize() * det.cpu_input_img_scale);
        det.cpu_input_img_resizer->FastImageResize(det.cpu_input_img, image, (int)CNNDetector::ImgResize::Bilinear, 1);
        image.clone(det.cpu_input_img);
    }

    det.cpu_img_gray.width = image.width;
    det.cpu_img_gray.height = image.height;
    if (SIMD::ImageConverter::Img8uToImg32fGRAY(det.cpu_img_gray, image, 1) < 0) return -2;

    SIMD::mm_erase((void*)det.data_transfer_flag, int(det.scales.size() * sizeof(det.data_transfer_flag[0])));
    det.RunCPUDetect();
    det.RunCheckDetectAsync();

    // intermediates
    *gray_w = det.cpu_img_gray.width;
    *gray_h = det.cpu_img_gray.height;
    if (gray_out)
        for (int y = 0; y < det.cpu_img_gray.height; ++y)
            memcpy(gray_out + (size_t)y * det.cpu_img_gray.width, det.cpu_img_gray.data + (size_t)y * det.cpu_img_gray.widthStep,
                   sizeof(float) * det.cpu_img_gray.width);

    int nl = 0;
    long loff = 0, roff = 0;
    for (int scl = 0; scl < (int)det.scales.size() && scl < level_cap; ++scl) {
        Size ls = det.cpu_img_gray.getSize() * det.scales[scl];
        if (ls.width < det.ext_pattern_size_cd.width || ls.height < det.ext_pattern_size_cd.height) break;
        scales_out[nl] = det.scales[scl];
        level_w[nl] = ls.width;
        level_h[nl] = ls.height;
        SIMD::Image_32f& li = det.cpu_img_scale[scl];
        if (levels_out) {
            if (loff + (long)ls.width * ls.height > levels_cap) return -3;
            if (det.scales[scl] != 1.f) {
                for (int y = 0; y < ls.height; ++y)
                    memcpy(levels_out + loff + (long)y * ls.width, li.data + (size_t)y * li.widthStep, sizeof(float) * ls.width);
            } else {
                for (int y = 0; y < ls.height; ++y)
                    memcpy(levels_out + loff + (long)y * ls.width, det.cpu_img_gray.data + (size_t)y * det.cpu_img_gray.widthStep,
                           sizeof(float) * ls.width);
            }
        }
        loff += (long)ls.width * ls.height;
        SIMD::Image_32f& rm = det.cpu_response_map[scl];
        resp_w[nl] = rm.width;
        resp_h[nl] = rm.height;
        if (resp_out) {
            if (roff + (long)rm.width * rm.height > resp_cap) return -4;
            for (int y = 0; y < rm.height; ++y)
                memcpy(resp_out + roff + (long)y * rm.width, rm.data + (size_t)y * rm.widthStep, sizeof(float) * rm.width);
        }
        roff += (long)rm.width * rm.height;
        ++nl;
    }
    *n_levels = nl;

    *n_raw = (int)det.cpu_detect_rect.size();
    for (int i = 0; i < (int)det.cpu_detect_rect.size() && i < raw_cap; ++i) copy_det(&raw_out[i], det.cpu_detect_rect[i]);

    // post-processing exactly as cnn_detector_v3.cpp:2745-2810
    std::vector<CNNDetector::Detection> detections;
    std::reverse_copy(det.cpu_detect_rect.begin(), det.cpu_detect_rect.end(), std::back_inserter(det.gpu_detect_rect));
    if (det.gpu_detect_rect.size() > 0) {
        std::sort(det.gpu_detect_rect.begin(), det.gpu_detect_rect.end(),
                  [](CNNDetector::Detection& a, CNNDetector::Detection& b) { return b.scale < a.scale; });
        if (det.advanced_param.merger_detect) {
            std::vector<CNNDetector::Detection> detections_temp = detections;
            det.Merger(detections_temp, det.gpu_detect_rect, 0.5f);
            if (det.advanced_param.min_num_detect > 1) {
                const int threshold = det.advanced_param.min_num_detect;
                detections_temp.erase(std::remove_if(detections_temp.begin(), detections_temp.end(),
                                                     [&threshold](const CNNDetector::Detection& d) { return d.num_detect < threshold; }),
                                      detections_temp.end());
            }
            if (detections_temp.size() > 0) {
                detections.clear();
                det.Merger(detections, detections_temp, 0.2f, true);
            }
        } else {
            detections.assign(det.gpu_detect_rect.begin(), det.gpu_detect_rect.end());
        }
        if (det.cpu_input_img_resizer != nullptr) {
            const float scale = (float)det.param.min_obj_size.height / (float)det.pattern_size.height;
            for (auto& d : detections)
                d.rect = Rect(int(float(d.rect.x) * scale), int(float(d.rect.y) * scale), int(float(d.rect.width) * scale),
                              int(float(d.rect.height) * scale));
        }
    }
    int nf = (int)detections.size();
    for (int i = 0; i < nf && i < final_cap; ++i) copy_det(&final_out[i], detections[i]);
    return nf;
}

// The reference's std::sort on detections keyed by scale (cnn_detector_v3.cpp:2750) applied
// to an arbitrary key sequence: returns the permutation (perm[i] = original index at slot i).
int ref_sort_by_scale_desc(const float* keys, int n, int* perm) {
    std::vector<std::pair<float, int>> v(n);
    for (int i = 0; i < n; ++i) v[i] = std::make_pair(keys[i], i);
    std::sort(v.begin(), v.end(), [](std::pair<float, int>& a, std::pair<float, int>& b) { return b.first < a.first; });
    for (int i = 0; i < n; ++i) perm[i] = v[i].second;
    return 0;
}

// The reference Merger (cnn_detector_v3.cpp:2814-2936) on a caller-given list.
int ref_merger(const ref_det* in, int n, float threshold, int del, ref_det* out, int cap) {
    std::vector<CNNDetector::Detection> rect, res;
    for (int i = 0; i < n; ++i) {
        CNNDetector::Detection d(in[i].x, in[i].y, in[i].w, in[i].h, in[i].score, in[i].scale, in[i].knn);
        d.num_detect = in[i].num_detect;
        rect.push_back(d);
    }
    CNNDetector* det = nullptr;
    // Merger touches no member state; call it through one long-lived detector object.
    static CNNDetector::Param dp;
    static CNNDetector::AdvancedParam dap;
    dap.detect_mode = CNNDetector::DetectMode::disable;
    static CNNDetector* holder = nullptr;
    if (!holder) holder = new CNNDetector(&dp, &dap);
    det = holder;
    det->Merger(res, rect, threshold, del != 0);
    int m = (int)res.size();
    for (int i = 0; i < m && i < cap; ++i) copy_det(&out[i], res[i]);
    return m;
}

// ---- the internal CNNDetector class (cnn_detector_v3.h:82-453), driven directly ----

// The same layout as ccnn_cnn_param / ccnn_cnn_advanced_param of include/ccnn_cnn.h.
typedef struct {
    int pipeline;
    int max_image_width, max_image_height;
    int min_obj_width, min_obj_height;
    int max_obj_width, max_obj_height;
    float scale_factor;
    int min_neighbors;
    int num_threads;
} ref_cnn_param;

typedef struct {
    int detect_mode, detect_precision, packet_detection, gray_image_only, facial_analysis;
    int equalize, reflection, type_check;
    float treshold_1, treshold_2, treshold_3;
    int adapt_min_neighbors, double_check, drop_detect, min_num_detect;
    int device_info, cuda_device_id, cl_platform_id, cl_device_id, concurrent_kernels, num_cnn_copy;
    int blur, img_resize, uniform_noise, merger_detect;
    int index_output[4];
} ref_cnn_advanced_param;

static void to_ref_params(const ref_cnn_param* p, const ref_cnn_advanced_param* a, CNNDetector::Param* q, CNNDetector::AdvancedParam* b) {
    q->pipeline = static_cast<CNNDetector::Pipeline>(p->pipeline);
    q->max_image_size = Size(p->max_image_width, p->max_image_height);
    q->min_obj_size = Size(p->min_obj_width, p->min_obj_height);
    q->max_obj_size = Size(p->max_obj_width, p->max_obj_height);
    q->scale_factor = p->scale_factor;
    q->min_neighbors = p->min_neighbors;
    q->num_threads = p->num_threads;
    b->detect_mode = static_cast<CNNDetector::DetectMode>(a->detect_mode);
    b->detect_precision = static_cast<CNNDetector::DetectPrecision>(a->detect_precision);
    b->packet_detection = a->packet_detection != 0;
    b->gray_image_only = a->gray_image_only != 0;
    b->facial_analysis = a->facial_analysis != 0;
    b->equalize = a->equalize != 0;
    b->reflection = a->reflection != 0;
    b->type_check = a->type_check;
    b->treshold_1 = a->treshold_1;
    b->treshold_2 = a->treshold_2;
    b->treshold_3 = a->treshold_3;
    b->adapt_min_neighbors = a->adapt_min_neighbors != 0;
    b->double_check = a->double_check != 0;
    b->drop_detect = a->drop_detect != 0;
    b->min_num_detect = a->min_num_detect;
    b->device_info = a->device_info != 0;
    b->cuda_device_id = a->cuda_device_id;
    b->cl_platform_id = a->cl_platform_id;
    b->cl_device_id = a->cl_device_id;
    b->concurrent_kernels = a->concurrent_kernels;
    b->num_cnn_copy = a->num_cnn_copy;
    b->blur = a->blur != 0;
    b->img_resize = static_cast<CNNDetector::ImgResize>(a->img_resize);
    b->uniform_noise = a->uniform_noise != 0;
    b->merger_detect = a->merger_detect != 0;
    for (int i = 0; i < 4; ++i) b->index_output[i] = a->index_output[i];
}

// CNNDetector(&param, &advanced_param) + Detect(detections, image) with `prior` already in the
// vector; returns the detection count and, when given, the parameters the detector then reports.
int ref_cnn_detect(const ref_cnn_param* p, const ref_cnn_advanced_param* a, const uint8_t* img, int w, int h, int ch, int step,
                   const ref_det* prior, int n_prior, ref_det* out, int cap, ref_cnn_param* p_after, ref_cnn_advanced_param* a_after) {
    std::lock_guard<std::mutex> lk(g_api_mutex);
    CNNDetector::Param q;
    CNNDetector::AdvancedParam b;
    to_ref_params(p, a, &q, &b);
    CNNDetector det(&q, &b);
    if (det.isEmpty()) return -1;
    std::vector<CNNDetector::Detection> dets;
    for (int i = 0; i < n_prior; ++i) {
        CNNDetector::Detection d(prior[i].x, prior[i].y, prior[i].w, prior[i].h, prior[i].score, prior[i].scale, prior[i].knn);
        d.num_detect = prior[i].num_detect;
        dets.push_back(d);
    }
    SIMD::Image_8u image(w, h, ch, const_cast<uint8_t*>(img), step);
    const int r = det.Detect(dets, image);
    if (r < 0) return r;
    const int n = (int)dets.size();
    for (int i = 0; i < n && i < cap; ++i) copy_det(&out[i], dets[i]);
    if (p_after) {
        const CNNDetector::Param g = det.getParam();
        *p_after = *p;
        p_after->pipeline = (int)g.pipeline;
        p_after->max_image_width = g.max_image_size.width;
        p_after->max_image_height = g.max_image_size.height;
    }
    if (a_after) {
        const CNNDetector::AdvancedParam g = det.getAdvancedParam();
        *a_after = *a;
        a_after->packet_detection = g.packet_detection;
        a_after->gray_image_only = g.gray_image_only;
        a_after->facial_analysis = g.facial_analysis;
        a_after->equalize = g.equalize;
        a_after->reflection = g.reflection;
        a_after->type_check = g.type_check;
        a_after->adapt_min_neighbors = g.adapt_min_neighbors;
        a_after->double_check = g.double_check;
        a_after->drop_detect = g.drop_detect;
        a_after->min_num_detect = g.min_num_detect;
        a_after->blur = g.blur;
        a_after->uniform_noise = g.uniform_noise;
        a_after->merger_detect = g.merger_detect;
    }
    return n;
}

}  // extern "C"
