// Header-only C++ facade with the reference's internal detector class
//   namespace NeuralNetworksLib { class CNNDetector }   (src/CNNObjectDetector/cnn_detector_v3.h:82-453)
// implemented over the C ABI of ccnn_cnn.h, so code written against the reference's CNNDetector
// recompiles against this header and links libccnn.so. Same nested types and field defaults
// (Param, AdvancedParam, Detection), the geometry types it uses (Size, Rect, SIMD::Image_8u) and the
// same methods: Detect, NMS, get/set of Param, AdvancedParam, max image size, min/max object size
// and thread count, getGrayImage.
//
// Differences a caller can observe:
//  * AdvancedParam::path_model[0..2] are honoured when set (the reference overwrites them with its
//    embedded models, the same files as the bundled defaults); path_model[3] is ignored;
//  * blur and uniform_noise (off unless set) are refused: Detect returns -1;
//  * Detection::facial_data stays empty (the public FaceDetector reports the attributes);
//  * getGrayImage fills an Image_32f whose data the facade owns (host memory), valid until the next
//    call on the detector.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

#include "ccnn_cnn.h"

namespace NeuralNetworksLib {

struct Size {
    int width = 0;
    int height = 0;
    Size() {}
    Size(int w, int h) : width(w), height(h) {}
};

struct Point {
    int x = 0;
    int y = 0;
    Point() {}
    Point(int _x, int _y) : x(_x), y(_y) {}
};

struct Rect {
    int x = 0, y = 0, width = 0, height = 0;
    int x2 = 0, y2 = 0, cx = 0, cy = 0;
    Rect() {}
    Rect(int _x, int _y, int _w, int _h) : x(_x), y(_y), width(_w), height(_h), x2(_x + _w), y2(_y + _h) {
        cx = (x2 + x) >> 1;
        cy = (y2 + y) >> 1;
    }
};

namespace SIMD {
// The fields of the reference's TmpImage (image.h:42-78) that a caller sets: an 8-bit image wrapping
// the caller's pixels (1 = gray, 3 = BGR, 4 = BGRA), widthStep in elements per row.
template <typename T>
struct TmpImage {
    int width = 0, height = 0, size = 0, widthStep = 0, nChannel = 1;
    T* data = nullptr;
    TmpImage() {}
    TmpImage(int w, int h, int ch, T* d, int step = 0)
        : width(w), height(h), size(w * h), widthStep(step ? step : w * ch), nChannel(ch), data(d) {}
    bool isEmpty() const { return data == nullptr; }
    Size getSize() const { return Size(width, height); }
};
typedef TmpImage<unsigned char> Image_8u;
typedef TmpImage<float> Image_32f;
}  // namespace SIMD

class CNNDetector {
   public:
    enum struct Pipeline { CPU = 0, GPU = 1, GPU_CPU = 2 };
    enum struct ImgResize { NearestNeighbor = 0, Bilinear = 1 };
    enum struct DetectMode { disable = 0, sync = 1, async = 2 };
    enum struct DetectPrecision { def = 0, low = 1, normal = 2, high = 3, ultra = 4 };

    struct Param {
        Pipeline pipeline = Pipeline::CPU;
        Size max_image_size = Size(1280, 720);
        Size min_obj_size = Size(48, 48);
        Size max_obj_size = Size(0, 0);
        float scale_factor = 1.2f;
        int min_neighbors = 2;
        int num_threads = 0;
    };
    struct AdvancedParam {
        DetectMode detect_mode = DetectMode::sync;
        DetectPrecision detect_precision = DetectPrecision::normal;
        bool packet_detection = false;
        bool gray_image_only = false;
        bool facial_analysis = false;
        bool equalize = true;
        bool reflection = true;
        int type_check = 1;
        float treshold_1 = 0.f;
        float treshold_2 = 0.f;
        float treshold_3 = 0.f;
        bool adapt_min_neighbors = false;
        bool double_check = true;
        bool drop_detect = true;
        int min_num_detect = 1;
        bool device_info = false;
        int cuda_device_id = 0;
        int cl_platform_id = -1;
        int cl_device_id = -1;
        int concurrent_kernels = 3;
        int num_cnn_copy = 1;
        bool blur = false;
        ImgResize img_resize = ImgResize::NearestNeighbor;
        bool uniform_noise = false;
        bool merger_detect = true;
        std::string path_model[4];
        int index_output[4];
        AdvancedParam() {
            index_output[0] = 1;
            index_output[1] = 0;
            index_output[2] = 0;
            index_output[3] = -1;
        }
    };
    struct FacialData {
        Point landmarks[5];
        int gender = -1;
        int smile = -1;
        int glasses = -1;
    };
    struct Detection {
        Rect rect;
        float score = 0.f;
        float scale = 0.f;
        int knn = 0;
        int num_detect = 0;
        std::vector<FacialData> facial_data;
        Detection() {}
        Detection(int x, int y, int w, int h, float s, float sc, int k) : rect(x, y, w, h), score(s), scale(sc), knn(k) {}
        Detection(Rect r, float s, float sc, int k) : rect(r), score(s), scale(sc), knn(k) {}
    };

    // CNNDetector(Param*, AdvancedParam*) initialises at once, as the reference does (cnn_detector_v3.cpp:45-61)
    explicit CNNDetector(Param* param = nullptr, AdvancedParam* advanced_param = nullptr) {
        if (param) param_ = *param;
        if (advanced_param) advanced_param_ = *advanced_param;
        Init();
    }
    ~CNNDetector() { Clear(); }
    CNNDetector(const CNNDetector&) = delete;
    CNNDetector& operator=(const CNNDetector&) = delete;

    bool isEmpty() const { return h_ == nullptr; }

    // Detect (cnn_detector_v3.cpp:2483-2813): 0 on success, -1 on failure. Detections already in the
    // vector stay in front of the new ones through the merges, as in the reference.
    int Detect(std::vector<Detection>& detections, SIMD::Image_8u& image) {
        if (isEmpty() && Init() < 0) return -1;
        ccnn_image im{image.width, image.height, image.nChannel, image.data, (size_t)image.widthStep};
        std::vector<ccnn_detection> prior(detections.size());
        for (size_t i = 0; i < detections.size(); ++i) prior[i] = to_c(detections[i]);
        std::vector<ccnn_detection> out(4096);
        int n = 0;
        ccnn_status st = ccnn_cnn_detect(h_, &im, prior.data(), (int)prior.size(), out.data(), (int)out.size(), &n);
        if (st == CCNN_TRUNCATED) {
            out.resize((size_t)n);
            st = ccnn_cnn_detect(h_, &im, prior.data(), (int)prior.size(), out.data(), (int)out.size(), &n);
        }
        if (st < 0) return -1;
        detections.clear();
        for (int i = 0; i < n; ++i) detections.push_back(from_c(out[i]));
        return 0;
    }

    // NMS(detections, rect) = Merger(detections, rect, 0.5): rect's clusters are appended to detections
    void NMS(std::vector<Detection>& detections, std::vector<Detection>& rect) {
        if (isEmpty() && Init() < 0) return;
        std::vector<ccnn_detection> in(rect.size()), out(rect.size() + 1);
        for (size_t i = 0; i < rect.size(); ++i) in[i] = to_c(rect[i]);
        int n = 0;
        if (ccnn_cnn_nms(h_, in.data(), (int)in.size(), out.data(), (int)out.size(), &n) < 0) return;
        for (int i = 0; i < n; ++i) detections.push_back(from_c(out[i]));
    }

    Param getParam() const {
        Param p = param_;
        if (isEmpty()) return p;
        ccnn_cnn_param c;
        if (ccnn_cnn_get_params(h_, &c, nullptr) == CCNN_OK) {
            p.pipeline = (Pipeline)c.pipeline;
            p.max_image_size = Size(c.max_image_width, c.max_image_height);
        }
        return p;
    }
    void setParam(Param& param) {
        param_ = param;
        set();
    }
    AdvancedParam getAdvancedParam() const {
        AdvancedParam a = advanced_param_;
        if (isEmpty()) return a;
        ccnn_cnn_advanced_param c;
        if (ccnn_cnn_get_params(h_, nullptr, &c) == CCNN_OK) {
            a.packet_detection = c.packet_detection != 0;
            a.gray_image_only = c.gray_image_only != 0;
            a.facial_analysis = c.facial_analysis != 0;
            a.equalize = c.equalize != 0;
            a.reflection = c.reflection != 0;
            a.type_check = c.type_check;
            a.adapt_min_neighbors = c.adapt_min_neighbors != 0;
            a.double_check = c.double_check != 0;
            a.drop_detect = c.drop_detect != 0;
            a.min_num_detect = c.min_num_detect;
            a.blur = c.blur != 0;
            a.uniform_noise = c.uniform_noise != 0;
            a.merger_detect = c.merger_detect != 0;
        }
        return a;
    }
    void setAdvancedParam(AdvancedParam& advanced_param) {
        advanced_param_ = advanced_param;
        set();
    }
    Size getMaxImageSize() const { return getParam().max_image_size; }
    void setMaxImageSize(Size s) {
        param_.max_image_size = s;
        set();
    }
    Size getMinObjectSize() const { return param_.min_obj_size; }
    void setMinObjectSize(Size s) {
        param_.min_obj_size = s;
        set();
    }
    Size getMaxObjectSize() const { return param_.max_obj_size; }
    void setMaxObjectSize(Size s) {
        param_.max_obj_size = s;
        set();
    }
    int getNumThreads() const { return param_.num_threads; }
    void setNumThreads(int n) {
        param_.num_threads = n;
        set();
    }

    // getGrayImage (cnn_detector_v3.cpp:2455-2470): the fp32 gray image of the last frame
    int getGrayImage(SIMD::Image_32f* image) const {
        if (isEmpty() || image == nullptr) return -1;
        const float* d = nullptr;
        int w = 0, h = 0;
        size_t step = 0;
        if (ccnn_get_gray_device(h_, &d, &w, &h, &step) != CCNN_OK) return -1;
        gray_.resize((size_t)w * h);
        if (ccnn_get_gray_host(h_, gray_.data(), (int)gray_.size(), &w, &h) != CCNN_OK) return -1;
        *image = SIMD::Image_32f(w, h, 1, gray_.data(), w);
        return 0;
    }

   private:
    ccnn_handle h_ = nullptr;
    Param param_;
    AdvancedParam advanced_param_;
    mutable std::vector<float> gray_;

    int Init() {
        ccnn_cnn_param p;
        ccnn_cnn_advanced_param a;
        to_c(param_, advanced_param_, &p, &a);
        const char* models[3];
        for (int i = 0; i < 3; ++i) models[i] = advanced_param_.path_model[i].empty() ? nullptr : advanced_param_.path_model[i].c_str();
        return ccnn_cnn_create(&p, &a, models, &h_) == CCNN_OK ? 0 : (h_ = nullptr, -1);
    }
    void Clear() {
        if (h_) ccnn_destroy(h_);
        h_ = nullptr;
    }
    // the setters clear the detector; the next Detect initialises it again (cnn_detector_v3.h:407-436)
    void set() { Clear(); }

    static void to_c(const Param& q, const AdvancedParam& b, ccnn_cnn_param* p, ccnn_cnn_advanced_param* a) {
        ccnn_cnn_default_params(p, a);
        p->pipeline = (int)q.pipeline;
        p->max_image_width = q.max_image_size.width;
        p->max_image_height = q.max_image_size.height;
        p->min_obj_width = q.min_obj_size.width;
        p->min_obj_height = q.min_obj_size.height;
        p->max_obj_width = q.max_obj_size.width;
        p->max_obj_height = q.max_obj_size.height;
        p->scale_factor = q.scale_factor;
        p->min_neighbors = q.min_neighbors;
        p->num_threads = q.num_threads;
        a->detect_mode = (int)b.detect_mode;
        a->detect_precision = (int)b.detect_precision;
        a->packet_detection = b.packet_detection;
        a->gray_image_only = b.gray_image_only;
        a->facial_analysis = b.facial_analysis;
        a->equalize = b.equalize;
        a->reflection = b.reflection;
        a->type_check = b.type_check;
        a->treshold_1 = b.treshold_1;
        a->treshold_2 = b.treshold_2;
        a->treshold_3 = b.treshold_3;
        a->adapt_min_neighbors = b.adapt_min_neighbors;
        a->double_check = b.double_check;
        a->drop_detect = b.drop_detect;
        a->min_num_detect = b.min_num_detect;
        a->device_info = b.device_info;
        a->cuda_device_id = b.cuda_device_id;
        a->cl_platform_id = b.cl_platform_id;
        a->cl_device_id = b.cl_device_id;
        a->concurrent_kernels = b.concurrent_kernels;
        a->num_cnn_copy = b.num_cnn_copy;
        a->blur = b.blur;
        a->img_resize = (int)b.img_resize;
        a->uniform_noise = b.uniform_noise;
        a->merger_detect = b.merger_detect;
        for (int i = 0; i < 4; ++i) a->index_output[i] = b.index_output[i];
    }
    static ccnn_detection to_c(const Detection& d) {
        ccnn_detection c;
        c.x = d.rect.x;
        c.y = d.rect.y;
        c.width = d.rect.width;
        c.height = d.rect.height;
        c.score = d.score;
        c.scale = d.scale;
        c.knn = d.knn;
        c.num_detect = d.num_detect;
        return c;
    }
    static Detection from_c(const ccnn_detection& c) {
        Detection d(c.x, c.y, c.width, c.height, c.score, c.scale, c.knn);
        d.num_detect = c.num_detect;
        return d;
    }
};

}  // namespace NeuralNetworksLib
