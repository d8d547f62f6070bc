// Header-only C++ facade with the reference's public class
//   namespace CompactCNNLib { class FaceDetector }   (src/CNNObjectDetector/CompactCNNLibAPI_v2.h:35-190)
// implemented over the C ABI of ccnn.h, so reference callers recompile against this header and link
// libccnn.so instead of the reference library. Same nested types, field names, defaults, method
// names and return conventions (0 / -1, Detect returns the face count or -1).
//
// Differences a caller can observe:
//  * instances are independent detectors by default. The reference shares one process-global
//    detector behind one mutex (CompactCNNLibAPI_v2.cpp:32-33): every instance's Init replaces it,
//    every Clear (and destructor) deletes it. FaceDetector::setSingleton(true), called before the
//    first Init, or defining CCNN_FACEDETECTOR_SINGLETON before including this header, gives exactly
//    those semantics;
//  * Param::models are honoured when set (the reference ignores them and always uses its embedded
//    models, which are the same files as the bundled defaults);
//  * Detect writes at most `capacity` faces (default 1000, the demos' buffer size) and returns the
//    total count; the reference has no capacity argument;
//  * getGrayImage32F(img, GPU) returns the device buffer, as the reference's GPU pipeline does;
//    with Pipeline::CPU it returns a host copy owned by the facade;
//  * CNTKDump2Binary reports nothing on failure, like the reference; ccnn_cntk_dump_to_binary returns a status.
#pragma once

#include <cstddef>
#include <mutex>
#include <vector>

#include "ccnn.h"
#include "ccnn_inspect.h"

namespace CompactCNNLib {

class FaceDetector {
   public:
    enum struct Pipeline { CPU = 0, GPU = 1, GPU_CPU = 2 };
    enum struct DetectMode { disable = 0, sync = 1, async = 2 };
    enum struct DetectPrecision { def = 0, low = 1, normal = 2, high = 3, ultra = 4 };

    struct Size {
        int width = 0;
        int height = 0;
        Size() = default;
        Size(int w, int h) : width(w), height(h) {}
    };
    struct Face {
        int x = 0, y = 0, width = 0, height = 0;
        float score = 0.f;
        int gender = -1, smile = -1, glasses = -1;
        Face() = default;
        Face(int _x, int _y, int _w, int _h, float _s = 0.f) : x(_x), y(_y), width(_w), height(_h), score(_s) {}
    };
    struct ImageData {
        int cols = 0, rows = 0, channels = 0;
        unsigned char* data = nullptr;
        size_t step = 0;
        ImageData() = default;
        ImageData(int c, int r, int ch, unsigned char* d, size_t s) : cols(c), rows(r), channels(ch), data(d), step(s) {}
    };
    struct Param {
        Size max_image_size = Size(1920, 1080);
        int min_face_height = 80;
        int max_face_height = 0;
        float scale_factor = 1.15f;
        int min_neighbors = 2;
        DetectPrecision detect_precision = DetectPrecision::high;
        float treshold[3];
        bool drop_detect = true;
        bool equalize = true;
        bool reflection = true;
        Pipeline pipeline = Pipeline::GPU;
        DetectMode detect_mode = DetectMode::async;
        int num_threads = 2;
        const char* models[3];
        int index_output[3];
        bool device_info = true;
        int cuda_device_id = 0;
        int cl_platform_id = -1;
        int cl_device_id = -1;
        bool facial_analysis = false;
        Param() {
            treshold[0] = -1.5f;
            treshold[1] = -1.25f;
            treshold[2] = -1.0f;
            models[0] = models[1] = models[2] = nullptr;
            index_output[0] = 1;
            index_output[1] = 0;
            index_output[2] = 0;
        }
    };

    FaceDetector() = default;
    ~FaceDetector() { Clear(); }
    FaceDetector(const FaceDetector&) = delete;
    FaceDetector& operator=(const FaceDetector&) = delete;

    // The reference's process-global detector (CompactCNNLibAPI_v2.cpp:32-33) instead of one detector
    // per instance; switch it before the first Init of the process.
    static void setSingleton(bool on) { global().singleton = on; }
    static bool isSingleton() { return global().singleton; }

    int Init(Param& param) {
        if (!isEmpty()) Clear();
        Lock lk(this);
        param_ = param;
        if (global().singleton) global().param = param;
        ccnn_params p = to_c(param);
        ccnn_handle& h = handle();
        return ccnn_create(&p, param.models, &h) == CCNN_OK ? 0 : (h = nullptr, -1);
    }

    int Detect(Face* faces, ImageData& img, int capacity = 1000) {
        if (isEmpty() || faces == nullptr) return -1;
        Lock lk(this);
        ccnn_image im{img.cols, img.rows, img.channels, img.data, img.step};
        std::vector<ccnn_face> out((size_t)(capacity > 0 ? capacity : 1));
        int n = 0;
        ccnn_status st = ccnn_detect(handle(), &im, out.data(), capacity, &n);
        if (st < 0) return -1;
        for (int i = 0; i < n && i < capacity; ++i) {
            faces[i] = Face(out[i].x, out[i].y, out[i].width, out[i].height, out[i].score);
            faces[i].gender = out[i].gender;  // facial analysis (else -1)
            faces[i].smile = out[i].smile;
            faces[i].glasses = out[i].glasses;
        }
        return n;
    }

    // FaceDetector::CNTKDump2Binary (CompactCNNLibAPI_v2.cpp:509-519)
    static void CNTKDump2Binary(const char* binary_file, const char* cntk_model_dump) {
        ccnn_cntk_dump_to_binary(binary_file, cntk_model_dump);
    }

    int Clear() {
        if (isEmpty()) return -1;
        Lock lk(this);
        ccnn_handle& h = handle();
        ccnn_destroy(h);
        h = nullptr;
        return 0;
    }

    bool isEmpty() const { return handle() == nullptr; }

    Param getParam() const {
        const Param& mine = global().singleton ? global().param : param_;
        if (isEmpty()) return mine;
        ccnn_params p;
        ccnn_get_params(handle(), &p);
        Param r = mine;
        r.max_image_size = Size(p.max_image_width, p.max_image_height);
        r.min_face_height = p.min_face_height;
        r.max_face_height = p.max_face_height;
        r.scale_factor = p.scale_factor;
        r.num_threads = p.num_threads;
        return r;
    }
    void setParam(Param& param) {
        param_ = param;
        if (global().singleton) global().param = param;
        if (isEmpty()) return;
        ccnn_params p = to_c(param);
        ccnn_set_params(handle(), &p);
    }

    Size getMaxImageSize() const { return getParam().max_image_size; }
    void setMaxImageSize(Size s) {
        if (!isEmpty()) ccnn_set_max_image_size(handle(), s.width, s.height);
    }
    int getMinObjectHeight() const { return getParam().min_face_height; }
    void setMinObjectHeight(int v) {
        if (!isEmpty()) ccnn_set_min_object_height(handle(), v);
    }
    int getMaxObjectHeight() const { return getParam().max_face_height; }
    void setMaxObjectHeight(int v) {
        if (!isEmpty()) ccnn_set_max_object_height(handle(), v);
    }
    int getNumThreads() const { return getParam().num_threads; }
    void setNumThreads(int v) {
        if (!isEmpty()) ccnn_set_num_threads(handle(), v);
    }

    int getGrayImage32F(ImageData* img, Pipeline pipeline) {
        if (isEmpty() || img == nullptr) return -1;
        const float* d = nullptr;
        int w = 0, h = 0;
        size_t step = 0;
        if (ccnn_get_gray_device(handle(), &d, &w, &h, &step) != CCNN_OK) return -1;
        if (pipeline == Pipeline::CPU) {
            gray_host_.resize((size_t)w * h);
            if (ccnn_get_gray_host(handle(), gray_host_.data(), (int)gray_host_.size(), &w, &h) != CCNN_OK) return -1;
            *img = ImageData(w, h, 1, reinterpret_cast<unsigned char*>(gray_host_.data()), sizeof(float) * (size_t)w);
        } else {
            *img = ImageData(w, h, 1, reinterpret_cast<unsigned char*>(const_cast<float*>(d)), step);
        }
        return 0;
    }

   private:
    ccnn_handle h_ = nullptr;
    Param param_;
    std::vector<float> gray_host_;

    // the process-global detector and its mutex, used when the singleton semantics are on
    struct Global {
#ifdef CCNN_FACEDETECTOR_SINGLETON
        bool singleton = true;
#else
        bool singleton = false;
#endif
        ccnn_handle h = nullptr;
        Param param;
        std::recursive_mutex mu;
    };
    static Global& global() {
        static Global g;
        return g;
    }
    ccnn_handle& handle() { return global().singleton ? global().h : h_; }
    ccnn_handle handle() const { return global().singleton ? global().h : h_; }
    // serialises Init / Detect / Clear across instances in singleton mode, as the reference's mutex does
    struct Lock {
        std::unique_lock<std::recursive_mutex> lk;
        explicit Lock(const FaceDetector*) {
            if (global().singleton) lk = std::unique_lock<std::recursive_mutex>(global().mu);
        }
    };

    static ccnn_params to_c(const Param& q) {
        ccnn_params p;
        ccnn_default_params(&p);
        p.max_image_width = q.max_image_size.width;
        p.max_image_height = q.max_image_size.height;
        p.min_face_height = q.min_face_height;
        p.max_face_height = q.max_face_height;
        p.scale_factor = q.scale_factor;
        p.min_neighbors = q.min_neighbors;
        p.detect_precision = (int)q.detect_precision;
        for (int i = 0; i < 3; ++i) {
            p.treshold[i] = q.treshold[i];
            p.index_output[i] = q.index_output[i];
        }
        p.drop_detect = q.drop_detect;
        p.equalize = q.equalize;
        p.reflection = q.reflection;
        p.pipeline = (int)q.pipeline;
        p.detect_mode = (int)q.detect_mode;
        p.num_threads = q.num_threads;
        p.device_info = q.device_info;
        p.cuda_device_id = q.cuda_device_id;
        p.cl_platform_id = q.cl_platform_id;
        p.cl_device_id = q.cl_device_id;
        p.facial_analysis = q.facial_analysis;
        return p;
    }
};

}  // namespace CompactCNNLib
