// Headless use of the C++ facade the way the reference's demo uses its library
// (src/FaceDetector/main.cpp: Param, Init, Detect into a caller-owned Face[1000] buffer), then every
// getter and setter, then the process-global (singleton) semantics.
// Prints "init <rc>", one "face x y w h score" line per face, and tagged lines for the rest.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "CompactCNNLib.h"
#include "../compactcnncascade_b200/csrc/synth_frame.h"

using namespace CompactCNNLib;

static void print_faces(const char* tag, FaceDetector& d, FaceDetector::ImageData& img) {
    FaceDetector::Face faces[1000];
    const int n = d.Detect(faces, img);
    printf("%s %d\n", tag, n);
    for (int i = 0; i < n; ++i) printf("face %d %d %d %d %.6f\n", faces[i].x, faces[i].y, faces[i].width, faces[i].height, faces[i].score);
}

int main(int argc, char** argv) {
    const int w = argc > 1 ? atoi(argv[1]) : 640, h = argc > 2 ? atoi(argv[2]) : 480;
    const unsigned long long seed = argc > 3 ? strtoull(argv[3], nullptr, 10) : 0;
    const char* mode = argc > 4 ? argv[4] : "basic";
    std::vector<unsigned char> frame((size_t)w * h * 3);
    ccnn_synth_frame(frame.data(), w, h, 3, w * 3, seed, 5, 40, 200, nullptr);
    FaceDetector::ImageData img(w, h, 3, frame.data(), (size_t)w * 3);

    FaceDetector::Param param;
    param.max_image_size = FaceDetector::Size(w, h);
    param.min_face_height = 40;
    param.max_face_height = 240;
    param.detect_mode = FaceDetector::DetectMode::sync;

    if (!strcmp(mode, "singleton")) {
        // the reference's process-global detector: one Init serves every instance, one Clear ends it
        FaceDetector::setSingleton(true);
        FaceDetector a, b;
        const int rc = a.Init(param);
        printf("init %d\n", rc);
        if (rc < 0) return 0;
        printf("shared %d %d\n", a.isEmpty() ? 0 : 1, b.isEmpty() ? 0 : 1);
        print_faces("b_detect", b, img);
        FaceDetector::Param q = param;
        q.min_face_height = 60;
        b.Init(q);  // replaces the detector `a` uses too
        printf("a_min %d\n", a.getMinObjectHeight());
        print_faces("a_detect", a, img);
        b.Clear();
        printf("after_clear %d %d\n", a.isEmpty() ? 1 : 0, b.isEmpty() ? 1 : 0);
        FaceDetector::Face f[4];
        printf("a_detect_cleared %d\n", a.Detect(f, img));
        return 0;
    }

    FaceDetector detector;
    const int rc = detector.Init(param);
    printf("init %d\n", rc);
    if (rc < 0) return 0;
    print_faces("detect", detector, img);
    FaceDetector::ImageData gray;
    const int grc = detector.getGrayImage32F(&gray, FaceDetector::Pipeline::CPU);
    printf("gray %d %d %dx%d\n", grc, gray.channels, gray.cols, gray.rows);
    if (!strcmp(mode, "setters")) {
        FaceDetector::Param g = detector.getParam();
        printf("param %d %d %d %d %.4f %d\n", g.max_image_size.width, g.max_image_size.height, g.min_face_height, g.max_face_height,
               g.scale_factor, g.num_threads);
        detector.setMinObjectHeight(60);
        printf("min %d\n", detector.getMinObjectHeight());
        print_faces("detect_min60", detector, img);
        detector.setMaxObjectHeight(120);
        printf("max %d\n", detector.getMaxObjectHeight());
        print_faces("detect_min60_max120", detector, img);
        detector.setNumThreads(3);
        printf("threads %d\n", detector.getNumThreads());
        detector.setMaxImageSize(FaceDetector::Size(w / 2, h / 2));
        FaceDetector::Size m = detector.getMaxImageSize();
        printf("maxsize %d %d\n", m.width, m.height);
        print_faces("detect_grown", detector, img);  // a larger frame re-initialises at its own size
        m = detector.getMaxImageSize();
        printf("maxsize_after %d %d\n", m.width, m.height);
        FaceDetector::Param q = param;
        q.scale_factor = 1.1f;
        q.min_face_height = 50;
        detector.setParam(q);
        g = detector.getParam();
        printf("param2 %d %.4f\n", g.min_face_height, g.scale_factor);
        print_faces("detect_param2", detector, img);
        const int crc = detector.Clear();
        printf("clear %d %d\n", crc, detector.isEmpty() ? 1 : 0);
        FaceDetector::Face f[4];
        printf("detect_cleared %d\n", detector.Detect(f, img));
    }
    return 0;
}
