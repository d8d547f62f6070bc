// Headless use of the C++ facade the way the reference's demo uses its library
// (src/FaceDetector/main.cpp: Param, Init, Detect into a caller-owned Face[1000] buffer).
// Prints "init <rc>" and then one line per face.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "CompactCNNLib.h"
#include "../compactcnncascade_b200/csrc/synth_frame.h"

using namespace CompactCNNLib;

int main(int argc, char** argv) {
    const int w = argc > 1 ? atoi(argv[1]) : 640, h = argc > 2 ? atoi(argv[2]) : 480;
    const unsigned long long seed = argc > 3 ? strtoull(argv[3], nullptr, 10) : 0;
    std::vector<unsigned char> frame((size_t)w * h * 3);
    ccnn_synth_frame(frame.data(), w, h, 3, w * 3, seed, 5, 40, 200, nullptr);

    FaceDetector::Param param;
    param.max_image_size = FaceDetector::Size(w, h);
    param.min_face_height = 40;
    param.max_face_height = 240;
    param.detect_mode = FaceDetector::DetectMode::sync;
    FaceDetector detector;
    const int rc = detector.Init(param);
    printf("init %d\n", rc);
    if (rc < 0) return 0;
    FaceDetector::Face faces[1000];
    FaceDetector::ImageData img(w, h, 3, frame.data(), (size_t)w * 3);
    const int n = detector.Detect(faces, img);
    for (int i = 0; i < n; ++i) printf("%d %d %d %d %.6f\n", faces[i].x, faces[i].y, faces[i].width, faces[i].height, faces[i].score);
    FaceDetector::ImageData gray;
    const int grc = detector.getGrayImage32F(&gray, FaceDetector::Pipeline::CPU);
    printf("gray %d %d %dx%d\n", grc, gray.channels, gray.cols, gray.rows);
    return 0;
}
