// Use of the internal-class facade (include/CNNDetector.h) the way code written against the
// reference's NeuralNetworksLib::CNNDetector does: Param + AdvancedParam, Detect into a vector of
// Detection (optionally holding detections already), NMS, the getters.
//   cnndetector_example W H SEED CHANNELS [key=value ...] [prior=x,y,w,h,score,scale,knn,num_detect ...] [nms=1]
// keys: min_obj, max_obj, sf, min_neighbors, precision, mode, t1, t2, t3, gray_only, equalize,
//       reflection, adapt, double_check, drop, min_num, merger, pipeline, packet
// Prints "rc <rc>", one "det x y w h score scale knn num_detect" line per detection, then the
// advanced parameters in force ("adv ..."), and with nms=1 the NMS clusters of the result ("nms ...").
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "CNNDetector.h"
#include "../compactcnncascade_b200/csrc/synth_frame.h"

using namespace NeuralNetworksLib;

static void print_det(const char* tag, const CNNDetector::Detection& d) {
    printf("%s %d %d %d %d %.9g %.9g %d %d\n", tag, d.rect.x, d.rect.y, d.rect.width, d.rect.height, d.score, d.scale, d.knn, d.num_detect);
}

int main(int argc, char** argv) {
    if (argc < 5) return 2;
    const int w = atoi(argv[1]), h = atoi(argv[2]), ch = atoi(argv[4]);
    const unsigned long long seed = strtoull(argv[3], nullptr, 10);
    std::vector<unsigned char> frame((size_t)w * h * ch);
    ccnn_synth_frame(frame.data(), w, h, ch, w * ch, seed, 5, 40, 200, nullptr);

    CNNDetector::Param p;
    CNNDetector::AdvancedParam a;
    p.max_image_size = Size(w, h);
    std::vector<CNNDetector::Detection> dets;
    bool nms = false;
    for (int i = 5; i < argc; ++i) {
        std::string kv = argv[i];
        const size_t eq = kv.find('=');
        if (eq == std::string::npos) return 2;
        const std::string k = kv.substr(0, eq);
        const char* v = kv.c_str() + eq + 1;
        if (k == "min_obj") p.min_obj_size = Size(atoi(v), atoi(v));
        else if (k == "max_obj") p.max_obj_size = Size(atoi(v), atoi(v));
        else if (k == "sf") p.scale_factor = (float)atof(v);
        else if (k == "min_neighbors") p.min_neighbors = atoi(v);
        else if (k == "pipeline") p.pipeline = (CNNDetector::Pipeline)atoi(v);
        else if (k == "precision") a.detect_precision = (CNNDetector::DetectPrecision)atoi(v);
        else if (k == "mode") a.detect_mode = (CNNDetector::DetectMode)atoi(v);
        else if (k == "t1") a.treshold_1 = (float)atof(v);
        else if (k == "t2") a.treshold_2 = (float)atof(v);
        else if (k == "t3") a.treshold_3 = (float)atof(v);
        else if (k == "gray_only") a.gray_image_only = atoi(v) != 0;
        else if (k == "equalize") a.equalize = atoi(v) != 0;
        else if (k == "reflection") a.reflection = atoi(v) != 0;
        else if (k == "adapt") a.adapt_min_neighbors = atoi(v) != 0;
        else if (k == "double_check") a.double_check = atoi(v) != 0;
        else if (k == "drop") a.drop_detect = atoi(v) != 0;
        else if (k == "min_num") a.min_num_detect = atoi(v);
        else if (k == "merger") a.merger_detect = atoi(v) != 0;
        else if (k == "packet") a.packet_detection = atoi(v) != 0;
        else if (k == "nms") nms = atoi(v) != 0;
        else if (k == "prior") {
            int x, y, ww, hh, knn, nd;
            float score, scale;
            if (sscanf(v, "%d,%d,%d,%d,%f,%f,%d,%d", &x, &y, &ww, &hh, &score, &scale, &knn, &nd) != 8) return 2;
            CNNDetector::Detection d(x, y, ww, hh, score, scale, knn);
            d.num_detect = nd;
            dets.push_back(d);
        } else
            return 2;
    }

    CNNDetector det(&p, &a);
    if (det.isEmpty()) {
        printf("rc -1\n");
        return 0;
    }
    SIMD::Image_8u image(w, h, ch, frame.data(), w * ch);
    const int rc = det.Detect(dets, image);
    printf("rc %d\n", rc);
    for (auto& d : dets) print_det("det", d);
    const CNNDetector::AdvancedParam g = det.getAdvancedParam();
    const CNNDetector::Param gp = det.getParam();
    printf("adv %d %d %d %d %d %d %d %d %d %d %d\n", g.type_check, g.drop_detect ? 1 : 0, g.gray_image_only ? 1 : 0, g.adapt_min_neighbors ? 1 : 0,
           g.double_check ? 1 : 0, g.min_num_detect, g.merger_detect ? 1 : 0, g.equalize ? 1 : 0, g.reflection ? 1 : 0,
           g.packet_detection ? 1 : 0, (int)gp.pipeline);
    printf("size %d %d\n", gp.max_image_size.width, gp.max_image_size.height);
    if (nms) {
        std::vector<CNNDetector::Detection> rect = dets, out;
        for (auto& d : dets) {  // shifted copies that merge with their originals
            CNNDetector::Detection e = d;
            e.rect = Rect(d.rect.x + d.rect.width / 10, d.rect.y + 1, d.rect.width, d.rect.height);
            rect.push_back(e);
        }
        det.NMS(out, rect);
        for (auto& d : out) print_det("nms", d);
    }
    SIMD::Image_32f gray;
    printf("gray %d %dx%d\n", det.getGrayImage(&gray), gray.width, gray.height);
    return 0;
}
