/* compactcnncascade_b200 — C ABI of the cascade's internal detector class
 *
 *   namespace NeuralNetworksLib { class CNNDetector }  (src/CNNObjectDetector/cnn_detector_v3.h:82-453)
 *
 * the class below the public FaceDetector: its own Param / AdvancedParam (every switch of the
 * cascade, not only what FaceDetector::Param exposes) and raw Detection results carrying the merged
 * scale, neighbour count (knn) and cluster size (num_detect). The header-only C++ facade
 * include/CNNDetector.h restores the class on top of these calls. Handles are the same ccnn_handle
 * as ccnn.h's, so ccnn_get_gray_device / ccnn_get_gray_host / ccnn_destroy apply to them too.
 */
#ifndef CCNN_CNN_H
#define CCNN_CNN_H

#include "ccnn.h"
#include "ccnn_inspect.h"

#ifdef __cplusplus
extern "C" {
#endif

/* CNNDetector::Param (cnn_detector_v3.h:114-123). Only the heights of the object sizes are used, as
 * in the reference (InitScales, cnn_detector_v3.cpp:289-346). */
typedef struct {
    int pipeline;                           /* CCNN_PIPELINE_*; every value runs on the GPU */
    int max_image_width, max_image_height;
    int min_obj_width, min_obj_height;
    int max_obj_width, max_obj_height;      /* 0 = no limit */
    float scale_factor;
    int min_neighbors;
    int num_threads;                        /* accepted and reported back; the cascade runs on the device */
} ccnn_cnn_param;

/* CNNDetector::AdvancedParam (cnn_detector_v3.h:124-175). The precision rules of CNNDetector::Init
 * (cnn_detector_v3.cpp:922-963) are applied on top, exactly as the reference does: detect_precision
 * sets type_check, `def` also resets most switches, `ultra` sets min_num_detect = 2, and detect_mode
 * disable or facial_analysis turn drop_detect off. */
typedef struct {
    int detect_mode;                        /* CCNN_DETECT_* */
    int detect_precision;                   /* CCNN_PRECISION_* */
    int packet_detection;                   /* all pyramid levels in one device launch per kernel: what the
                                               reference's level atlas is for; results are those of the
                                               level-by-level cascade */
    int gray_image_only;
    int facial_analysis;
    int equalize, reflection;
    int type_check;                         /* overridden by detect_precision, as in the reference */
    float treshold_1, treshold_2, treshold_3;
    int adapt_min_neighbors, double_check, drop_detect, min_num_detect;
    int device_info, cuda_device_id, cl_platform_id, cl_device_id;
    int concurrent_kernels, num_cnn_copy;   /* accepted and reported back */
    int blur;                               /* must be 0 (CCNN_ERR_UNSUPPORTED otherwise) */
    int img_resize;                         /* accepted; the level resize follows the scale, as in the reference */
    int uniform_noise;                      /* must be 0 (CCNN_ERR_UNSUPPORTED otherwise) */
    int merger_detect;
    int index_output[4];                    /* output neuron of stage 1, 2, 3 and the landmark net */
} ccnn_cnn_advanced_param;

/* The member defaults of CNNDetector::Param and AdvancedParam (cnn_detector_v3.h:114-175). */
CCNN_API void ccnn_cnn_default_params(ccnn_cnn_param* p, ccnn_cnn_advanced_param* ap);

/* CNNDetector::CNNDetector(Param*, AdvancedParam*) followed by Init (cnn_detector_v3.cpp:42-61,
 * 907-985). model_paths[0..2] (nullable, or the whole array NULL) are the three cascade stages, as
 * AdvancedParam::path_model[0..2]; empty entries take the bundled models (the reference embeds the
 * same files). The landmark net of facial analysis is always the bundled one. */
CCNN_API ccnn_status ccnn_cnn_create(const ccnn_cnn_param* p, const ccnn_cnn_advanced_param* ap, const char* const* model_paths,
                                     ccnn_handle* out);

/* CNNDetector::Detect(std::vector<Detection>& detections, Image_8u& image) (cnn_detector_v3.cpp:2483-2813).
 * `prior` / `n_prior` are the detections the caller's vector already holds: the reference keeps them
 * in front of the new clusters of the first merge, so they take part in the min_num_detect filter and
 * the second merge (and are rescaled with the rest when the input frame is shrunk); with no new raw
 * detection they are returned unchanged. At most `capacity` detections are written to `out`, the
 * total goes to *n (CCNN_TRUNCATED if it did not fit). `prior` may alias `out`. */
CCNN_API ccnn_status ccnn_cnn_detect(ccnn_handle h, const ccnn_image* img, const ccnn_detection* prior, int n_prior, ccnn_detection* out,
                                     int capacity, int* n);

/* CNNDetector::NMS(detections, rect) = Merger(detections, rect, 0.5) (cnn_detector_v3.h:401-404,
 * cnn_detector_v3.cpp:2814-2936), run on the handle's device: the clusters of `rect` in the
 * reference's order (the caller appends them to its vector). */
CCNN_API ccnn_status ccnn_cnn_nms(ccnn_handle h, const ccnn_detection* rect, int n_rect, ccnn_detection* out, int capacity, int* n_out);

/* getParam / getAdvancedParam and setParam / setAdvancedParam (cnn_detector_v3.h:406-416): a setter
 * clears the detector and the next Detect initialises it again. Either pointer may be NULL. The
 * getters report the values in force, after Init's precision rules and Detect's re-initialisations
 * (max image size, gray_image_only). */
CCNN_API ccnn_status ccnn_cnn_get_params(ccnn_handle h, ccnn_cnn_param* p, ccnn_cnn_advanced_param* ap);
CCNN_API ccnn_status ccnn_cnn_set_params(ccnn_handle h, const ccnn_cnn_param* p, const ccnn_cnn_advanced_param* ap);

#ifdef __cplusplus
}
#endif
#endif /* CCNN_CNN_H */
