/* compactcnncascade_b200 — C ABI of the B200 face-detection cascade.
 *
 * This is the drop-in boundary for the reference's public API
 *   namespace CompactCNNLib { class FaceDetector }  (src/CNNObjectDetector/CompactCNNLibAPI_v2.h:35-190,
 *   identical shape in prebuild/include/CompactCNNLib.h:36-194)
 * flattened to plain C: opaque handles instead of the process-global singleton, explicit output
 * capacities, status codes instead of -1/printf. The header-only C++ facade include/CompactCNNLib.h
 * restores the reference's class on top of these calls.
 *
 * All compute runs on one CUDA device through hand-written sm_100a kernels; there is no CPU
 * fallback: calls fail with CCNN_ERR_CUDA when the device or the kernels are unavailable.
 */
#ifndef CCNN_H
#define CCNN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCNN_API __attribute__((visibility("default")))

typedef enum {
    CCNN_OK = 0,
    CCNN_TRUNCATED = 1,          /* more faces than the output capacity; the first `capacity` were written */
    CCNN_PENDING = 2,            /* serving loop: the frame is not finished yet (ccnn_server_poll) */
    CCNN_BUSY = 3,               /* serving loop: the request queue is full; submit again later */
    CCNN_ERR_INVALID_ARG = -1,
    CCNN_ERR_MODEL = -2,         /* model file missing, truncated, wrong format version or unsupported shape */
    CCNN_ERR_CONFIG = -3,        /* parameters give an empty scale list (reference: "Invalid configuration") */
    CCNN_ERR_CUDA = -4,          /* CUDA runtime / device failure; see ccnn_last_error() */
    CCNN_ERR_OOM = -5,           /* device memory exhausted */
    CCNN_ERR_UNSUPPORTED = -6    /* e.g. an image with other than 1, 3 or 4 channels */
} ccnn_status;

typedef struct ccnn_detector* ccnn_handle;

/* FaceDetector::Pipeline / DetectMode / DetectPrecision values (CompactCNNLibAPI_v2.h:38-57) */
enum { CCNN_PIPELINE_CPU = 0, CCNN_PIPELINE_GPU = 1, CCNN_PIPELINE_GPU_CPU = 2 };
enum { CCNN_DETECT_DISABLE = 0, CCNN_DETECT_SYNC = 1, CCNN_DETECT_ASYNC = 2 };
enum { CCNN_PRECISION_DEF = 0, CCNN_PRECISION_LOW = 1, CCNN_PRECISION_NORMAL = 2, CCNN_PRECISION_HIGH = 3, CCNN_PRECISION_ULTRA = 4 };

/* FaceDetector::Param (CompactCNNLibAPI_v2.h:97-161). `pipeline`, `detect_mode == async`,
 * `num_threads`, `device_info`, `cl_*` are accepted for drop-in fidelity; every pipeline runs the
 * cascade on the GPU, and async/sync give identical results. */
typedef struct {
    int max_image_width, max_image_height;  /* buffers are sized for this; larger frames re-initialise */
    int min_face_height;
    int max_face_height;                    /* 0 = no limit */
    float scale_factor;
    int min_neighbors;
    int detect_precision;
    float treshold[3];                      /* stage thresholds, range [-1.7159, 1.7159] */
    int drop_detect;
    int equalize;
    int reflection;
    int pipeline;
    int detect_mode;
    int num_threads;
    int index_output[3];                    /* output neuron of each stage's net */
    int device_info;
    int cuda_device_id;
    int cl_platform_id, cl_device_id;
    int facial_analysis;                    /* 1: run the landmark network (bundled cnn4landmarks_cntk.bin) on
                                               accepted windows: gender/smile/glasses, and drop_detect off */
} ccnn_params;

/* FaceDetector::Face (CompactCNNLibAPI_v2.h:66-82) */
typedef struct {
    int x, y, width, height;
    float score;
    int gender, smile, glasses;             /* facial analysis: median over the merged windows; else -1 */
} ccnn_face;

/* FaceDetector::ImageData (CompactCNNLibAPI_v2.h:84-95): 1 = gray, 3 = BGR, 4 = BGRA, row pitch in bytes */
typedef struct {
    int cols, rows, channels;
    const unsigned char* data;
    size_t step;
} ccnn_image;

/* FaceDetector::Param::Param() defaults of CompactCNNLibAPI_v2.h:97-161 (source header:
 * detect_precision = high, pipeline = GPU, detect_mode = async, min_face_height = 80). */
CCNN_API void ccnn_default_params(ccnn_params* p);

/* FaceDetector::Init (CompactCNNLibAPI_v2.cpp:373-407). model_paths[i] may be NULL (or the whole
 * array NULL) for the bundled cnn4face{1,2,3}_cntk.bin; unlike the reference, given paths are
 * honoured. Only the CNTK format (version 1.1) is accepted. */
CCNN_API ccnn_status ccnn_create(const ccnn_params* params, const char* const* model_paths, ccnn_handle* out);

/* FaceDetector::Clear + destructor */
CCNN_API ccnn_status ccnn_destroy(ccnn_handle h);

/* FaceDetector::Detect (CompactCNNLibAPI_v2.cpp:409-544) on a host image. Writes at most
 * `capacity` faces and the total count to *n_faces; returns CCNN_TRUNCATED if it did not fit.
 * The image buffer may be pageable or pinned host memory. */
CCNN_API ccnn_status ccnn_detect(ccnn_handle h, const ccnn_image* img, ccnn_face* faces, int capacity, int* n_faces);

/* Same, for an image already in device memory (img->data is a device pointer). `stream` is a
 * cudaStream_t (NULL = the handle's own stream); the call returns after the result is on the host.
 * A frame whose base and row step are multiples of 64 bytes is read in place (not copied). */
CCNN_API ccnn_status ccnn_detect_device(ccnn_handle h, const ccnn_image* img, void* stream, ccnn_face* faces, int capacity,
                                        int* n_faces);

/* Several host frames of the same size and channel count, pipelined over the handle's frame
 * slots (upload of frame k+1 overlaps the cascade of frame k). faces is n_images x
 * capacity_per_image; n_faces[i] gets each frame's count. Results equal n_images ccnn_detect calls. */
CCNN_API ccnn_status ccnn_detect_batch(ccnn_handle h, const ccnn_image* imgs, int n_images, ccnn_face* faces, int capacity_per_image,
                                       int* n_faces);

/* Several device frames (img[i].data are device pointers) of one size, pipelined like
 * ccnn_detect_batch. gpu_ms (nullable) receives the device time of the whole batch, measured with
 * CUDA events on the handle's streams from before the first frame to after the last. */
CCNN_API ccnn_status ccnn_detect_device_batch(ccnn_handle h, const ccnn_image* imgs, int n_images, ccnn_face* faces,
                                              int capacity_per_image, int* n_faces, float* gpu_ms);

/* FaceDetector::getGrayImage32F (CompactCNNLibAPI_v2.cpp:464-505), GPU pipeline: the internal fp32
 * gray image of the last frame, as a device pointer with its size and row pitch in bytes.
 * Valid until the next call on the handle. */
CCNN_API ccnn_status ccnn_get_gray_device(ccnn_handle h, const float** data, int* cols, int* rows, size_t* step);
/* The same image copied to host memory (cols x rows floats, dense). */
CCNN_API ccnn_status ccnn_get_gray_host(ccnn_handle h, float* out, int capacity, int* cols, int* rows);

/* getParam / setParam / get|setMaxImageSize / get|setMin|MaxObjectHeight / get|setNumThreads
 * (CompactCNNLibAPI_v2.h:171-185). Setters re-initialise lazily, as the reference's do. */
CCNN_API ccnn_status ccnn_get_params(ccnn_handle h, ccnn_params* out);
CCNN_API ccnn_status ccnn_set_params(ccnn_handle h, const ccnn_params* p);
CCNN_API ccnn_status ccnn_set_max_image_size(ccnn_handle h, int width, int height);
CCNN_API ccnn_status ccnn_set_min_object_height(ccnn_handle h, int v);
CCNN_API ccnn_status ccnn_set_max_object_height(ccnn_handle h, int v);
CCNN_API ccnn_status ccnn_set_num_threads(ccnn_handle h, int v);

/* Message of the last failing call on this thread ("" if none). */
CCNN_API const char* ccnn_last_error(void);

/* Library version string. */
CCNN_API const char* ccnn_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CCNN_H */
