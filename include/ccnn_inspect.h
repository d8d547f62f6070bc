/* compactcnncascade_b200 — inspection entry points of the detection path.
 *
 * These expose the path's internal steps so that each can be checked against the reference's
 * own objects on the same inputs: the gray converter (ImageConverter::Img8uToImg32fGRAY,
 * src/CNNObjectDetector/image_proc.cpp:299-317), the pyramid resizer
 * (ImageResizer::FastImageResize, image_resize.cpp:564-584), the stage-1 net
 * (ConvNeuralNetwork::Forward, cnn_simd_cntk.cpp:964-995), the per-level response maps and
 * candidate scan (CNNDetector::RunCheckDetect, cnn_detector_v3.cpp:1842-2011) and the raw
 * detection list before clustering (cpu_detect_rect, cnn_detector_v3.cpp:2745-2750).
 * They are not needed to run the detector.
 */
#ifndef CCNN_INSPECT_H
#define CCNN_INSPECT_H

#include "ccnn.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int width, height;           /* level image size */
    float scale;
    int resp_width, resp_height; /* stage-1 response map size */
} ccnn_level_info;

typedef struct {
    int level;                   /* level index (0 = largest scale) */
    int x, y;                    /* point in level pixels (4 x response index) */
    float score;                 /* stage-1 response */
    int accepted;                /* stage-2/3 verdict: 0 no, 1 first window, 2 shrunken retry window */
    float check_score;           /* score of an accepted window */
    int knn;
} ccnn_candidate;

typedef struct {
    int x, y, width, height;
    float score, scale;
    int knn, num_detect;
} ccnn_detection;

/* fp32 gray from 8-bit gray/BGR/BGRA; both pointers device memory, steps in bytes. The source
 * step must be a multiple of 64 and both pointers 64-byte aligned. */
CCNN_API ccnn_status ccnn_gray_u8_to_f32(const unsigned char* d_src, int cols, int rows, int channels, size_t src_step, float* d_dst,
                                         size_t dst_step, void* stream);

/* fp32 resize; type 0 = nearest neighbour, 1 = bilinear (ImgResize enum). Device pointers. */
CCNN_API ccnn_status ccnn_resize_f32(const float* d_src, int src_cols, int src_rows, size_t src_step, float* d_dst, int dst_cols,
                                     int dst_rows, size_t dst_step, int type, void* stream);

/* Stage-1 net of the handle on one fp32 device image (treated as a single pyramid level at
 * scale 1). The response map (dense, resp_cols floats per row) goes to d_resp. */
CCNN_API ccnn_status ccnn_stage1_forward(ccnn_handle h, const float* d_img, int cols, int rows, size_t step, float* d_resp, int resp_cap,
                                         int* resp_cols, int* resp_rows, void* stream);

/* Stage-1 response map of one fp32 device image, allocating no device memory. No counterpart in
 * the reference: it serves callers that may not call cudaMalloc — plug-in hosts that budget all
 * device memory up front and pass a component only its input and output buffers, or processes whose
 * device memory is already held by another framework's caching allocator, where a new allocation
 * would fail or stall the device. Instead of per-handle buffers it uses one fixed scratch array
 * compiled into the library (9 MiB + 256 B per GPU that loads the library, held until exit):
 * images up to 2,359,296 floats of L1 planes (about 1920x1080, 2^21 pixels) are accepted, larger
 * ones are refused with CCNN_ERR_INVALID_ARG and a message naming the limit. model_path may be NULL
 * for the bundled cnn4face1_cntk.bin. The first call in each CUDA context (on each device, and again
 * after a device reset) looks up the array's device address (cudaGetSymbolAddress, with that device
 * current); make that first call before any stream capture.
 * All calls share the array and it keeps the last call's contents; calls that overlap on the GPU
 * (other streams or threads) race on it. Returns after the response map is written. */
CCNN_API ccnn_status ccnn_stage1_forward_static(const char* model_path, const float* d_img, int cols, int rows, size_t step,
                                                float* d_resp, int resp_cap, int* resp_cols, int* resp_rows, void* stream);

/* Measured ceiling of the fp32 pipe on the current device for the instructions the exact kernels
 * issue (packed add.rn.f32x2 and the packed product fma.rn.f32x2 with a (-0, -0) addend): lane
 * operations per second, each packed instruction counting two per thread, best of `reps` timed
 * launches of `iters` loop trips after one warm-up launch. No counterpart in the reference: it is the
 * denominator of the stage-1 kernels' roofline. Allocates a small sink buffer; synchronous. */
CCNN_API ccnn_status ccnn_measure_fp32_peak(int iters, int reps, double* lane_ops_per_s, float* best_ms);

/* Intermediates of the handle's last frame. */
CCNN_API ccnn_status ccnn_inspect_levels(ccnn_handle h, ccnn_level_info* out, int capacity, int* n_levels);
CCNN_API ccnn_status ccnn_inspect_response(ccnn_handle h, int level, float* out, int capacity);
CCNN_API ccnn_status ccnn_inspect_candidates(ccnn_handle h, ccnn_candidate* out, int capacity, int* n);
CCNN_API ccnn_status ccnn_inspect_raw_detections(ccnn_handle h, ccnn_detection* out, int capacity, int* n);

/* The pyramid a freshly created handle (with the CNTK models) processes for a frame of this size and channel count
 * (CNNDetector::InitScales, cnn_detector_v3.cpp:289-346, with the level-size rule of RunCPUDetect
 * :2080-2088 and the re-initialisation rules of Detect :2499-2546). Host-only; needs no GPU. */
CCNN_API ccnn_status ccnn_plan_levels(const ccnn_params* p, int cols, int rows, int channels, ccnn_level_info* out, int capacity,
                                      int* n_levels);

/* Re-runs the handle's last frame `iters` times (CCNN_ERR_UNSUPPORTED when that frame was read in
 * place from device memory) and writes the mean duration (ms, CUDA events) of each kernel of the
 * chain: [0] gray, [1] pyramid (the legacy family only; the CNTK stage-1 front kernel resamples the
 * levels from the gray frame itself, so this entry is an empty gap), [2] stage-1 front, [3] stage-1 back (which also counts the
 * candidates), [4] candidate write, [5] stage-2/3 windows, [6] replay/sort/merge, [7] the learned gate
 * (when on), [8] the pyramid and stage 1 as one persistent launch (the batched form's kernel on this
 * frame). n_kernels entries are written. */
CCNN_API ccnn_status ccnn_profile_last_frame(ccnn_handle h, int iters, float* kernel_ms, int n_kernels);

/* Compares, on the current device, the packed reciprocal the kernels use in the rational tanh with the
 * IEEE reciprocal for every float from 1.0 to +infinity (and the first NaN); *mismatches must be 0.
 * No reference counterpart: the evidence behind replacing the division (cnnpp_cplusplus.cpp:662-666). */
CCNN_API ccnn_status ccnn_check_reciprocal(long long* mismatches, long long* checked);

/* FaceDetector::CNTKDump2Binary (src/CNNObjectDetector/CompactCNNLibAPI_v2.cpp:509-519): converts a
 * CNTK text dump of a trained cascade network into the binary model format (version 1.1) that
 * ccnn_create loads. ".bin" is appended to binary_file when it has no such extension. Host-only. */
CCNN_API ccnn_status ccnn_cntk_dump_to_binary(const char* binary_file, const char* cntk_model_dump);

/* The seeded synthetic frame of the benchmarks and tests, rendered on the device into d_out
 * (channels 1, 3 = BGR or 4 = BGRA interleaved, row pitch `step` bytes) on `stream`; byte-identical
 * to the host generator for every seed and size. faces_out (host, may be NULL) receives n_faces
 * records {int cx, cy, w, h; float angle_deg, contrast}. Returns when the frame is written.
 * No reference counterpart (the reference publishes no benchmark inputs). */
CCNN_API ccnn_status ccnn_synth_frame_device(void* d_out, int width, int height, int channels, size_t step, unsigned long long seed,
                                             int n_faces, int min_face, int max_face, void* faces_out, void* stream);

/* Schedule of a handle, as the autotuner (compactcnncascade_b200/autotune.py) picks it per frame size:
 * frames in flight (1-64, default 8) and resident blocks per SM of the persistent stage-2/3 window
 * kernel (1-6, default 4; 5 and 6 select builds with fewer registers a thread); 0 keeps a value. Rebuilds the handle's device state (as a re-Init does).
 * Results do not depend on the schedule. No reference counterpart (the reference has no GPU
 * schedule to tune). */
CCNN_API ccnn_status ccnn_set_schedule(ccnn_handle h, int frame_slots, int window_ctas_per_sm);
CCNN_API ccnn_status ccnn_get_schedule(ccnn_handle h, int* frame_slots, int* window_ctas_per_sm);

/* The full schedule: the two knobs above, the register budget of the two stage-1 kernels
 * (resident 256-thread blocks per SM, 3 or 4: more blocks hide more latency, fewer registers
 * may spill), and the batched form: batch_frames > 1 runs groups of that many frames of one size
 * through ccnn_detect_batch / ccnn_detect_device_batch as one graph each (the pyramid and stage 1
 * of every level of every frame of the group in one persistent launch fed by a device work queue,
 * then the candidates, windows and replays of the group in one launch each); frame_slots must be at
 * least batch_frames, and frame_slots / batch_frames groups are in flight. batch_blocks_per_sm is
 * the persistent kernel's resident blocks per SM (its grid, 1-4; 4 selects the 64-register build,
 * 1-3 the 80-register one; fewer blocks leave SMs to other frames' kernels). 0 keeps a value
 * (batch_frames: -1 keeps it, 0 turns the batched form off). Same rules as ccnn_set_schedule. */
typedef struct {
    int frame_slots;
    int window_ctas_per_sm;
    int front_blocks_per_sm;
    int back_blocks_per_sm;
    int batch_frames;
    int batch_blocks_per_sm;
} ccnn_schedule;
CCNN_API ccnn_status ccnn_set_schedule_ex(ccnn_handle h, const ccnn_schedule* s);
CCNN_API ccnn_status ccnn_get_schedule_ex(ccnn_handle h, ccnn_schedule* s);

/* Legacy cascade networks (model format 1.0, the cnn4face{1,2,3}_new.bin family: tanh activations,
 * max or average pooling; reader SIMD::ConvNeuralNetwork::Init, src/CNNObjectDetector/cnn_simd.cpp:40-336,
 * forward pass Run_single_thread, cnn_simd.cpp:551-874, in the reference's plain-C++ build).
 * ccnn_legacy_model_info parses a model file (host only) into info[10] = {max_pool, min_w, min_h,
 * maps L1, maps L2, maps L3, L3 kernel width, L3 kernel height, fully connected hidden layer,
 * hidden neurons}. ccnn_legacy_net_forward runs the network on a device fp32 image (step in bytes)
 * and writes the dense ow x oh response map to d_resp (device memory of resp_cap floats);
 * returns when the map is written. */
CCNN_API ccnn_status ccnn_legacy_model_info(const char* model_path, int* info, int n_info);
CCNN_API ccnn_status ccnn_legacy_net_forward(const char* model_path, const float* d_img, int cols, int rows, size_t step, float* d_resp,
                                             int resp_cap, int* ow, int* oh, void* stream);

/* The permutation the detector's device sort applies to detections with the given scales
 * (perm[i] = input index placed at slot i); equals std::sort with comp(a, b) = b < a. */
CCNN_API ccnn_status ccnn_sort_permutation(const float* scales, int n, int* perm);
/* The same permutation computed on the device by the replay kernel's block-wide sort (partition
 * rounds in parallel, leaf insertion sorts in parallel); scales and perm are host memory, synchronous.
 * No reference counterpart: it exists so tests can compare the block-wide form with std::sort. */
CCNN_API ccnn_status ccnn_sort_permutation_device(const float* scales, int n, int* perm);

#ifdef __cplusplus
}
#endif
#endif /* CCNN_INSPECT_H */
