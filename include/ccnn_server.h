/* compactcnncascade_b200 — serving loop (continuous batching of frames of mixed resolutions).
 *
 * No reference counterpart: the reference's CNNDetector processes one frame per call behind a
 * process-global mutex (src/CNNObjectDetector/CompactCNNLibAPI_v2.cpp:223-224, 419). The server keeps
 * the per-frame pipeline of ccnn_detect, but many frames are on the device at once: requests are
 * admitted as frame slots free up, frames of different resolutions run side by side on their own
 * streams and captured graphs, and results are collected as they finish.
 *
 *  - Resolution classes: every distinct (cols, rows, channels) gets its own detector, created
 *    for exactly that frame size with `slots_per_class` frame slots, when the HBM budget allows
 *    (idle classes are evicted, least recently used first, to make room).
 *  - Admission: a request is launched as soon as a slot of its class is free, in arrival order
 *    among the requests that can run; a request whose class can never fit the budget fails with
 *    CCNN_ERR_OOM.
 *  - Results: each frame's faces are exactly those of ccnn_detect on a fresh handle created with
 *    the server's parameters and max_image_size = the frame's size (no state carries over from
 *    other frames), so a frame gives the same result alone and in any mix.
 *  - Memory: the image data must stay valid until the request's result has been taken
 *    (ccnn_server_wait / a non-pending ccnn_server_poll); page-locked frames
 *    (ccnn_host_alloc) upload asynchronously.
 */
#ifndef CCNN_SERVER_H
#define CCNN_SERVER_H

#include "ccnn.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ccnn_server_s* ccnn_server;

typedef struct {
    size_t hbm_budget_bytes; /* device memory the frame slots may hold (0: 8 GiB) */
    int slots_per_class;     /* frames of one resolution class in flight at once (0: 4) */
    int max_queue;           /* requests waiting for a slot before submit answers CCNN_BUSY (0: 65536) */
} ccnn_server_config;

typedef struct {
    long long submitted, completed, failed;
    int queued;              /* waiting for a slot */
    int in_flight;           /* on the device */
    int classes;             /* resolution classes resident */
    size_t hbm_bytes;        /* device bytes held by frame slots */
} ccnn_server_stats;

CCNN_API ccnn_status ccnn_server_create(const ccnn_params* params, const char* const* model_paths, const ccnn_server_config* config,
                                        ccnn_server* out);
CCNN_API ccnn_status ccnn_server_destroy(ccnn_server s);
/* Turns the learned gate (include/ccnn_gate.h, ccnn_gate_set) on for every resolution class the
 * server creates; only before the first frame is submitted (CCNN_ERR_INVALID_ARG after). */
CCNN_API ccnn_status ccnn_server_set_gate(ccnn_server s, const float* params, int n_params, float threshold, float fallback_fraction);
/* The gate's candidate margin (ccnn_gate_set_margin, pixels 0-64, default 16) for every class; only
 * before the first frame is submitted. */
CCNN_API ccnn_status ccnn_server_set_gate_margin(ccnn_server s, int pixels);
/* Queues one frame; *ticket identifies its result. CCNN_BUSY when max_queue requests wait. */
CCNN_API ccnn_status ccnn_server_submit(ccnn_server s, const ccnn_image* img, long long* ticket);
/* Result of a ticket: CCNN_PENDING while unfinished (poll), or blocks until it is done (wait).
 * latency_ms (optional) = submit to completion. A ticket's result can be taken once. */
CCNN_API ccnn_status ccnn_server_poll(ccnn_server s, long long ticket, ccnn_face* faces, int capacity, int* n_faces, double* latency_ms);
CCNN_API ccnn_status ccnn_server_wait(ccnn_server s, long long ticket, ccnn_face* faces, int capacity, int* n_faces, double* latency_ms);
CCNN_API ccnn_status ccnn_server_stats_get(ccnn_server s, ccnn_server_stats* out);

/* Page-locked host memory for frames (cudaMallocHost / cudaFreeHost). */
CCNN_API void* ccnn_host_alloc(size_t bytes);
CCNN_API void ccnn_host_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* CCNN_SERVER_H */
