/* compactcnncascade_b200 — learned scale/region gate in front of the stage-1 scan.
 *
 * No reference counterpart: the reference scans every pyramid level in full
 * (CNNDetector::RunCPUDetect, src/CNNObjectDetector/cnn_detector_v3.cpp:2063-2235). The gate is
 * an addition evaluated against that full scan by box recall: a small network on an 8x8-averaged
 * copy of the gray frame predicts, for each pyramid octave and each 16x16-pixel cell of the
 * frame, whether the cascade will accept a window centred in that cell. Stage-1 tiles whose
 * candidates' window centres lie in no likely cell (with one cell of margin) are skipped; a frame
 * with many cells close below the threshold is scanned in full.
 *
 * Network (700 fp32 parameters, fp16 activations):
 *   f  = (8x8 box average of the gray frame - 128) / 64   (cols/8 x rows/8)
 *   a1 = LReLU_0.1(conv3x3(f, 1 -> 8 maps) + b1)        (zero padding)
 *   a2 = LReLU_0.1(conv3x3(a1, 8 -> 8 maps) + b2)
 *   q  = 2x2 average of a2                              (one vector per 16x16 cell)
 *   p  = sigmoid(W3 q + b3), one probability per octave
 * Parameter layout: W1[8][9], b1[8], W2[8 out][8 in][9], b2[8], W3[4][8], b3[4] (taps row-major).
 * The octave of a level is floor(log2(scale of level 0 / scale of the level)), clamped to 3.
 * Labels: uint8 [frame][octave][cell row][cell column], cells (cols/16) x (rows/16).
 */
#ifndef CCNN_GATE_H
#define CCNN_GATE_H

#include "ccnn.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CCNN_GATE_PARAMS 700
#define CCNN_GATE_OCTAVES 4

/* Turns the gate on for every later frame of the handle: n_params must be CCNN_GATE_PARAMS;
 * threshold in (0, 1) is the probability a cell needs; a frame in which more than
 * fallback_fraction of all (octave, cell) probabilities lie in [threshold / 4, threshold) runs the
 * full scan. Frames smaller than 32x32 gray pixels always run the full scan. */
CCNN_API ccnn_status ccnn_gate_set(ccnn_handle h, const float* params, int n_params, float threshold, float fallback_fraction);
/* Back to the full scan. */
CCNN_API ccnn_status ccnn_gate_disable(ccnn_handle h);

/* How far (in frame pixels along each axis, 0-64, default 16: the centre's cell and one cell on
 * either side) from a stage-1 candidate's window centre the gate looks for a likely cell of the
 * candidate's octave; the stage-1 tiles are kept by the same rule. A smaller margin skips more work
 * and keeps fewer of the plain cascade's boxes. */
CCNN_API ccnn_status ccnn_gate_set_margin(ccnn_handle h, int pixels);

/* Stage-1 tiles of the handle's last frame: how many of the front (pooled layer-1) and back
 * (response) tiles ran, of how many, and whether the frame fell back to the full scan. With the
 * gate off every tile runs. */
CCNN_API ccnn_status ccnn_gate_stats(ccnn_handle h, int* front_run, int* front_total, int* back_run, int* back_total, int* fallback);

/* The gate's probabilities for the handle's last frame (run with the gate on): 4 octaves x
 * (rows/16) x (cols/16) floats in host memory, octave-major, cell rows in order. *n gets the count;
 * returns CCNN_TRUNCATED when capacity is smaller (the first `capacity` are written). */
CCNN_API ccnn_status ccnn_gate_probabilities(ccnn_handle h, float* out, int capacity, int* n);

/* Training labels from the handle's last frame (run with the gate off): 1 at the (octave, cell) of
 * the window centre of every candidate that stage 3 accepted, else 0; d_labels is device memory of
 * 4 x (rows/16) x (cols/16) bytes for the frame's gray size, written on `stream`. */
CCNN_API ccnn_status ccnn_gate_labels(ccnn_handle h, unsigned char* d_labels, void* stream);

/* f for one gray frame (device fp32, step in bytes) into d_feat (device fp16, (cols/8) x (rows/8)
 * packed rows), on `stream` (a cudaStream_t, or NULL). */
CCNN_API ccnn_status ccnn_gate_features(const float* d_gray, int cols, int rows, size_t step, void* d_feat, void* stream);

/* Mean positive-weighted binary cross-entropy over n frames of features (d_feat, fp16
 * [n][h8][w8]) and labels (d_labels, uint8 [n][4][h8/2][w8/2]) and its gradient with respect to
 * the parameters (d_params, device fp32). grad_out and loss_out are host memory. Synchronous. */
CCNN_API ccnn_status ccnn_gate_gradient(const float* d_params, const void* d_feat, const unsigned char* d_labels, int n, int w8, int h8,
                                        float pos_weight, float* grad_out, float* loss_out);

/* Adam (beta 0.9 / 0.999, eps 1e-8) over consecutive mini-batches of `batch` frames, `epochs`
 * passes. params (host fp32) is the start point and receives the result; losses (host, `epochs`
 * floats, may be NULL) receives each pass's mean loss. Synchronous. */
CCNN_API ccnn_status ccnn_gate_train(float* params, const void* d_feat, const unsigned char* d_labels, int n, int w8, int h8, int batch,
                                     int epochs, float lr, float pos_weight, float* losses);

#ifdef __cplusplus
}
#endif

#endif /* CCNN_GATE_H */
