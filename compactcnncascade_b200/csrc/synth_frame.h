/* Seeded synthetic frames for benchmarks and tests (no reference counterpart: the reference
 * publishes no benchmark inputs). */
#ifndef CCNN_SYNTH_FRAME_H
#define CCNN_SYNTH_FRAME_H
#include <stdint.h>

#include "synth_common.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int cx, cy;      /* patch centre (pixels) */
    int w, h;        /* patch size (pixels) */
    float angle_deg; /* in-plane rotation */
    float contrast;  /* 0.6 .. 1.4 */
} ccnn_synth_face;

/* Writes a width x height frame with `channels` (1, 3 = BGR, 4 = BGRA) interleaved bytes per
 * pixel and row pitch `step` into `out`. Face heights are drawn from [min_face, max_face].
 * `faces_out` (nullable) receives the n_faces placed patches. Returns n_faces, or < 0 on bad
 * arguments (-1) or allocation failure (-2). */
int ccnn_synth_frame(uint8_t* out, int width, int height, int channels, int step, uint64_t seed, int n_faces,
                     int min_face, int max_face, ccnn_synth_face* faces_out);

/* The host half of the generator, shared with the device renderer: the background tables
 * (`tables`: cos/sin of the 4 column phases [4][width] x2, then of the 4 row phases [4][height]
 * x2, 8 * (width + height) doubles), each face's geometry (`geom`, n_faces entries), the channel
 * jitter (4 ints) and the PCG32 state (state, inc) from which the noise takes two draws per pixel
 * in raster order. Returns n_faces or -1. */
int ccnn_synth_plan(int width, int height, uint64_t seed, int n_faces, int min_face, int max_face, double* tables,
                    ccnn_synth_geom* geom, int* jitter, uint64_t* noise_state, ccnn_synth_face* faces_out);

#ifdef __cplusplus
}
#endif
#endif
