/* Seeded synthetic frames for benchmarks and tests (no reference counterpart: the reference
 * publishes no benchmark inputs). */
#ifndef CCNN_SYNTH_FRAME_H
#define CCNN_SYNTH_FRAME_H
#include <stdint.h>
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

#ifdef __cplusplus
}
#endif
#endif
