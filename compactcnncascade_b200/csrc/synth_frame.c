/* Seeded synthetic BGR frames for the face-detection benchmarks and tests.
 *
 * The detection benchmarks are quoted on generated frames (no dataset is available): a
 * low-frequency background (4 random 2-D cosines, summed amplitude 60, offset 128), Gaussian-like
 * noise (sigma 8), and N face-like patches (shaded ellipse with Gaussian eyes, brows, nose and
 * mouth and a dark hair cap, rotated by up to +/-15 degrees, contrast 0.6-1.4, heights drawn from
 * [min, max]).
 *
 * Determinism: every value comes from integer PCG32 draws and IEEE double arithmetic with no
 * libm calls (cos, sin and exp are evaluated by our own range reduction + Taylor series), so a given
 * seed produces the same bytes on every x86-64 host. Build with -ffp-contract=off.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "synth_common.h"
#include "synth_frame.h"

int ccnn_synth_plan(int width, int height, uint64_t seed, int n_faces, int min_face, int max_face, double* tables,
                    ccnn_synth_geom* geom, int* jitter, uint64_t* noise_state, ccnn_synth_face* faces_out) {
    if (width <= 0 || height <= 0 || n_faces < 0 || min_face <= 0 || max_face < min_face || !tables || (n_faces && !geom) || !jitter ||
        !noise_state)
        return -1;
    pcg32_t rng;
    pcg32_seed(&rng, seed, 0x9e3779b97f4a7c15ULL);

    /* background: 4 cosines, amplitude 15 each (sum 60), 0.5-3 cycles per frame */
    double fx[4], fy[4], ph[4];
    for (int k = 0; k < 4; ++k) {
        fx[k] = unif_range(&rng, 0.5, 3.0) * (pcg32_next(&rng) & 1 ? 1.0 : -1.0);
        fy[k] = unif_range(&rng, 0.5, 3.0);
        ph[k] = unif_range(&rng, 0.0, 2.0 * SYNTH_PI);
    }
    for (int c = 0; c < 4; ++c) jitter[c] = (int)(pcg32_next(&rng) % 11u) - 5;

    /* separable evaluation: cos(a + b) = cos a cos b - sin a sin b */
    double* ca = tables;
    double* sa = ca + 4 * (size_t)width;
    double* cb = sa + 4 * (size_t)width;
    double* sb = cb + 4 * (size_t)height;
    for (int k = 0; k < 4; ++k)
        for (int x = 0; x < width; ++x) {
            double a = 2.0 * SYNTH_PI * fx[k] * (double)x / (double)width + ph[k];
            ca[k * width + x] = synth_cos(a);
            sa[k * width + x] = synth_sin(a);
        }
    for (int y = 0; y < height; ++y)
        for (int k = 0; k < 4; ++k) {
            double b = 2.0 * SYNTH_PI * fy[k] * (double)y / (double)height;
            cb[k * height + y] = synth_cos(b);
            sb[k * height + y] = synth_sin(b);
        }

    /* faces, drawn in order over their rotated bounding boxes */
    for (int i = 0; i < n_faces; ++i) {
        int fh = min_face + (int)(pcg32_next(&rng) % (uint32_t)(max_face - min_face + 1));
        int fw = (int)(0.759 * fh);
        ccnn_synth_face f;
        f.h = fh;
        f.w = fw;
        int mx = width - fw, my = height - fh;
        f.cx = (mx > 0 ? (int)(pcg32_next(&rng) % (uint32_t)mx) : 0) + fw / 2;
        f.cy = (my > 0 ? (int)(pcg32_next(&rng) % (uint32_t)my) : 0) + fh / 2;
        f.angle_deg = (float)unif_range(&rng, -15.0, 15.0);
        f.contrast = (float)unif_range(&rng, 0.6, 1.4);
        if (faces_out) faces_out[i] = f;

        ccnn_synth_geom* g = geom + i;
        double th = (double)f.angle_deg * SYNTH_PI / 180.0;
        g->ct = synth_cos(th);
        g->st = synth_sin(th);
        g->contrast = (double)f.contrast;
        g->cx = f.cx;
        g->cy = f.cy;
        g->fw = fw;
        g->fh = fh;
        int rad = (fw > fh ? fw : fh) / 2 + 2;
        g->x0 = f.cx - rad < 0 ? 0 : f.cx - rad;
        g->y0 = f.cy - rad < 0 ? 0 : f.cy - rad;
        g->x1 = f.cx + rad > width - 1 ? width - 1 : f.cx + rad;
        g->y1 = f.cy + rad > height - 1 ? height - 1 : f.cy + rad;
    }
    /* the noise takes two draws per pixel in raster order from here */
    noise_state[0] = rng.state;
    noise_state[1] = rng.inc;
    return n_faces;
}

int ccnn_synth_frame(uint8_t* out, int width, int height, int channels, int step, uint64_t seed, int n_faces,
                     int min_face, int max_face, ccnn_synth_face* faces_out) {
    if (!out || width <= 0 || height <= 0 || (channels != 1 && channels != 3 && channels != 4) || step < width * channels)
        return -1;
    if (n_faces < 0 || min_face <= 0 || max_face < min_face) return -1;

    double* tables = (double*)malloc(sizeof(double) * 8 * ((size_t)width + (size_t)height));
    float* lum = (float*)malloc(sizeof(float) * (size_t)width * (size_t)height);
    ccnn_synth_geom* geom = (ccnn_synth_geom*)malloc(sizeof(ccnn_synth_geom) * (size_t)(n_faces > 0 ? n_faces : 1));
    if (!tables || !lum || !geom) {
        free(tables);
        free(lum);
        free(geom);
        return -2;
    }
    int jitter[4];
    uint64_t ns[2];
    ccnn_synth_plan(width, height, seed, n_faces, min_face, max_face, tables, geom, jitter, ns, faces_out);
    const double* ca = tables;
    const double* sa = ca + 4 * (size_t)width;
    const double* cb = sa + 4 * (size_t)width;
    const double* sb = cb + 4 * (size_t)height;
    for (int y = 0; y < height; ++y) {
        float* lrow = lum + (size_t)y * width;
        for (int x = 0; x < width; ++x) {
            double bg = 128.0;
            for (int k = 0; k < 4; ++k) bg += 15.0 * (ca[k * width + x] * cb[k * height + y] - sa[k * width + x] * sb[k * height + y]);
            lrow[x] = (float)bg;
        }
    }
    for (int i = 0; i < n_faces; ++i) {
        const ccnn_synth_geom* g = geom + i;
        for (int y = g->y0; y <= g->y1; ++y)
            for (int x = g->x0; x <= g->x1; ++x) lum[(size_t)y * width + x] = synth_draw_face(g, x, y, lum[(size_t)y * width + x]);
    }
    pcg32_t rng;
    rng.state = ns[0];
    rng.inc = ns[1];
    for (int y = 0; y < height; ++y) {
        uint8_t* row = out + (size_t)y * (size_t)step;
        const float* lrow = lum + (size_t)y * width;
        for (int x = 0; x < width; ++x) {
            uint32_t r0 = pcg32_next(&rng), r1 = pcg32_next(&rng);
            synth_pixel_out(lrow[x], r0, r1, jitter, channels, row + x * channels);
        }
    }
    free(tables);
    free(lum);
    free(geom);
    return n_faces;
}
