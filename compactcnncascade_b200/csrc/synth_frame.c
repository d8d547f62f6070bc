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

#include "synth_frame.h"

typedef struct {
    uint64_t state, inc;
} pcg32_t;

static uint32_t pcg32_next(pcg32_t* r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((-rot) & 31u));
}

static void pcg32_seed(pcg32_t* r, uint64_t seed, uint64_t seq) {
    r->state = 0u;
    r->inc = (seq << 1u) | 1u;
    pcg32_next(r);
    r->state += seed;
    pcg32_next(r);
}

/* uniform double in [0, 1) with 32 random bits */
static double unif(pcg32_t* r) { return (double)pcg32_next(r) * (1.0 / 4294967296.0); }
static double unif_range(pcg32_t* r, double a, double b) { return a + (b - a) * unif(r); }

static const double kPi = 3.14159265358979323846;

static double floor_d(double x) {
    double t = (double)(int64_t)x;
    return (t > x) ? t - 1.0 : t;
}

/* cos on any argument: reduce to [-pi, pi], then to [0, pi/2] by symmetry, Taylor to x^20. */
static double synth_cos(double x) {
    double k = floor_d(x / (2.0 * kPi) + 0.5);
    double r = x - k * (2.0 * kPi);
    if (r < 0) r = -r;
    double sign = 1.0;
    if (r > 0.5 * kPi) {
        r = kPi - r;
        sign = -1.0;
    }
    double r2 = r * r, term = 1.0, sum = 1.0;
    for (int n = 1; n <= 10; ++n) {
        term = -term * r2 / (double)((2 * n - 1) * (2 * n));
        sum += term;
    }
    return sign * sum;
}
static double synth_sin(double x) { return synth_cos(x - 0.5 * kPi); }

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* exp(-t) for t >= 0: t = n ln2 + r, Taylor series of exp(-r) on [0, ln2), exact halvings. */
static double synth_exp_neg(double t) {
    if (t > 60.0) return 0.0;
    const double ln2 = 0.69314718055994530942;
    int n = (int)(t / ln2);
    double r = t - (double)n * ln2;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k <= 14; ++k) {
        term = -term * r / (double)k;
        sum += term;
    }
    for (int k = 0; k < n; ++k) sum *= 0.5;
    return sum;
}

static double gauss2(double du, double dv, double sx, double sy) { return synth_exp_neg(du * du / (sx * sx) + dv * dv / (sy * sy)); }

/* Face model in the patch frame: u across, v top to bottom, both in [-1, 1] on the ellipse.
 * Smooth shading with Gaussian eyes, brows, cheeks, nose, mouth and a dark hair cap; the
 * proportions were tuned so that the cascade's three stages accept most patches. */
static double face_value(double u, double v) {
    const double eye_x = 0.384, eye_y = -0.212;
    double val = 174.1 + 24.7 * (1.0 - (u * u + v * v)) - 27.8 * u * u;
    for (int s = -1; s <= 1; s += 2) {
        val -= 182.0 * gauss2(u - eye_x * s, v - eye_y, 0.175, 0.08);
        val -= 20.0 * gauss2(u - eye_x * s, v + 0.557, 0.167, 0.0266);
        val += 15.3 * gauss2(u - eye_x * s, v - eye_y - 0.35, 0.2, 0.15);
    }
    val -= 81.5 * gauss2(u, v - 0.254, 0.124, 0.0647);
    val += 8.4 * gauss2(u, v - (eye_y + 0.254) * 0.5, 0.06, 0.2);
    val -= 83.8 * gauss2(u, v - 0.580, 0.349, 0.0438);
    if (v < -0.80) val = 30.0;
    return clampd(val, 0.0, 255.0);
}

int ccnn_synth_frame(uint8_t* out, int width, int height, int channels, int step, uint64_t seed, int n_faces,
                     int min_face, int max_face, ccnn_synth_face* faces_out) {
    if (!out || width <= 0 || height <= 0 || (channels != 1 && channels != 3 && channels != 4) || step < width * channels)
        return -1;
    if (n_faces < 0 || min_face <= 0 || max_face < min_face) return -1;

    pcg32_t rng;
    pcg32_seed(&rng, seed, 0x9e3779b97f4a7c15ULL);

    /* background: 4 cosines, amplitude 15 each (sum 60), 0.5-3 cycles per frame */
    double fx[4], fy[4], ph[4];
    for (int k = 0; k < 4; ++k) {
        fx[k] = unif_range(&rng, 0.5, 3.0) * (pcg32_next(&rng) & 1 ? 1.0 : -1.0);
        fy[k] = unif_range(&rng, 0.5, 3.0);
        ph[k] = unif_range(&rng, 0.0, 2.0 * kPi);
    }
    int jitter[4];
    for (int c = 0; c < 4; ++c) jitter[c] = (int)(pcg32_next(&rng) % 11u) - 5;

    /* separable evaluation: cos(a + b) = cos a cos b - sin a sin b */
    double* ca = (double*)malloc(sizeof(double) * 8 * (size_t)width);
    float* lum = (float*)malloc(sizeof(float) * (size_t)width * (size_t)height);
    if (!ca || !lum) {
        free(ca);
        free(lum);
        return -2;
    }
    double* sa = ca + 4 * (size_t)width;
    for (int k = 0; k < 4; ++k)
        for (int x = 0; x < width; ++x) {
            double a = 2.0 * kPi * fx[k] * (double)x / (double)width + ph[k];
            ca[k * width + x] = synth_cos(a);
            sa[k * width + x] = synth_sin(a);
        }
    for (int y = 0; y < height; ++y) {
        double cb[4], sb[4];
        for (int k = 0; k < 4; ++k) {
            double b = 2.0 * kPi * fy[k] * (double)y / (double)height;
            cb[k] = synth_cos(b);
            sb[k] = synth_sin(b);
        }
        float* lrow = lum + (size_t)y * width;
        for (int x = 0; x < width; ++x) {
            double bg = 128.0;
            for (int k = 0; k < 4; ++k) bg += 15.0 * (ca[k * width + x] * cb[k] - sa[k * width + x] * sb[k]);
            lrow[x] = (float)bg;
        }
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

        double th = (double)f.angle_deg * kPi / 180.0;
        double ct = synth_cos(th), st = synth_sin(th);
        int rad = (fw > fh ? fw : fh) / 2 + 2;
        int x0 = f.cx - rad, x1 = f.cx + rad, y0 = f.cy - rad, y1 = f.cy + rad;
        if (x0 < 0) x0 = 0;
        if (y0 < 0) y0 = 0;
        if (x1 > width - 1) x1 = width - 1;
        if (y1 > height - 1) y1 = height - 1;
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                /* 2x2 supersampling: coverage alpha and the mean face value of covered samples */
                double acc = 0.0;
                int inside = 0;
                for (int sy = 0; sy < 2; ++sy)
                    for (int sx = 0; sx < 2; ++sx) {
                        double dx = (double)x + (sx ? 0.25 : -0.25) - (double)f.cx;
                        double dy = (double)y + (sy ? 0.25 : -0.25) - (double)f.cy;
                        double u = (ct * dx + st * dy) / (0.5 * (double)fw);
                        double w = (-st * dx + ct * dy) / (0.5 * (double)fh);
                        if (u * u + w * w < 1.0) {
                            acc += face_value(u, w);
                            inside++;
                        }
                    }
                if (inside > 0) {
                    double alpha = (double)inside / 4.0;
                    double fv = acc / (double)inside;
                    double cur = (double)lum[(size_t)y * width + x];
                    double target = cur + (double)f.contrast * (fv - cur);
                    lum[(size_t)y * width + x] = (float)(cur + alpha * (target - cur));
                }
            }
    }

    /* noise (sum of 4 uniforms scaled to sigma 8), per-channel jitter, quantisation */
    for (int y = 0; y < height; ++y) {
        uint8_t* row = out + (size_t)y * (size_t)step;
        const float* lrow = lum + (size_t)y * width;
        for (int x = 0; x < width; ++x) {
            uint32_t r0 = pcg32_next(&rng), r1 = pcg32_next(&rng);
            double n = ((double)(r0 & 0xffffu) + (double)(r0 >> 16) + (double)(r1 & 0xffffu) + (double)(r1 >> 16)) / 65536.0 - 2.0;
            double v = (double)lrow[x] + n * 8.0 * 1.7320508075688772; /* var of a sum of 4 U(0,1) is 1/3 */
            for (int c = 0; c < channels; ++c) {
                double vc = (c < 3) ? v + (double)jitter[c] : 255.0;
                vc = clampd(vc, 0.0, 255.0);
                row[x * channels + c] = (uint8_t)(int)(vc + 0.5);
            }
        }
    }
    free(ca);
    free(lum);
    return n_faces;
}
