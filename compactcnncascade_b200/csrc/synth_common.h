/* Arithmetic shared by the host and device synthetic-frame generators: PCG32 draws and IEEE
 * double evaluation with no libm calls (cos, sin and exp by range reduction + Taylor series), so
 * both produce the same bytes. Compile without contraction (-ffp-contract=off, nvcc -fmad=false). */
#ifndef CCNN_SYNTH_COMMON_H
#define CCNN_SYNTH_COMMON_H
#include <stdint.h>

#ifdef __CUDACC__
#define SYNTH_FN static __host__ __device__ __forceinline__
#else
#define SYNTH_FN static inline
#endif

typedef struct {
    uint64_t state, inc;
} pcg32_t;

SYNTH_FN uint32_t pcg32_next(pcg32_t* r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((-rot) & 31u));
}

SYNTH_FN void pcg32_seed(pcg32_t* r, uint64_t seed, uint64_t seq) {
    r->state = 0u;
    r->inc = (seq << 1u) | 1u;
    pcg32_next(r);
    r->state += seed;
    pcg32_next(r);
}

/* uniform double in [0, 1) with 32 random bits */
SYNTH_FN double unif(pcg32_t* r) { return (double)pcg32_next(r) * (1.0 / 4294967296.0); }
SYNTH_FN double unif_range(pcg32_t* r, double a, double b) { return a + (b - a) * unif(r); }

#define SYNTH_PI 3.14159265358979323846

SYNTH_FN double floor_d(double x) {
    double t = (double)(int64_t)x;
    return (t > x) ? t - 1.0 : t;
}

/* cos on any argument: reduce to [-pi, pi], then to [0, pi/2] by symmetry, Taylor to x^20. */
SYNTH_FN double synth_cos(double x) {
    double k = floor_d(x / (2.0 * SYNTH_PI) + 0.5);
    double r = x - k * (2.0 * SYNTH_PI);
    if (r < 0) r = -r;
    double sign = 1.0;
    if (r > 0.5 * SYNTH_PI) {
        r = SYNTH_PI - r;
        sign = -1.0;
    }
    double r2 = r * r, term = 1.0, sum = 1.0;
    for (int n = 1; n <= 10; ++n) {
        term = -term * r2 / (double)((2 * n - 1) * (2 * n));
        sum += term;
    }
    return sign * sum;
}
SYNTH_FN double synth_sin(double x) { return synth_cos(x - 0.5 * SYNTH_PI); }

SYNTH_FN double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* exp(-t) for t >= 0: t = n ln2 + r, Taylor series of exp(-r) on [0, ln2), exact halvings. */
SYNTH_FN double synth_exp_neg(double t) {
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

SYNTH_FN double gauss2(double du, double dv, double sx, double sy) { return synth_exp_neg(du * du / (sx * sx) + dv * dv / (sy * sy)); }

/* Face model in the patch frame: u across, v top to bottom, both in [-1, 1] on the ellipse.
 * Smooth shading with Gaussian eyes, brows, cheeks, nose, mouth and a dark hair cap; the
 * proportions were tuned so that the cascade's three stages accept most patches. */
SYNTH_FN double face_value(double u, double v) {
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


/* Per-face drawing geometry (the rotated bounding box clipped to the frame). */
typedef struct {
    int cx, cy, fw, fh;
    int x0, x1, y0, y1;
    double ct, st, contrast;
} ccnn_synth_geom;

/* One pixel of the face layer: blends face `g` over the current luminance `cur` (2x2
 * supersampled coverage), as the generator draws faces in order. */
SYNTH_FN float synth_draw_face(const ccnn_synth_geom* g, int x, int y, float lum) {
    double acc = 0.0;
    int inside = 0;
    for (int sy = 0; sy < 2; ++sy)
        for (int sx = 0; sx < 2; ++sx) {
            double dx = (double)x + (sx ? 0.25 : -0.25) - (double)g->cx;
            double dy = (double)y + (sy ? 0.25 : -0.25) - (double)g->cy;
            double u = (g->ct * dx + g->st * dy) / (0.5 * (double)g->fw);
            double w = (-g->st * dx + g->ct * dy) / (0.5 * (double)g->fh);
            if (u * u + w * w < 1.0) {
                acc += face_value(u, w);
                inside++;
            }
        }
    if (inside == 0) return lum;
    double alpha = (double)inside / 4.0;
    double fv = acc / (double)inside;
    double cur = (double)lum;
    double target = cur + g->contrast * (fv - cur);
    return (float)(cur + alpha * (target - cur));
}

/* Noise, per-channel jitter and quantisation of one pixel from its two PCG32 draws. */
SYNTH_FN void synth_pixel_out(float lum, uint32_t r0, uint32_t r1, const int* jitter, int channels, uint8_t* px) {
    double n = ((double)(r0 & 0xffffu) + (double)(r0 >> 16) + (double)(r1 & 0xffffu) + (double)(r1 >> 16)) / 65536.0 - 2.0;
    double v = (double)lum + n * 8.0 * 1.7320508075688772; /* var of a sum of 4 U(0,1) is 1/3 */
    for (int c = 0; c < channels; ++c) {
        double vc = (c < 3) ? v + (double)jitter[c] : 255.0;
        vc = clampd(vc, 0.0, 255.0);
        px[c] = (uint8_t)(int)(vc + 0.5);
    }
}

/* The PCG32 state `delta` draws ahead, by the logarithmic-time LCG jump of F. Brown, "Random
 * number generation with arbitrary strides" (Trans. Am. Nucl. Soc., 1994). */
SYNTH_FN pcg32_t pcg32_advanced(pcg32_t r, uint64_t delta) {
    uint64_t cur_mult = 6364136223846793005ULL, cur_plus = r.inc, acc_mult = 1u, acc_plus = 0u;
    while (delta > 0) {
        if (delta & 1u) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1u) * cur_plus;
        cur_mult *= cur_mult;
        delta >>= 1;
    }
    r.state = acc_mult * r.state + acc_plus;
    return r;
}

#endif /* CCNN_SYNTH_COMMON_H */
