// Test infrastructure only: a plain CPU restatement of the reference's face-detection path.
// It is the checker for the CUDA path (tests/, the smoke check, bench.py's CPU baseline), never the
// measured or shipped code. Compiled by oracle/Makefile with -O2 -ffp-contract=off (IEEE single
// precision, no contraction), the arithmetic the reference's plain C++ path performs.
//
// Each function names the reference code it restates (paths under src/CNNObjectDetector/).
#include "ccnn_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------- gray (image_proc.cpp:299-317)
void gray_image(const uint8_t* img, int w, int h, int ch, int step, float* out, int ostride) {
    for (int y = 0; y < h; ++y) {
        const uint8_t* p = img + (size_t)y * step;
        float* o = out + (size_t)y * ostride;
        for (int x = 0; x < w; ++x) {
            if (ch == 1) {
                o[x] = (float)p[x];  // Img8uToImg32f (:99-102)
            } else {
                const float b = (float)p[x * ch], g = (float)p[x * ch + 1], r = (float)p[x * ch + 2];
                o[x] = 0.114f * b + 0.587f * g + 0.299f * r;  // (:195-201), BGRA (:287-293)
            }
        }
    }
}

// ---------------------------------------------------------------- resize (image_resize.cpp)
struct Lut {
    std::vector<uint32_t> px, py;
    std::vector<float> fx, cx, fy, cy;
};

// ImageResizer::preprocessing (:46-122): 12-bit fixed point, weights from the unclamped position
Lut make_lut(int sw, int sh, int dw, int dh) {
    Lut L;
    const uint32_t sclx = ((uint32_t)sw << 12) / (uint32_t)dw + 1, scly = ((uint32_t)sh << 12) / (uint32_t)dh + 1;
    for (int iy = 0; iy < dh; ++iy) {
        const uint32_t y = (uint32_t)iy * scly, p = y >> 12;
        const float f = (float)(y - (p << 12)), c = 4096.f - f;
        L.py.push_back(std::min(p, (uint32_t)(sh - 1)));
        L.fy.push_back(f / 16777216.f);
        L.cy.push_back(c / 16777216.f);
    }
    for (int ix = 0; ix < dw; ++ix) {
        const uint32_t x = (uint32_t)ix * sclx, p = x >> 12;
        const float f = (float)(x - (p << 12));
        L.px.push_back(std::min(p, (uint32_t)(sw - 2)));
        L.fx.push_back(f);
        L.cx.push_back(4096.f - f);
    }
    return L;
}

// FastImageResize (:564-584): equal sizes copy; 0 = nearest neighbour (:328-392), 1 = bilinear (:393-541)
void resize_f32(const float* src, int sw, int sh, int ss, float* dst, int dw, int dh, int ds, int type) {
    if (sw == dw && sh == dh) {
        for (int y = 0; y < dh; ++y) memcpy(dst + (size_t)y * ds, src + (size_t)y * ss, sizeof(float) * dw);
        return;
    }
    const Lut L = make_lut(sw, sh, dw, dh);
    for (int iy = 0; iy < dh; ++iy) {
        uint32_t py = L.py[iy];
        if (type == 0) {
            for (int ix = 0; ix < dw; ++ix) dst[(size_t)iy * ds + ix] = src[(size_t)py * ss + L.px[ix]];
        } else {
            if (py + 1 >= (uint32_t)sh) py--;
            const float* r0 = src + (size_t)py * ss;
            const float* r1 = r0 + ss;
            for (int ix = 0; ix < dw; ++ix) {
                const uint32_t px = L.px[ix];
                const float t = r0[px] * L.cx[ix] + r0[px + 1] * L.fx[ix];
                const float b = r1[px] * L.cx[ix] + r1[px + 1] * L.fx[ix];
                dst[(size_t)iy * ds + ix] = t * L.cy[iy] + b * L.fy[iy];
            }
        }
    }
}

// bilinear on bytes (:197-326): the float result is truncated to a byte
void resize_u8_bilinear(const uint8_t* src, int sw, int sh, int ss, uint8_t* dst, int dw, int dh, int ds) {
    if (sw == dw && sh == dh) {
        for (int y = 0; y < dh; ++y) memcpy(dst + (size_t)y * ds, src + (size_t)y * ss, dw);
        return;
    }
    const Lut L = make_lut(sw, sh, dw, dh);
    for (int iy = 0; iy < dh; ++iy) {
        uint32_t py = L.py[iy];
        if (py + 1 >= (uint32_t)sh) py--;
        const uint8_t* r0 = src + (size_t)py * ss;
        const uint8_t* r1 = r0 + ss;
        for (int ix = 0; ix < dw; ++ix) {
            const uint32_t px = L.px[ix];
            const float t = (float)r0[px] * L.cx[ix] + (float)r0[px + 1] * L.fx[ix];
            const float b = (float)r1[px] * L.cx[ix] + (float)r1[px + 1] * L.fx[ix];
            dst[(size_t)iy * ds + ix] = (uint8_t)(int)(t * L.cy[iy] + b * L.fy[iy]);
        }
    }
}

// ---------------------------------------------------------------- equalisation (image_proc.cpp:720-799)
void equalize(uint8_t* img, int w, int h, int stride) {
    int hist[256] = {0}, cf[256];
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) hist[img[(size_t)y * stride + x]]++;
    cf[0] = hist[0];
    for (int k = 1; k < 256; ++k) cf[k] = cf[k - 1] + hist[k];
    const float lo = (float)cf[0], hi = (float)cf[255];
    if (lo == hi) return;
    const float d = 255.f / (hi - lo);
    int lut[256];
    for (int k = 0; k < 256; ++k) lut[k] = (int)(((float)cf[k] - lo) * d + 0.5f);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) img[(size_t)y * stride + x] = (uint8_t)lut[img[(size_t)y * stride + x]];
}

// ---------------------------------------------------------------- networks (cnn_simd_cntk.cpp)
struct Net {
    int min_w = 0, min_h = 0;
    int maps[3] = {0, 0, 0}, kw[3] = {0, 0, 0}, kh[3] = {0, 0, 0};
    std::vector<float> k[3], act[3];
    float af = 0.f;
    int hl = 0, conn = 0, hs = 0, nout = 0;
    std::vector<float> hw, hb, htw, hbn, ow, ob;
    float otw = 0.f;
    int index = 0;
    bool ok = false;
};

template <class T>
bool rd(const std::string& s, size_t& off, T* v) {
    if (off + sizeof(T) > s.size()) return false;
    memcpy(v, s.data() + off, sizeof(T));
    off += sizeof(T);
    return true;
}

bool rdv(const std::string& s, size_t& off, std::vector<float>& v, long long n) {
    if (n < 0 || off + 4 * (size_t)n > s.size()) return false;
    v.resize((size_t)n);
    memcpy(v.data(), s.data() + off, 4 * (size_t)n);
    off += 4 * (size_t)n;
    return true;
}

// the binary layout read by ConvNeuralNetwork::Init (:42-404)
Net load_net(const std::string& path, int index_output) {
    Net n;
    std::ifstream f(path, std::ios::binary);
    if (!f) return n;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string s = ss.str();
    size_t o = 0;
    float ver;
    uint8_t mp, full;
    int layers;
    if (!rd(s, o, &ver) || ver < 1.0f || ver > 1.1f) return n;
    if (!rd(s, o, &mp) || !rd(s, o, &n.min_w) || !rd(s, o, &n.min_h) || !rd(s, o, &layers) || layers != 3) return n;
    for (int i = 0; i < 3; ++i)
        if (!rd(s, o, &n.maps[i])) return n;
    for (int l = 0; l < 3; ++l)
        if (!rd(s, o, &n.kw[l]) || !rd(s, o, &n.kh[l]) || !rdv(s, o, n.k[l], (long long)n.maps[l] * n.kw[l] * n.kh[l])) return n;
    if (!rd(s, o, &n.af)) return n;
    for (int l = 0; l < 3; ++l)
        if (!rdv(s, o, n.act[l], 5LL * n.maps[l])) return n;
    if (!rd(s, o, &full) || !rd(s, o, &n.hl) || !rd(s, o, &n.conn) || !rd(s, o, &n.hs)) return n;
    if (!mp || full || n.kw[1] * n.kh[1] != 9) return n;
    if (!rdv(s, o, n.hw, (long long)n.hl * n.conn) || !rdv(s, o, n.hb, n.hl) || !rdv(s, o, n.htw, n.hl / n.hs) ||
        !rdv(s, o, n.hbn, 2LL * n.hs) || !rd(s, o, &n.nout) || !rdv(s, o, n.ow, (long long)n.nout * n.hl) || !rdv(s, o, n.ob, n.nout) ||
        !rd(s, o, &n.otw))
        return n;
    n.index = std::min(index_output, n.nout - 1);
    if (n.index == 0) n.af = -n.af;
    n.ok = true;
    return n;
}

inline float tanh_approx(float c) {  // cnnpp_cplusplus.cpp:662-666
    const float a = 1.41645f;
    const float sgn = c < 0.f ? -1.f : 1.f;
    return sgn * (1.f - 1.f / (1.f + fabsf(c) + c * c + a * c * c * c * c));
}

inline float act(float x, const float* p) {  // lrelu_bn (:604-605): bias, w1, w2, (bn_w unused), bn_b
    const float c = x + p[0];
    return p[1] * c + p[2] * std::max(0.f, c) + p[4];
}

// valid convolution of one map: row-major taps accumulated left to right, except the 5x4 kernel
// whose rows are summed separately and then added in order (conv_5x4, :158-187)
std::vector<float> conv(const std::vector<float>& src, int sw, int sh, const float* k, int kw, int kh, int* ow, int* oh) {
    *ow = sw - kw + 1;
    *oh = sh - kh + 1;
    std::vector<float> out((size_t)std::max(0, *ow) * std::max(0, *oh));
    const bool row_sums = (kw == 4 && kh == 5);
    for (int y = 0; y < *oh; ++y)
        for (int x = 0; x < *ow; ++x) {
            float acc = 0.f;
            if (row_sums) {
                for (int r = 0; r < kh; ++r) {
                    float rs = src[(size_t)(y + r) * sw + x] * k[r * kw];
                    for (int c = 1; c < kw; ++c) rs = rs + src[(size_t)(y + r) * sw + x + c] * k[r * kw + c];
                    acc = r == 0 ? rs : acc + rs;
                }
            } else {
                acc = src[(size_t)y * sw + x] * k[0];
                for (int t = 1; t < kw * kh; ++t) acc = acc + src[(size_t)(y + t / kw) * sw + x + t % kw] * k[t];
            }
            out[(size_t)y * *ow + x] = acc;
        }
    return out;
}

// activation + 2x2 max pooling over the floor(size/2) cells (lrelu_bn_max, :593-622)
std::vector<float> act_pool(const std::vector<float>& c, int w, int h, const float* p, int* pw, int* ph) {
    *pw = w >> 1;
    *ph = h >> 1;
    std::vector<float> out((size_t)*pw * *ph);
    for (int y = 0; y < *ph; ++y)
        for (int x = 0; x < *pw; ++x) {
            const float a = act(c[(size_t)(2 * y) * w + 2 * x], p), b = act(c[(size_t)(2 * y) * w + 2 * x + 1], p);
            const float d = act(c[(size_t)(2 * y + 1) * w + 2 * x], p), e = act(c[(size_t)(2 * y + 1) * w + 2 * x + 1], p);
            out[(size_t)y * *pw + x] = fmaxf(fmaxf(a, b), fmaxf(d, e));
        }
    return out;
}

// neighbour-map sums feeding the next layer (add / add2, Run :705-731, :758-785)
std::vector<std::vector<float>> map_sums(const std::vector<std::vector<float>>& P) {
    const int n = (int)P.size();
    std::vector<std::vector<float>> S(n, std::vector<float>(P[0].size()));
    for (size_t i = 0; i < P[0].size(); ++i) {
        S[0][i] = P[0][i] + P[1][i];
        for (int m = 1; m < n - 1; ++m) S[m][i] = P[m - 1][i] + P[m][i] + P[m + 1][i];
        S[n - 1][i] = P[n - 2][i] + P[n - 1][i];
    }
    return S;
}

// ConvNeuralNetwork::Run (:640-963) on a w x h image; writes the response map
bool net_forward(const Net& N, const float* img, int w, int h, int stride, std::vector<float>& out, int* ow, int* oh) {
    if (w < N.min_w || h < N.min_h) return false;
    std::vector<float> in((size_t)w * h);
    for (int y = 0; y < h; ++y) memcpy(&in[(size_t)y * w], img + (size_t)y * stride, sizeof(float) * w);
    int cw, ch, pw = 0, ph = 0;
    std::vector<std::vector<float>> P1;
    for (int m = 0; m < N.maps[0]; ++m) {
        std::vector<float> c = conv(in, w, h, &N.k[0][(size_t)m * N.kw[0] * N.kh[0]], N.kw[0], N.kh[0], &cw, &ch);
        P1.push_back(act_pool(c, cw, ch, &N.act[0][5 * m], &pw, &ph));
    }
    std::vector<std::vector<float>> S1 = map_sums(P1), P2;
    int p2w = 0, p2h = 0;
    for (int m = 0; m < N.maps[1]; ++m) {
        std::vector<float> c = conv(S1[m / 2], pw, ph, &N.k[1][(size_t)m * 9], 3, 3, &cw, &ch);
        P2.push_back(act_pool(c, cw, ch, &N.act[1][5 * m], &p2w, &p2h));
    }
    std::vector<std::vector<float>> S2 = map_sums(P2), A3;
    int w3 = 0, h3 = 0;
    for (int m = 0; m < N.maps[2]; ++m) {
        std::vector<float> c = conv(S2[m / 2], p2w, p2h, &N.k[2][(size_t)m * N.kw[2] * N.kh[2]], N.kw[2], N.kh[2], &w3, &h3);
        for (auto& v : c) v = act(v, &N.act[2][5 * m]);
        A3.push_back(c);
    }
    *ow = w3;
    *oh = h3;
    out.assign((size_t)w3 * h3, 0.f);
    const int G = N.hl / N.hs;
    for (size_t px = 0; px < out.size(); ++px) {
        float acc = 0.f;
        for (int i = 0; i < G; ++i)
            for (int t = 0; t < N.hs; ++t) {
                const int nn = N.hs * i + t;
                float s = N.hb[nn];  // mulCN_add_tanhW (:646-672)
                for (int j = 0; j < N.conn; ++j) s = s + A3[i + j][px] * N.hw[(size_t)nn * N.conn + j];
                s = s * N.htw[i];
                s = tanh_approx(s);
                s = 0.5f * s + 0.5f;
                const float hv = N.hbn[2 * t] * s + N.hbn[2 * t + 1];
                const float wgt = N.ow[(size_t)N.index * N.hl + t * G + i];  // (:885-900)
                acc = (nn == 0) ? hv * wgt : hv * wgt + acc;
            }
        float c = (acc + N.ob[N.index]) * N.otw;  // tanhW (:673-690)
        c = tanh_approx(c);
        out[px] = N.af == 0.f ? 0.5f * c + 0.5f : N.af * c;
    }
    return true;
}

// ---------------------------------------------------------------- boxes (type.h:239-328)
struct Box {
    int x, y, w, h, x2, y2;
    float score = 0.f, scale = 0.f;
    int knn = 0, num = 0;
    bool checked = false;
};

Box mk(int x, int y, int w, int h, float score, float scale, int knn) {
    Box b;
    b.x = x;
    b.y = y;
    b.w = w;
    b.h = h;
    b.x2 = x + w;
    b.y2 = y + h;
    b.score = score;
    b.scale = scale;
    b.knn = knn;
    return b;
}

bool apart(const Box& a, const Box& b) { return a.x > b.x2 || b.x > a.x2 || a.y > b.y2 || b.y > a.y2; }

float overlap(const Box& a, const Box& b) {  // Rect::overlap: intersection over bounding box
    if (apart(a, b)) return 0.f;
    const int X0 = std::min(a.x, b.x), X1 = std::max(a.x, b.x), X2 = std::min(a.x2, b.x2), X3 = std::max(a.x2, b.x2);
    const int Y0 = std::min(a.y, b.y), Y1 = std::max(a.y, b.y), Y2 = std::min(a.y2, b.y2), Y3 = std::max(a.y2, b.y2);
    return (float)((X2 - X1) * (Y2 - Y1)) / (float)((X3 - X0) * (Y3 - Y0));
}

int intersection(const Box& a, const Box& b) {  // Rect::intersects
    if (apart(a, b)) return 0;
    return (std::min(a.x2, b.x2) - std::max(a.x, b.x)) * (std::min(a.y2, b.y2) - std::max(a.y, b.y));
}

Box shrink(const Box& r, float s) {  // Rect::operator*
    s = 1.f - s;
    const int sx = (int)((float)r.w * s), sy = (int)((float)r.h * s);
    return mk(r.x + (sx >> 1), r.y + (sy >> 1), r.w - sx, r.h - sy, 0.f, 0.f, 0);
}

// CNNDetector::Merger (cnn_detector_v3.cpp:2814-2936)
std::vector<Box> merger(std::vector<Box> in, float thr, bool del) {
    std::vector<Box> out;
    for (size_t i = 0; i < in.size(); ++i) {
        if (in[i].checked) continue;
        Box mx = in[i], mn = in[i];
        bool drop = false;
        for (size_t j = i + 1; j < in.size(); ++j) {
            Box& e = in[j];
            if (e.checked) continue;
            int X[4] = {mx.x, mx.x2, e.x, e.x2}, Y[4] = {mx.y, mx.y2, e.y, e.y2};
            if (X[0] >= X[3] || X[1] <= X[2] || Y[0] >= Y[3] || Y[1] <= Y[2]) continue;
            const float s1 = (float)((X[1] - X[0]) * (Y[1] - Y[0])), s2 = (float)((X[3] - X[2]) * (Y[3] - Y[2]));
            std::sort(X, X + 4);
            std::sort(Y, Y + 4);
            const float su = (float)((X[3] - X[0]) * (Y[3] - Y[0])), si = (float)((X[2] - X[1]) * (Y[2] - Y[1]));
            const float r1 = si / s1, r2 = si / s2, r3 = si / su;
            float ratio = std::min(r1, r2);
            const int cx1 = X[0] + ((X[3] - X[0]) >> 1), cy1 = Y[0] + ((Y[3] - Y[0]) >> 1);
            const int cx2 = X[1] + ((X[2] - X[1]) >> 1), cy2 = Y[1] + ((Y[2] - Y[1]) >> 1);
            const int tc = std::min(X[3] - X[0], X[2] - X[1]) >> 1;
            if (r3 > 0.75f * thr && std::max(r1, r2) > 0.7f && std::abs(cx1 - cx2) < tc && std::abs(cy1 - cy2) < tc) ratio = 1.f;
            if (!(ratio > thr)) continue;
            if (del) {
                if (s1 > s2) {
                    e.checked = true;
                    continue;
                }
                drop = true;
                break;
            }
            mx.x = std::min(mx.x, X[0]);
            mx.y = std::min(mx.y, Y[0]);
            mx.x2 = std::max(mx.x2, X[3]);
            mx.y2 = std::max(mx.y2, Y[3]);
            mn.x = std::max(mn.x, X[1]);
            mn.y = std::max(mn.y, Y[1]);
            mn.x2 = std::min(mn.x2, X[2]);
            mn.y2 = std::min(mn.y2, Y[2]);
            mx.score = mx.score < e.score ? e.score : mx.score;
            mx.knn = std::max(mx.knn, e.knn);
            mx.scale = mx.scale > e.scale ? e.scale : mx.scale;
            mx.num++;
            e.checked = true;
        }
        if (drop) continue;
        Box r = mx;
        r.x = (mn.x + mx.x) >> 1;
        r.y = (mn.y + mx.y) >> 1;
        r.x2 = (mn.x2 + mx.x2) >> 1;
        r.y2 = (mn.y2 + mx.y2) >> 1;
        r.w = r.x2 - r.x;
        r.h = r.y2 - r.y;
        r.checked = false;
        out.push_back(r);
    }
    return out;
}

// ---------------------------------------------------------------- the cascade (cnn_detector_v3.cpp)
struct Cascade {
    orc_params p;
    Net n1, n2, n3;
    int type_check = 1, min_num_detect = 1;
    bool adapt_mn = false, drop = true, detect = true, merge = true, double_check = true;
    bool gray_only = true, input_down = false;
    float input_scale = 0.f;
    std::vector<float> scales;
    int ext_w = 47, ext_h = 51;

    // Init precision rules (:922-963) after the API's conversion (CompactCNNLibAPI_v2.cpp:300-326)
    void rules() {
        type_check = 1;
        min_num_detect = 1;
        drop = p.drop_detect != 0;
        adapt_mn = false;
        double_check = true;
        detect = p.detect_mode != 0;
        merge = detect;
        if (p.detect_precision == 0) {
            gray_only = true;
            adapt_mn = true;
            drop = false;
            merge = true;
            p.equalize = 1;
            p.reflection = 1;
        }
        switch (p.detect_precision) {
            case 1: type_check = 0; drop = false; break;
            case 2: type_check = 1; break;
            case 3: type_check = 2; break;
            case 4: type_check = 2; min_num_detect = 2; break;
            default: break;
        }
        if (!detect) drop = false;
    }

    // InitScales (:289-346)
    bool init_scales() {
        scales.clear();
        input_down = false;
        const int ph = n1.min_h;
        float mx = 1.f;
        if (p.min_face_height > 0) {
            mx = std::min(3.f, (float)ph / (float)p.min_face_height);
            if (gray_only && mx < 0.8f) {
                input_down = true;
                input_scale = mx;
                mx = 1.f;
            }
        }
        float mn = p.max_face_height > 0 ? (float)ph / (float)p.max_face_height : (float)ph / (float)p.max_image_h;
        mn = std::min(mx, mn);
        if (p.scale_factor < 1.f) p.scale_factor = 1.1f;
        float s = mx;
        if (p.scale_factor != 1.f)
            while (s > mn) {
                scales.push_back(s);
                s /= p.scale_factor;
            }
        else
            scales.push_back(s);
        ext_w = detect ? n2.min_w + 11 : n1.min_w;
        ext_h = detect ? n2.min_h + 11 : n1.min_h;
        return !scales.empty();
    }
};

struct Verdict {
    bool accept;
    float score;
    int knn;
};

// CPUCheckDetect's window evaluation (:1489-1800) for one candidate and window (mod 0 / 1)
Verdict check_window(const Cascade& C, const std::vector<float>& gray, int gw, int gh, int px, int py, float score0, float scale, int mod) {
    const float inv = 1.f / scale;
    int x = (int)((float)(px - 6) * inv), y = (int)((float)(py - 5) * inv);
    int width = (int)((float)36 * inv), height = (int)((float)38 * inv);
    if (mod == 1) {
        const float k = 0.15f;
        x = (int)(x + width * k / 2.f);
        width = (int)(width - width * k);
        y = (int)(y + height * k / 2.f);
        height = (int)(height - height * k);
    }
    const int rx = std::min(std::max(x, 0), gw), ry = std::min(std::max(y, 0), gh);
    const int rc = std::min(std::max(x + width, 0), gw) - rx, rr = std::min(std::max(y + height, 0), gh) - ry;
    std::vector<float> crop(49 * 51);
    resize_f32(&gray[(size_t)ry * gw + rx], rc, rr, gw, crop.data(), 49, 51, 49, 0);
    std::vector<uint8_t> u8(49 * 51);
    for (int i = 0; i < 49 * 51; ++i) u8[i] = (uint8_t)(int)(crop[i] + 0.5f);  // FloatToUChar (image_proc.cpp:365)
    if (C.p.equalize) equalize(u8.data(), 49, 51, 49);
    const int mn = (C.adapt_mn && scale > 0.7f && C.p.min_neighbors > 1) ? C.p.min_neighbors - 1 : C.p.min_neighbors;
    float max1 = -10.f, max2 = -10.f;
    int k1 = 0, k2 = 0;
    std::vector<float> in(47 * 51), out;
    int ow, oh;
    for (int stage = 0; stage < 2; ++stage) {
        for (int yy = 0; yy < 51; ++yy)
            for (int xx = 0; xx < 47; ++xx) {
                int col = stage == 0 ? xx + 2 : (C.p.reflection ? 46 - xx : xx);  // UCharToFloat(offset 2) / _inv
                in[(size_t)yy * 47 + xx] = (float)u8[(size_t)yy * 49 + col];
            }
        net_forward(stage == 0 ? C.n2 : C.n3, in.data(), 47, 51, 47, out, &ow, &oh);
        for (float d : out) {
            if (stage == 0) {
                max1 = max1 < d ? d : max1;
                if (d > C.p.treshold[1]) k1++;
            } else {
                max2 = max2 < d ? d : max2;
                if (d > C.p.treshold[2]) k2++;
            }
        }
        if (C.type_check == 0 && k1 >= mn) break;
        if (C.type_check > 0 && k1 <= 0) break;
        if (C.type_check == 2 && k1 < mn) break;
    }
    bool flag = false;
    if (C.type_check == 0) flag = k1 >= mn || k2 >= mn;
    if (C.type_check == 1) flag = (k1 >= mn && k2 > 0) || (k1 > 0 && k2 >= mn);
    if (C.type_check == 2) flag = k1 >= mn && k2 >= mn;
    Verdict v;
    v.accept = flag;
    v.score = score0 + (float)k1 * std::max(-1.7159f, max1) + (float)k2 * std::max(-1.7159f, max2);
    v.knn = std::min(k1, k2);
    return v;
}

}  // namespace

extern "C" {

int orc_gray(const uint8_t* img, int w, int h, int ch, int step, float* out) {
    if (ch != 1 && ch != 3 && ch != 4) return -1;
    gray_image(img, w, h, ch, step, out, w);
    return 0;
}

int orc_resize_f32(const float* src, int sw, int sh, int sstride, float* dst, int dw, int dh, int type) {
    resize_f32(src, sw, sh, sstride, dst, dw, dh, dw, type);
    return 0;
}

int orc_equalize(uint8_t* img, int w, int h) {
    equalize(img, w, h, w);
    return 0;
}

int orc_net_forward(const char* model_path, int index_output, const float* img, int w, int h, int stride, float* out, int cap, int* ow,
                    int* oh) {
    Net n = load_net(model_path, index_output);
    if (!n.ok) return -1;
    std::vector<float> r;
    if (!net_forward(n, img, w, h, stride, r, ow, oh)) return -2;
    if ((int)r.size() > cap) return -3;
    memcpy(out, r.data(), sizeof(float) * r.size());
    return 0;
}

int orc_sort_perm(const float* keys, int n, int* perm) {
    std::vector<std::pair<float, int>> v(n);
    for (int i = 0; i < n; ++i) v[i] = std::make_pair(keys[i], i);
    std::sort(v.begin(), v.end(), [](const std::pair<float, int>& a, const std::pair<float, int>& b) { return b.first < a.first; });
    for (int i = 0; i < n; ++i) perm[i] = v[i].second;
    return 0;
}

// CNNDetector::Detect (:2483-2813) on the CPU pipeline, for one frame on a fresh detector
// (colour frames start from the state the reference reaches after its gray_image_only re-Init).
int orc_detect(const orc_params* prm, const char* model_dir, const uint8_t* img, int w, int h, int ch, int step, float* gray_out,
               int* gray_w, int* gray_h, int level_cap, int* n_levels, float* scales_out, int* level_w, int* level_h, float* resp_out,
               long resp_cap, int* resp_w, int* resp_h, orc_cand* cands_out, int cand_cap, int* n_cands, orc_det* raw, int raw_cap,
               int* n_raw, orc_det* final_out, int final_cap) {
    Cascade C;
    C.p = *prm;
    if (C.p.max_image_w < w) C.p.max_image_w = w;
    if (C.p.max_image_h < h) C.p.max_image_h = h;
    const std::string dir(model_dir);
    C.n1 = load_net(dir + "/cnn4face1_cntk.bin", 1);
    C.n2 = load_net(dir + "/cnn4face2_cntk.bin", 0);
    C.n3 = load_net(dir + "/cnn4face3_cntk.bin", 0);
    if (!C.n1.ok || !C.n2.ok || !C.n3.ok) return -1;
    C.gray_only = true;
    C.rules();
    if (ch != 1) C.gray_only = false;
    if (!C.init_scales()) return -2;
    *n_levels = 0;
    *n_cands = 0;
    *n_raw = 0;
    if (w < C.ext_w || h < C.ext_h) return 0;

    // gray image (with the 8-bit bilinear shrink for 1-channel input, :2531-2538)
    int gw = w, gh = h;
    std::vector<float> gray;
    if (C.input_down && ch == 1) {
        gw = (int)((float)w * C.input_scale);
        gh = (int)((float)h * C.input_scale);
        std::vector<uint8_t> small((size_t)gw * gh);
        resize_u8_bilinear(img, w, h, step, small.data(), gw, gh, gw);
        gray.resize((size_t)gw * gh);
        gray_image(small.data(), gw, gh, 1, gw, gray.data(), gw);
    } else {
        gray.resize((size_t)gw * gh);
        gray_image(img, w, h, ch, step, gray.data(), gw);
    }
    *gray_w = gw;
    *gray_h = gh;
    if (gray_out) memcpy(gray_out, gray.data(), sizeof(float) * gray.size());

    // levels and stage 1 (RunCPUDetect :2063-2233)
    struct Level {
        int w, h, rw, rh;
        float s;
        std::vector<float> resp;
    };
    std::vector<Level> lv;
    for (size_t scl = 0; scl < C.scales.size(); ++scl) {
        Level L;
        L.s = C.scales[scl];
        L.w = (int)((float)gw * L.s);
        L.h = (int)((float)gh * L.s);
        if (L.w < C.ext_w || L.h < C.ext_h) break;
        std::vector<float> li((size_t)L.w * L.h);
        resize_f32(gray.data(), gw, gh, gw, li.data(), L.w, L.h, L.w, L.s > 0.7f ? 0 : 1);
        net_forward(C.n1, li.data(), L.w, L.h, L.w, L.resp, &L.rw, &L.rh);
        lv.push_back(std::move(L));
    }
    const int nl = (int)lv.size();
    *n_levels = nl;
    long roff = 0;
    for (int i = 0; i < nl && i < level_cap; ++i) {
        scales_out[i] = lv[i].s;
        level_w[i] = lv[i].w;
        level_h[i] = lv[i].h;
        resp_w[i] = lv[i].rw;
        resp_h[i] = lv[i].rh;
        if (resp_out && roff + (long)lv[i].resp.size() <= resp_cap) memcpy(resp_out + roff, lv[i].resp.data(), sizeof(float) * lv[i].resp.size());
        roff += (long)lv[i].resp.size();
    }

    // candidates and stages 2/3, smallest level first (RunCheckDetect :1842-2011)
    std::vector<Box> det;
    int nc = 0;
    for (int scl = nl - 1; scl >= 0; --scl) {
        const Level& L = lv[scl];
        const float inv = 1.f / L.s;
        std::vector<std::pair<int, int>> pts;
        std::vector<float> sc;
        for (int j = 0; j < L.rh; ++j)
            for (int i = 0; i < L.rw; ++i) {
                const float r = L.resp[(size_t)j * L.rw + i];
                if (!(r > C.p.treshold[0])) continue;
                const int px = 4 * i, py = 4 * j;
                if (nc < cand_cap) {
                    cands_out[nc].level = scl;
                    cands_out[nc].x = px;
                    cands_out[nc].y = py;
                    cands_out[nc].score = r;
                }
                nc++;
                const Box nr = mk((int)((float)px * inv), (int)((float)py * inv), (int)((float)23 * inv), (int)((float)27 * inv), 0.f,
                                  L.s, 0);
                if (C.drop) {  // DropDetection (:1820-1840) against everything gathered so far
                    const Box ex = shrink(nr, 0.7f);
                    bool dropped = false;
                    for (size_t k = 0; k < det.size(); ++k) {
                        const float ov = overlap(nr, det[k]);
                        if (ov == 0.f) continue;
                        if (ov > 0.5f) {
                            det.push_back(mk(nr.x, nr.y, nr.w, nr.h, det[k].score, L.s, det[k].knn));
                            dropped = true;
                            break;
                        }
                        if (intersection(det[k], ex) == ex.w * ex.h) {
                            dropped = true;
                            break;
                        }
                    }
                    if (dropped) continue;
                }
                pts.push_back(std::make_pair(px, py));
                sc.push_back(r);
            }
        const size_t rect_size = det.size();
        for (size_t q = 0; q < pts.size(); ++q) {
            const int px = pts[q].first, py = pts[q].second;
            const Box nr = mk((int)((float)px * inv), (int)((float)py * inv), (int)((float)23 * inv), (int)((float)27 * inv), 0.f, L.s, 0);
            if (!C.detect) {
                det.push_back(mk(nr.x, nr.y, nr.w, nr.h, sc[q], L.s, 0));
                continue;
            }
            if (C.drop) {  // copy of an overlapping box found at this level (:1507-1527)
                bool hit = false;
                for (size_t k = rect_size; k < det.size(); ++k)
                    if (overlap(nr, det[k]) > 0.5f) {
                        det.push_back(mk(nr.x, nr.y, nr.w, nr.h, det[k].score, L.s, det[k].knn));
                        hit = true;
                        break;
                    }
                if (hit) continue;
            }
            for (int mod = 0; mod < (C.double_check ? 2 : 1); ++mod) {
                const Verdict v = check_window(C, gray, gw, gh, px, py, sc[q], L.s, mod);
                if (v.accept) {
                    det.push_back(mk(nr.x, nr.y, nr.w, nr.h, v.score, L.s, v.knn));
                    break;
                }
            }
        }
    }
    *n_cands = nc;
    *n_raw = (int)det.size();
    for (int i = 0; i < (int)det.size() && i < raw_cap; ++i) {
        raw[i].x = det[i].x;
        raw[i].y = det[i].y;
        raw[i].w = det[i].w;
        raw[i].h = det[i].h;
        raw[i].score = det[i].score;
        raw[i].scale = det[i].scale;
        raw[i].knn = det[i].knn;
        raw[i].num_detect = det[i].num;
    }

    // post-processing (:2745-2810)
    std::vector<Box> all(det.rbegin(), det.rend()), fin;
    if (!all.empty()) {
        std::sort(all.begin(), all.end(), [](const Box& a, const Box& b) { return b.scale < a.scale; });
        if (C.merge) {
            std::vector<Box> t = merger(all, 0.5f, false);
            if (C.min_num_detect > 1)
                t.erase(std::remove_if(t.begin(), t.end(), [&](const Box& b) { return b.num < C.min_num_detect; }), t.end());
            if (!t.empty()) fin = merger(t, 0.2f, true);
        } else {
            fin = all;
        }
        if (C.input_down && ch == 1) {
            const float s = (float)C.p.min_face_height / (float)C.n1.min_h;
            for (auto& b : fin) {
                const int x = (int)((float)b.x * s), y = (int)((float)b.y * s), ww = (int)((float)b.w * s), hh = (int)((float)b.h * s);
                b = mk(x, y, ww, hh, b.score, b.scale, b.knn);
            }
        }
    }
    for (int i = 0; i < (int)fin.size() && i < final_cap; ++i) {
        final_out[i].x = fin[i].x;
        final_out[i].y = fin[i].y;
        final_out[i].w = fin[i].w;
        final_out[i].h = fin[i].h;
        final_out[i].score = fin[i].score;
        final_out[i].scale = fin[i].scale;
        final_out[i].knn = fin[i].knn;
        final_out[i].num_detect = fin[i].num;
    }
    return (int)fin.size();
}

}  // extern "C"
