// CNTK-format model reader and packer. The byte layout is the reference's
// (SIMD::ConvNeuralNetwork::Init, src/CNNObjectDetector/cnn_simd_cntk.cpp:42-404, plain-C++
// branch): version f32, max_pool u8, min size 2 x i32, layer count i32, maps per layer, then per
// conv layer (kw, kh) and maps x kw*kh kernels, af_scale, per map (bias, lrelu_w1, lrelu_w2,
// bn_weight, bn_bias), snn_full_connect u8, hidden size, connections, hl_scale, hidden weights,
// biases, per-group tanh slopes, hl_scale x (bn_weight, bn_bias), output neuron count, output
// weights and biases, output tanh slope.
#include "model.h"

#include <dlfcn.h>

#include <cstring>
#include <fstream>
#include <sstream>

namespace ccnn {

namespace {
struct Reader {
    const uint8_t* p;
    size_t n, off = 0;
    bool ok = true;
    template <class T>
    T get() {
        T v{};
        if (off + sizeof(T) > n) {
            ok = false;
            return v;
        }
        std::memcpy(&v, p + off, sizeof(T));
        off += sizeof(T);
        return v;
    }
    bool floats(std::vector<float>& v, long long count) {
        if (count < 0 || count > (1 << 24)) return ok = false;
        v.resize((size_t)count);
        for (auto& x : v) x = get<float>();
        return ok;
    }
};
}  // namespace

bool parse_model(const uint8_t* data, size_t n, RawModel* m, std::string* err) {
    Reader r{data, n};
    m->version = r.get<float>();
    if (!r.ok || m->version < 1.0f || m->version > 1.1f) {
        *err = "model format version is not supported (CNTK format 1.0-1.1 expected)";
        return false;
    }
    m->max_pool = r.get<uint8_t>() != 0;
    m->min_w = r.get<int32_t>();
    m->min_h = r.get<int32_t>();
    m->layers = r.get<int32_t>();
    if (!r.ok || m->layers != 3) {
        *err = "model must have 3 convolution layers";
        return false;
    }
    for (int i = 0; i < 3; ++i) m->maps[i] = r.get<int32_t>();
    for (int l = 0; l < 3; ++l) {
        m->kw[l] = r.get<int32_t>();
        m->kh[l] = r.get<int32_t>();
        if (!r.ok || m->kw[l] <= 0 || m->kh[l] <= 0 || m->maps[l] <= 0 || m->maps[l] > 4096) {
            *err = "malformed convolution layer";
            return false;
        }
        if (!r.floats(m->kernels[l], (long long)m->maps[l] * m->kw[l] * m->kh[l])) break;
    }
    m->af_scale = r.get<float>();
    for (int l = 0; l < 3; ++l) r.floats(m->act[l], 5LL * m->maps[l]);
    m->full_connect = r.get<uint8_t>() != 0;
    m->hl = r.get<int32_t>();
    m->conn = r.get<int32_t>();
    m->hs = r.get<int32_t>();
    if (!r.ok) {
        *err = "model file is truncated";
        return false;
    }
    if (!m->max_pool || m->kw[1] * m->kh[1] != 9) {
        // the reference refuses the same (cnn_simd_cntk.cpp:322-329)
        *err = "this configuration of cnn models is not supported (max pooling and a 3x3 second layer required)";
        return false;
    }
    if (m->hl <= 0 || m->hs <= 0 || m->hl % m->hs != 0 || m->conn <= 0) {
        *err = "malformed hidden layer";
        return false;
    }
    const long long per = m->full_connect ? m->maps[2] : m->conn;
    r.floats(m->hw, (long long)m->hl * per);
    r.floats(m->hb, m->hl);
    r.floats(m->htw, m->hl / m->hs);
    r.floats(m->hbn, 2LL * m->hs);
    m->nout = r.get<int32_t>();
    if (!r.ok || m->nout <= 0 || m->nout > 4096) {
        *err = "malformed output layer";
        return false;
    }
    r.floats(m->ow, (long long)m->nout * m->hl);
    r.floats(m->ob, m->nout);
    m->otw = r.get<float>();
    if (!r.ok) {
        *err = "model file is truncated";
        return false;
    }
    return true;
}

bool load_model_file(const std::string& path, RawModel* m, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) {
        *err = "model file not found: " + path;
        return false;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string s = ss.str();
    if (!parse_model(reinterpret_cast<const uint8_t*>(s.data()), s.size(), m, err)) {
        *err += " (" + path + ")";
        return false;
    }
    return true;
}

template <class NW>
bool pack_model(const RawModel& m, int index_output, NW* o, std::string* err) {
    const bool shape_ok = m.maps[0] == NW::kM1 && m.maps[1] == NW::kM2 && m.maps[2] == NW::kM3 && m.kw[0] == NW::kK1W &&
                          m.kh[0] == NW::kK1H && m.kw[1] == NW::kK2W && m.kh[1] == NW::kK2H && m.kw[2] == NW::kK3W &&
                          m.kh[2] == NW::kK3H && m.hl == NW::kHL && m.conn == NW::kConn && m.hs == NW::kHS && !m.full_connect;
    if (!shape_ok) {
        *err = "model shape differs from the cascade prototype this build supports (cntk/stage_{1,2,3}.cntk)";
        return false;
    }
    if (index_output < 0) {
        *err = "index_output must be >= 0";
        return false;
    }
    std::memset(o, 0, sizeof(NW));
    auto tap = [&](int l, int mm, int k) { return m.kernels[l][(size_t)mm * m.kw[l] * m.kh[l] + k]; };
    for (int mm = 0; mm < NW::kM1; ++mm)
        for (int k = 0; k < NW::kK1W * NW::kK1H; ++k) o->k1d[mm][k] = make_float2(tap(0, mm, k), tap(0, mm, k));
    for (int i = 0; i < NW::kM1 / 2; ++i)
        for (int k = 0; k < NW::kK1W * NW::kK1H; ++k) o->k1p[i][k] = make_float2(tap(0, 2 * i, k), tap(0, 2 * i + 1, k));
    for (int i = 0; i < NW::kM2 / 2; ++i)
        for (int k = 0; k < NW::kK2W * NW::kK2H; ++k) o->k2p[i][k] = make_float2(tap(1, 2 * i, k), tap(1, 2 * i + 1, k));
    for (int i = 0; i < NW::kM3 / 2; ++i)
        for (int k = 0; k < NW::kK3W * NW::kK3H; ++k) o->k3p[i][k] = make_float2(tap(2, 2 * i, k), tap(2, 2 * i + 1, k));
    auto act = [&](int l, int mm, int field) { return m.act[l][5 * mm + field]; };
    for (int mm = 0; mm < NW::kM1; ++mm) {
        o->b1[mm] = act(0, mm, 0);
        o->w1a[mm] = act(0, mm, 1);
        o->w1b[mm] = act(0, mm, 2);
        o->bn1[mm] = act(0, mm, 4);  // bn_weight is folded into w1/w2 by the converter and unused
    }
    for (int mm = 0; mm < NW::kM2; ++mm) {
        o->b2[mm] = act(1, mm, 0);
        o->w2a[mm] = act(1, mm, 1);
        o->w2b[mm] = act(1, mm, 2);
        o->bn2[mm] = act(1, mm, 4);
    }
    for (int mm = 0; mm < NW::kM3; ++mm) {
        o->b3[mm] = act(2, mm, 0);
        o->w3a[mm] = act(2, mm, 1);
        o->w3b[mm] = act(2, mm, 2);
        o->bn3[mm] = act(2, mm, 4);
    }
    for (int mm = 0; mm < NW::kM1; ++mm) {
        const float v[4] = {o->b1[mm], o->w1a[mm], o->w1b[mm], o->bn1[mm]};
        for (int f = 0; f < 4; ++f) o->a1d[mm][f] = make_float2(v[f], v[f]);
    }
    for (int i = 0; i < NW::kM1 / 2; ++i) {
        o->a1p[i][0] = make_float2(o->b1[2 * i], o->b1[2 * i + 1]);
        o->a1p[i][1] = make_float2(o->w1a[2 * i], o->w1a[2 * i + 1]);
        o->a1p[i][2] = make_float2(o->w1b[2 * i], o->w1b[2 * i + 1]);
        o->a1p[i][3] = make_float2(o->bn1[2 * i], o->bn1[2 * i + 1]);
    }
    for (int i = 0; i < NW::kM2 / 2; ++i) {
        o->a2p[i][0] = make_float2(o->b2[2 * i], o->b2[2 * i + 1]);
        o->a2p[i][1] = make_float2(o->w2a[2 * i], o->w2a[2 * i + 1]);
        o->a2p[i][2] = make_float2(o->w2b[2 * i], o->w2b[2 * i + 1]);
        o->a2p[i][3] = make_float2(o->bn2[2 * i], o->bn2[2 * i + 1]);
    }
    for (int i = 0; i < NW::kM3 / 2; ++i) {
        o->a3p[i][0] = make_float2(o->b3[2 * i], o->b3[2 * i + 1]);
        o->a3p[i][1] = make_float2(o->w3a[2 * i], o->w3a[2 * i + 1]);
        o->a3p[i][2] = make_float2(o->w3b[2 * i], o->w3b[2 * i + 1]);
        o->a3p[i][3] = make_float2(o->bn3[2 * i], o->bn3[2 * i + 1]);
    }
    for (int n = 0; n < NW::kHL; ++n) o->hb[n] = m.hb[n];
    for (int q = 0; q < NW::kHL / 2; ++q)
        for (int j = 0; j < NW::kConn; ++j)
            o->hwp[q][j] = make_float2(m.hw[(size_t)(2 * q) * NW::kConn + j], m.hw[(size_t)(2 * q + 1) * NW::kConn + j]);
    for (int i = 0; i < NW::kGroups; ++i) o->htw[i] = m.htw[i];
    for (int t = 0; t < NW::kHS; ++t) {
        o->hbnw[t] = m.hbn[2 * t];
        o->hbnb[t] = m.hbn[2 * t + 1];
    }
    const int idx = index_output < m.nout - 1 ? index_output : m.nout - 1;
    // output sum visits n = HS*i + t with weight t*G + i (cnn_simd_cntk.cpp:885-900)
    for (int i = 0; i < NW::kGroups; ++i)
        for (int t = 0; t < NW::kHS; ++t) o->ow[NW::kHS * i + t] = m.ow[(size_t)idx * m.hl + t * NW::kGroups + i];
    o->ob = m.ob[idx];
    o->otw = m.otw;
    o->af = idx == 0 ? -m.af_scale : m.af_scale;
    o->negzero = make_float2(-0.f, -0.f);
    return true;
}

template bool pack_model<Stage1W>(const RawModel&, int, Stage1W*, std::string*);
template bool pack_model<Stage2W>(const RawModel&, int, Stage2W*, std::string*);
template bool pack_model<Stage3W>(const RawModel&, int, Stage3W*, std::string*);

bool pack_landmarks(const RawModel& m, LandmarkNet* o, std::string* err) {
    using LN = LandmarkNet;
    const bool shape_ok = m.min_w == LN::kInW && m.min_h == LN::kInH && m.maps[0] == LN::kM1 && m.maps[1] == LN::kM2 &&
                          m.maps[2] == LN::kM3 && m.kw[0] == 4 && m.kh[0] == 4 && m.kw[1] == 3 && m.kh[1] == 3 &&
                          m.kw[2] == LN::kK3W && m.kh[2] == LN::kK3H && m.full_connect && m.hl == LN::kHL && m.hs == LN::kHL &&
                          m.nout == LN::kOut;
    if (!shape_ok) {
        *err = "facial-analysis model shape differs from cnn4landmarks_cntk.bin";
        return false;
    }
    std::memset(o, 0, sizeof(LN));
    auto tap = [&](int l, int mm, int k) { return m.kernels[l][(size_t)mm * m.kw[l] * m.kh[l] + k]; };
    auto act = [&](int l, int mm, int field) { return m.act[l][5 * mm + field]; };
    auto act_pair = [&](int l, int i, float2* out4) {
        const int f[4] = {0, 1, 2, 4};  // conv bias, lrelu w1, lrelu w2, bn bias (bn weight folded)
        for (int q = 0; q < 4; ++q) out4[q] = make_float2(act(l, 2 * i, f[q]), act(l, 2 * i + 1, f[q]));
    };
    for (int i = 0; i < LN::kM1 / 2; ++i) {
        for (int k = 0; k < 16; ++k) o->k1p[i][k] = make_float2(tap(0, 2 * i, k), tap(0, 2 * i + 1, k));
        act_pair(0, i, o->a1p[i]);
    }
    for (int i = 0; i < LN::kM2 / 2; ++i) {
        for (int k = 0; k < 9; ++k) o->k2p[i][k] = make_float2(tap(1, 2 * i, k), tap(1, 2 * i + 1, k));
        act_pair(1, i, o->a2p[i]);
    }
    for (int i = 0; i < LN::kM3 / 2; ++i) {
        for (int k = 0; k < LN::kK3W * LN::kK3H; ++k) o->k3p[i][k] = make_float2(tap(2, 2 * i, k), tap(2, 2 * i + 1, k));
        act_pair(2, i, o->a3p[i]);
    }
    for (int q = 0; q < LN::kHL / 2; ++q) {
        for (int j = 0; j < LN::kM3; ++j)
            o->hwp[q][j] = make_float2(m.hw[(size_t)(2 * q) * LN::kM3 + j], m.hw[(size_t)(2 * q + 1) * LN::kM3 + j]);
        o->hbp[q] = make_float2(m.hb[2 * q], m.hb[2 * q + 1]);
        o->hbnwp[q] = make_float2(m.hbn[2 * (2 * q)], m.hbn[2 * (2 * q + 1)]);
        o->hbnbp[q] = make_float2(m.hbn[2 * (2 * q) + 1], m.hbn[2 * (2 * q + 1) + 1]);
    }
    o->htw = m.htw[0];
    // one group, so the output sum visits the hidden neurons in order with weight index t
    for (int k = 0; k < LN::kOut; ++k) {
        for (int t = 0; t < LN::kHL; ++t) o->ow[k][t] = m.ow[(size_t)k * m.hl + t];
        o->ob[k] = m.ob[k];
    }
    o->otw = m.otw;
    o->af = m.af_scale;  // index_output -1: every output, no sign flip (cnn_simd_cntk.cpp:396-397)
    o->negzero = make_float2(-0.f, -0.f);
    return true;
}

std::string bundled_model_dir() {
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&bundled_model_dir), &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        size_t s = p.rfind('/');
        std::string dir = (s == std::string::npos) ? std::string(".") : p.substr(0, s);
        return dir + "/models";
    }
    return "models";
}

}  // namespace ccnn
