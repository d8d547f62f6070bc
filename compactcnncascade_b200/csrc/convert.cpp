// CNTK model dump -> cascade model file (format 1.1), the reference's
// FaceDetector::CNTKDump2Binary (src/CNNObjectDetector/CompactCNNLibAPI_v2.cpp:509-519), which runs
// CNNModelsConverter::LoadCNTKModel with preprocessing on and SaveToBinaryFile
// (src/CNNObjectDetector/cnn_models_converter.cpp:79-746).
//
// The dump is CNTK's text listing of a trained network: node headers such as
//   z.c11.W=LearnableParameter [4 x 4 x 3 x 1]   followed by value lines up to a line holding '#'
// The conversion, restated:
//   * layer and map counts: the highest l with a line containing "z.c<l>", per layer the highest s
//     with "z.c<l><s>"; kernel sizes from the "Kernel:" field of the z.c<l>1.c node;
//   * L1 kernels: the three input-channel planes of each row summed, transposed, then scaled by
//     1/128, the conv bias lowered by the sum of the unscaled kernel (input normalisation folded);
//   * L2/L3 kernels transposed; batch norm folded: w = scale / sqrtf(var + 1e-5),
//     b = bias - mean * scale / sqrtf(var + 1e-5), and the LeakyReLU weights multiplied by w;
//   * hidden layer: groups z.h<i>, connections and group size from the z.h1.c "Kernel:" field,
//     weights transposed per group, one tanh slope per group, batch norm per slot (one line each);
//   * outputs from z.z.arrayOfFunctions[0] (W, b) and the output tanh slope; more than three
//     outputs select the sigmoid form (af_scale 0), else 1.7159.
// Every step keeps the reference's float arithmetic (sqrtf, division, the double-precision sum of
// the L1 correction) so the written bytes are identical.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ccnn_inspect.h"

namespace ccnn {
void set_error(const std::string& msg);
}

namespace {

using Lines = std::vector<std::string>;

bool any_line_has(const Lines& d, const std::string& key) {
    for (const auto& s : d)
        if (s.find(key) != std::string::npos) return true;
    return false;
}

std::vector<std::string> tokens_after(const std::string& s, const char* mark) {
    const size_t p = s.find(mark);
    std::istringstream iss(p == std::string::npos ? std::string() : s.substr(p));
    return std::vector<std::string>{std::istream_iterator<std::string>{iss}, std::istream_iterator<std::string>{}};
}

// values of node `z.<node>.<param>=`: every token of the following lines up to one holding '#';
// line >= 0 keeps only that line's tokens
bool node_values(const Lines& d, const std::string& node, const std::string& param, int line, std::vector<float>* out) {
    out->clear();
    const std::string key = "z." + node + "." + param + "=";
    for (size_t i = 0; i < d.size(); ++i) {
        if (d[i].find(key) == std::string::npos) continue;
        int k = 0;
        for (size_t j = i + 1; j < d.size() && d[j].find('#') == std::string::npos; ++j, ++k) {
            std::istringstream iss(d[j]);
            std::string tok;
            while (iss >> tok)
                if (line < 0 || k == line) out->push_back(std::stof(tok));
        }
        return true;
    }
    return false;
}

// the two numbers after "Kernel:" of node `z.<node>.c=` (width, height)
bool kernel_size(const Lines& d, const std::string& node, int* w, int* h) {
    const std::string key = "z." + node + ".c=";
    for (const auto& s : d)
        if (s.find(key) != std::string::npos) {
            const auto t = tokens_after(s, "Kernel:");
            if (t.size() < 4) return false;
            *w = std::stoi(t[1]);
            *h = std::stoi(t[3]);
            return true;
        }
    return false;
}

struct Model {
    bool max_pool = false;
    int min_w = 0, min_h = 0;
    std::vector<int> maps;
    int kw[3] = {0, 0, 0}, kh[3] = {0, 0, 0};
    std::vector<std::vector<float>> kernels[3];
    float af = 1.7159f;
    std::vector<std::vector<float>> bias, w1, w2, bnw, bnb;
    bool full_connect = false;
    int hl = 0, conn = 0, hs = 0;
    std::vector<std::vector<float>> hw;
    std::vector<float> hb, htw, hbnw, hbnb;
    std::vector<std::vector<float>> ow;
    std::vector<float> ob;
    float otw = 0.f;
};

bool fail(const std::string& m) {
    ccnn::set_error("CNTK dump: " + m);
    return false;
}

bool load_dump(const std::string& path, Model* m) {
    std::ifstream f(path);
    if (!f.is_open()) return fail("file not found: " + path);
    Lines d;
    std::string s;
    while (std::getline(f, s)) {
        for (size_t p = s.find("._"); p != std::string::npos; p = s.find("._")) s.erase(p, 2);
        d.push_back(s);
    }
    // input size and pooling type
    bool got = false;
    for (const auto& line : d)
        if (line.find("features") != std::string::npos) {
            const auto t = tokens_after(line, "[");
            if (t.size() < 4) return fail("features node without a size");
            m->min_w = std::stoi(t[1]);
            m->min_h = std::stoi(t[3]);
            got = true;
            break;
        }
    if (!got) return fail("no features node");
    for (size_t i = 0; i + 1 < d.size(); ++i)
        if (d[i].find("Pooling") != std::string::npos) {
            std::istringstream iss(d[i + 1]);
            std::string a, b;
            iss >> a >> b;
            m->max_pool = !b.empty() && std::stoi(b) == 1;
            break;
        }
    // structure
    int layers = 1;
    while (any_line_has(d, "z.c" + std::to_string(layers))) ++layers;
    --layers;
    if (layers != 3) return fail("the cascade format needs 3 convolution layers");
    for (int l = 1; l <= layers; ++l) {
        int sf = 1;
        while (any_line_has(d, "z.c" + std::to_string(l) + std::to_string(sf))) ++sf;
        m->maps.push_back(sf - 1);
    }
    std::vector<float> v;
    std::vector<double> preproc(m->maps[0], 0.0);
    for (int l = 0; l < 3; ++l) {
        if (!kernel_size(d, "c" + std::to_string(l + 1) + "1", &m->kw[l], &m->kh[l])) return fail("no kernel size of layer " + std::to_string(l + 1));
        const int kw = m->kw[l], kh = m->kh[l], n = kw * kh;
        for (int k = 0; k < m->maps[l]; ++k) {
            if (!node_values(d, "c" + std::to_string(l + 1) + std::to_string(k + 1), "W", -1, &v)) return fail("missing kernel");
            std::vector<float> plane(n);
            if (l == 0) {  // three input channels summed per row
                if ((int)v.size() < 3 * n) return fail("short layer-1 kernel");
                for (int y = 0; y < kh; ++y)
                    for (int x = 0; x < kw; ++x)
                        plane[y * kw + x] = v[3 * kw * y + 0 * kw + x] + v[3 * kw * y + 1 * kw + x] + v[3 * kw * y + 2 * kw + x];
            } else {
                if ((int)v.size() < n) return fail("short kernel");
                plane.assign(v.begin(), v.begin() + n);
            }
            std::vector<float> t(n);
            for (int e = 0; e < n; ++e) t[e] = plane[kh * (e % kw) + e / kw];  // transpose
            if (l == 0)
                for (int e = 0; e < n; ++e) {
                    preproc[k] += -1.0 * (double)t[e];
                    t[e] *= 0.0078125f;
                }
            m->kernels[l].push_back(t);
        }
    }
    // per-map activation and folded batch norm
    m->bias.resize(3);
    m->w1.resize(3);
    m->w2.resize(3);
    m->bnw.resize(3);
    m->bnb.resize(3);
    for (int l = 0; l < 3; ++l)
        for (int j = 0; j < m->maps[l]; ++j) {
            const std::string c = "c" + std::to_string(l + 1) + std::to_string(j + 1);
            const std::string bn = "bn" + std::to_string(l + 1) + std::to_string(j + 1);
            float a1, a2, b, sc, bb, mean, var;
            if (!node_values(d, c, "res.PlusArgs[0].ElementTimesArgs[0]", -1, &v) || v.empty()) return fail("missing " + c + " w1");
            a1 = v[0];
            if (!node_values(d, c, "res.PlusArgs[1].ElementTimesArgs[0]", -1, &v) || v.empty()) return fail("missing " + c + " w2");
            a2 = v[0];
            if (!node_values(d, c, "b", -1, &v) || v.empty()) return fail("missing " + c + " bias");
            b = v[0];
            if (!node_values(d, bn, "scale", -1, &v) || v.empty()) return fail("missing " + bn);
            sc = v[0];
            if (!node_values(d, bn, "bias", -1, &v) || v.empty()) return fail("missing " + bn);
            bb = v[0];
            if (!node_values(d, bn, "runMean", -1, &v) || v.empty()) return fail("missing " + bn);
            mean = v[0];
            if (!node_values(d, bn, "runVariance", -1, &v) || v.empty()) return fail("missing " + bn);
            var = v[0] + 0.00001f;
            const float bw = sc / sqrtf(var);
            const float bnbias = bb - mean * sc / sqrtf(var);
            if (l == 0) b += (float)preproc[j];
            m->bias[l].push_back(b);
            m->w1[l].push_back(a1 * bw);
            m->w2[l].push_back(a2 * bw);
            m->bnw[l].push_back(bw);
            m->bnb[l].push_back(bnbias);
        }
    // hidden layer
    int groups = 1;
    while (any_line_has(d, "z.h" + std::to_string(groups))) ++groups;
    --groups;
    bool hk = false;
    for (const auto& line : d)
        if (line.find("z.h1.c=Convolution") != std::string::npos) {
            const auto t = tokens_after(line, "Kernel:");
            if (t.size() < 8) return fail("z.h1.c kernel field");
            m->conn = std::stoi(t[1]);
            m->hs = std::stoi(t[7]);
            const int last = m->maps[2];
            m->full_connect = std::stoi(t[1]) == last || std::stoi(t[3]) == last;
            hk = true;
            break;
        }
    if (!hk || groups <= 0 || m->hs <= 0 || m->conn <= 0) return fail("no hidden layer");
    m->hl = m->hs * groups;
    m->hw.assign(m->hl, std::vector<float>(m->conn));
    for (int i = 0; i < groups; ++i) {
        if (!node_values(d, "h" + std::to_string(i + 1), "W", -1, &v) || (int)v.size() < m->hs * m->conn) return fail("hidden weights");
        for (int j = 0; j < m->hs; ++j)
            for (int k = 0; k < m->conn; ++k) {
                const int n = j * m->conn + k;  // transposed index
                m->hw[m->hs * i + j][k] = v[m->hs * (n % m->conn) + n / m->conn];
            }
    }
    m->hb.assign(m->hl, 0.f);
    for (int i = 0; i < groups; ++i) {
        if (!node_values(d, "h" + std::to_string(i + 1), "b", -1, &v) || (int)v.size() < m->hs) return fail("hidden bias");
        for (int j = 0; j < m->hs; ++j) m->hb[m->hs * i + j] = v[j];
        if (!node_values(d, "h" + std::to_string(i + 1), "res.PlusArgs[0].ElementTimesArgs[1].x.ElementTimesArgs[0]", -1, &v) || v.empty())
            return fail("hidden tanh slope");
        m->htw.push_back(v[0]);
    }
    for (int t = 0; t < m->hs; ++t) {
        float sc, bb, mean, var;
        if (!node_values(d, "bn_h", "scale", t, &v) || v.empty()) return fail("bn_h scale");
        sc = v[0];
        if (!node_values(d, "bn_h", "bias", t, &v) || v.empty()) return fail("bn_h bias");
        bb = v[0];
        if (!node_values(d, "bn_h", "runMean", t, &v) || v.empty()) return fail("bn_h runMean");
        mean = v[0];
        if (!node_values(d, "bn_h", "runVariance", t, &v) || v.empty()) return fail("bn_h runVariance");
        var = v[0] + 0.00001f;
        m->hbnw.push_back(sc / sqrtf(var));
        m->hbnb.push_back(bb - mean * sc / sqrtf(var));
    }
    // outputs
    if (!node_values(d, "z", "arrayOfFunctions[0].W", -1, &v) || v.empty()) return fail("output weights");
    const int nout = (int)v.size() / m->hl;
    for (int i = 0; i < nout; ++i) m->ow.emplace_back(v.begin() + (size_t)i * m->hl, v.begin() + (size_t)(i + 1) * m->hl);
    if (!node_values(d, "z", "arrayOfFunctions[0].b", -1, &v)) return fail("output bias");
    m->ob = v;
    if ((int)m->ob.size() > 3) m->af = 0.f;
    if (!node_values(d, "z", "PlusArgs[0].ElementTimesArgs[1].x.ElementTimesArgs[0]", -1, &v) || v.empty()) return fail("output tanh slope");
    m->otw = v[0];
    return true;
}

template <class T>
void put(std::ofstream& f, T v) {
    f.write(reinterpret_cast<const char*>(&v), sizeof(T));
}

bool save(const std::string& path, const Model& m) {
    std::ofstream f(path, std::ios::binary);
    if (!f.is_open()) return fail("cannot write " + path);
    put<float>(f, 1.1f);
    put<bool>(f, m.max_pool);
    put<int32_t>(f, m.min_w);
    put<int32_t>(f, m.min_h);
    put<int32_t>(f, 3);
    for (int l = 0; l < 3; ++l) put<int32_t>(f, m.maps[l]);
    for (int l = 0; l < 3; ++l) {
        put<int32_t>(f, m.kw[l]);
        put<int32_t>(f, m.kh[l]);
        for (const auto& k : m.kernels[l])
            for (float x : k) put<float>(f, x);
    }
    put<float>(f, fabsf(m.af));
    for (int l = 0; l < 3; ++l)
        for (int j = 0; j < m.maps[l]; ++j) {
            put<float>(f, m.bias[l][j]);
            put<float>(f, m.w1[l][j]);
            put<float>(f, m.w2[l][j]);
            put<float>(f, m.bnw[l][j]);
            put<float>(f, m.bnb[l][j]);
        }
    put<bool>(f, m.full_connect);
    put<int32_t>(f, m.hl);
    put<int32_t>(f, m.conn);
    put<int32_t>(f, m.hs);
    const int per = m.full_connect ? m.maps[2] : m.conn;
    for (int i = 0; i < m.hl; ++i)
        for (int j = 0; j < per; ++j) put<float>(f, j < m.conn ? m.hw[i][j] : 0.f);
    for (float x : m.hb) put<float>(f, x);
    for (float x : m.htw) put<float>(f, x);
    for (int t = 0; t < m.hs; ++t) {
        put<float>(f, m.hbnw[t]);
        put<float>(f, m.hbnb[t]);
    }
    put<int32_t>(f, (int32_t)m.ob.size());
    for (const auto& w : m.ow)
        for (float x : w) put<float>(f, x);
    for (float x : m.ob) put<float>(f, x);
    put<float>(f, m.otw);
    return (bool)f;
}

}  // namespace

extern "C" CCNN_API ccnn_status ccnn_cntk_dump_to_binary(const char* binary_file, const char* cntk_model_dump) {
    if (!binary_file || !binary_file[0] || !cntk_model_dump) {
        ccnn::set_error("invalid arguments");
        return CCNN_ERR_INVALID_ARG;
    }
    Model m;
    if (!load_dump(cntk_model_dump, &m)) return CCNN_ERR_MODEL;
    std::string out(binary_file);
    if (out.find(".bin") == std::string::npos) out += ".bin";  // SaveToBinaryFile appends the extension
    if (!save(out, m)) return CCNN_ERR_INVALID_ARG;
    return CCNN_OK;
}
