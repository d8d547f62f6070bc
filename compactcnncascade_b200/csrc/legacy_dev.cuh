// Device arithmetic of the legacy (format 1.0) networks, shared by the standalone forward pass
// and the stage-2/3 window kernel. Every operation is the reference's plain-C++ one
// (src/CNNObjectDetector/cnnpp_cplusplus.cpp), in the same order.
#pragma once

#include "ccnn_common.cuh"
#include "legacy.h"

namespace ccnn {

// tanh(c + b) of the four convolution outputs of a 2x2 window, their max or sum, then
// tanh(w * pooled + b) * af (max_tanh_tanh :473, tanh_avr_tanh :411)
__device__ __forceinline__ float lg_pool_tanh(const float c[4], int max_pool, float cb, float sw, float sb, float af) {
    float t[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) t[d] = tanh_rational(fadd(c[d], cb));
    const float p = max_pool ? fmaxf(fmaxf(t[0], t[1]), fmaxf(t[2], t[3])) : fadd(fadd(fadd(t[0], t[1]), t[2]), t[3]);
    return fmul(af, tanh_rational(fadd(fmul(sw, p), sb)));
}

// neighbouring-map sum i of `count` pooled maps (planes `plane` floats apart, element o), with the
// reference's additions: maps 0+1, (i-1)+i+(i+1), and (count-2)+(count-1) (add :916, add2 :933)
__device__ __forceinline__ float lg_map_sum(const float* __restrict__ planes, long long plane, int count, int i, long long o) {
    if (i == 0) return fadd(planes[o], planes[plane + o]);
    if (i == count - 1) return fadd(planes[(count - 2) * plane + o], planes[(count - 1) * plane + o]);
    return fadd(fadd(planes[(i - 1) * plane + o], planes[i * plane + o]), planes[(i + 1) * plane + o]);
}

// L3 map m at one output: the convolution chain over the kernel taps (`in(t)` is tap t's input,
// row-major; conv_6x5 :212, conv_8x7 :292), then tanh_tanh (:778) for a fully connected net, or
// tanh_tanh_2tanh (:692) with the map's two hidden neurons
template <class In>
__device__ __forceinline__ float lg_l3_value(const LegacyNet& N, int m, In in) {
    const float* k = N.k3[m];
    const int kt = N.k3w * N.k3h;
    float c = fmul(in(0), k[0]);
    for (int t = 1; t < kt; ++t) c = fadd(c, fmul(in(t), k[t]));
    c = tanh_rational(fadd(c, N.cb[2][m]));
    c = tanh_rational(fadd(fmul(N.sw[2][m], c), N.sb[2][m]));
    if (N.full_connect) return fmul(N.af, c);
    const float c1 = tanh_rational(fadd(fmul(fmul(N.af, N.hw[2 * m]), c), N.hb[2 * m]));
    const float c2 = tanh_rational(fadd(fmul(fmul(N.af, N.hw[2 * m + 1]), c), N.hb[2 * m + 1]));
    return fmul(N.af, fadd(fmul(N.ow[2 * m], c1), fmul(N.ow[2 * m + 1], c2)));
}

// fully connected hidden neuron n from the L3 values: mulC24_add_tanh (:1003) for 24 maps, else
// mulC2_add / mulC1_add / tanh (:968-1002, :868), which leave out the output weight
__device__ __forceinline__ float lg_hidden_fc(const LegacyNet& N, int n, const float* vals) {
    if (N.m2 == 24) {
        float s = N.hb[n];
        for (int j = 0; j < 24; ++j) s = fadd(s, fmul(vals[j], N.hwfc[n][j]));
        return fmul(fmul(N.af, tanh_rational(s)), N.ow[n]);
    }
    float s = fadd(fmul(vals[0], N.hwfc[n][0]), fmul(vals[1], N.hwfc[n][1]));
    for (int j = 2; j < N.m2; ++j) s = fadd(fmul(vals[j], N.hwfc[n][j]), s);
    return fmul(N.af, tanh_rational(fadd(s, N.hb[n])));
}

// the output neuron on the summed hidden values (tanh :868)
__device__ __forceinline__ float lg_finish(const LegacyNet& N, float acc) { return fmul(N.af, tanh_rational(fadd(acc, N.ob))); }

}  // namespace ccnn
