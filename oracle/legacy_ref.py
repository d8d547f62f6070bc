"""CPU restatement of the legacy (format 1.0, `_new.bin`) cascade networks in float32 numpy
(test infrastructure: a checker, never a product path).

Follows SIMD::ConvNeuralNetwork of the reference's plain-C++ build: the reader
(src/CNNObjectDetector/cnn_simd.cpp:40-336) and Run_single_thread (cnn_simd.cpp:551-874) over the
CNNPP operations of src/CNNObjectDetector/cnnpp_cplusplus.cpp (conv_4x4 :92, conv_3x3 :36,
conv_6x5 :212, conv_8x7 :292, max_tanh_tanh :473, tanh_avr_tanh :411, tanh_tanh_2tanh :692,
tanh_tanh :778, mulC24_add_tanh :1003, mulC1_add / mulC2_add :968-1002, tanh :868, add :916,
add2 :933). Every operation is one float32 operation in the reference's order, applied to whole
maps, so the result is bit-exact.
"""
import struct

import numpy as np

F = np.float32
TANH_A = F(1.41645)


def load(path):
    """Parse a format-1.0 model file into a dict of float32 arrays."""
    with open(path, "rb") as f:
        b = f.read()
    o = [0]

    def rd(fmt):
        v = struct.unpack_from("<" + fmt, b, o[0])
        o[0] += struct.calcsize(fmt)
        return v if len(v) > 1 else v[0]

    def floats(n):
        v = np.frombuffer(b, "<f4", n, o[0]).astype(F)
        o[0] += 4 * n
        return v

    if rd("f") != 1.0:
        raise ValueError("not a format-1.0 model")
    net = {"max_pool": rd("B") != 0, "min": rd("ii")}
    if rd("i") != 3:
        raise ValueError("three layers expected")
    maps = [rd("i") for _ in range(3)]
    net["maps"] = maps
    ks = []
    for m in maps:
        kw, kh = rd("ii")
        ks.append(floats(m * kw * kh).reshape(m, kh, kw))
    net["k"] = ks
    net["af"] = F(rd("f"))
    net["act"] = [floats(3 * m).reshape(m, 3) for m in maps]  # conv bias, pooling weight, pooling bias
    net["fc"] = rd("B") != 0
    hl = rd("i")
    net["hw"] = floats(hl * maps[2]).reshape(hl, maps[2]) if net["fc"] else floats(hl)
    net["hb"] = floats(hl)
    net["ow"] = floats(hl)
    net["ob"] = F(rd("f"))
    return net


def tanh_r(c):
    """sgn(c) (1 - 1 / (((1 + |c|) + c c) + a c c c c)) (USE_FAST_TANH)."""
    c = np.asarray(c, F)
    sgn = np.where(c < 0, F(-1), F(1)).astype(F)
    d = (F(1) + np.abs(c)) + c * c
    d = d + (((TANH_A * c) * c) * c) * c
    return sgn * (F(1) - F(1) / d)


def _conv(img, k):
    """Valid convolution, taps accumulated left to right in row-major order."""
    kh, kw = k.shape
    h, w = img.shape
    oh, ow = h - kh + 1, w - kw + 1
    acc = img[0:oh, 0:ow] * k[0, 0]
    for t in range(1, kh * kw):
        r, c = divmod(t, kw)
        acc = acc + img[r:r + oh, c:c + ow] * k[r, c]
    return acc


def _pool_tanh(conv, max_pool, cb, sw, sb, af):
    """tanh(c + b) of each position of the 2x2 windows, max or sum, then tanh(w p + b) af."""
    h, w = conv.shape[0] // 2 * 2, conv.shape[1] // 2 * 2
    t = tanh_r(conv[:h, :w] + cb)
    c1, c2, c3, c4 = t[0::2, 0::2], t[0::2, 1::2], t[1::2, 0::2], t[1::2, 1::2]
    p = np.maximum(np.maximum(c1, c2), np.maximum(c3, c4)) if max_pool else ((c1 + c2) + c3) + c4
    return af * tanh_r(sw * p + sb)


def _sums(maps):
    n = len(maps)
    out = [maps[0] + maps[1]]
    out += [(maps[i - 1] + maps[i]) + maps[i + 1] for i in range(1, n - 1)]
    out.append(maps[n - 2] + maps[n - 1])
    return out


def forward(net, img):
    """Response map of the network on a float32 H x W image."""
    img = np.asarray(img, F)
    m0, m1, m2 = net["maps"]
    af = net["af"]
    r1c, r1r = img.shape[1] - 3, img.shape[0] - 3
    p1 = []
    for m in range(m0):
        conv = _conv(img, net["k"][0][m])[: r1r // 2 * 2, : r1c // 2 * 2]
        cb, sw, sb = net["act"][0][m]
        p1.append(_pool_tanh(conv, net["max_pool"], cb, sw, sb, af))
    s1 = _sums(p1)
    r2c, r2r = r1c // 2 - 2, r1r // 2 - 2
    p2 = []
    for m in range(m1):
        conv = _conv(s1[m // 2], net["k"][1][m])[: r2r // 2 * 2, : r2c // 2 * 2]
        cb, sw, sb = net["act"][1][m]
        p2.append(_pool_tanh(conv, net["max_pool"], cb, sw, sb, af))
    s2 = _sums(p2)
    vals = []
    for m in range(m2):
        c = _conv(s2[m // 2], net["k"][2][m])
        cb, sw, sb = net["act"][2][m]
        c = tanh_r(c + cb)
        c = tanh_r(sw * c + sb)
        if net["fc"]:
            vals.append(af * c)
        else:
            c1 = tanh_r((af * net["hw"][2 * m]) * c + net["hb"][2 * m])
            c2 = tanh_r((af * net["hw"][2 * m + 1]) * c + net["hb"][2 * m + 1])
            vals.append(af * (net["ow"][2 * m] * c1 + net["ow"][2 * m + 1] * c2))
    if not net["fc"]:
        acc = vals[1] + vals[0]
        for i in range(1, m2 // 2):
            acc = acc + (vals[2 * i + 1] + vals[2 * i])
    else:
        hs = []
        for n in range(len(net["hb"])):
            w = net["hw"][n]
            if m2 == 24:
                s = net["hb"][n] + vals[0] * w[0]
                for j in range(1, 24):
                    s = s + vals[j] * w[j]
                hs.append((af * tanh_r(s)) * net["ow"][n])
            else:
                s = vals[0] * w[0] + vals[1] * w[1]
                for j in range(2, m2):
                    s = vals[j] * w[j] + s
                hs.append(af * tanh_r(s + net["hb"][n]))
        acc = hs[0]
        for h in hs[1:]:
            acc = acc + h
    return af * tanh_r(acc + net["ob"])
