"""CPU restatement of the learned gate's network, loss and gradient in float64 (test
infrastructure: the checker for the device training kernels, never a product path).

The gate has no reference counterpart (the reference scans every level in full); this follows the
network the library documents in include/ccnn_gate.h:
  f  -> a1 = LReLU_0.1(conv3x3(f; W1) + b1) -> a2 = LReLU_0.1(conv3x3(a1; W2) + b2)
     -> q = 2x2 average -> p = sigmoid(W3 q + b3),
  loss = mean over (frame, octave, cell) of  -pw*y*log(p) - (1-y)*log(1-p),
with each log term limited to 30 (p clamped to 1e-7), as the device head does. With
fp16=True the features and both activation maps are rounded to binary16 where the device stores
them, so the gradient matches the device's up to fp32 accumulation order.
"""
import numpy as np

N_PARAMS = 700
K, C = 4, 8
W1, B1, W2, B2, W3, B3 = 0, 72, 80, 656, 664, 696


def _unpack(p):
    p = np.asarray(p, np.float64)
    return (p[W1:B1].reshape(C, 1, 3, 3), p[B1:W2], p[W2:B2].reshape(C, C, 3, 3), p[B2:W3], p[W3:B3].reshape(K, C), p[B3:])


def _conv(x, w):
    """3x3 convolution with zero padding: x [n][cin][h][w], w [cout][cin][3][3]."""
    n, cin, h, wd = x.shape
    xp = np.zeros((n, cin, h + 2, wd + 2))
    xp[:, :, 1:-1, 1:-1] = x
    out = np.zeros((n, w.shape[0], h, wd))
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("oc,nchw->nohw", w[:, :, dy, dx], xp[:, :, dy:dy + h, dx:dx + wd])
    return out


def _wgrad(g, x):
    """d/dW of sum(g * conv(x, W)): g [n][cout][h][w], x [n][cin][h][w] -> [cout][cin][3][3]."""
    n, cin, h, wd = x.shape
    xp = np.zeros((n, cin, h + 2, wd + 2))
    xp[:, :, 1:-1, 1:-1] = x
    out = np.zeros((g.shape[1], cin, 3, 3))
    for dy in range(3):
        for dx in range(3):
            out[:, :, dy, dx] = np.einsum("nohw,nchw->oc", g, xp[:, :, dy:dy + h, dx:dx + wd])
    return out


def _xgrad(g, w):
    """d/dx of sum(g * conv(x, W)) (the transposed convolution)."""
    n, cout, h, wd = g.shape
    gp = np.zeros((n, cout, h + 2, wd + 2))
    gp[:, :, 1:-1, 1:-1] = g
    out = np.zeros((n, w.shape[1], h, wd))
    for dy in range(3):
        for dx in range(3):
            # out(y, x) += g(y - dy + 1, x - dx + 1) * w(dy, dx)
            out += np.einsum("oc,nohw->nchw", w[:, :, dy, dx], gp[:, :, 2 - dy:2 - dy + h, 2 - dx:2 - dx + wd])
    return out


def _lrelu(z):
    return np.where(z > 0, z, 0.1 * z)


def _r16(x, on):
    return x.astype(np.float16).astype(np.float64) if on else x


def forward(params, feat, fp16=False):
    """Probabilities [n][K][h8/2][w8/2] for features [n][h8][w8]."""
    return _run(params, feat, None, 1.0, fp16)[0]


def loss_and_grad(params, feat, labels, pos_weight, fp16=False):
    """(loss, gradient[700]) over all frames; labels uint8 [n][K][h8/2][w8/2]."""
    _, loss, grad = _run(params, feat, labels, pos_weight, fp16)
    return loss, grad


def _run(params, feat, labels, pw, fp16):
    w1, b1, w2, b2, w3, b3 = _unpack(params)
    f = _r16(np.asarray(feat, np.float64), fp16)[:, None]
    n, _, h8, w8 = f.shape
    h16, w16 = h8 // 2, w8 // 2
    a1 = _r16(_lrelu(_conv(f, w1) + b1[None, :, None, None]), fp16)
    a2 = _r16(_lrelu(_conv(a1, w2) + b2[None, :, None, None]), fp16)
    t = a2[:, :, :2 * h16, :2 * w16]
    q = 0.25 * (t[:, :, 0::2, 0::2] + t[:, :, 0::2, 1::2] + t[:, :, 1::2, 0::2] + t[:, :, 1::2, 1::2])  # [n][C][h16][w16]
    z = np.einsum("kc,nchw->nkhw", w3, q) + b3[None, :, None, None]
    p = 1.0 / (1.0 + np.exp(-z))
    if labels is None:
        return p, None, None
    y = np.asarray(labels, np.float64)
    inv = 1.0 / (n * K * h16 * w16)
    lp = np.minimum(-np.log(np.maximum(p, 1e-7)), 30.0)
    ln = np.minimum(-np.log(np.maximum(1.0 - p, 1e-7)), 30.0)
    loss = float(np.sum(pw * y * lp + (1.0 - y) * ln) * inv)
    gz = (p * (pw * y + 1.0 - y) - pw * y) * inv  # d loss / d z (the limits are not differentiated)
    g = np.zeros(N_PARAMS)
    g[W3:B3] = np.einsum("nkhw,nchw->kc", gz, q).ravel()
    g[B3:] = gz.sum(axis=(0, 2, 3))
    gq = np.einsum("nkhw,kc->nchw", gz, w3)
    gz2 = np.zeros_like(a2)
    up = 0.25 * np.repeat(np.repeat(gq, 2, axis=2), 2, axis=3)
    gz2[:, :, :2 * h16, :2 * w16] = up
    gz2 *= np.where(a2 > 0, 1.0, 0.1)
    g[W2:B2] = _wgrad(gz2, a1).ravel()
    g[B2:W3] = gz2.sum(axis=(0, 2, 3))
    gz1 = _xgrad(gz2, w2) * np.where(a1 > 0, 1.0, 0.1)
    g[W1:B1] = _wgrad(gz1, f).ravel()
    g[B1:W2] = gz1.sum(axis=(0, 2, 3))
    return p, loss, g
