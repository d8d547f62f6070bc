"""Learned scale/region gate in front of the stage-1 scan (include/ccnn_gate.h).

The plain cascade labels its own frames: every window that stage 3 accepts marks the pyramid
octave of its level and the 16x16 cell of the frame that holds its centre. A 700-parameter network
on the 8x8-averaged gray frame (two 3x3 convolutions with 8 maps, a 2x2 average and a sigmoid per
octave) learns those labels with the library's own device kernels (fp16 activations, fp32
accumulation, Adam). At detection time the stage-1 tiles whose candidates' window centres fall in
no cell above the threshold are skipped, and a frame with many cells just below the threshold is
scanned in full.

No reference counterpart: the reference scans every level in full (CNNDetector::RunCPUDetect,
src/CNNObjectDetector/cnn_detector_v3.cpp:2063-2235); the gate is evaluated against that full scan by
box recall.

    python -m compactcnncascade_b200.gate --train-frames 20000 --eval-frames 1000 --out weights.bin
"""
import argparse
import ctypes
import json
import math
import os
import struct
import sys
import time

import numpy as np

from . import _capi

N_PARAMS = 700
OCTAVES = 4
# parameter layout: W1[8][9], b1[8], W2[8 out][8 in][9], b2[8], W3[4][8], b3[4]
W1, B1, W2, B2, W3, B3 = 0, 72, 80, 656, 664, 696
WEIGHTS_1080P = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "gate_1080p.bin")
_MAGIC = b"CCGT"

# the 1080p workload the shipped weights were trained on
FRAME_W, FRAME_H, N_FACES, MIN_PATCH, MAX_PATCH = 1920, 1080, 20, 30, 300
MIN_FACE, MAX_FACE, SCALE_FACTOR = 40, 240, 1.15
TRAIN_SEED0, EVAL_SEED0 = 5_000_000, 9_000_000  # disjoint from the benchmark's and the tests' seeds


def init_params(seed=0, prior=0.02):
    """He-initialised weights and a head bias at the logit of the expected positive rate."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[W1:B1] = rng.normal(0.0, math.sqrt(2.0 / 9.0), B1 - W1)
    p[W2:B2] = rng.normal(0.0, math.sqrt(2.0 / 72.0), B2 - W2)
    p[W3:B3] = rng.normal(0.0, math.sqrt(1.0 / 8.0), B3 - W3)
    p[B3:] = math.log(prior / (1.0 - prior))
    return p


def save(path, params, meta=None):
    """Weight file: b"CCGT", u32 version 1, u32 count, count fp32 (little endian), then an
    optional JSON description of how the weights were made."""
    p = np.ascontiguousarray(params, np.float32)
    if p.size != N_PARAMS:
        raise ValueError(f"the gate has {N_PARAMS} parameters, got {p.size}")
    with open(path, "wb") as f:
        f.write(_MAGIC + struct.pack("<II", 1, p.size) + p.astype("<f4").tobytes())
        if meta:
            f.write(json.dumps(meta, sort_keys=True).encode())


def load(path=WEIGHTS_1080P):
    with open(path, "rb") as f:
        blob = f.read()
    if blob[:4] != _MAGIC:
        raise ValueError(f"{path}: not a gate weight file")
    ver, n = struct.unpack("<II", blob[4:12])
    if ver != 1 or n != N_PARAMS:
        raise ValueError(f"{path}: version {ver} with {n} parameters is not supported")
    return np.frombuffer(blob[12:12 + 4 * n], "<f4").astype(np.float32)


def load_meta(path=WEIGHTS_1080P):
    with open(path, "rb") as f:
        blob = f.read()
    tail = blob[12 + 4 * N_PARAMS:]
    return json.loads(tail.decode()) if tail else {}


def detector_params():
    from . import default_params
    p = default_params()
    p.min_face_height, p.max_face_height, p.scale_factor = MIN_FACE, MAX_FACE, SCALE_FACTOR
    p.max_image_width, p.max_image_height = FRAME_W, FRAME_H
    return p


class Dataset:
    """Features (fp16 [n][rows/8][cols/8]) and labels (uint8 [n][4][rows/16][cols/16]) on the device."""

    def __init__(self, feat, labels, positives):
        self.feat, self.labels, self.positives = feat, labels, positives

    @property
    def n(self):
        return self.feat.shape[0]

    @property
    def w8(self):
        return self.feat.shape[2]

    @property
    def h8(self):
        return self.feat.shape[1]


def collect(det, seeds, width=FRAME_W, height=FRAME_H, n_faces=N_FACES, min_patch=MIN_PATCH, max_patch=MAX_PATCH):
    """Runs the plain cascade (gate off) on the seeded frames, rendered on the device, and keeps
    each frame's gate features and the labels from stage 3's accepts."""
    import torch
    from . import synth_frame_device
    L = _capi.lib()
    det.disableGate()
    frame = torch.empty((height, width, 3), dtype=torch.uint8, device="cuda")
    w8 = h8 = None
    feat = labels = None
    for i, s in enumerate(seeds):
        synth_frame_device(frame.data_ptr(), width, height, s, n_faces, min_patch, max_patch)
        det.DetectDevice(frame.data_ptr(), width, height, 3, width * 3)
        gptr, gw, gh, gstep = det.grayDevice()
        if feat is None:
            w8, h8 = gw // 8, gh // 8
            feat = torch.empty((len(seeds), h8, w8), dtype=torch.float16, device="cuda")
            labels = torch.empty((len(seeds), OCTAVES, h8 // 2, w8 // 2), dtype=torch.uint8, device="cuda")
        elif (gw // 8, gh // 8) != (w8, h8):
            raise ValueError("every frame of a gate dataset must have the same gray size")
        _capi.check(L.ccnn_gate_features(gptr, gw, gh, gstep, feat[i].data_ptr(), None), "ccnn_gate_features")
        _capi.check(L.ccnn_gate_labels(det._h, labels[i].data_ptr(), None), "ccnn_gate_labels")
    torch.cuda.synchronize()
    return Dataset(feat, labels, int(labels.sum().item()))


def gradient(params, ds, pos_weight):
    """(loss, gradient) of the device kernels over the whole dataset."""
    import torch
    P = torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
    g = np.zeros(N_PARAMS, np.float32)
    loss = ctypes.c_float()
    _capi.check(_capi.lib().ccnn_gate_gradient(P.data_ptr(), ds.feat.data_ptr(), ds.labels.data_ptr(), ds.n, ds.w8, ds.h8, pos_weight,
                                                g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(loss)),
                "ccnn_gate_gradient")
    return float(loss.value), g


def train(ds, params=None, epochs=20, batch=64, lr=3e-3, pos_weight=20.0, seed=0):
    """Adam on the device over consecutive mini-batches; returns (params, per-epoch mean loss)."""
    p = init_params(seed) if params is None else np.array(params, np.float32)
    losses = np.zeros(epochs, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    _capi.check(_capi.lib().ccnn_gate_train(p.ctypes.data_as(fp), ds.feat.data_ptr(), ds.labels.data_ptr(), ds.n, ds.w8, ds.h8,
                                             min(batch, ds.n), epochs, lr, pos_weight, losses.ctypes.data_as(fp)),
                "ccnn_gate_train")
    return p, losses


def _iou(a, b):
    ax1, ay1, ax2, ay2 = a[0], a[1], a[0] + a[2], a[1] + a[3]
    bx1, by1, bx2, by2 = b[0], b[1], b[0] + b[2], b[1] + b[3]
    iw, ih = min(ax2, bx2) - max(ax1, bx1), min(ay2, by2) - max(ay1, by1)
    if iw <= 0 or ih <= 0:
        return 0.0
    inter = iw * ih
    return inter / float(a[2] * a[3] + b[2] * b[3] - inter)


def box_recall(ref, got, iou=0.5):
    """(matched, total): boxes of `ref` that a distinct box of `got` overlaps by IoU >= iou."""
    used = [False] * len(got)
    hit = 0
    for r in ref:
        best, bi = iou, -1
        for j, g in enumerate(got):
            if not used[j]:
                v = _iou(r, g)
                if v >= best:
                    best, bi = v, j
        if bi >= 0:
            used[bi] = True
            hit += 1
    return hit, len(ref)


def evaluate(det, seeds, params, thresholds, fallback_fraction=0.25, width=FRAME_W, height=FRAME_H, n_faces=N_FACES,
             min_patch=MIN_PATCH, max_patch=MAX_PATCH, margin=16):
    """Box recall of the gated cascade against the plain one on the seeded frames, and the share
    of stage-1 tiles that ran, per threshold (candidate margin `margin` pixels)."""
    import torch
    from . import synth_frame_device
    frame = torch.empty((height, width, 3), dtype=torch.uint8, device="cuda")
    det.disableGate()
    plain = []
    for s in seeds:
        synth_frame_device(frame.data_ptr(), width, height, s, n_faces, min_patch, max_patch)
        plain.append(det.DetectDevice(frame.data_ptr(), width, height, 3, width * 3))
    out = []
    for thr in thresholds:
        det.setGate(params, thr, fallback_fraction)
        det.setGateMargin(margin)
        hit = tot = 0
        fr = ft = br = bt = fb = 0
        frames_full = 0
        for s, ref in zip(seeds, plain):
            synth_frame_device(frame.data_ptr(), width, height, s, n_faces, min_patch, max_patch)
            got = det.DetectDevice(frame.data_ptr(), width, height, 3, width * 3)
            h, t = box_recall(ref, got)
            hit, tot = hit + h, tot + t
            a, b, c, d, e = det.gateStats()
            fr, ft, br, bt, fb = fr + a, ft + b, br + c, bt + d, fb + e
            frames_full += int(h == t)
        out.append({"threshold": thr, "margin": margin, "box_recall": hit / max(1, tot), "boxes": tot, "frames_all_boxes": frames_full,
                    "front_tiles_run": fr / max(1, ft), "back_tiles_run": br / max(1, bt), "fallback_frames": fb})
    det.setGateMargin(16)
    det.disableGate()
    return out


def _operating_point(ev, thresholds):
    """(threshold, margin): of the evaluated pairs that kept >= 99.5% of the plain boxes on the
    held-out frames (half a point over the 99% recall target, for frames outside the evaluation
    set), the one that runs the fewest stage-1 back tiles (ties: the higher threshold)."""
    ok = [r for r in ev if r["box_recall"] >= 0.995]
    if not ok:
        return min(thresholds), 16
    best = min(ok, key=lambda r: (r["back_tiles_run"], -r["threshold"]))
    return best["threshold"], best.get("margin", 16)


def main(argv=None):
    ap = argparse.ArgumentParser(description="train the learned gate on frames labelled by the plain cascade")
    ap.add_argument("--train-frames", type=int, default=20000)
    ap.add_argument("--eval-frames", type=int, default=1000)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--pos-weight", type=float, default=80.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--thresholds", default="0.02,0.05,0.1,0.2,0.3,0.4,0.5")
    ap.add_argument("--margins", default="8,16", help="candidate margins (pixels) to evaluate")
    ap.add_argument("--fallback", type=float, default=0.25)
    ap.add_argument("--out", default=WEIGHTS_1080P)
    ap.add_argument("--report", default=None, help="write the evaluation as JSON here")
    ap.add_argument("--eval-only", action="store_true",
                    help="keep the weights in --out, evaluate them again and rewrite their description")
    a = ap.parse_args(argv)
    from . import FaceDetector
    det = FaceDetector()
    if det.Init(detector_params()) != 0:
        raise RuntimeError(_capi.last_error())
    thr = [float(x) for x in a.thresholds.split(",")]
    margins = [int(x) for x in a.margins.split(",")]

    def evaluate_all(params):
        ev = []
        for m in margins:
            ev += evaluate(det, range(EVAL_SEED0, EVAL_SEED0 + a.eval_frames), params, thr, a.fallback, margin=m)
        for r in ev:
            print(json.dumps(r), flush=True)
        return ev

    if a.eval_only:
        params, meta = load(a.out), load_meta(a.out)
        ev = evaluate_all(params)
        op_thr, op_margin = _operating_point(ev, thr)
        meta.update(eval=ev, eval_frames=a.eval_frames, eval_seeds=[EVAL_SEED0, EVAL_SEED0 + a.eval_frames],
                    operating_threshold=op_thr, operating_margin=op_margin)
        print(f"operating threshold {op_thr}, margin {op_margin} px", flush=True)
        save(a.out, params, meta)
        if a.report:
            with open(a.report, "w") as f:
                json.dump({"weights": os.path.basename(a.out), "eval_frames": a.eval_frames,
                           "eval_seeds": meta["eval_seeds"], "fallback_fraction": a.fallback,
                           "operating_threshold": op_thr, "operating_margin": op_margin, "eval": ev,
                           "workload": meta.get("workload"), "reference": "plain cascade boxes matched at IoU >= 0.5"}, f, indent=1)
        return 0
    t0 = time.time()
    ds = collect(det, range(TRAIN_SEED0, TRAIN_SEED0 + a.train_frames))
    t1 = time.time()
    print(f"collected {ds.n} frames ({ds.positives} positive cells of {ds.labels.numel()}) in {t1 - t0:.1f} s", flush=True)
    params, losses = train(ds, epochs=a.epochs, batch=a.batch, lr=a.lr, pos_weight=a.pos_weight, seed=a.seed)
    t2 = time.time()
    print(f"trained {a.epochs} epochs in {t2 - t1:.1f} s; loss {losses[0]:.4f} -> {losses[-1]:.4f}", flush=True)
    del ds
    ev = evaluate_all(params)
    op, op_margin = _operating_point(ev, thr)
    print(f"operating threshold {op}, margin {op_margin} px", flush=True)
    meta = {"operating_threshold": op, "operating_margin": op_margin, "train_frames": a.train_frames, "train_seeds": [TRAIN_SEED0, TRAIN_SEED0 + a.train_frames], "epochs": a.epochs,
            "batch": a.batch, "lr": a.lr, "pos_weight": a.pos_weight, "init_seed": a.seed,
            "loss_first_last": [float(losses[0]), float(losses[-1])],
            "workload": f"{FRAME_W}x{FRAME_H} synthetic, {N_FACES} patches {MIN_PATCH}-{MAX_PATCH} px, min face {MIN_FACE}, "
                        f"max face {MAX_FACE}, scale {SCALE_FACTOR}",
            "eval_frames": a.eval_frames, "eval_seeds": [EVAL_SEED0, EVAL_SEED0 + a.eval_frames], "eval": ev}
    save(a.out, params, meta)
    if a.report:
        with open(a.report, "w") as f:
            json.dump({"losses": [float(x) for x in losses], **meta}, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
