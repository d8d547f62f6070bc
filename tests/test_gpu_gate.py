"""Learned gate on the GPU: the device gradient against the float64 restatement, the skip path
(gate fully on = plain cascade, fully off = nothing scanned, ambiguous = full-scan fallback),
training on frames the plain cascade labels, and what the shipped trained weights gain over the
full scan at >= 99% box recall."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import gate  # noqa: E402
from oracle import gate_ref  # noqa: E402


def _det(w=640, h=480):
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    return d


def _const_params(prob):
    p = np.zeros(700, np.float32)
    p[gate.B3:] = np.log(prob / (1 - prob))
    return p


@pytest.mark.parametrize("pos_weight", [1.0, 12.0])
def test_device_gradient_matches_restatement(pos_weight):
    rng = np.random.default_rng(5)
    n, h8, w8 = 3, 30, 40
    feat = rng.uniform(-2, 2, (n, h8, w8)).astype(np.float16)
    lab = (rng.random((n, 4, h8 // 2, w8 // 2)) < 0.1).astype(np.uint8)
    params = gate.init_params(4)
    params[gate.B3:] = -1.5
    ds = gate.Dataset(torch.from_numpy(feat).cuda(), torch.from_numpy(lab).cuda(), int(lab.sum()))
    loss, g = gate.gradient(params, ds, pos_weight)
    want_loss, want = gate_ref.loss_and_grad(params, feat.astype(np.float64), lab, pos_weight, fp16=True)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    # fp32 accumulation in a different order (and rare fp16 rounding flips of activations)
    assert np.linalg.norm(g - want) <= 2e-3 * np.linalg.norm(want)
    assert np.allclose(g, want, rtol=2e-2, atol=2e-3 * np.abs(want).max())


def test_features_are_normalised_8x8_means():
    d = _det()
    img = ccnn.synth_frame(640, 480, 11, 5, 40, 200)[0]
    d.Detect(img)
    gptr, gw, gh, step = d.grayDevice()
    feat = torch.empty((gh // 8, gw // 8), dtype=torch.float16, device="cuda")
    ccnn._capi.check(ccnn._capi.lib().ccnn_gate_features(gptr, gw, gh, step, feat.data_ptr(), None), "features")
    torch.cuda.synchronize()
    gray = d.getGrayImage32F().astype(np.float64)
    want = (gray[: gh // 8 * 8, : gw // 8 * 8].reshape(gh // 8, 8, gw // 8, 8).mean(axis=(1, 3)) - 128) / 64
    assert np.allclose(feat.cpu().numpy().astype(np.float64), want, atol=2e-3)


@pytest.mark.parametrize("w,h", [(1920, 1080), (333, 211), (640, 480)])
def test_detector_probabilities_follow_the_network(w, h):
    """The features the gray-conversion launch writes for the gate inside the frame's graph give the
    probabilities of the network restated in float64 on the features of the standalone feature
    kernel (fp16 storage points; fp32 accumulation order differs)."""
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    params = gate.load() if os.path.exists(gate.WEIGHTS_1080P) else gate.init_params(3)
    d.setGate(params, 0.5, 1.0)
    imgs = [ccnn.synth_frame(w, h, 60 + k, 5, 30, max(31, min(w, h) // 2))[0] for k in range(3)]
    d.DetectBatch(imgs[:2])
    d.Detect(imgs[2])
    got = d.gateProbabilities()
    gptr, gw, gh, step = d.grayDevice()
    feat = torch.empty((gh // 8, gw // 8), dtype=torch.float16, device="cuda")
    ccnn._capi.check(ccnn._capi.lib().ccnn_gate_features(gptr, gw, gh, step, feat.data_ptr(), None), "features")
    torch.cuda.synchronize()
    want = gate_ref.forward(params.astype(np.float64), feat.cpu().numpy()[None].astype(np.float64), fp16=True)[0]
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 2e-3


@pytest.mark.parametrize("seed", [21, 22])
def test_gate_fully_on_is_the_plain_cascade(seed):
    d = _det()
    img = ccnn.synth_frame(640, 480, seed, 5, 40, 200)[0]
    plain = d.Detect(img)
    d.setGate(_const_params(0.999), 0.5, 0.25)
    gated = d.Detect(img)
    fr, ft, br, bt, fb = d.gateStats()
    assert gated == plain and len(plain) > 0
    assert (fr, br, fb) == (ft, bt, 0)


def test_gate_fully_off_scans_nothing():
    d = _det()
    img = ccnn.synth_frame(640, 480, 23, 5, 40, 200)[0]
    assert len(d.Detect(img)) > 0
    d.setGate(_const_params(1e-6), 0.5, 0.25)
    assert d.Detect(img) == []
    fr, ft, br, bt, fb = d.gateStats()
    assert fr == 0 and br == 0 and ft > 0 and bt > 0 and fb == 0
    d.disableGate()
    assert len(d.Detect(img)) > 0


def test_ambiguous_frame_falls_back_to_full_scan():
    d = _det()
    img = ccnn.synth_frame(640, 480, 24, 5, 40, 200)[0]
    plain = d.Detect(img)
    d.setGate(_const_params(0.3), 0.5, 0.25)  # every cell in [thr/4, thr): ambiguous
    assert d.Detect(img) == plain
    fr, ft, br, bt, fb = d.gateStats()
    assert fb == 1 and (fr, br) == (ft, bt)


def _brightness_params(level, gain=8.0):
    """A hand-set gate that passes the feature through one channel: probability >= 0.5 in the
    cells whose 2x2-averaged feature is at least `level` (the brightest parts of the frame)."""
    p = np.zeros(700, np.float32)
    p[gate.W1 + 4] = 1.0  # W1[0] centre tap
    p[gate.W2 + 4] = 1.0  # W2[0][0] centre tap
    for k in range(4):
        p[gate.W3 + 8 * k] = gain
        p[gate.B3 + k] = -gain * level
    return p


@pytest.mark.parametrize("seeds", [(40, 41), (42, 43)])
def test_partial_gate_recomputes_every_active_tile(seeds):
    """Frame A runs in full, then frame B with a gate that keeps only part of the tiles: every
    response of B is either the plain cascade's own value or the skipped-tile marker, so no active
    tile read stage-1 data left over from frame A."""
    d = _det(1920, 1080)
    a, b = (ccnn.synth_frame(1920, 1080, s, 20, 30, 300)[0] for s in seeds)
    d.Detect(b)
    want = [d.response_map(i) for i in range(len(d.levels()))]
    gray = d.getGrayImage32F().astype(np.float64)
    f = (gray[:1080 // 8 * 8].reshape(135, 8, 240, 8).mean(axis=(1, 3)) - 128) / 64
    q = f[:134].reshape(67, 2, 120, 2).mean(axis=(1, 3))
    d.Detect(a)
    d.setGate(_brightness_params(float(np.quantile(np.maximum(q, 0), 0.97))), 0.5, 1.0)
    d.Detect(b)
    fr, ft, br, bt, fb = d.gateStats()
    assert 0 < br < bt and 0 < fr <= ft and fb == 0
    skipped = 0
    for i, w in enumerate(want):
        g = d.response_map(i)
        off = g == np.float32(-1e30)
        skipped += int(off.sum())
        assert np.array_equal(g[~off], w[~off]), i
    assert skipped > 0


@pytest.mark.parametrize("w,h", [(47, 51), (64, 64), (100, 80), (333, 211)])
def test_gate_on_small_and_odd_frames(w, h):
    """Frames down to the stage-2/3 window: a gate that keeps every tile changes nothing, one that keeps
    none leaves no face (frames under 32x32 gray pixels would always run in full)."""
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    img = ccnn.synth_frame(w, h, 90 + w, 2, 40, max(41, min(w, h) - 2))[0]
    plain = d.Detect(img)
    d.setGate(_const_params(0.999), 0.5, 0.25)
    assert d.Detect(img) == plain
    fr, ft, br, bt, fb = d.gateStats()
    assert (fr, br) == (ft, bt)
    d.setGate(_const_params(1e-6), 0.5, 0.25)
    assert d.Detect(img) == []


def test_gate_rejects_bad_arguments():
    d = _det()
    with pytest.raises(ccnn.CCNNError):
        d.setGate(np.zeros(10, np.float32))
    with pytest.raises(ccnn.CCNNError):
        d.setGate(np.zeros(700, np.float32), threshold=1.5)
    with pytest.raises(ccnn.CCNNError):
        d.setGateMargin(65)


def test_wider_margin_keeps_more():
    """The candidate margin only widens or narrows the search: a wider margin runs a superset of the
    tiles and keeps at least the boxes of a narrower one; the default (16 px) is the one-cell rule."""
    params = gate.load() if os.path.exists(gate.WEIGHTS_1080P) else gate.init_params(3)
    imgs = [ccnn.synth_frame(1920, 1080, 70 + i, 20, 30, 300)[0] for i in range(3)]
    d0 = _det(1920, 1080)
    d0.setGate(params, 0.3, 0.25)
    default = [d0.Detect(im) for im in imgs]
    d = _det(1920, 1080)
    d.setGate(params, 0.3, 0.25)
    runs = {}
    for m in (0, 8, 16, 64):
        d.setGateMargin(m)
        got = [d.Detect(im) for im in imgs]
        runs[m] = d.gateStats()
        if m == 16:
            assert got == default
    for a, b in ((0, 8), (8, 16), (16, 64)):
        assert runs[a][0] <= runs[b][0] and runs[a][2] <= runs[b][2]
    assert runs[0][2] < runs[64][2]


def test_batch_path_uses_the_gate():
    d = _det()
    imgs = [ccnn.synth_frame(640, 480, 30 + i, 5, 40, 200)[0] for i in range(4)]
    plain = [d.Detect(im) for im in imgs]
    d.setGate(_const_params(0.999), 0.5, 0.25)
    assert d.DetectBatch(imgs) == plain
    d.setGate(_const_params(1e-6), 0.5, 0.25)
    assert d.DetectBatch(imgs) == [[] for _ in imgs]


def test_training_on_cascade_labels_lowers_the_loss():
    d = _det()
    ds = gate.collect(d, range(700, 740), width=640, height=480, n_faces=5, min_patch=40, max_patch=200)
    assert ds.n == 40 and ds.positives > 0 and ds.feat.shape == (40, 60, 80) and ds.labels.shape == (40, 4, 30, 40)
    p0 = gate.init_params(0)
    l0, _ = gate.gradient(p0, ds, 20.0)
    p1, losses = gate.train(ds, p0, epochs=15, batch=8, lr=3e-3, pos_weight=20.0)
    l1, _ = gate.gradient(p1, ds, 20.0)
    assert np.all(np.isfinite(p1)) and np.all(np.isfinite(losses))
    assert l1 < 0.7 * l0


@pytest.mark.skipif(not os.path.exists(gate.WEIGHTS_1080P), reason="no trained weights in the package")
def test_trained_gate_keeps_recall_and_skips_work():
    """The shipped weights, on 1080p frames none of them was trained on: >= 99% of the plain
    cascade's boxes are found while well under half of the stage-1 tiles run. The untrained
    network at the same threshold does not get both."""
    meta = gate.load_meta()
    thr, margin = meta.get("operating_threshold", 0.1), meta.get("operating_margin", 16)
    d = ccnn.FaceDetector()
    assert d.Init(gate.detector_params()) == 0
    seeds = range(gate.EVAL_SEED0 + 5000, gate.EVAL_SEED0 + 5040)
    trained = gate.evaluate(d, seeds, gate.load(), [thr], margin=margin)[0]
    assert trained["box_recall"] >= 0.99
    assert trained["back_tiles_run"] <= 0.5
    untrained = gate.evaluate(d, seeds, gate.init_params(0), [thr], margin=margin)[0]
    assert untrained["box_recall"] < 0.99 or untrained["back_tiles_run"] > 0.5
