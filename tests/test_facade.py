"""The header-only C++ facades compile against the C ABI like the reference's own demo code and
give the reference's results (its strict IEEE build, oracle/_ref/libccnn_ref.so):
include/CompactCNNLib.h (FaceDetector: Detect, every getter and setter, the process-global
singleton semantics) and include/CNNDetector.h (the internal CNNDetector class: Param /
AdvancedParam, raw Detection results with scale / knn / num_detect, detections already in the
caller's vector, NMS, the parameters the detector reports after Init's precision rules)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "compactcnncascade_b200")


def _build(tmp_path_factory, src, name):
    exe = str(tmp_path_factory.mktemp("facade") / name)
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", src), os.path.join(PKG, "csrc", "synth_frame.c"),
                           "-x", "none", "-L", PKG, "-lccnn", f"-Wl,-rpath,{PKG}", "-o", exe])
    return exe


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    return _build(tmp_path_factory, "facade_example.cpp", "facade_example")


@pytest.fixture(scope="module")
def cnn_example(tmp_path_factory):
    return _build(tmp_path_factory, "cnndetector_example.cpp", "cnndetector_example")


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _run(exe, *args):
    return subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, check=True).stdout.splitlines()


def test_facades_build_and_fail_cleanly_without_gpu(example, cnn_example):
    if _cuda():
        pytest.skip("covered by the GPU variants")
    assert _run(example) == ["init -1"]
    assert _run(cnn_example, 640, 480, 1, 3) == ["rc -1"]


def _sections(lines):
    """'tag n' headers followed by n 'face ...' lines -> {tag: [(x, y, w, h, score)]}, other lines by tag."""
    out, i = {}, 0
    while i < len(lines):
        parts = lines[i].split()
        if len(parts) == 2 and parts[0].startswith(("detect", "b_detect", "a_detect")) and lines[i + 1:i + 2] and \
                (int(parts[1]) <= 0 or lines[i + 1].startswith("face ")):
            n = max(0, int(parts[1]))
            out[parts[0]] = [tuple(float(v) for v in l.split()[1:]) for l in lines[i + 1:i + 1 + n]]
            out[parts[0] + "_n"] = int(parts[1])
            i += 1 + n
        else:
            out[parts[0]] = parts[1:]
            i += 1
    return out


def _ref_faces(img, **kw):
    from oracle import ref
    h, w = img.shape[:2]
    kw.setdefault("max_w", w)
    kw.setdefault("max_h", h)
    return [tuple(float(v) for v in f) for f in ref.face_detect(np.ascontiguousarray(img), ref.params(**kw))]


def _close(got, exp):
    """Boxes identical, scores equal to the printed precision (%.6f)."""
    assert len(got) == len(exp), (got, exp)
    for g, e in zip(got, exp):
        assert g[:4] == e[:4], (g, e)
        assert abs(g[4] - e[4]) <= 5e-7 * max(1.0, abs(e[4])), (g, e)


@pytest.mark.gpu
def test_face_detector_facade_matches_reference(example):
    if not _cuda():
        pytest.skip("no CUDA device")
    import compactcnncascade_b200 as ccnn
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build not present")
    w, h = 640, 480
    img, _ = ccnn.synth_frame(w, h, 1, 5, 40, 200)
    out = _sections(_run(example, w, h, 1, "setters"))
    assert out["init"] == ["0"]
    _close(out["detect"], _ref_faces(img, min_face=40, max_face=240))
    assert len(out["detect"]) > 0
    assert out["gray"] == ["0", "1", f"{w}x{h}"]
    assert out["param"][:4] == [str(w), str(h), "40", "240"] and out["param"][4] == "1.1500"
    assert out["min"] == ["60"]
    _close(out["detect_min60"], _ref_faces(img, min_face=60, max_face=240))
    assert out["max"] == ["120"]
    _close(out["detect_min60_max120"], _ref_faces(img, min_face=60, max_face=120))
    assert out["threads"] == ["3"]
    assert out["maxsize"] == [str(w // 2), str(h // 2)]
    _close(out["detect_grown"], _ref_faces(img, min_face=60, max_face=120, max_w=w // 2, max_h=h // 2))
    assert out["maxsize_after"] == [str(w), str(h)]
    assert out["param2"] == ["50", "1.1000"]
    _close(out["detect_param2"], _ref_faces(img, min_face=50, max_face=240, scale_factor=1.1))
    assert out["clear"] == ["0", "1"]
    assert out["detect_cleared"] == ["-1"]


@pytest.mark.gpu
def test_face_detector_facade_singleton_semantics(example):
    if not _cuda():
        pytest.skip("no CUDA device")
    import compactcnncascade_b200 as ccnn
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build not present")
    w, h = 640, 480
    img, _ = ccnn.synth_frame(w, h, 1, 5, 40, 200)
    out = _sections(_run(example, w, h, 1, "singleton"))
    assert out["init"] == ["0"]
    assert out["shared"] == ["1", "1"]  # one Init serves every instance
    _close(out["b_detect"], _ref_faces(img, min_face=40, max_face=240))
    assert out["a_min"] == ["60"]  # b's Init replaced the detector a uses
    _close(out["a_detect"], _ref_faces(img, min_face=60, max_face=240))
    assert out["after_clear"] == ["1", "1"]  # b's Clear ended it for a too
    assert out["a_detect_cleared"] == ["-1"]


# (args to the example, the same configuration for the reference)
CNN_CASES = [
    ("defaults", {}),
    ("high", {"min_obj": 40, "max_obj": 240, "sf": 1.15, "precision": 3, "t1": -1.5, "t2": -1.25, "t3": -1.0}),
    ("normal_adapt", {"min_obj": 40, "max_obj": 240, "sf": 1.15, "precision": 2, "t1": -1.5, "t2": -1.25, "t3": -1.0, "adapt": 1,
                      "double_check": 0, "drop": 0, "min_num": 2}),
    ("no_merger", {"min_obj": 40, "max_obj": 240, "sf": 1.15, "precision": 3, "t1": -1.5, "t2": -1.25, "t3": -1.0, "merger": 0}),
    ("ultra", {"min_obj": 40, "sf": 1.15, "precision": 4, "t1": -1.5, "t2": -1.25, "t3": -1.0}),
    # precision `def` with a colour frame needs min_obj < 34: above it the reference recurses forever
    ("def", {"min_obj": 30, "max_obj": 240, "precision": 0, "t1": -1.5, "t2": -1.25, "t3": -1.0}),
    ("low_gray_shrunk", {"min_obj": 60, "precision": 1, "t1": -1.5, "t2": -1.25, "t3": -1.0, "gray_only": 1}),
    ("packet_gpu", {"min_obj": 40, "max_obj": 240, "precision": 3, "t1": -1.5, "t2": -1.25, "t3": -1.0, "packet": 1, "pipeline": 1}),
]
PRIORS = [(10, 12, 50, 60, 1.0, 0.5, 3, 2), (300, 200, 80, 90, 2.5, 0.25, 1, 0), (305, 204, 80, 90, 0.5, 0.3, 2, 1)]


def _cnn_ref(img, cfg, prior=()):
    from compactcnncascade_b200 import _capi
    from oracle import ref
    p, ap = _capi.CnnParam(), _capi.CnnAdvancedParam()
    _capi.lib().ccnn_cnn_default_params(p, ap)
    p.max_image_height, p.max_image_width = img.shape[:2]
    keymap = {"min_neighbors": "min_neighbors", "precision": "detect_precision", "mode": "detect_mode", "t1": "treshold_1",
              "t2": "treshold_2", "t3": "treshold_3", "gray_only": "gray_image_only", "equalize": "equalize",
              "reflection": "reflection", "adapt": "adapt_min_neighbors", "double_check": "double_check", "drop": "drop_detect",
              "min_num": "min_num_detect", "merger": "merger_detect", "packet": "packet_detection"}
    for k, v in cfg.items():
        if k == "min_obj":
            p.min_obj_width = p.min_obj_height = v
        elif k == "max_obj":
            p.max_obj_width = p.max_obj_height = v
        elif k == "sf":
            p.scale_factor = v
        elif k == "pipeline":
            p.pipeline = v
        else:
            setattr(ap, keymap[k], v)
    return ref.cnn_detect(img, p, ap, prior)


def _dets(lines, tag):
    out = []
    for l in lines:
        parts = l.split()
        if parts[0] == tag:
            v = parts[1:]
            out.append((int(v[0]), int(v[1]), int(v[2]), int(v[3]), float(np.float32(v[4])), float(np.float32(v[5])), int(v[6]), int(v[7])))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name,cfg", CNN_CASES, ids=[c[0] for c in CNN_CASES])
@pytest.mark.parametrize("with_prior", [False, True], ids=["empty", "prior"])
def test_cnn_detector_facade_matches_reference(cnn_example, name, cfg, with_prior):
    if not _cuda():
        pytest.skip("no CUDA device")
    import compactcnncascade_b200 as ccnn
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build not present")
    w, h = 640, 480
    ch = 1 if name == "low_gray_shrunk" else 3
    img, _ = ccnn.synth_frame(w, h, 7, 5, 40, 200, channels=ch)
    prior = PRIORS if with_prior else []
    args = [f"{k}={v}" for k, v in cfg.items()] + [f"prior={','.join(str(x) for x in d)}" for d in prior] + ["nms=1"]
    lines = _run(cnn_example, w, h, 7, ch, *args)
    assert lines[0] == "rc 0"
    exp, pa, apa = _cnn_ref(img, cfg, prior)
    got = _dets(lines, "det")
    assert got == exp
    assert len(exp) > 0 or name == "defaults"
    adv = [int(v) for v in next(l.split()[1:] for l in lines if l.startswith("adv "))]
    assert adv[:9] == [apa.type_check, apa.drop_detect, apa.gray_image_only, apa.adapt_min_neighbors, apa.double_check,
                       apa.min_num_detect, apa.merger_detect, apa.equalize, apa.reflection]
    # packet mode and pipeline as a CUDA build of the reference reports them (InitDevice,
    # cnn_detector_v3.cpp:67-84; precision `def` turns packet mode off first, :922-925); the CPU
    # reference build here turns every pipeline into CPU instead
    pipeline = cfg.get("pipeline", 0)
    packet = 1 if (cfg.get("packet", 0) and pipeline > 0 and cfg.get("precision", 2) != 0) else 0
    assert adv[9:] == [packet, 1 if packet else pipeline]
    size = next(l.split()[1:] for l in lines if l.startswith("size "))
    assert [int(v) for v in size] == [pa.max_image_width, pa.max_image_height]
    # NMS of the result and shifted copies of it, against the reference Merger(0.5)
    rect = exp + [(x + wd // 10, y + 1, wd, ht, s, sc, k, nd) for (x, y, wd, ht, s, sc, k, nd) in exp]
    assert _dets(lines, "nms") == ref.merger(rect, 0.5)
