"""Loader for tests/golden/golden.json (fixtures generated from the reference by
tests/golden/make_golden.py)."""
import hashlib
import json
import os
import struct

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")
_G = None


def golden():
    global _G
    if _G is None:
        with open(PATH) as f:
            _G = json.load(f)
    return _G


def fbits(x):
    return struct.pack("<f", float(x)).hex()


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def case_names():
    return [c["name"] for c in golden()["cases"]]


def case(name):
    return next(c for c in golden()["cases"] if c["name"] == name)


def frame(c):
    import compactcnncascade_b200 as ccnn
    f = c["frame"]
    img, _ = ccnn.synth_frame(f["w"], f["h"], f["seed"], f["n"], f["mn"], f["mx"], channels=f["ch"])
    return img


def oracle_params(c):
    from oracle import oracle as orc
    d = dict(c["params"])
    if "thr" in d:
        d["thr"] = tuple(d["thr"])
    return orc.params(max_w=c["max_image"][0], max_h=c["max_image"][1], **d)


def ccnn_params(c):
    """The same configuration as FaceDetector::Param of the package."""
    import compactcnncascade_b200 as ccnn
    d = c["params"]
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = c["max_image"]
    p.min_face_height = d.get("min_face", 40)
    p.max_face_height = d.get("max_face", 240)
    p.scale_factor = d.get("scale_factor", 1.15)
    p.detect_precision = d.get("precision", 3)
    thr = d.get("thr", (-1.5, -1.25, -1.0))
    for i in range(3):
        p.treshold[i] = thr[i]
    p.drop_detect = d.get("drop_detect", 1)
    p.equalize = d.get("equalize", 1)
    p.reflection = d.get("reflection", 1)
    p.detect_mode = d.get("detect_mode", 1)
    p.min_neighbors = d.get("min_neighbors", 2)
    return p


def primitive_inputs():
    """Regenerates the seeded primitive inputs in make_golden.py's order."""
    rng = np.random.default_rng(golden()["primitive_seed"])
    grays = [rng.integers(0, 256, size=(53, 67) if ch == 1 else (53, 67, ch), dtype=np.uint8) for ch in (1, 3, 4)]
    src = (rng.random((211, 173), dtype=np.float32) * 255).astype(np.float32)
    nets = []
    for st, idx, (w, h) in [(1, 1, (23, 27)), (1, 1, (131, 97)), (2, 0, (47, 51)), (3, 0, (47, 51)), (2, 1, (47, 51))]:
        nets.append((st, idx, (rng.random((h, w), dtype=np.float32) * 255).astype(np.float32)))
    return grays, src, nets
