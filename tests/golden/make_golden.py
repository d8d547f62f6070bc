"""Generates tests/golden/golden.json from the reference's own CPU path (oracle/_ref, built from the
unmodified reference sources by oracle/Makefile). Run on a machine where the reference is present:

    make -C oracle ref && python tests/golden/make_golden.py

Frames come from the package's seeded generator; the fixture stores each frame's SHA-256 so the
tests can confirm the generator reproduces the same bytes. Float results are stored as IEEE bit
patterns (hex) or as SHA-256 of the raw float32 arrays, so comparisons are bit-exact.
"""
import hashlib
import json
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import compactcnncascade_b200 as ccnn  # noqa: E402
from oracle import ref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def fbits(x):
    return struct.pack("<f", float(x)).hex()


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# (name, frame spec, detector params)
CASES = [
    ("vga_bgr_s0", dict(w=640, h=480, seed=0, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240)),
    ("vga_bgr_s1", dict(w=640, h=480, seed=1, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240)),
    ("vga_bgr_s2", dict(w=640, h=480, seed=2, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240)),
    ("vga_bgr_s3", dict(w=640, h=480, seed=3, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240)),
    ("hd_bgr_s0", dict(w=1920, h=1080, seed=0, n=20, mn=30, mx=300, ch=3), dict(min_face=40, max_face=240)),
    ("hd_bgr_s7", dict(w=1920, h=1080, seed=7, n=20, mn=30, mx=300, ch=3), dict(min_face=40, max_face=240)),
    ("vga_gray_downscale", dict(w=640, h=480, seed=5, n=5, mn=60, mx=200, ch=1), dict(min_face=80, max_face=0)),
    ("vga_gray_full", dict(w=640, h=480, seed=6, n=5, mn=40, mx=200, ch=1), dict(min_face=30, max_face=200)),
    ("vga_bgra", dict(w=640, h=480, seed=11, n=5, mn=40, mx=200, ch=4), dict(min_face=40, max_face=240)),
    ("prec_low", dict(w=640, h=480, seed=12, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240, precision=1)),
    ("prec_normal", dict(w=640, h=480, seed=12, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240, precision=2)),
    ("prec_ultra", dict(w=640, h=480, seed=12, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240, precision=4)),
    ("prec_def", dict(w=640, h=480, seed=12, n=5, mn=40, mx=200, ch=3), dict(min_face=30, max_face=240, precision=0)),
    ("no_drop", dict(w=640, h=480, seed=13, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240, drop_detect=0)),
    ("no_equalize_no_reflection", dict(w=640, h=480, seed=13, n=5, mn=40, mx=200, ch=3),
     dict(min_face=40, max_face=240, equalize=0, reflection=0)),
    ("stage1_only", dict(w=640, h=480, seed=14, n=5, mn=40, mx=200, ch=3), dict(min_face=40, max_face=240, detect_mode=0)),
    ("upsample_sf105", dict(w=320, h=240, seed=15, n=4, mn=20, mx=120, ch=3), dict(min_face=20, max_face=0, scale_factor=1.05)),
    ("odd_97x61", dict(w=97, h=61, seed=16, n=1, mn=30, mx=50, ch=3), dict(min_face=20, max_face=0)),
    ("exact_47x51", dict(w=47, h=51, seed=17, n=1, mn=30, mx=40, ch=3), dict(min_face=30, max_face=0)),
    ("too_small_40x40", dict(w=40, h=40, seed=18, n=1, mn=20, mx=30, ch=3), dict(min_face=20, max_face=0)),
    ("low_threshold", dict(w=640, h=480, seed=19, n=5, mn=40, mx=200, ch=3),
     dict(min_face=40, max_face=240, thr=(-1.7, -1.5, -1.3))),
]


def frame(spec):
    img, _ = ccnn.synth_frame(spec["w"], spec["h"], spec["seed"], spec["n"], spec["mn"], spec["mx"], channels=spec["ch"])
    return img


def main():
    if not ref.available():
        raise SystemExit("oracle/_ref/libccnn_ref.so is missing: build it with `make -C oracle ref` first")
    out = {"generator": "compactcnncascade_b200.synth_frame", "reference": "oracle/_ref/libccnn_ref.so (strict IEEE build)",
           "cases": []}
    for name, spec, dp in CASES:
        img = frame(spec)
        mw, mh = max(spec["w"], 64), max(spec["h"], 64)
        p = ref.params(max_w=mw, max_h=mh, **dp)
        steps = ref.detect_steps(img, p)
        api = ref.face_detect(img, p)
        assert steps["final"] == api, name  # the step-wise replay equals the genuine API
        cands = []
        for li in reversed(range(len(steps["resp"]))):
            r = steps["resp"][li]
            ys, xs = np.nonzero(r > np.float32(dp.get("thr", (-1.5,))[0]))
            cands += [[li, int(x) * 4, int(y) * 4, fbits(r[y, x])] for y, x in zip(ys, xs)]
        out["cases"].append({
            "name": name, "frame": spec, "params": dp, "max_image": [mw, mh], "frame_sha256": sha(img),
            "gray_sha256": sha(steps["gray"]), "gray_shape": list(steps["gray"].shape),
            "levels": [[l[0], l[1], fbits(l[2])] for l in steps["levels"]],
            "level_sha256": [sha(l[3]) for l in steps["levels"]],
            "resp_shapes": [list(r.shape) for r in steps["resp"]],
            "resp_sha256": [sha(r) for r in steps["resp"]],
            "candidates": cands,
            "raw": [[d[0], d[1], d[2], d[3], fbits(d[4]), fbits(d[5]), d[6], d[7]] for d in steps["raw"]],
            "final": [[f[0], f[1], f[2], f[3], fbits(f[4])] for f in api],
        })
        print(f"{name}: {len(steps['levels'])} levels, {len(cands)} candidates, {len(steps['raw'])} raw, {len(api)} faces")

    # primitives on seeded random inputs
    rng = np.random.default_rng(1234)
    prim = {"gray": [], "resize": [], "net": []}
    for ch in (1, 3, 4):
        img = rng.integers(0, 256, size=(53, 67) if ch == 1 else (53, 67, ch), dtype=np.uint8)
        prim["gray"].append({"ch": ch, "shape": [53, 67], "input_sha256": sha(img), "out_sha256": sha(ref.gray(img))})
    src = (rng.random((211, 173), dtype=np.float32) * 255).astype(np.float32)
    prim["resize_src_sha256"] = sha(src)
    for (dw, dh) in [(50, 60), (173, 211), (300, 401), (100, 201)]:
        for t in (0, 1):
            prim["resize"].append({"dw": dw, "dh": dh, "type": t, "out_sha256": sha(ref.resize_f32(src, dw, dh, t))})
    for st, idx, (w, h) in [(1, 1, (23, 27)), (1, 1, (131, 97)), (2, 0, (47, 51)), (3, 0, (47, 51)), (2, 1, (47, 51))]:
        img = (rng.random((h, w), dtype=np.float32) * 255).astype(np.float32)
        r = ref.net_forward(st, img, idx)
        prim["net"].append({"stage": st, "index": idx, "w": w, "h": h, "input_sha256": sha(img), "out_sha256": sha(r),
                            "out_shape": list(r.shape), "first": [fbits(v) for v in r.ravel()[:4]]})
    out["primitives"] = prim
    out["primitive_seed"] = 1234

    # std::sort permutations on tie-heavy keys (the device replicates this order)
    srt = []
    for n in (5, 16, 17, 33, 64, 200, 513):
        keys = rng.integers(0, 4, size=n).astype(np.float32) * np.float32(0.25) + np.float32(0.1)
        srt.append({"keys": [fbits(k) for k in keys], "perm": ref.sort_perm(keys).tolist()})
    out["sort"] = srt

    with open(OUT, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
