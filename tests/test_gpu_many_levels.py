"""Many uneven pyramid levels and crowded candidate lists, bit-identical to the reference's own
cascade (the strict IEEE build of the unmodified sources, oracle/_ref/libccnn_ref.so).

* The batched-pyramid settings (scale factor 1.05, min face 20, no max face, so the largest level
  is an upsampled 1.35x copy): more levels than one launch's level table holds.
* Hundreds of small faces and a low stage-1 threshold: thousands of candidates, more than the replay keeps in shared memory,
  and levels with more candidates than its bit matrices cover.
"""
import time

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import numpy as np  # noqa: E402

import compactcnncascade_b200 as ccnn  # noqa: E402
from oracle import ref  # noqa: E402

if not ref.available():
    pytest.skip("reference build oracle/_ref/libccnn_ref.so not present", allow_module_level=True)


def _reference(img, thr1=-1.5, **kw):
    """The reference cascade's levels, candidates (levels last to first, raster order, response >
    treshold_1), raw detections and final boxes."""
    h, w = img.shape[:2]
    steps = ref.detect_steps(img, ref.params(max_w=w, max_h=h, thr=(thr1, -1.25, -1.0), **kw), with_levels=False,
                             resp_cap=2 * w * h)
    cands = []
    for li in reversed(range(len(steps["resp"]))):
        r = steps["resp"][li]
        ys, xs = np.nonzero(r > np.float32(thr1))
        cands += [(li, int(x) * 4, int(y) * 4) for y, x in zip(ys, xs)]
    return {"levels": [(a, b) for a, b, _, _ in steps["levels"]], "candidates": cands, "raw": steps["raw"],
            "final": steps["final"]}


def _run(img, p):
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    faces = d.Detect(img)
    out = {"faces": faces, "levels": d.levels(), "cands": d.candidates(), "raw": d.raw_detections()}
    d.Clear()
    return out


def test_1080p_sf105_min20_matches_reference():
    w, h = 1920, 1080
    img = ccnn.synth_frame(w, h, 4242, 30, 20, 600)[0]
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 20, 0, 1.05
    p.detect_mode = 1
    g = _run(img, p)
    exp = _reference(img, min_face=20, max_face=0, scale_factor=1.05)
    assert len(g["levels"]) == len(exp["levels"]) and len(g["levels"]) > 32
    assert [(lv[0], lv[1]) for lv in g["levels"]] == exp["levels"]
    assert [(c[0], c[1], c[2]) for c in g["cands"]] == exp["candidates"]
    assert len(g["cands"]) > 500
    assert g["raw"] == exp["raw"]
    assert g["faces"] == exp["final"] and len(g["faces"]) > 0


@pytest.mark.parametrize("n_faces,thr1", [(300, -1.5), (400, -1.7)])
def test_crowded_candidates_match_reference(n_faces, thr1):
    w, h = 1920, 1080
    img = ccnn.synth_frame(w, h, 77, n_faces, 30, 90)[0]
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    p.treshold[0] = thr1
    p.detect_mode = 1
    g = _run(img, p)
    t = time.time()
    exp = _reference(img, thr1=thr1)
    per_level = {}
    for c in g["cands"]:
        per_level[c[0]] = per_level.get(c[0], 0) + 1
    print(f"thr1 {thr1}: reference {time.time() - t:.1f} s, {len(g['cands'])} candidates "
          f"(max {max(per_level.values())} in one level), {len(g['raw'])} raw, {len(g['faces'])} faces")
    assert [(c[0], c[1], c[2]) for c in g["cands"]] == exp["candidates"]
    assert g["raw"] == exp["raw"]
    assert g["faces"] == exp["final"]
