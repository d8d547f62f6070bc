"""Many uneven pyramid levels and crowded candidate lists, bit-identical to the oracle.

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

import compactcnncascade_b200 as ccnn  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def _run(img, p):
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    faces = d.Detect(img)
    out = {"faces": faces, "levels": d.levels(), "cands": d.candidates(), "raw": d.raw_detections()}
    d.Clear()
    return out


def test_1080p_sf105_min20_matches_oracle():
    w, h = 1920, 1080
    img = ccnn.synth_frame(w, h, 4242, 30, 20, 600)[0]
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 20, 0, 1.05
    p.detect_mode = 1
    g = _run(img, p)
    ref = orc.detect(img, orc.params(max_w=w, max_h=h, min_face=20, max_face=0, scale_factor=1.05))
    assert len(g["levels"]) == len(ref["levels"]) and len(g["levels"]) > 32
    assert [(lv[0], lv[1]) for lv in g["levels"]] == [(a, b) for a, b, _ in ref["levels"]]
    assert [(c[0], c[1], c[2]) for c in g["cands"]] == [(c[0], c[1], c[2]) for c in ref["candidates"]]
    assert len(g["cands"]) > 500
    assert g["raw"] == ref["raw"]
    assert g["faces"] == ref["final"] and len(g["faces"]) > 0


@pytest.mark.parametrize("n_faces,thr1", [(300, -1.5), (400, -1.7)])
def test_crowded_candidates_match_oracle(n_faces, thr1):
    w, h = 1920, 1080
    img = ccnn.synth_frame(w, h, 77, n_faces, 30, 90)[0]
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    p.treshold[0] = thr1
    p.detect_mode = 1
    g = _run(img, p)
    t = time.time()
    ref = orc.detect(img, orc.params(max_w=w, max_h=h, thr=(thr1, -1.25, -1.0)))
    per_level = {}
    for c in g["cands"]:
        per_level[c[0]] = per_level.get(c[0], 0) + 1
    print(f"thr1 {thr1}: oracle {time.time() - t:.1f} s, {len(g['cands'])} candidates "
          f"(max {max(per_level.values())} in one level), {len(g['raw'])} raw, {len(g['faces'])} faces")
    assert [(c[0], c[1], c[2]) for c in g["cands"]] == [(c[0], c[1], c[2]) for c in ref["candidates"]]
    assert g["raw"] == ref["raw"]
    assert g["faces"] == ref["final"]
