"""The stage-1 front kernel resamples every level tile from the gray frame (the pyramid is not stored).
The reference picks the resampling per level (RunCPUDetect, cnn_detector_v3.cpp:2090-2104): a copy at
scale 1, nearest neighbour above 0.7, bilinear below. Min face 27 at scale factor 1.15 gives all three
(level 0 at scale 1.0, levels 1-2 at 0.87 and 0.76, the rest bilinear), and min face 24 an upsampled
nearest-neighbour level 0 (1.125); every response map must equal the reference build's bit for bit, and
so must the candidates, the raw detections and the final boxes, for BGR and gray frames."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402
from oracle import ref  # noqa: E402
from tests.goldens import fbits, sha  # noqa: E402

if not ref.available():
    pytest.skip("reference build oracle/_ref/libccnn_ref.so not present", allow_module_level=True)

RESP_RTOL = 1e-4  # stated bar for fp32 response maps; they are also checked bit-exact


@pytest.mark.parametrize("min_face,channels,seed", [(27, 3, 31), (27, 1, 32), (24, 3, 33)])
def test_copy_nearest_and_bilinear_levels_match_reference(min_face, channels, seed):
    w, h = 640, 480
    img = ccnn.synth_frame(w, h, seed, 6, 30, 200)[0]
    if channels == 1:
        img = np.ascontiguousarray(img[:, :, 1])
    rp = ref.params(min_face=min_face, max_face=240, scale_factor=1.15, max_w=w, max_h=h)
    exp = ref.detect_steps(img, rp, with_levels=False, resp_cap=2 * w * h)
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = min_face, 240, 1.15
    det = ccnn.FaceDetector()
    assert det.Init(p) == 0, _capi.last_error()
    faces = det.Detect(img)
    levels = det.levels()
    assert [(lv[0], lv[1], fbits(lv[2])) for lv in levels] == [(a, b, fbits(s)) for a, b, s, _ in exp["levels"]]
    scales = [lv[2] for lv in levels]
    assert scales[0] >= 1.0 and any(0.7 < s < 1.0 for s in scales) and scales[-1] < 0.7
    for i, r_exp in enumerate(exp["resp"]):
        r = det.response_map(i)
        assert r.shape == r_exp.shape
        assert np.allclose(r, r_exp, rtol=RESP_RTOL, atol=0), i
        assert sha(r) == sha(r_exp), i
    assert det.raw_detections() == exp["raw"]
    assert faces == exp["final"]
    det.Clear()
