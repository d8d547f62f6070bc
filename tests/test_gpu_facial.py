"""Facial analysis (the landmark network as a fourth stage) on the GPU against the reference's
own cascade with facial_analysis on: same boxes, scores, gender, smile and glasses."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from oracle import ref  # noqa: E402

if not ref.available():
    pytest.skip("reference build (oracle/_ref) not available", allow_module_level=True)


def _params(w, h, precision=3):
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    p.detect_precision = precision
    p.detect_mode = 1
    p.facial_analysis = 1
    return p


CASES = [(640, 480, 100 + i, 5, 40, 200, 3) for i in range(4)] + [(640, 480, 200, 5, 40, 200, 2), (640, 480, 201, 5, 40, 200, 4),
                                                                   (1920, 1080, 7, 20, 30, 300, 3)]


@pytest.mark.parametrize("w,h,seed,nf,lo,hi,prec", CASES)
def test_facial_analysis_matches_reference(w, h, seed, nf, lo, hi, prec):
    img = ccnn.synth_frame(w, h, seed, nf, lo, hi)[0]
    d = ccnn.FaceDetector()
    assert d.Init(_params(w, h, prec)) == 0
    got = d.Detect(img, attributes=True)
    d.Clear()
    want = ref.face_detect_fa(img, ref.params(max_w=w, max_h=h, precision=prec))
    assert got == want
    assert len(got) > 0 and all(f[5] in (0, 1) for f in got)


def test_facial_analysis_off_keeps_attributes_unset():
    img = ccnn.synth_frame(640, 480, 100, 5, 40, 200)[0]
    p = _params(640, 480)
    p.facial_analysis = 0
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    faces = d.Detect(img, attributes=True)
    assert faces and all(f[5:] == (-1, -1, -1) for f in faces)
