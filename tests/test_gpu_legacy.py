"""Legacy model family (format 1.0, cnn4face{1,2,3}_new.bin) on the GPU: the device forward pass of
each network equals the reference's own (SIMD::ConvNeuralNetwork of src/CNNObjectDetector/cnn_simd.cpp,
plain-C++ build with strict IEEE float) bit for bit, on random images and on gray synthetic frames.
Each reference call runs in a fresh process: the reference's fully connected route keeps the buffers
of the first network that ran it (a function-local static), so only one network per process is right."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402
from oracle import ref  # noqa: E402

if not ref.legacy_available():
    pytest.skip("legacy reference build (oracle/_ref/libccnn_ref_legacy.so) not available", allow_module_level=True)

MODELS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "compactcnncascade_b200", "models")


def _device_forward(name, img, pitch_pad=0):
    h, w = img.shape
    pitch = w + pitch_pad
    buf = torch.zeros((h, pitch), dtype=torch.float32, device="cuda")
    buf[:, :w] = torch.from_numpy(img).cuda()
    out = torch.full((w * h,), np.nan, dtype=torch.float32, device="cuda")
    ow, oh = ctypes.c_int(), ctypes.c_int()
    st = _capi.lib().ccnn_legacy_net_forward(os.path.join(MODELS, name).encode(), buf.data_ptr(), w, h, pitch * 4, out.data_ptr(), out.numel(),
                                             ctypes.byref(ow), ctypes.byref(oh), None)
    _capi.check(st, "ccnn_legacy_net_forward")
    return out[: ow.value * oh.value].cpu().numpy().reshape(oh.value, ow.value)


def _gray(w, h, seed, nf, lo, hi):
    img = ccnn.synth_frame(w, h, seed, nf, lo, hi, channels=1)[0]
    return img.astype(np.float32)


RNG = np.random.default_rng(3)
CASES = [
    ("cnn4face1_new.bin", RNG.uniform(0, 255, (150, 200)).astype(np.float32), 0),
    ("cnn4face1_new.bin", RNG.uniform(0, 255, (31, 27)).astype(np.float32), 5),
    ("cnn4face1_new.bin", _gray(640, 480, 11, 5, 40, 200), 0),
    ("cnn4face1_new.bin", _gray(333, 211, 12, 3, 30, 90), 3),
    ("cnn4face2_new.bin", RNG.uniform(0, 255, (51, 47)).astype(np.float32), 0),
    ("cnn4face2_new.bin", _gray(47, 51, 13, 1, 40, 45), 0),
    ("cnn4face2_new.bin", RNG.uniform(0, 255, (64, 80)).astype(np.float32), 1),
    ("cnn4face3_new.bin", RNG.uniform(0, 255, (51, 47)).astype(np.float32), 0),
    ("cnn4face3_new.bin", _gray(47, 51, 14, 1, 40, 45), 2),
    ("cnn4face3_new.bin", RNG.uniform(0, 255, (70, 90)).astype(np.float32), 0),
]


@pytest.mark.parametrize("name,img,pad", CASES, ids=[f"{c[0]}-{c[1].shape[1]}x{c[1].shape[0]}" for c in CASES])
def test_legacy_forward_matches_reference(name, img, pad):
    got = _device_forward(name, img, pad)
    want = ref.legacy_net_forward_isolated(os.path.join(MODELS, name), img)
    assert got.shape == want.shape and got.size > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), float(np.abs(got - want).max())


def test_legacy_forward_rejects_small_images():
    with pytest.raises(ccnn.CCNNError):
        _device_forward("cnn4face2_new.bin", np.zeros((39, 35), np.float32))


def _legacy_detector(w, h, min_face=40, max_face=240, scale=1.15):
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = min_face, max_face, scale
    p.detect_mode = 1
    d = ccnn.FaceDetector()
    assert d.Init(p, models=[os.path.join(MODELS, f"cnn4face{i}_new.bin") for i in (1, 2, 3)]) == 0, _capi.last_error()
    return d


DETECT_CASES = [(640, 480, 1, 5, 40, 200, 3), (640, 480, 2, 5, 40, 200, 3), (640, 480, 3, 5, 40, 200, 3), (640, 480, 4, 5, 40, 200, 1),
                (1280, 720, 5, 10, 30, 300, 3), (1920, 1080, 7, 20, 30, 300, 3)]


@pytest.mark.parametrize("w,h,seed,nf,lo,hi,ch", DETECT_CASES)
def test_legacy_cascade_matches_reference(w, h, seed, nf, lo, hi, ch):
    """The whole cascade with the legacy models gives the reference's own faces (built for the legacy
    family) on the same frame, box for box and score for score."""
    img = ccnn.synth_frame(w, h, seed, nf, lo, hi, channels=ch)[0]
    d = _legacy_detector(w, h)
    got = d.Detect(img)
    d.Clear()
    want = ref.legacy_face_detect(img, max_w=w, max_h=h)
    assert got == want
    assert len(want) > 0 or seed == 4


def test_legacy_detector_refuses_mixed_families_and_the_gate():
    p = ccnn.default_params()
    d = ccnn.FaceDetector()
    mixed = [os.path.join(MODELS, "cnn4face1_new.bin"), os.path.join(MODELS, "cnn4face2_cntk.bin"), os.path.join(MODELS, "cnn4face3_new.bin")]
    assert d.Init(p, models=mixed) == -1
    d = _legacy_detector(640, 480)
    with pytest.raises(ccnn.CCNNError):
        d.setGate(np.zeros(700, np.float32), 0.5)
