"""Parity of the CUDA path with the reference's own CPU implementation, step by step.

Bar (see the module docstrings of each kernel): gray image, pyramid levels, candidate indices and
raw detections bit-exact; response maps within 1e-4 relative (they are in fact bit-exact, which is
also asserted); final boxes identical.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402

RESP_RTOL = 1e-4


def _dev_u8(img, pitch_mult=64):
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    pitch = (w * ch + pitch_mult - 1) // pitch_mult * pitch_mult
    t = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
    t[:, : w * ch] = torch.from_numpy(img.reshape(h, w * ch)).cuda()
    return t, pitch


def test_gray_bitexact(ref):
    rng = np.random.default_rng(1)
    L = _capi.lib()
    for (w, h) in [(17, 5), (1023, 1077), (1920, 1080), (47, 51)]:
        for ch in (1, 3, 4):
            img = rng.integers(0, 256, size=(h, w) if ch == 1 else (h, w, ch), dtype=np.uint8)
            src, sp = _dev_u8(img)
            dpitch = (w + 15) // 16 * 16
            dst = torch.zeros((h, dpitch), dtype=torch.float32, device="cuda")
            st = L.ccnn_gray_u8_to_f32(src.data_ptr(), w, h, ch, sp, dst.data_ptr(), dpitch * 4, None)
            assert st == 0, _capi.last_error()
            got = dst[:, :w].cpu().numpy()
            exp = ref.gray(np.ascontiguousarray(img))
            assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (w, h, ch)


def test_resize_bitexact(ref):
    rng = np.random.default_rng(2)
    L = _capi.lib()
    src = (rng.random((1017, 1017), dtype=np.float32) * 255).astype(np.float32)
    dsrc = torch.from_numpy(src).cuda()
    for (dw, dh) in [(50, 50), (200, 150), (509, 1000), (1017, 1017), (1400, 1100)]:
        for typ in (0, 1):
            dst = torch.zeros((dh, dw), dtype=torch.float32, device="cuda")
            st = L.ccnn_resize_f32(dsrc.data_ptr(), 1017, 1017, 1017 * 4, dst.data_ptr(), dw, dh, dw * 4, typ, None)
            assert st == 0, _capi.last_error()
            exp = ref.resize_f32(src, dw, dh, typ)
            assert np.array_equal(dst.cpu().numpy().view(np.uint32), exp.view(np.uint32)), (dw, dh, typ)


@pytest.fixture(scope="module")
def det():
    p = ccnn.default_params()
    p.min_face_height, p.max_face_height = 40, 240
    p.detect_mode = 1
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0, _capi.last_error()
    yield d
    d.Clear()


def test_stage1_forward(ref, det):
    rng = np.random.default_rng(3)
    L = _capi.lib()
    for (w, h) in [(23, 27), (24, 28), (47, 51), (97, 61), (300, 211), (1296, 729)]:
        img = (rng.random((h, w), dtype=np.float32) * 255).astype(np.float32)
        dimg = torch.from_numpy(img).cuda()
        cap = w * h
        resp = torch.zeros(cap, dtype=torch.float32, device="cuda")
        rw, rh = ctypes.c_int(), ctypes.c_int()
        st = L.ccnn_stage1_forward(det._h, dimg.data_ptr(), w, h, w * 4, resp.data_ptr(), cap, ctypes.byref(rw),
                                   ctypes.byref(rh), None)
        assert st == 0, _capi.last_error()
        got = resp[: rw.value * rh.value].cpu().numpy().reshape(rh.value, rw.value)
        exp = ref.net_forward(1, img, 1)
        assert got.shape == exp.shape
        rel = np.abs(got - exp) / np.maximum(np.abs(exp), 1e-6)
        assert rel.max() <= RESP_RTOL
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (w, h, float(np.abs(got - exp).max()))


CASES = [(640, 480, 0, 5, 40, 200), (640, 480, 1, 5, 40, 200), (1920, 1080, 0, 20, 30, 300), (1920, 1080, 7, 20, 30, 300)]


@pytest.mark.parametrize("w,h,seed,nf,mn,mx", CASES)
def test_detect_pipeline_matches_reference(ref, det, w, h, seed, nf, mn, mx):
    img, _ = ccnn.synth_frame(w, h, seed, nf, mn, mx)
    got_faces = det.Detect(img)
    p = ref.params(min_face=40, max_face=240, scale_factor=1.15)
    steps = ref.detect_steps(img, p)
    # gray
    assert np.array_equal(det.getGrayImage32F().view(np.uint32), steps["gray"].view(np.uint32))
    # levels and response maps
    lv = det.levels()
    assert [(a[0], a[1]) for a in lv] == [(b[0], b[1]) for b in steps["levels"]]
    assert [a[2] for a in lv] == [b[2] for b in steps["levels"]]
    for i, r in enumerate(steps["resp"]):
        g = det.response_map(i)
        assert g.shape == r.shape
        assert np.allclose(g, r, rtol=RESP_RTOL, atol=0)
        assert np.array_equal(g.view(np.uint32), r.view(np.uint32)), i
    # candidate indices: raster scan, smallest level first
    exp_c = []
    for i in reversed(range(len(steps["resp"]))):
        ys, xs = np.nonzero(steps["resp"][i] > np.float32(-1.5))
        exp_c += [(i, int(x) * 4, int(y) * 4) for y, x in zip(ys, xs)]
    got_c = [(c[0], c[1], c[2]) for c in det.candidates()]
    assert got_c == exp_c
    # raw detections (cpu_detect_rect order) and final boxes
    assert det.raw_detections() == [tuple(r) for r in steps["raw"]]
    assert [tuple(f) for f in got_faces] == [tuple(f) for f in steps["final"]]
    api = ref.face_detect(img, p)
    assert [tuple(f) for f in got_faces] == [tuple(f) for f in api]
