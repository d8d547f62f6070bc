"""ccnn_stage1_forward_static: the stage-1 entry point for callers that may not allocate device
memory (their host budgets all device memory up front, or another framework's allocator holds it).
It must give the same response maps as the regular handle-based entry point, on consecutive calls
that share its fixed scratch array, for vector-aligned and odd image widths and padded row pitches,
and refuse images beyond the array's stated limit and unreadable model files. This file is
collected last so a failure here comes after every other test has run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402

RESP_RTOL = 1e-4  # the response-map tolerance of the parity tests (results are in fact bit-exact)


def _forward(fn_static, handle, img, pitch):
    """Response map of `img` (h x w floats) stored on the device with a row pitch of `pitch` floats."""
    L = _capi.lib()
    h, w = img.shape
    buf = np.full((h, pitch), np.float32(-7.0), dtype=np.float32)  # padding the kernels must not read
    buf[:, :w] = img
    dimg = torch.from_numpy(buf).cuda()
    cap = w * h
    resp = torch.full((cap,), float("nan"), dtype=torch.float32, device="cuda")
    rw, rh = ctypes.c_int(), ctypes.c_int()
    if fn_static:
        st = L.ccnn_stage1_forward_static(None, dimg.data_ptr(), w, h, pitch * 4, resp.data_ptr(), cap, ctypes.byref(rw),
                                          ctypes.byref(rh), None)
    else:
        st = L.ccnn_stage1_forward(handle, dimg.data_ptr(), w, h, pitch * 4, resp.data_ptr(), cap, ctypes.byref(rw),
                                   ctypes.byref(rh), None)
    assert st == 0, _capi.last_error()
    return resp[: rw.value * rh.value].cpu().numpy().reshape(rh.value, rw.value)


def test_static_scratch_entry_matches_regular_entry():
    p = ccnn.default_params()
    p.min_face_height = 40
    det = ccnn.FaceDetector()
    assert det.Init(p) == 0, _capi.last_error()
    rng = np.random.default_rng(2024)
    # two calls in a row (the second reuses the scratch left by the first), a smaller image, an odd
    # width (scalar loads), and padded row pitches with vector and scalar loads
    cases = [(1296, 729, 1296), (1920, 1080, 1920), (300, 211, 300), (301, 211, 301), (1296, 729, 1300), (301, 211, 305)]
    for (w, h, pitch) in cases:
        img = (rng.random((h, w), dtype=np.float32) * 255).astype(np.float32)
        got = _forward(True, None, img, pitch)
        exp = _forward(False, det._h, img, pitch)
        assert got.shape == exp.shape
        assert np.all(np.isfinite(got))
        assert np.allclose(got, exp, rtol=RESP_RTOL, atol=0)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (w, h, pitch)
    det.Clear()


def test_static_scratch_entry_refuses_oversize_images():
    L = _capi.lib()
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    rw, rh = ctypes.c_int(), ctypes.c_int()
    st = L.ccnn_stage1_forward_static(None, dummy.data_ptr(), 4096, 2160, 4096 * 4, dummy.data_ptr(), 16, ctypes.byref(rw),
                                      ctypes.byref(rh), None)
    assert st == _capi.ERR_INVALID_ARG
    assert "static scratch" in _capi.last_error() and "2359296" in _capi.last_error()


def test_static_scratch_entry_refuses_missing_model(tmp_path):
    L = _capi.lib()
    dummy = torch.zeros(64 * 64, dtype=torch.float32, device="cuda")
    rw, rh = ctypes.c_int(), ctypes.c_int()
    st = L.ccnn_stage1_forward_static(str(tmp_path / "no_such_model.bin").encode(), dummy.data_ptr(), 64, 64, 64 * 4,
                                      dummy.data_ptr(), 64 * 64, ctypes.byref(rw), ctypes.byref(rh), None)
    assert st == _capi.ERR_MODEL, _capi.last_error()
