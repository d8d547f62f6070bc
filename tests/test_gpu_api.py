"""Behaviour of the public API on the GPU: batching, device input, the reference's
re-initialisation rules and cross-frame state, capacities and errors, independent handles."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def _params(w=640, h=480, min_face=40, max_face=240, sf=1.15):
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = min_face, max_face, sf
    p.detect_mode = 1
    return p


@pytest.fixture(scope="module")
def frames():
    return [ccnn.synth_frame(640, 480, 100 + i, 5, 40, 200)[0] for i in range(7)]


def test_batch_equals_single_frames(frames):
    d = ccnn.FaceDetector()
    assert d.Init(_params()) == 0
    single = [d.Detect(f) for f in frames]
    assert d.DetectBatch(frames) == single
    assert d.DetectBatch(frames[::-1]) == single[::-1]
    for f, s in zip(frames, single):
        assert s == orc.detect(f, orc.params(max_w=640, max_h=480))["final"]


def test_device_input_equals_host_input(frames):
    d = ccnn.FaceDetector()
    assert d.Init(_params()) == 0
    L = _capi.lib()
    cap = 256
    faces = (_capi.Face * (cap * len(frames)))()
    ns = (ctypes.c_int * len(frames))()
    dev = [torch.from_numpy(f).cuda() for f in frames]
    imgs = (_capi.Image * len(frames))(*[_capi.Image(640, 480, 3, t.data_ptr(), 640 * 3) for t in dev])
    ms = ctypes.c_float()
    assert L.ccnn_detect_device_batch(d._h, imgs, len(frames), faces, cap, ns, ctypes.byref(ms)) == 0
    assert ms.value > 0
    got = [[(f.x, f.y, f.width, f.height, f.score) for f in faces[i * cap: i * cap + ns[i]]] for i in range(len(frames))]
    assert got == [d.Detect(f) for f in frames]
    one = (_capi.Face * cap)()
    n = ctypes.c_int()
    im = _capi.Image(640, 480, 3, dev[0].data_ptr(), 640 * 3)
    assert L.ccnn_detect_device(d._h, ctypes.byref(im), None, one, cap, ctypes.byref(n)) == 0
    assert [(f.x, f.y, f.width, f.height, f.score) for f in one[: n.value]] == got[0]


def test_larger_frame_reinitialises_like_the_reference():
    img, _ = ccnn.synth_frame(1280, 720, 5, 8, 40, 200)
    small = ccnn.FaceDetector()
    assert small.Init(_params(640, 480)) == 0
    got = small.Detect(img)  # max_image_size grows to the frame (cnn_detector_v3.cpp:2499-2513)
    assert small.getMaxImageSize() == (1280, 720)
    assert got == orc.detect(img, orc.params(max_w=1280, max_h=720))["final"]


def test_level_count_state_carries_over_frames():
    """RunCPUDetect lowers num_scales when a level is too small and Detect only resets it for
    frames whose size differs from max_image_size: a max-size frame after a small one keeps the
    small frame's level count."""
    d = ccnn.FaceDetector()
    assert d.Init(_params(640, 480, min_face=40, max_face=0)) == 0
    big, _ = ccnn.synth_frame(640, 480, 9, 5, 40, 200)
    small, _ = ccnn.synth_frame(200, 150, 9, 1, 40, 60)
    d.Detect(big)
    n_big = len(d.levels())
    d.Detect(small)
    n_small = len(d.levels())
    assert n_small < n_big
    d.Detect(big)
    assert len(d.levels()) == n_small


def test_capacity_truncation_and_errors(frames):
    d = ccnn.FaceDetector()
    assert d.Init(_params(min_face=40, max_face=240)) == 0
    L = _capi.lib()
    img, _ = ccnn.synth_frame(640, 480, 1, 5, 40, 200)  # three faces (golden vga_bgr_s1)
    full = d.Detect(img)
    assert len(full) >= 2
    one = (_capi.Face * 1)()
    n = ctypes.c_int()
    im = _capi.Image(640, 480, 3, img.ctypes.data, 640 * 3)
    assert L.ccnn_detect(d._h, ctypes.byref(im), one, 1, ctypes.byref(n)) == _capi.TRUNCATED
    assert n.value == len(full) and (one[0].x, one[0].y) == full[0][:2]
    bad = _capi.Image(640, 480, 2, img.ctypes.data, 640 * 2)
    assert L.ccnn_detect(d._h, ctypes.byref(bad), one, 1, ctypes.byref(n)) == _capi.ERR_UNSUPPORTED
    tiny = np.zeros((20, 20, 3), np.uint8)
    assert d.Detect(tiny) == []


def test_independent_handles_and_setters(frames):
    a, b = ccnn.FaceDetector(), ccnn.FaceDetector()
    assert a.Init(_params(min_face=40)) == 0 and b.Init(_params(min_face=60, max_face=200)) == 0
    for f in frames[:3]:
        assert a.Detect(f) == orc.detect(f, orc.params(max_w=640, max_h=480, min_face=40))["final"]
        assert b.Detect(f) == orc.detect(f, orc.params(max_w=640, max_h=480, min_face=60, max_face=200))["final"]
    a.setMinObjectHeight(60)
    a.setMaxObjectHeight(200)
    assert (a.getMinObjectHeight(), a.getMaxObjectHeight()) == (60, 200)
    assert a.Detect(frames[0]) == b.Detect(frames[0])


def test_gray_device_pointer(frames):
    d = ccnn.FaceDetector()
    assert d.Init(_params()) == 0
    d.Detect(frames[0])
    ptr, w, h, step = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
    assert _capi.lib().ccnn_get_gray_device(d._h, ctypes.byref(ptr), ctypes.byref(w), ctypes.byref(h), ctypes.byref(step)) == 0
    assert ptr.value and (w.value, h.value) == (640, 480) and step.value % 64 == 0
    # read the device buffer by address
    n = h.value * step.value // 4
    buf = torch.empty(n, dtype=torch.float32, device="cuda")
    cudart = ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert cudart.cudaMemcpy(buf.data_ptr(), ptr.value, n * 4, 3) == 0  # cudaMemcpyDeviceToDevice
    dev = buf.view(h.value, step.value // 4)[:, : w.value].cpu().numpy()
    assert np.array_equal(dev, d.getGrayImage32F())
    assert np.array_equal(dev, orc.gray(frames[0]))
