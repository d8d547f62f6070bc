"""Device frames are read only after the caller's pending work that writes them: on the legacy
default stream when no stream is given (where torch writes by default), or on the stream the caller
passes. Each frame is written by a torch copy queued behind a long GPU spin, right before the call;
a detector that read early would see the blank frame left there before."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402

W, H = 1280, 720
SPIN_CYCLES = 200_000_000  # about 0.1 s of GPU time before the frame is written


def _detector():
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = W, H
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0, _capi.last_error()
    return d


def _frames():
    imgs = [ccnn.synth_frame(W, H, 4100 + i, 10, 30, 300)[0] for i in range(3)]
    return imgs, [torch.from_numpy(im).cuda() for im in imgs]


def test_device_frame_waits_for_default_stream_writer():
    d = _detector()
    imgs, src = _frames()
    want = [d.Detect(im) for im in imgs]
    assert all(len(f) > 0 for f in want)
    for aligned in (True, False):
        for k in range(len(imgs)):
            base = torch.zeros(H * W * 3 + 64, dtype=torch.uint8, device="cuda")
            frame = base[: H * W * 3] if aligned else base[1: 1 + H * W * 3]  # read in place / copied
            torch.cuda.synchronize()
            torch.cuda._sleep(SPIN_CYCLES)  # default stream: busy, then the frame is written
            frame.copy_(src[k].view(-1))
            got = d.DetectDevice(frame.data_ptr(), W, H, 3, W * 3)
            assert got == want[k], (aligned, k)
    d.Clear()


def test_device_frame_waits_for_given_stream_writer():
    d = _detector()
    imgs, src = _frames()
    want = [d.Detect(im) for im in imgs]
    s = torch.cuda.Stream()
    for k in range(len(imgs)):
        frame = torch.zeros(H * W * 3, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            torch.cuda._sleep(SPIN_CYCLES)
            frame.copy_(src[k].view(-1))
        got = d.DetectDevice(frame.data_ptr(), W, H, 3, W * 3, stream=ctypes.c_void_p(s.cuda_stream))
        assert got == want[k], k
    d.Clear()


def test_device_batch_waits_for_default_stream_writer():
    d = _detector()
    imgs, src = _frames()
    want = [d.Detect(im) for im in imgs]
    n_img = 6
    frames = [torch.zeros(H * W * 3, dtype=torch.uint8, device="cuda") for _ in range(n_img)]
    torch.cuda.synchronize()
    torch.cuda._sleep(SPIN_CYCLES)
    for i, f in enumerate(frames):
        f.copy_(src[i % len(src)].view(-1))
    arr = (_capi.Image * n_img)(*[_capi.Image(W, H, 3, f.data_ptr(), W * 3) for f in frames])
    cap = 256
    faces = (_capi.Face * (n_img * cap))()
    n = (ctypes.c_int * n_img)()
    assert _capi.lib().ccnn_detect_device_batch(d._h, arr, n_img, faces, cap, n, None) >= 0, _capi.last_error()
    got = [[(f.x, f.y, f.width, f.height, f.score) for f in faces[i * cap: i * cap + n[i]]] for i in range(n_img)]
    assert got == [want[i % len(want)] for i in range(n_img)]
    d.Clear()
