"""Device frames are read where they are when aligned (the graph's gray node is pointed at them) and
copied otherwise; either way, and mixed with host frames on the same handle, the faces are the
ones the host path gives."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402


def test_in_place_and_copied_device_frames_agree():
    w, h = 1280, 720
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    imgs = [ccnn.synth_frame(w, h, 300 + i, 10, 30, 300)[0] for i in range(3)]
    want = [d.Detect(im) for im in imgs]
    assert sum(len(f) for f in want) > 0
    for k, im in enumerate(imgs):
        row = w * 3
        aligned = torch.from_numpy(im).cuda()  # 64-byte aligned, step 3840: read in place
        assert d.DetectDevice(aligned.data_ptr(), w, h, 3, row) == want[k]
        big = torch.zeros(h * (row + 64) + 64, dtype=torch.uint8, device="cuda")
        shifted = big[1:1 + h * row].view(h, row)  # misaligned base: copied
        shifted.copy_(torch.from_numpy(im.reshape(h, row)))
        assert d.DetectDevice(shifted.data_ptr(), w, h, 3, row) == want[k]
        padded = big[: h * (row + 8)].view(h, row + 8)  # step not a multiple of 64: copied
        padded[:, :row].copy_(torch.from_numpy(im.reshape(h, row)))
        assert d.DetectDevice(padded.data_ptr(), w, h, 3, row + 8) == want[k]
        assert d.DetectDevice(aligned.data_ptr(), w, h, 3, row) == want[k]
        assert d.Detect(im) == want[k]  # the node points back at the staging buffer
    # an in-place frame cannot be re-run later by the profiler; a host frame can
    aligned = torch.from_numpy(imgs[0]).cuda()
    d.DetectDevice(aligned.data_ptr(), w, h, 3, w * 3)
    ms = (ctypes.c_float * 8)()
    assert _capi.lib().ccnn_profile_last_frame(d._h, 2, ms, 8) == _capi.ERR_UNSUPPORTED
    d.Detect(imgs[0])
    assert _capi.lib().ccnn_profile_last_frame(d._h, 2, ms, 8) == _capi.OK
    batch = [torch.from_numpy(im).cuda() for im in imgs]
    arr = (_capi.Image * 3)(*[_capi.Image(w, h, 3, t.data_ptr(), w * 3) for t in batch])
    faces = (_capi.Face * (3 * 256))()
    n = (ctypes.c_int * 3)()
    assert _capi.lib().ccnn_detect_device_batch(d._h, arr, 3, faces, 256, n, None) >= 0
    got = [[(f.x, f.y, f.width, f.height, f.score) for f in faces[i * 256: i * 256 + n[i]]] for i in range(3)]
    assert got == want
