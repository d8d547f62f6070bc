"""The batched form (schedule knob batch_frames): groups of frames run as one graph each, with the
pyramid and stage 1 of every level of every frame of a group in one persistent launch fed by a
device work queue. Every frame's faces must equal the per-frame path's (itself bit-exact against the
reference): host and device frames, frames read in place and copied, leftover frames after the last
full group, the learned gate, pyramids deeper than one launch's level table, and the largest
batched-pyramid frames."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi, autotune  # noqa: E402


def _params(w, h, min_face=40, max_face=240, sf=1.15):
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = min_face, max_face, sf
    p.detect_mode = 1
    return p


def _device_batch(det, frames, w, h, steps=None, cap=512):
    L = _capi.lib()
    n = len(frames)
    arr = (_capi.Image * n)(*[_capi.Image(w, h, 3, t.data_ptr(), steps[i] if steps else w * 3) for i, t in enumerate(frames)])
    faces = (_capi.Face * (n * cap))()
    nf = (ctypes.c_int * n)()
    st = L.ccnn_detect_device_batch(det._h, arr, n, faces, cap, nf, None)
    assert st >= 0, _capi.last_error()
    return [[(f.x, f.y, f.width, f.height, f.score) for f in faces[i * cap: i * cap + nf[i]]] for i in range(n)]


@pytest.mark.parametrize("batch,slots,bpsm", [(2, 4, 3), (4, 8, 4), (8, 8, 3), (8, 16, 4), (4, 8, 1)])
def test_batched_host_frames_equal_per_frame(batch, slots, bpsm):
    w, h = 1280, 720
    imgs = [ccnn.synth_frame(w, h, 5000 + i, 10, 30, 300)[0] for i in range(11)]  # leftovers after the last full group
    d = ccnn.FaceDetector()
    assert d.Init(_params(w, h)) == 0
    want = [d.Detect(im) for im in imgs]
    assert sum(len(f) for f in want) > 0
    autotune.set_schedule(d, {"frame_slots": slots, "batch_frames": batch, "batch_blocks_per_sm": bpsm})
    assert autotune.get_schedule(d)["batch_frames"] == batch
    assert d.DetectBatch(imgs) == want
    assert d.DetectBatch(imgs[::-1]) == want[::-1]  # the contexts' graphs are replayed
    assert [d.Detect(im) for im in imgs[:3]] == want[:3]  # single frames still run on the slots
    d.Clear()


def test_batched_device_frames_in_place_and_copied():
    w, h = 1920, 1080
    imgs = [ccnn.synth_frame(w, h, 6000 + i, 20, 30, 300)[0] for i in range(8)]
    d = ccnn.FaceDetector()
    assert d.Init(_params(w, h)) == 0
    want = [d.Detect(im) for im in imgs]
    autotune.set_schedule(d, {"frame_slots": 8, "batch_frames": 4})
    frames, steps = [], []
    for i, im in enumerate(imgs):
        if i % 3 == 1:  # misaligned base: packed into the slot
            big = torch.zeros(h * w * 3 + 64, dtype=torch.uint8, device="cuda")
            t = big[1:1 + h * w * 3]
            t.copy_(torch.from_numpy(im).view(-1))
            frames.append(t)
            steps.append(w * 3)
        elif i % 3 == 2:  # pitch not a multiple of 64: packed
            t = torch.zeros((h, w * 3 + 8), dtype=torch.uint8, device="cuda")
            t[:, : w * 3] = torch.from_numpy(im.reshape(h, w * 3))
            frames.append(t)
            steps.append(w * 3 + 8)
        else:  # read in place
            frames.append(torch.from_numpy(im).cuda())
            steps.append(w * 3)
    assert _device_batch(d, frames, w, h, steps) == want
    d.Clear()


def test_batched_gated_equals_per_frame_gated():
    from compactcnncascade_b200 import gate
    w, h = 1920, 1080
    imgs = [ccnn.synth_frame(w, h, 7000 + i, 20, 30, 300)[0] for i in range(8)]
    d = ccnn.FaceDetector()
    assert d.Init(_params(w, h)) == 0
    d.setGate(gate.load(), 0.1, 0.25)
    want = [d.Detect(im) for im in imgs]
    autotune.set_schedule(d, {"frame_slots": 8, "batch_frames": 4})
    d.setGate(gate.load(), 0.1, 0.25)
    assert d.DetectBatch(imgs) == want
    d.Clear()


def test_batched_many_levels_equal_per_frame():
    w, h = 1920, 1080
    imgs = [ccnn.synth_frame(w, h, 4242 + i, 30, 20, 600)[0] for i in range(4)]
    d = ccnn.FaceDetector()
    assert d.Init(_params(w, h, min_face=20, max_face=0, sf=1.05)) == 0
    want = [d.Detect(im) for im in imgs]
    assert len(d.levels()) > 32
    autotune.set_schedule(d, {"frame_slots": 4, "batch_frames": 2})
    assert d.DetectBatch(imgs) == want
    d.Clear()


def test_batched_largest_frames_equal_per_frame():
    w, h = 4800, 2400
    frames = []
    for i in range(2):
        t = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda")
        ccnn.synth_frame_device(t.data_ptr(), w, h, 700_000 + 1000 * w + i, 60, 20, 600)
        frames.append(t)
    d = ccnn.FaceDetector()
    assert d.Init(_params(w, h, min_face=20, max_face=0, sf=1.05)) == 0
    want = [d.DetectDevice(t.data_ptr(), w, h, 3, w * 3) for t in frames]
    assert len(d.levels()) == 86 and sum(len(f) for f in want) > 0
    autotune.set_schedule(d, {"frame_slots": 2, "batch_frames": 2})
    assert _device_batch(d, frames, w, h) == want
    d.Clear()


def test_single_launch_stage1_equals_per_frame():
    """batch_frames = 1 (and packet mode of the CNNDetector API): every frame keeps its own graph, with
    the pyramid and stage 1 of all its levels in one persistent launch."""
    from compactcnncascade_b200 import gate
    for (w, h, mn, mx, sf, nf, lo, hi) in [(1280, 720, 40, 240, 1.15, 10, 30, 300), (1920, 1080, 20, 0, 1.05, 30, 20, 600)]:
        imgs = [ccnn.synth_frame(w, h, 8000 + i, nf, lo, hi)[0] for i in range(3)]
        d = ccnn.FaceDetector()
        assert d.Init(_params(w, h, min_face=mn, max_face=mx, sf=sf)) == 0
        want = [d.Detect(im) for im in imgs]
        autotune.set_schedule(d, {"batch_frames": 1})
        assert [d.Detect(im) for im in imgs] == want
        assert d.DetectBatch(imgs) == want
        if sf == 1.15:
            d.setGate(gate.load(), 0.1, 0.25)
            gated = [d.Detect(im) for im in imgs]
            autotune.set_schedule(d, {"batch_frames": 0})
            d.setGate(gate.load(), 0.1, 0.25)
            assert [d.Detect(im) for im in imgs] == gated
        d.Clear()
