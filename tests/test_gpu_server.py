"""Serving loop (include/ccnn_server.h) on the GPU: frames of mixed resolutions in flight
together give exactly the result each gives alone on a fresh handle sized for it; admission by
the HBM budget (eviction, refusal); a bounded request queue."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402
from oracle import ref  # noqa: E402


def _params():
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = 1920, 1080
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    p.detect_mode = 1
    return p


def _alone(img):
    """ccnn_detect on a fresh handle whose max_image_size is the frame's size."""
    p = _params()
    p.max_image_width, p.max_image_height = img.shape[1], img.shape[0]
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    faces = d.Detect(img)
    d.Clear()
    return faces


@pytest.fixture(scope="module")
def mix():
    frames = []
    for i, (w, h, nf) in enumerate([(640, 480, 5), (1280, 720, 10), (1920, 1080, 20), (960, 540, 8)]):
        img = ccnn.synth_frame(w, h, 500 + i, nf, 30, min(300, h // 2))[0]
        pf = ccnn.pinned_frame(img.shape)
        pf[...] = img
        frames.append(pf)
    gray = ccnn.synth_frame(640, 480, 777, 5, 40, 200, channels=1)[0]
    frames.append(gray)
    return frames


def test_mixed_resolutions_match_alone(mix):
    alone = [_alone(f) for f in mix]
    assert sum(len(a) for a in alone) > 0
    srv = ccnn.FaceServer(_params(), slots_per_class=3)
    order = [i for _ in range(4) for i in (2, 0, 4, 1, 3, 2, 1)]
    tickets = [(i, srv.submit(mix[i])) for i in order]
    assert all(t is not None for _, t in tickets)
    for i, t in tickets:
        faces, lat = srv.wait(t)
        assert faces == alone[i], f"frame {i} differs in the mix"
        assert lat > 0.0
    st = srv.stats()
    assert st["completed"] == len(order) and st["failed"] == 0 and st["queued"] == 0 and st["in_flight"] == 0
    assert st["classes"] == len(mix)
    srv.close()


def test_gated_server_matches_gated_detector(mix):
    """With the learned gate on, every frame of a mixed stream gives what a gated detector sized for
    it gives alone; the gate cannot be changed once frames were submitted."""
    from compactcnncascade_b200 import gate
    if not __import__("os").path.exists(gate.WEIGHTS_1080P):
        pytest.skip("no trained gate weights in the package")
    w, thr = gate.load(), 0.2
    alone = []
    for f in mix:
        p = _params()
        p.max_image_width, p.max_image_height = f.shape[1], f.shape[0]
        d = ccnn.FaceDetector()
        assert d.Init(p) == 0
        d.setGate(w, thr, 0.25)
        alone.append(d.Detect(f))
        d.Clear()
    srv = ccnn.FaceServer(_params(), slots_per_class=2)
    srv.set_gate(w, thr, 0.25)
    tickets = [(i, srv.submit(mix[i])) for i in (2, 0, 1, 4, 3, 2, 0)]
    for i, t in tickets:
        assert srv.wait(t)[0] == alone[i], f"frame {i} differs in the mix"
    with pytest.raises(ccnn.CCNNError):
        srv.set_gate(w, thr, 0.25)
    srv.close()


def test_server_frame_matches_reference(mix):
    """A served frame against the reference's own cascade (strict IEEE build of its sources)."""
    if not ref.available():
        pytest.skip("reference build oracle/_ref/libccnn_ref.so not present")
    srv = ccnn.FaceServer(_params())
    t = srv.submit(mix[0])
    faces, _ = srv.wait(t)
    img = np.ascontiguousarray(mix[0])
    p = ref.params(max_w=img.shape[1], max_h=img.shape[0])
    assert faces == ref.face_detect(img, p)
    srv.close()


def test_poll_and_ticket_rules(mix):
    srv = ccnn.FaceServer(_params())
    t = srv.submit(mix[1])
    res = None
    for _ in range(200000):
        res = srv.poll(t)
        if res is not None:
            break
    assert res is not None and res[0] == _alone(mix[1])
    with pytest.raises(ccnn.CCNNError):
        srv.wait(t)  # a result is taken once
    with pytest.raises(ccnn.CCNNError):
        srv.wait(123456789)
    srv.close()


def test_budget_evicts_idle_classes(mix):
    # room for one 1080p class with one slot: other classes evict it when idle
    probe = ccnn.FaceServer(_params(), slots_per_class=1)
    probe.wait(probe.submit(mix[2]))
    one = probe.stats()["hbm_bytes"]
    probe.close()
    srv = ccnn.FaceServer(_params(), hbm_budget_bytes=int(one * 1.05), slots_per_class=1)
    alone = {i: _alone(mix[i]) for i in (0, 1, 2)}
    for i in (2, 0, 1, 2, 0):
        faces, _ = srv.wait(srv.submit(mix[i]))
        assert faces == alone[i]
        assert srv.stats()["hbm_bytes"] <= int(one * 1.05)
    srv.close()


def test_budget_refuses_oversize_class(mix):
    srv = ccnn.FaceServer(_params(), hbm_budget_bytes=1 << 20)
    t = srv.submit(mix[2])
    with pytest.raises(ccnn.CCNNError) as e:
        srv.wait(t)
    assert e.value.status == _capi.ERR_OOM
    assert srv.stats()["failed"] == 1
    srv.close()


def test_queue_bound(mix):
    srv = ccnn.FaceServer(_params(), slots_per_class=1, max_queue=2)
    tickets, busy = [], 0
    for _ in range(64):
        t = srv.submit(mix[2])
        if t is None:
            busy += 1
        else:
            tickets.append(t)
    assert busy > 0
    ref = _alone(mix[2])
    for t in tickets:
        assert srv.wait(t)[0] == ref
    srv.close()
