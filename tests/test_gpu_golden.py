"""The CUDA path against golden fixtures generated from the reference's own code: every stage
bit-exact (gray, pyramid levels, stage-1 response maps, candidate indices and scores, raw
detections in the reference's order, final boxes) for every recorded configuration."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402
from tests.goldens import case, case_names, ccnn_params, fbits, frame, golden, primitive_inputs, sha  # noqa: E402

RESP_RTOL = 1e-4  # stated bar for fp32 response maps; they are also checked bit-exact below


@pytest.mark.parametrize("name", case_names())
def test_detector_matches_reference_golden(name):
    c = case(name)
    img = frame(c)
    assert sha(img) == c["frame_sha256"]
    det = ccnn.FaceDetector()
    assert det.Init(ccnn_params(c)) == 0, _capi.last_error()
    faces = det.Detect(img)
    assert [[f[0], f[1], f[2], f[3], fbits(f[4])] for f in faces] == c["final"]
    if not c["levels"]:
        det.Clear()
        return
    assert [[l[0], l[1], fbits(l[2])] for l in det.levels()] == c["levels"]
    assert sha(det.getGrayImage32F()) == c["gray_sha256"]
    for i, h in enumerate(c["resp_sha256"]):
        r = det.response_map(i)
        assert list(r.shape) == c["resp_shapes"][i]
        assert sha(r) == h, (name, i)
    got_c = [[a[0], a[1], a[2], fbits(a[3])] for a in det.candidates()]
    assert got_c == c["candidates"]
    got_raw = [[d[0], d[1], d[2], d[3], fbits(d[4]), fbits(d[5]), d[6], d[7]] for d in det.raw_detections()]
    assert got_raw == c["raw"]
    det.Clear()


def test_primitives_match_reference_golden():
    g = golden()["primitives"]
    grays, src, nets = primitive_inputs()
    L = _capi.lib()
    for img, rec in zip(grays, g["gray"]):
        h, w = img.shape[:2]
        ch = rec["ch"]
        pitch = (w * ch + 63) // 64 * 64
        d = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
        d[:, : w * ch] = torch.from_numpy(img.reshape(h, w * ch)).cuda()
        dp = (w + 15) // 16 * 16
        out = torch.zeros((h, dp), dtype=torch.float32, device="cuda")
        assert L.ccnn_gray_u8_to_f32(d.data_ptr(), w, h, ch, pitch, out.data_ptr(), dp * 4, None) == 0
        assert sha(out[:, :w].cpu().numpy()) == rec["out_sha256"], ch
    ds = torch.from_numpy(src).cuda()
    for rec in g["resize"]:
        out = torch.zeros((rec["dh"], rec["dw"]), dtype=torch.float32, device="cuda")
        assert L.ccnn_resize_f32(ds.data_ptr(), src.shape[1], src.shape[0], src.shape[1] * 4, out.data_ptr(), rec["dw"], rec["dh"],
                                 rec["dw"] * 4, rec["type"], None) == 0
        assert sha(out.cpu().numpy()) == rec["out_sha256"], rec
    p = ccnn.default_params()
    p.min_face_height = 40
    det = ccnn.FaceDetector()
    assert det.Init(p) == 0
    for (st, idx, img), rec in zip(nets, g["net"]):
        if st != 1 or idx != 1:
            continue  # the stage-1 entry point runs the handle's stage-1 net (output neuron 1)
        h, w = img.shape
        di = torch.from_numpy(img).cuda()
        resp = torch.zeros(w * h, dtype=torch.float32, device="cuda")
        rw, rh = ctypes.c_int(), ctypes.c_int()
        assert L.ccnn_stage1_forward(det._h, di.data_ptr(), w, h, w * 4, resp.data_ptr(), w * h, ctypes.byref(rw),
                                     ctypes.byref(rh), None) == 0
        r = resp[: rw.value * rh.value].cpu().numpy().reshape(rh.value, rw.value)
        assert list(r.shape) == rec["out_shape"] and sha(r) == rec["out_sha256"]
    det.Clear()
