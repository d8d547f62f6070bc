"""Host-side logic of the package that needs no GPU: the C ABI surface, the device sort's order,
the scale planner, parameter defaults and error behaviour."""
import ctypes
import os
import re
import shutil

import numpy as np
import pytest

import compactcnncascade_b200 as ccnn
from compactcnncascade_b200 import _capi
from oracle import oracle as orc
from tests.goldens import case, case_names, ccnn_params, fbits, golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"CCNN_API\s+[\w\s\*]+?\b(ccnn_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert sorted(set(_capi.EXPORTED)) == names
    assert b"sm_100a" in L.ccnn_version()


def test_cnn_detector_defaults_are_the_reference_defaults():
    p, ap = _capi.CnnParam(), _capi.CnnAdvancedParam()
    _capi.lib().ccnn_cnn_default_params(p, ap)
    # CNNDetector::Param (cnn_detector_v3.h:114-123)
    assert (p.pipeline, p.max_image_width, p.max_image_height) == (0, 1280, 720)
    assert (p.min_obj_width, p.min_obj_height, p.max_obj_width, p.max_obj_height) == (48, 48, 0, 0)
    assert abs(p.scale_factor - 1.2) < 1e-6 and p.min_neighbors == 2 and p.num_threads == 0
    # CNNDetector::AdvancedParam (cnn_detector_v3.h:124-175)
    assert (ap.detect_mode, ap.detect_precision, ap.packet_detection, ap.gray_image_only, ap.facial_analysis) == (1, 2, 0, 0, 0)
    assert (ap.equalize, ap.reflection, ap.type_check) == (1, 1, 1)
    assert (ap.treshold_1, ap.treshold_2, ap.treshold_3) == (0.0, 0.0, 0.0)
    assert (ap.adapt_min_neighbors, ap.double_check, ap.drop_detect, ap.min_num_detect) == (0, 1, 1, 1)
    assert (ap.device_info, ap.cuda_device_id, ap.cl_platform_id, ap.cl_device_id) == (0, 0, -1, -1)
    assert (ap.concurrent_kernels, ap.num_cnn_copy, ap.blur, ap.img_resize, ap.uniform_noise, ap.merger_detect) == (3, 1, 0, 0, 0, 1)
    assert list(ap.index_output) == [1, 0, 0, -1]


def test_default_params_are_the_reference_defaults():
    p = ccnn.default_params()
    # FaceDetector::Param (CompactCNNLibAPI_v2.h:97-161)
    assert (p.max_image_width, p.max_image_height) == (1920, 1080)
    assert (p.min_face_height, p.max_face_height, p.min_neighbors) == (80, 0, 2)
    assert abs(p.scale_factor - 1.15) < 1e-7 and p.detect_precision == 3
    assert list(p.treshold) == [np.float32(-1.5), np.float32(-1.25), np.float32(-1.0)]
    assert (p.drop_detect, p.equalize, p.reflection, p.pipeline, p.detect_mode, p.num_threads) == (1, 1, 1, 1, 2, 2)
    assert list(p.index_output) == [1, 0, 0]
    assert (p.cuda_device_id, p.cl_platform_id, p.cl_device_id, p.facial_analysis) == (0, -1, -1, 0)


def _perm(keys):
    keys = np.ascontiguousarray(keys, np.float32)
    perm = np.empty(len(keys), np.int32)
    assert _capi.lib().ccnn_sort_permutation(keys.ctypes.data, len(keys), perm.ctypes.data) == 0
    return perm


def test_device_sort_order_is_std_sort_golden():
    for rec in golden()["sort"]:
        keys = np.array([np.frombuffer(bytes.fromhex(k), "<f4")[0] for k in rec["keys"]], np.float32)
        assert _perm(keys).tolist() == rec["perm"]


def test_device_sort_order_is_std_sort_random():
    rng = np.random.default_rng(3)
    for trial in range(3000):
        n = int(rng.integers(0, 400))
        kind = trial % 4
        if kind == 0:
            keys = rng.integers(0, 3, n).astype(np.float32)
        elif kind == 1:
            keys = np.sort(rng.integers(0, 13, n))[::-1].astype(np.float32)  # the detector's case: sorted runs
        elif kind == 2:
            keys = rng.random(n).astype(np.float32)
        else:
            keys = np.repeat(rng.random(max(1, n // 20)).astype(np.float32), 20)[:n]
        assert _perm(keys).tolist() == orc.sort_perm(keys).tolist(), (trial, n)


@pytest.mark.parametrize("name", case_names())
def test_plan_levels_match_reference(name):
    c = case(name)
    p = ccnn_params(c)
    buf = (_capi.LevelInfo * 1024)()
    n = ctypes.c_int()
    f = c["frame"]
    assert _capi.lib().ccnn_plan_levels(ctypes.byref(p), f["w"], f["h"], f["ch"], buf, 1024, ctypes.byref(n)) == 0
    got = [[b.width, b.height, fbits(b.scale)] for b in buf[: n.value]]
    assert got == c["levels"]
    assert [[b.resp_height, b.resp_width] for b in buf[: n.value]] == c["resp_shapes"]


def test_plan_levels_large_pyramid():
    """4800x2400, min face 20, scale 1.05: the reference's 86 levels of the batched-pyramid workload."""
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = 4800, 2400
    p.min_face_height, p.max_face_height, p.scale_factor = 20, 0, 1.05
    buf = (_capi.LevelInfo * 1024)()
    n = ctypes.c_int()
    assert _capi.lib().ccnn_plan_levels(ctypes.byref(p), 4800, 2400, 3, buf, 1024, ctypes.byref(n)) == 0
    assert n.value == 86
    assert (buf[0].width, buf[0].height) == (6480, 3240)  # scale min(3, 27/20) = 1.35: upsampled


def test_invalid_configuration_is_reported():
    p = ccnn.default_params()
    p.min_face_height, p.max_face_height = 40, 20  # max face below min face: empty scale list
    p.max_face_height = 10
    n = ctypes.c_int()
    st = _capi.lib().ccnn_plan_levels(ctypes.byref(p), 640, 480, 3, None, 0, ctypes.byref(n))
    assert st in (0, _capi.ERR_CONFIG)


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda_available(), reason="checks the behaviour without a GPU")
def test_create_without_gpu_fails_loudly():
    p = ccnn.default_params()
    h = ctypes.c_void_p()
    st = _capi.lib().ccnn_create(ctypes.byref(p), None, ctypes.byref(h))
    assert st == _capi.ERR_CUDA
    assert "no CUDA device" in _capi.last_error()
    d = ccnn.FaceDetector()
    assert d.Init(p) == -1 and d.isEmpty()


def _create(paths):
    p = ccnn.default_params()
    arr = (ctypes.c_char_p * 3)(*[x.encode() if x else None for x in paths])
    h = ctypes.c_void_p()
    st = _capi.lib().ccnn_create(ctypes.byref(p), arr, ctypes.byref(h))
    if st == 0:
        _capi.lib().ccnn_destroy(h)
    return st, _capi.last_error()


def test_model_file_errors(tmp_path):
    models = os.path.join(ROOT, "compactcnncascade_b200", "models")
    m1 = os.path.join(models, "cnn4face1_cntk.bin")
    st, msg = _create([str(tmp_path / "missing.bin"), None, None])
    assert st == _capi.ERR_MODEL and "not found" in msg
    data = open(m1, "rb").read()
    trunc = tmp_path / "trunc.bin"
    trunc.write_bytes(data[: len(data) // 2])
    st, msg = _create([str(trunc), None, None])
    assert st == _capi.ERR_MODEL and "truncated" in msg
    oldver = tmp_path / "v09.bin"
    oldver.write_bytes(np.float32(0.9).tobytes() + data[4:])
    st, msg = _create([str(oldver), None, None])
    assert st == _capi.ERR_MODEL and "version" in msg
    # a stage-2 net where the stage-1 net belongs: shape mismatch
    st, msg = _create([os.path.join(models, "cnn4face2_cntk.bin"), None, None])
    assert st == _capi.ERR_MODEL and "prototype" in msg


def test_bundled_models_load_then_need_a_gpu():
    st, msg = _create([None, None, None])
    if _cuda_available():
        assert st == 0
    else:
        assert st == _capi.ERR_CUDA
