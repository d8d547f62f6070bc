"""Legacy model family (format 1.0, cnn4face{1,2,3}_new.bin), host side: the reader's view of the
three shipped files and its refusals."""
import ctypes
import os

import pytest

from compactcnncascade_b200 import _capi

MODELS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "compactcnncascade_b200", "models")


def _info(name):
    info = (ctypes.c_int * 10)()
    st = _capi.lib().ccnn_legacy_model_info(os.path.join(MODELS, name).encode(), info, 10)
    return st, list(info)


@pytest.mark.parametrize("name,want", [
    # max_pool, min w, min h, maps L1/L2/L3, L3 kernel w x h, fully connected, hidden neurons
    ("cnn4face1_new.bin", [1, 27, 31, 4, 8, 16, 5, 6, 0, 32]),
    ("cnn4face2_new.bin", [0, 36, 40, 6, 12, 24, 7, 8, 0, 48]),
    ("cnn4face3_new.bin", [0, 36, 40, 6, 12, 24, 7, 8, 1, 48]),
])
def test_reader_shapes(name, want):
    st, info = _info(name)
    assert st == _capi.OK and info == want


def test_reader_refuses_other_files(tmp_path):
    st, _ = _info("cnn4face1_cntk.bin")
    assert st == _capi.ERR_MODEL and "format 1.0" in _capi.last_error()
    blob = open(os.path.join(MODELS, "cnn4face2_new.bin"), "rb").read()
    cut = tmp_path / "cut.bin"
    cut.write_bytes(blob[: len(blob) - 100])
    info = (ctypes.c_int * 10)()
    assert _capi.lib().ccnn_legacy_model_info(str(cut).encode(), info, 10) == _capi.ERR_MODEL
    assert "truncated" in _capi.last_error()
    assert _capi.lib().ccnn_legacy_model_info(b"/nonexistent/model.bin", info, 10) == _capi.ERR_MODEL


# ---- the float32 restatement (oracle/legacy_ref.py) against the reference's legacy build ----

import numpy as np  # noqa: E402

from oracle import legacy_ref, ref  # noqa: E402


@pytest.mark.skipif(not ref.legacy_available(), reason="legacy reference build (oracle/_ref) not available")
@pytest.mark.parametrize("name,shape,seed", [("cnn4face1_new.bin", (150, 200), 1), ("cnn4face1_new.bin", (31, 27), 2),
                                             ("cnn4face2_new.bin", (51, 47), 3), ("cnn4face2_new.bin", (64, 80), 4),
                                             ("cnn4face3_new.bin", (51, 47), 5), ("cnn4face3_new.bin", (70, 90), 6)])
def test_restatement_matches_reference(name, shape, seed):
    img = np.random.default_rng(seed).uniform(0, 255, shape).astype(np.float32)
    path = os.path.join(MODELS, name)
    got = legacy_ref.forward(legacy_ref.load(path), img)
    want = ref.legacy_net_forward_isolated(path, img)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), float(np.abs(got - want).max())
