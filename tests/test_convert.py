"""CNTK dump -> binary model conversion (FaceDetector::CNTKDump2Binary): byte-identical to the
reference's own converter on synthetic dumps of the three cascade shapes and the landmark shape,
and the converted files load in the detector's model reader."""
import ctypes
import os

import pytest

from compactcnncascade_b200 import _capi
from tests.cntk_dump import make_dump

SHAPES = {
    "stage1": dict(win=(23, 27), maps=(4, 8, 16), kernels=((4, 4), (3, 3), (4, 5)), hs=4, conn=4, n_out=3),
    "stage2": dict(win=(36, 40), maps=(6, 12, 24), kernels=((4, 4), (3, 3), (7, 8)), hs=4, conn=4, n_out=3),
    "stage3": dict(win=(36, 40), maps=(6, 12, 24), kernels=((4, 4), (3, 3), (7, 8)), hs=2, conn=8, n_out=3),
    "landmarks": dict(win=(49, 51), maps=(24, 48, 96), kernels=((4, 4), (3, 3), (10, 11)), hs=384, conn=96, n_out=13, full=True),
}


@pytest.mark.parametrize("name", sorted(SHAPES))
@pytest.mark.parametrize("seed", [1, 2])
def test_conversion_matches_reference(ref, tmp_path, name, seed):
    dump = tmp_path / f"{name}.txt"
    dump.write_text(make_dump(seed, **SHAPES[name]))
    ours, theirs = str(tmp_path / "ours.bin"), str(tmp_path / "theirs.bin")
    st = _capi.lib().ccnn_cntk_dump_to_binary(ours.encode(), str(dump).encode())
    assert st == 0, _capi.last_error()
    ref.cntk_dump2binary(theirs, str(dump))
    a, b = open(ours, "rb").read(), open(theirs, "rb").read()
    assert len(a) > 1000 and a == b


def test_extension_and_errors(tmp_path):
    dump = tmp_path / "d.txt"
    dump.write_text(make_dump(3, **SHAPES["stage1"]))
    L = _capi.lib()
    assert L.ccnn_cntk_dump_to_binary(str(tmp_path / "noext").encode(), str(dump).encode()) == 0
    assert os.path.exists(tmp_path / "noext.bin")
    assert L.ccnn_cntk_dump_to_binary(str(tmp_path / "x.bin").encode(), str(tmp_path / "missing.txt").encode()) == _capi.ERR_MODEL
    assert b"not found" in _capi.lib().ccnn_last_error()


@pytest.mark.gpu
def test_converted_models_load_in_detector(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import compactcnncascade_b200 as ccnn
    paths = []
    for i, name in enumerate(("stage1", "stage2", "stage3")):
        dump = tmp_path / f"{name}.txt"
        dump.write_text(make_dump(10 + i, **SHAPES[name]))
        out = str(tmp_path / f"{name}.bin")
        assert _capi.lib().ccnn_cntk_dump_to_binary(out.encode(), str(dump).encode()) == 0
        paths.append(out)
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = 640, 480
    d = ccnn.FaceDetector()
    assert d.Init(p, models=paths) == 0
    img = ccnn.synth_frame(640, 480, 5, 5, 40, 200)[0]
    assert isinstance(d.Detect(img), list)
