"""The header-only C++ facade (include/CompactCNNLib.h) compiles against the C ABI like the
reference's demo code and behaves like the Python API."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "compactcnncascade_b200")


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("facade") / "facade_example")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "facade_example.cpp"), os.path.join(PKG, "csrc", "synth_frame.c"),
                           "-x", "none", "-L", PKG, "-lccnn", f"-Wl,-rpath,{PKG}", "-o", exe])
    return exe


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_facade_builds_and_fails_cleanly_without_gpu(example):
    if _cuda():
        pytest.skip("covered by the GPU variant")
    out = subprocess.run([example], capture_output=True, text=True, check=True).stdout
    assert out.strip() == "init -1"


@pytest.mark.gpu
def test_facade_detects_like_python_api(example):
    import compactcnncascade_b200 as ccnn
    out = subprocess.run([example, "640", "480", "1"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[0] == "init 0"
    faces = [tuple(float(v) for v in l.split()) for l in out[1:-1]]
    img, _ = ccnn.synth_frame(640, 480, 1, 5, 40, 200)
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height, p.min_face_height, p.max_face_height, p.detect_mode = 640, 480, 40, 240, 1
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    exp = d.Detect(img)
    assert [f[:4] for f in faces] == [tuple(float(v) for v in e[:4]) for e in exp]
    assert out[-1] == "gray 0 1 640x480"
