"""The oracle (CPU restatement, oracle/ccnn_oracle.cpp) pinned against golden fixtures generated
from the reference's own code, and against the reference build itself when it is present."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.goldens import case, case_names, fbits, frame, golden, oracle_params, primitive_inputs, sha


def test_generator_is_deterministic():
    for c in golden()["cases"]:
        assert sha(frame(c)) == c["frame_sha256"], c["name"]


@pytest.mark.parametrize("name", case_names())
def test_oracle_matches_reference_golden(name):
    c = case(name)
    if c["frame"]["w"] * c["frame"]["h"] > 1_000_000:
        pytest.skip("full-HD cases are covered on the GPU path (oracle takes seconds)")
    out = orc.detect(frame(c), oracle_params(c))
    assert [[l[0], l[1], fbits(l[2])] for l in out["levels"]] == c["levels"]
    if c["levels"]:
        assert sha(out["gray"]) == c["gray_sha256"]
    assert [sha(r) for r in out["resp"]] == c["resp_sha256"]
    assert [[a[0], a[1], a[2], fbits(a[3])] for a in out["candidates"]] == c["candidates"]
    assert [[d[0], d[1], d[2], d[3], fbits(d[4]), fbits(d[5]), d[6], d[7]] for d in out["raw"]] == c["raw"]
    assert [[f[0], f[1], f[2], f[3], fbits(f[4])] for f in out["final"]] == c["final"]


def test_oracle_primitives_match_golden():
    g = golden()["primitives"]
    grays, src, nets = primitive_inputs()
    for img, rec in zip(grays, g["gray"]):
        assert sha(img) == rec["input_sha256"]
        assert sha(orc.gray(img)) == rec["out_sha256"], rec["ch"]
    assert sha(src) == g["resize_src_sha256"]
    for rec in g["resize"]:
        assert sha(orc.resize_f32(src, rec["dw"], rec["dh"], rec["type"])) == rec["out_sha256"], rec
    for (st, idx, img), rec in zip(nets, g["net"]):
        assert sha(img) == rec["input_sha256"]
        r = orc.net_forward(st, img, idx)
        assert list(r.shape) == rec["out_shape"] and sha(r) == rec["out_sha256"], rec


def test_oracle_sort_is_std_sort():
    for rec in golden()["sort"]:
        keys = np.array([np.frombuffer(bytes.fromhex(k), "<f4")[0] for k in rec["keys"]], np.float32)
        assert orc.sort_perm(keys).tolist() == rec["perm"]


def test_oracle_vs_reference_live(ref):
    """Random shapes and values, straight against the reference build (when present)."""
    rng = np.random.default_rng(7)
    for _ in range(20):
        w, h = int(rng.integers(23, 160)), int(rng.integers(27, 160))
        img = (rng.random((h, w), dtype=np.float32) * 255).astype(np.float32)
        a, b = orc.net_forward(1, img, 1), ref.net_forward(1, img, 1)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        dw, dh = int(rng.integers(2, 300)), int(rng.integers(2, 300))
        for t in (0, 1):
            assert np.array_equal(orc.resize_f32(img, dw, dh, t).view(np.uint32), ref.resize_f32(img, dw, dh, t).view(np.uint32))
    for st in (2, 3):
        img = (rng.random((51, 47), dtype=np.float32) * 255).astype(np.float32)
        assert np.array_equal(orc.net_forward(st, img, 0).view(np.uint32), ref.net_forward(st, img, 0).view(np.uint32))
