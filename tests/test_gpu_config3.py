"""The batched-pyramid workload's frames against the reference's own cascade (the strict IEEE build
of the unmodified sources, oracle/_ref/libccnn_ref.so): 3840x2160 and 4800x2400 seeded frames with 60
face patches of 20-600 px, scale factor 1.05, min face 20, no max face. The largest level is an
upsampled 1.35x copy of the frame and the pyramid has 83 / 86 levels of uneven sizes, more than one
launch's level table holds. Level sizes and scales, every response map (bit for bit), the candidate
indices and scores, the raw detections in the reference's order and the final boxes must be identical.

The reference takes 15-25 s per frame on one core; both frames run in parallel spawned processes."""
import multiprocessing as mp

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import _capi  # noqa: E402
from oracle import ref  # noqa: E402
from tests.goldens import fbits, sha  # noqa: E402

if not ref.available():
    pytest.skip("reference build oracle/_ref/libccnn_ref.so not present", allow_module_level=True)

SIZES = [(3840, 2160), (4800, 2400)]
N_PATCHES, MIN_PATCH, MAX_PATCH = 60, 20, 600
RESP_RTOL = 1e-4  # stated bar for fp32 response maps; they are also checked bit-exact


def _seed(w):
    return 700_000 + 1000 * w  # the seeds of the benchmark's batched-pyramid frames


def _frame(w, h):
    return ccnn.synth_frame(w, h, _seed(w), N_PATCHES, MIN_PATCH, MAX_PATCH)[0]


def _reference(size):
    """The reference's cascade on one frame (run in a spawned worker): levels, response-map hashes,
    candidates in its visiting order (levels last to first, raster order, response > treshold_1),
    raw detections and final boxes."""
    w, h = size
    img = _frame(w, h)
    p = ref.params(min_face=20, max_face=0, scale_factor=1.05, max_w=w, max_h=h)
    # response pixels are at most about 1/16 of each level; the levels sum to under 20x the frame
    steps = ref.detect_steps(img, p, with_levels=False, resp_cap=2 * w * h)
    cands = []
    for li in reversed(range(len(steps["resp"]))):
        r = steps["resp"][li]
        ys, xs = np.nonzero(r > np.float32(-1.5))
        cands += [(li, int(x) * 4, int(y) * 4, fbits(r[y, x])) for y, x in zip(ys, xs)]
    return {"levels": [(a, b, fbits(s)) for a, b, s, _ in steps["levels"]],
            "resp_shapes": [r.shape for r in steps["resp"]], "resp_sha": [sha(r) for r in steps["resp"]],
            "resp_sample": [r.ravel()[:: max(1, r.size // 4096)].copy() for r in steps["resp"]],
            "cands": cands, "raw": steps["raw"], "final": steps["final"]}


@pytest.fixture(scope="module")
def reference_results():
    with mp.get_context("spawn").Pool(len(SIZES)) as pool:
        return dict(zip(SIZES, pool.map(_reference, SIZES)))


@pytest.mark.parametrize("size", SIZES, ids=[f"{w}x{h}" for w, h in SIZES])
def test_batched_pyramid_frame_matches_reference(size, reference_results):
    w, h = size
    exp = reference_results[size]
    img = _frame(w, h)
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = w, h
    p.min_face_height, p.max_face_height, p.scale_factor = 20, 0, 1.05
    p.detect_mode = 1
    det = ccnn.FaceDetector()
    assert det.Init(p) == 0, _capi.last_error()
    faces = det.Detect(img)
    levels = det.levels()
    assert [(lv[0], lv[1], fbits(lv[2])) for lv in levels] == exp["levels"]
    assert len(levels) > 80 and levels[0][0] > w  # the upsampled 1.35x level leads the pyramid
    for i, (shape, hsh, sample) in enumerate(zip(exp["resp_shapes"], exp["resp_sha"], exp["resp_sample"])):
        r = det.response_map(i)
        assert r.shape == shape
        got_sample = r.ravel()[:: max(1, r.size // 4096)]
        assert np.allclose(got_sample, sample, rtol=RESP_RTOL, atol=0), i
        assert sha(r) == hsh, i
    cands = [(c[0], c[1], c[2], fbits(c[3])) for c in det.candidates()]
    assert len(cands) == len(exp["cands"]) and len(cands) > 1000
    assert cands == exp["cands"]
    assert det.raw_detections() == exp["raw"]
    assert faces == exp["final"] and len(faces) > 10
    det.Clear()
