"""Schedules (ccnn_set_schedule) change throughput only: every schedule gives the same faces."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import compactcnncascade_b200 as ccnn  # noqa: E402
from compactcnncascade_b200 import autotune  # noqa: E402


def test_results_do_not_depend_on_the_schedule():
    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = 1280, 720
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    imgs = [ccnn.synth_frame(1280, 720, 60 + i, 10, 30, 300)[0] for i in range(5)]
    d = ccnn.FaceDetector()
    assert d.Init(p) == 0
    assert autotune.get_schedule(d) == (8, 4)
    want = d.DetectBatch(imgs)
    assert sum(len(f) for f in want) > 0
    for sched in [(1, 1), (3, 2), (16, 3), (5, 4)]:
        autotune.set_schedule(d, *sched)
        assert autotune.get_schedule(d) == sched
        assert d.DetectBatch(imgs) == want
        assert [d.Detect(im) for im in imgs] == want
    with pytest.raises(ccnn.CCNNError):
        autotune.set_schedule(d, 65, 4)
    with pytest.raises(ccnn.CCNNError):
        autotune.set_schedule(d, 8, 5)
    d2 = ccnn.FaceDetector()
    assert d2.Init(p, schedule=(2, 2)) == 0 and autotune.get_schedule(d2) == (2, 2)
