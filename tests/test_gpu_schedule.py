"""Schedules (ccnn_set_schedule_ex) change throughput only: every schedule gives the same faces."""
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
    assert autotune.get_schedule(d) == autotune.DEFAULTS
    want = d.DetectBatch(imgs)
    assert sum(len(f) for f in want) > 0
    names = [k for k, _ in autotune.KNOBS]
    for sched in [(1, 1, 3, 3, 0, 3), (3, 2, 4, 4, 2, 4), (16, 3, 3, 4, 4, 3), (5, 4, 4, 3, 5, 3), (2, 2, 3, 4, 1, 4), (12, 5, 4, 4, 0, 3),
                  (8, 6, 3, 4, 0, 3)]:
        sd = dict(zip(names, sched))
        autotune.set_schedule(d, sd)
        assert autotune.get_schedule(d) == sd
        assert d.DetectBatch(imgs) == want
        assert [d.Detect(im) for im in imgs] == want
    for bad in [{"frame_slots": 65}, {"window_ctas_per_sm": 7}, {"front_blocks_per_sm": 2}, {"back_blocks_per_sm": 5},
                {"batch_frames": 17}, {"frame_slots": 4, "batch_frames": 8}, {"batch_blocks_per_sm": 5}]:
        with pytest.raises(ccnn.CCNNError):
            autotune.set_schedule(d, bad)
    d2 = ccnn.FaceDetector()
    assert d2.Init(p, schedule={"frame_slots": 2, "window_ctas_per_sm": 2}) == 0
    assert autotune.get_schedule(d2) == dict(autotune.DEFAULTS, frame_slots=2, window_ctas_per_sm=2)
