"""Schedule autotuner, host side: table keys and lookups."""
import json

from compactcnncascade_b200 import autotune, default_params


def test_key_and_lookup(tmp_path):
    p = default_params()
    p.max_image_width, p.max_image_height = 1920, 1080
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    k = autotune.key(1920, 1080, 1.15, 40, 240)
    assert k == "1920x1080/sf1.15/min40/max240"
    path = tmp_path / "t.json"
    assert autotune.lookup(p, str(path)) is None  # no table
    path.write_text(json.dumps({k: {"frame_slots": 12, "window_ctas_per_sm": 3, "back_blocks_per_sm": 4, "frames_per_s": 1.0}}))
    assert autotune.lookup(p, str(path)) == {"frame_slots": 12, "window_ctas_per_sm": 3, "back_blocks_per_sm": 4}
    p.scale_factor = 1.05
    assert autotune.lookup(p, str(path)) is None
    path.write_text("not json")
    assert autotune.load_table(str(path)) == {}
