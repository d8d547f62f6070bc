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


def test_gated_entries_are_separate(tmp_path):
    """A detector with the learned gate on has table entries of its own (the gate changes which kernels
    dominate); the plain entry is not used for it and the other way round."""
    p = default_params()
    p.max_image_width, p.max_image_height = 1920, 1080
    p.min_face_height, p.max_face_height, p.scale_factor = 40, 240, 1.15
    k = autotune.key(1920, 1080, 1.15, 40, 240)
    kg = autotune.key(1920, 1080, 1.15, 40, 240, gated=True)
    assert kg == k + "/gate"
    path = tmp_path / "t.json"
    path.write_text(json.dumps({kg: {"frame_slots": 16, "window_ctas_per_sm": 5, "gate_threshold": 0.4, "frames_per_s": 2.0}}))
    assert autotune.lookup(p, str(path)) is None
    assert autotune.lookup(p, str(path), gated=True) == {"frame_slots": 16, "window_ctas_per_sm": 5}


def test_shipped_table_is_consistent():
    """Every entry of the shipped table names only known knobs with values the library accepts."""
    table = autotune.load_table()
    assert table
    allowed = dict(autotune.KNOBS)
    for name, e in table.items():
        sched = {k: e[k] for k in allowed if k in e}
        assert sched, name
        for k, v in sched.items():
            assert v in allowed[k], (name, k, v)
        assert e["frames_per_s"] > 0
