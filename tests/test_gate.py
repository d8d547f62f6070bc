"""Learned gate, host side: the float64 restatement of its loss gradient against central finite
differences, the weight-file format, parameter layout and the box-recall measure."""
import numpy as np
import pytest

from compactcnncascade_b200 import gate
from oracle import gate_ref


def _case(seed=1):
    rng = np.random.default_rng(seed)
    p = gate.init_params(seed + 2).astype(np.float64)
    p[gate.B3:] = -1.0
    f = rng.normal(0, 1, (2, 10, 12))
    lab = (rng.random((2, 4, 5, 6)) < 0.2).astype(np.uint8)
    return p, f, lab


def test_layout_matches_header():
    assert gate.N_PARAMS == gate_ref.N_PARAMS == 700
    assert (gate.W1, gate.B1, gate.W2, gate.B2, gate.W3, gate.B3) == (gate_ref.W1, gate_ref.B1, gate_ref.W2, gate_ref.B2, gate_ref.W3,
                                                                      gate_ref.B3)
    assert gate.B3 + gate.OCTAVES == gate.N_PARAMS


@pytest.mark.parametrize("pos_weight", [1.0, 5.0])
def test_restated_gradient_matches_finite_differences(pos_weight):
    p, f, lab = _case()
    _, g = gate_ref.loss_and_grad(p, f, lab, pos_weight)
    eps = 1e-6
    idx = list(range(0, 72, 7)) + list(range(72, 80)) + list(range(80, 656, 23)) + list(range(656, 700))
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        num = (gate_ref.loss_and_grad(pp, f, lab, pos_weight)[0] - gate_ref.loss_and_grad(pm, f, lab, pos_weight)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-7 + 1e-6 * abs(g[i]), i


def test_forward_is_probability_map():
    p, f, _ = _case()
    pr = gate_ref.forward(p, f)
    assert pr.shape == (2, 4, 5, 6) and np.all((pr > 0) & (pr < 1))


def test_weight_file_round_trip(tmp_path):
    p = gate.init_params(7)
    path = str(tmp_path / "g.bin")
    gate.save(path, p, {"note": "x"})
    assert np.array_equal(gate.load(path), p)
    assert gate.load_meta(path) == {"note": "x"}
    with pytest.raises(ValueError):
        gate.save(path, p[:10])
    with open(path, "r+b") as fh:
        fh.write(b"XXXX")
    with pytest.raises(ValueError):
        gate.load(path)


def test_box_recall():
    ref = [(0, 0, 10, 10), (100, 100, 20, 20), (50, 50, 10, 10)]
    got = [(1, 1, 10, 10), (100, 100, 20, 20)]
    assert gate.box_recall(ref, got) == (2, 3)
    assert gate.box_recall(ref, []) == (0, 3)
    assert gate.box_recall([], got) == (0, 0)
    # one gated box can match one plain box only
    assert gate.box_recall([(0, 0, 10, 10), (0, 0, 10, 10)], [(0, 0, 10, 10)]) == (1, 2)


def test_shipped_weights_load():
    import os
    if not os.path.exists(gate.WEIGHTS_1080P):
        pytest.skip("no trained weights in the package")
    p = gate.load()
    assert p.shape == (700,) and np.all(np.isfinite(p))
    meta = gate.load_meta()
    assert meta["train_frames"] >= 1000 and meta["eval_frames"] >= 100


def test_operating_point_rule():
    """Of the evaluated (threshold, margin) pairs with >= 99.5 % box recall, the one that runs the fewest
    back tiles (ties: the higher threshold); none reaching it: the lowest threshold, one cell of margin."""
    ev = [{"threshold": 0.1, "margin": 8, "box_recall": 0.999, "back_tiles_run": 0.30},
          {"threshold": 0.3, "margin": 8, "box_recall": 0.996, "back_tiles_run": 0.26},
          {"threshold": 0.5, "margin": 8, "box_recall": 0.990, "back_tiles_run": 0.22},
          {"threshold": 0.4, "margin": 16, "box_recall": 0.997, "back_tiles_run": 0.26}]
    assert gate._operating_point(ev, [0.1, 0.3, 0.4, 0.5]) == (0.4, 16)
    assert gate._operating_point(ev[:3], [0.1, 0.3, 0.5]) == (0.3, 8)
    assert gate._operating_point([dict(r, box_recall=0.98) for r in ev], [0.1, 0.3, 0.4, 0.5]) == (0.1, 16)


def test_shipped_operating_point_follows_its_evaluation():
    """The operating point recorded with the shipped weights is the rule's choice on the committed
    1,000-frame held-out evaluation, and it keeps at least 99.5 % of the plain cascade's boxes there."""
    import json
    import os
    rec = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles", "gate_heldout_eval_1080p.json")
    if not os.path.exists(gate.WEIGHTS_1080P) or not os.path.exists(rec):
        pytest.skip("no trained weights or evaluation record")
    with open(rec) as fh:
        r = json.load(fh)
    thr = sorted({e["threshold"] for e in r["eval"]})
    op = gate._operating_point(r["eval"], thr)
    assert op == (r["operating_threshold"], r["operating_margin"])
    meta = gate.load_meta()
    assert (meta["operating_threshold"], meta["operating_margin"]) == op
    chosen = [e for e in r["eval"] if (e["threshold"], e["margin"]) == op]
    assert len(chosen) == 1 and chosen[0]["box_recall"] >= 0.995 and r["eval_frames"] >= 1000
