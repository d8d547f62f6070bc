"""Synthetic CNTK text dumps of cascade networks, in the layout the reference's dump parser reads
(src/CNNObjectDetector/cnn_models_converter.cpp:79-268): node headers `z.<node>.<param>=...`
followed by value lines and a closing line holding '#'. Used to compare the converters."""
import numpy as np


def _f(x):
    return "%.9g" % np.float32(x)


def _node(lines, name, values, per_line=None):
    lines.append(f"z.{name}=LearnableParameter")
    vals = [_f(v) for v in np.asarray(values, np.float32).ravel()]
    if per_line is None:
        lines.append(" ".join(vals))
    else:
        for i in range(0, len(vals), per_line):
            lines.append(" ".join(vals[i:i + per_line]))
    lines.append("#")


def make_dump(seed, win=(23, 27), maps=(4, 8, 16), kernels=((4, 4), (3, 3), (4, 5)), hs=4, conn=4, n_out=3, full=False):
    rng = np.random.default_rng(seed)
    L = [f"features=InputValue [ {win[0]} x {win[1]} x 3 ]", "Pooling", " pool 1"]
    for l in range(3):
        kw, kh = kernels[l]
        for k in range(maps[l]):
            c = f"c{l + 1}{k + 1}"
            L.append(f"z.{c}.c=Convolution Kernel: {kw} x {kh} x 1")
            n = kw * kh * (3 if l == 0 else 1)
            _node(L, f"{c}.W", rng.normal(0, 0.3, n), per_line=3 * kw if l == 0 else kw)
            _node(L, f"{c}.b", rng.normal(0, 0.2, 1))
            _node(L, f"{c}.res.PlusArgs[0].ElementTimesArgs[0]", rng.uniform(0.05, 0.3, 1))
            _node(L, f"{c}.res.PlusArgs[1].ElementTimesArgs[0]", rng.uniform(0.5, 1.0, 1))
            bn = f"bn{l + 1}{k + 1}"
            _node(L, f"{bn}.scale", rng.uniform(0.5, 2.0, 1))
            _node(L, f"{bn}.bias", rng.normal(0, 0.5, 1))
            _node(L, f"{bn}.runMean", rng.normal(0, 1.0, 1))
            _node(L, f"{bn}.runVariance", rng.uniform(0.1, 3.0, 1))
    c_in = maps[2] if full else conn
    groups = 1 if full else maps[2] - conn + 1
    for i in range(groups):
        h = f"h{i + 1}"
        if i == 0:
            L.append(f"z.{h}.c=Convolution Kernel: {c_in} x 1 x 1 x {hs}")
        _node(L, f"{h}.W", rng.normal(0, 0.3, hs * c_in), per_line=hs)
        _node(L, f"{h}.b", rng.normal(0, 0.2, hs))
        _node(L, f"{h}.res.PlusArgs[0].ElementTimesArgs[1].x.ElementTimesArgs[0]", rng.uniform(0.5, 1.5, 1))
    for p in ("scale", "bias", "runMean", "runVariance"):
        lo, hi = {"scale": (0.5, 2.0), "bias": (-0.5, 0.5), "runMean": (-1, 1), "runVariance": (0.1, 3.0)}[p]
        _node(L, f"bn_h.{p}", rng.uniform(lo, hi, hs), per_line=1)
    _node(L, "z.arrayOfFunctions[0].W", rng.normal(0, 0.3, n_out * hs * groups), per_line=hs * groups)
    _node(L, "z.arrayOfFunctions[0].b", rng.normal(0, 0.2, n_out))
    _node(L, "z.PlusArgs[0].ElementTimesArgs[1].x.ElementTimesArgs[0]", rng.uniform(0.5, 1.0, 1))
    return "\n".join(L) + "\n"
