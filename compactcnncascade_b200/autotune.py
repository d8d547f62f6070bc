"""Schedule autotuner: for a frame size and detector settings, times the cascade on seeded synthetic
frames (rendered on the device) under each candidate schedule -- frames in flight and resident
stage-2/3 blocks per SM (include/ccnn_inspect.h, ccnn_set_schedule) -- and keeps the fastest in a
JSON table keyed by the workload. FaceDetector.Init(..., schedule="auto") applies a table entry.
Results never depend on the schedule; only throughput does.

    python -m compactcnncascade_b200.autotune --width 1920 --height 1080
"""
import argparse
import ctypes
import json
import os
import sys

from . import _capi

TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "schedules.json")
SLOTS = (4, 8, 12, 16)
WINDOW_CTAS = (2, 3, 4)


def key(width, height, scale_factor, min_face, max_face):
    return f"{width}x{height}/sf{scale_factor:g}/min{min_face}/max{max_face}"


def load_table(path=TABLE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(p, path=TABLE):
    """(frame_slots, window_ctas_per_sm) tuned for these parameters, or None."""
    e = load_table(path).get(key(p.max_image_width, p.max_image_height, p.scale_factor, p.min_face_height, p.max_face_height))
    return (e["frame_slots"], e["window_ctas_per_sm"]) if e else None


def set_schedule(det, frame_slots, window_ctas_per_sm):
    _capi.check(_capi.lib().ccnn_set_schedule(det._h, int(frame_slots), int(window_ctas_per_sm)), "ccnn_set_schedule")


def get_schedule(det):
    a, b = ctypes.c_int(), ctypes.c_int()
    _capi.check(_capi.lib().ccnn_get_schedule(det._h, ctypes.byref(a), ctypes.byref(b)), "ccnn_get_schedule")
    return a.value, b.value


def measure(det, frames, width, height, batch=64, steps=8, warmup=3):
    """Frames/s of pipelined batches of the device frames (device time from the library's events)."""
    L = _capi.lib()
    cap = 256
    faces = (_capi.Face * (batch * cap))()
    nf = (ctypes.c_int * batch)()
    gms = ctypes.c_float()

    def step(k):
        arr = (_capi.Image * batch)()
        for j in range(batch):
            t = frames[(k * batch + j) % len(frames)]
            arr[j] = _capi.Image(width, height, 3, t.data_ptr(), width * 3)
        _capi.check(L.ccnn_detect_device_batch(det._h, arr, batch, faces, cap, nf, ctypes.byref(gms)), "ccnn_detect_device_batch")
        return gms.value

    for k in range(warmup):
        step(k)
    return steps * batch / (sum(step(warmup + k) for k in range(steps)) / 1e3)


def tune(width, height, scale_factor=1.15, min_face=40, max_face=240, n_faces=20, min_patch=30, max_patch=300, distinct=16,
         slots=SLOTS, window_ctas=WINDOW_CTAS, rounds=2):
    """Times every candidate schedule `rounds` times (interleaved) and returns the table entry."""
    import torch
    from . import FaceDetector, default_params, synth_frame_device
    p = default_params()
    p.max_image_width, p.max_image_height = width, height
    p.min_face_height, p.max_face_height, p.scale_factor = min_face, max_face, scale_factor
    p.detect_mode = 1
    det = FaceDetector()
    if det.Init(p) != 0:
        raise RuntimeError(_capi.last_error())
    frames = []
    for s in range(distinct):
        t = torch.empty((height, width, 3), dtype=torch.uint8, device="cuda")
        synth_frame_device(t.data_ptr(), width, height, 800_000 + s, n_faces, min_patch, max_patch)
        frames.append(t)
    best = {}
    for _ in range(rounds):
        for sl in slots:
            for wc in window_ctas:
                set_schedule(det, sl, wc)
                fps = measure(det, frames, width, height)
                best[(sl, wc)] = max(best.get((sl, wc), 0.0), fps)
    (sl, wc), fps = max(best.items(), key=lambda kv: kv[1])
    det.Clear()
    return {"frame_slots": sl, "window_ctas_per_sm": wc, "frames_per_s": round(fps, 1),
            "tried": {f"{a}x{b}": round(v, 1) for (a, b), v in sorted(best.items())}}


def main(argv=None):
    ap = argparse.ArgumentParser(description="pick the fastest schedule for a frame size and store it")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--scale-factor", type=float, default=1.15)
    ap.add_argument("--min-face", type=int, default=40)
    ap.add_argument("--max-face", type=int, default=240)
    ap.add_argument("--faces", type=int, default=20)
    ap.add_argument("--table", default=TABLE)
    a = ap.parse_args(argv)
    entry = tune(a.width, a.height, a.scale_factor, a.min_face, a.max_face, n_faces=a.faces)
    table = load_table(a.table)
    table[key(a.width, a.height, a.scale_factor, a.min_face, a.max_face)] = entry
    with open(a.table, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    print(json.dumps(entry), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
