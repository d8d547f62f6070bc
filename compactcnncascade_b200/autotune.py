"""Schedule autotuner: for a frame size and detector settings, times the cascade on seeded synthetic
frames (rendered on the device) under candidate schedules and keeps the fastest in a JSON table
keyed by the workload. FaceDetector.Init(..., schedule="auto") applies a table entry. Results never
depend on the schedule; only throughput does.

The knobs (include/ccnn_inspect.h, ccnn_schedule):
  frame_slots          frames in flight, each with its own stream, buffers and captured graph
  window_ctas_per_sm   resident blocks per SM of the persistent stage-2/3 window kernel (5, 6: builds
                       with 48 and 40 registers a thread)
  front_blocks_per_sm  register budget of the stage-1 front kernel (3: 80 registers, 4: 64)
  back_blocks_per_sm   register budget of the stage-1 back kernel (3: 80 registers, 4: 64)
  batch_frames         frames per batched graph (0: every frame its own graph; 1: the same with the
                       pyramid and stage 1 of all levels in one persistent launch); the batched form
                       runs the pyramid and stage 1 of a whole group in one persistent launch
  batch_blocks_per_sm  resident blocks per SM of that persistent kernel (its grid; 4: 64 registers,
                       1-3: 80; fewer leave SMs to other frames' kernels)

The search is coordinate descent from the defaults: each knob in turn takes the value that times
fastest with the others held, for two passes (a full product of the knobs would be 960 timings).

    python -m compactcnncascade_b200.autotune --width 1920 --height 1080 [--gate]
"""
import argparse
import ctypes
import json
import os
import sys

from . import _capi

TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "schedules.json")
KNOBS = (("frame_slots", (4, 8, 12, 16, 24, 32)), ("window_ctas_per_sm", (2, 3, 4, 5, 6)), ("front_blocks_per_sm", (3, 4)),
         ("back_blocks_per_sm", (3, 4)), ("batch_frames", (0, 1, 2, 4, 8)), ("batch_blocks_per_sm", (1, 2, 3, 4)))
DEFAULTS = {"frame_slots": 8, "window_ctas_per_sm": 4, "front_blocks_per_sm": 3, "back_blocks_per_sm": 4, "batch_frames": 0,
            "batch_blocks_per_sm": 3}


def key(width, height, scale_factor, min_face, max_face, gated=False):
    """Table key of a workload; the learned gate changes which kernels dominate, so a gated detector
    has entries of its own."""
    return f"{width}x{height}/sf{scale_factor:g}/min{min_face}/max{max_face}" + ("/gate" if gated else "")


def load_table(path=TABLE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(p, path=TABLE, gated=False):
    """The tuned schedule (knob -> value) for these parameters (with the learned gate on, when
    gated), or None."""
    e = load_table(path).get(key(p.max_image_width, p.max_image_height, p.scale_factor, p.min_face_height, p.max_face_height, gated))
    if not e:
        return None
    return {k: e[k] for k, _ in KNOBS if k in e}


def set_schedule(det, schedule):
    """Applies a schedule (dict of knobs; missing knobs keep their value) to a FaceDetector."""
    s = _capi.Schedule(*[int(schedule.get(k, -1 if k == "batch_frames" else 0)) for k, _ in KNOBS])
    _capi.check(_capi.lib().ccnn_set_schedule_ex(det._h, ctypes.byref(s)), "ccnn_set_schedule_ex")


def get_schedule(det):
    s = _capi.Schedule()
    _capi.check(_capi.lib().ccnn_get_schedule_ex(det._h, ctypes.byref(s)), "ccnn_get_schedule_ex")
    return {k: getattr(s, k) for k, _ in KNOBS}


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
         knobs=KNOBS, passes=2, batch=64, gate=None):
    """Coordinate descent over the knobs; returns the table entry (the schedule, its frames/s and
    every timing taken). gate: (parameters, threshold, margin in pixels) of the learned gate to time
    with, or None."""
    import torch
    from . import FaceDetector, default_params, synth_frame_device
    p = default_params()
    p.max_image_width, p.max_image_height = width, height
    p.min_face_height, p.max_face_height, p.scale_factor = min_face, max_face, scale_factor
    p.detect_mode = 1
    det = FaceDetector()
    if det.Init(p) != 0:
        raise RuntimeError(_capi.last_error())
    if gate is not None:
        det.setGate(gate[0], gate[1])
        det.setGateMargin(gate[2] if len(gate) > 2 else 16)
    frames = []
    for s in range(distinct):
        t = torch.empty((height, width, 3), dtype=torch.uint8, device="cuda")
        synth_frame_device(t.data_ptr(), width, height, 800_000 + s, n_faces, min_patch, max_patch)
        frames.append(t)
    timings = {}

    def timed(sched):
        name = "/".join(f"{sched[k]}" for k, _ in knobs)
        set_schedule(det, sched)
        fps = measure(det, frames, width, height, batch=batch)
        timings[name] = round(max(timings.get(name, 0.0), fps), 1)
        return fps

    best = dict(DEFAULTS)
    best_fps = timed(best)
    for _ in range(passes):
        for k, values in knobs:
            for v in values:
                if v == best[k]:
                    continue
                trial = dict(best, **{k: v})
                if trial["batch_frames"] > trial["frame_slots"]:
                    continue
                fps = timed(trial)
                if fps > best_fps:
                    best, best_fps = trial, fps
    det.Clear()
    entry = dict(best, frames_per_s=round(best_fps, 1), knobs=[k for k, _ in knobs], tried=timings)
    if gate is not None:
        entry["gate_threshold"] = gate[1]
        entry["gate_margin"] = gate[2] if len(gate) > 2 else 16
    return entry


def main(argv=None):
    ap = argparse.ArgumentParser(description="pick the fastest schedule for a frame size and store it")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--scale-factor", type=float, default=1.15)
    ap.add_argument("--min-face", type=int, default=40)
    ap.add_argument("--max-face", type=int, default=240)
    ap.add_argument("--faces", type=int, default=20)
    ap.add_argument("--min-patch", type=int, default=30)
    ap.add_argument("--max-patch", type=int, default=300)
    ap.add_argument("--batch", type=int, default=64, help="frames per timed batch")
    ap.add_argument("--table", default=TABLE)
    ap.add_argument("--gate", action="store_true", help="tune with the shipped learned gate at its operating threshold")
    a = ap.parse_args(argv)
    gate = None
    if a.gate:
        from . import gate as gate_mod
        meta = gate_mod.load_meta()
        gate = (gate_mod.load(), meta.get("operating_threshold", 0.1), meta.get("operating_margin", 16))
    entry = tune(a.width, a.height, a.scale_factor, a.min_face, a.max_face, n_faces=a.faces, min_patch=a.min_patch,
                 max_patch=a.max_patch, batch=a.batch, gate=gate)
    table = load_table(a.table)
    table[key(a.width, a.height, a.scale_factor, a.min_face, a.max_face, gate is not None)] = entry
    with open(a.table, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    print(json.dumps(entry), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
