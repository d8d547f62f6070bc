"""Throughput of the plain face-detection cascade on 1920x1080 BGR frames.

A step is one pass of the detection path over a batch of B synthetic 1080p frames (seeded
generator: 20 face patches of 30-300 px), detector settings min face 40, max face 240,
scale factor 1.15, precision high, drop_detect/equalize/reflection on.

  value  frames/s over all ranks, inputs resident in device memory when timing starts;
         device time from CUDA events recorded by the library on its own streams
         (ccnn_detect_device_batch), summed over the K timed steps, max over ranks.
  e2e    the same frames through the public host-memory API (ccnn_detect_batch) from pinned
         host buffers: upload, the cascade and the result download inside the timed region
         (host wall clock around the synchronous calls).

Multi-GPU: frames are independent, so N ranks are N replicas on disjoint frame seeds, with no
data-path collective; value = all ranks' frames / the slowest rank's time.

`--impl reference` times the reference's own CPU cascade (oracle/_ref, built from the
unmodified sources with the reference's shipped flags) on all host cores on the same workload.
"""
import argparse
import ctypes
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 1920, 1080
N_FACES, MIN_PATCH, MAX_PATCH = 20, 30, 300
MIN_FACE, MAX_FACE, SCALE_FACTOR = 40, 240, 1.15
WORKLOAD = "plain cascade, 1920x1080 BGR synthetic frames (20 face patches 30-300 px), min face 40, max face 240, scale 1.15"
METRIC = "1080p frames/s & p99 ms, batched+gated vs plain cascade at >=99% box recall"
KERNELS = ["gray", "pyramid", "stage1_front", "stage1_back", "cand_write", "stage23_windows", "replay_merge"]


def _gen_frame(seed):
    import compactcnncascade_b200 as ccnn
    img, _ = ccnn.synth_frame(W, H, seed, N_FACES, MIN_PATCH, MAX_PATCH)
    return img


def _frames(seeds, workers):
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(workers, len(seeds))) as pool:
        return pool.map(_gen_frame, seeds)


# ---------------- serving workload ----------------

SERVE_MIX = [((640, 480), 0.3, 5, 40, 200), ((1280, 720), 0.3, 10, 30, 300), ((1920, 1080), 0.3, 20, 30, 300),
             ((3840, 2160), 0.1, 60, 20, 600)]


def _gen_serve_frame(args):
    import compactcnncascade_b200 as ccnn
    (w, h), seed, nf, lo, hi = args
    return ccnn.synth_frame(w, h, seed, nf, lo, hi)[0]


def serve_frames(per_res, seed0=900_000):
    jobs = [(m[0], seed0 + 1000 * r + i, m[2], m[3], m[4]) for r, m in enumerate(SERVE_MIX) for i in range(per_res)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(len(jobs), os.cpu_count() or 4)) as pool:
        imgs = pool.map(_gen_serve_frame, jobs)
    out = {}
    for (res, *_), img in zip(jobs, imgs):
        out.setdefault(res, []).append(img)
    return out


def run_serving(frames_by_res, rate, n_frames, seed=1, gate=None):
    """Poisson arrivals (seeded exponential inter-arrival times) of frames drawn from the
    resolution mix; every frame goes through the serving loop (ccnn_server_*). Returns latency
    percentiles (submit -> result on the device side, measured by the server) and throughput."""
    import compactcnncascade_b200 as ccnn
    rng = np.random.default_rng(seed)
    p = ccnn.default_params()
    p.min_face_height, p.max_face_height, p.scale_factor = MIN_FACE, MAX_FACE, SCALE_FACTOR
    p.detect_mode = 1
    srv = ccnn.FaceServer(p, hbm_budget_bytes=32 << 30, slots_per_class=4)
    if gate is not None:
        srv.set_gate(*gate)
    pinned = {res: [] for res in frames_by_res}
    for res, imgs in frames_by_res.items():
        for img in imgs:
            pf = ccnn.pinned_frame(img.shape)
            pf[...] = img
            pinned[res].append(pf)
    # warm-up: every class once (detector creation and graph capture are not part of serving)
    for res in pinned:
        srv.wait(srv.submit(pinned[res][0]))
    weights = np.array([m[1] for m in SERVE_MIX])
    kinds = rng.choice(len(SERVE_MIX), size=n_frames, p=weights / weights.sum())
    gaps = rng.exponential(1.0 / rate, size=n_frames)
    tickets = []
    t0 = time.perf_counter()
    due = t0
    for k, g in zip(kinds, gaps):
        due += g
        while time.perf_counter() < due:
            pass
        res = SERVE_MIX[k][0]
        imgs = pinned[res]
        t = None
        while t is None:  # a full queue pushes back on the client
            t = srv.submit(imgs[len(tickets) % len(imgs)])
        tickets.append((res, t))
    lat = {res: [] for res in pinned}
    for res, t in tickets:
        lat[res].append(srv.wait(t)[1])
    wall = time.perf_counter() - t0
    srv.close()
    allv = np.concatenate([np.array(v) for v in lat.values() if v])
    out = {"rate_per_s": rate, "frames": n_frames, "fps": round(n_frames / wall, 1),
           "p50_ms": round(float(np.percentile(allv, 50)), 3), "p99_ms": round(float(np.percentile(allv, 99)), 3),
           "per_resolution": {f"{r[0]}x{r[1]}": {"frames": len(v), "p50_ms": round(float(np.percentile(v, 50)), 3),
                                                 "p99_ms": round(float(np.percentile(v, 99)), 3)} for r, v in lat.items() if v}}
    return out


# ---------------- batched pyramid: many uneven levels ----------------

BATCHED = [((3840, 2160), 60, 20, 600), ((4800, 2400), 60, 20, 600)]
RECALL_SEED0 = 20_000_000  # frames of the gated phase's recall sample (disjoint from the gate's training and evaluation)


def launches_per_frames(n_frames, n_levels, batch_frames, gated=False):
    """Kernels the library launches for n_frames frames of one size. Per frame: gray, stage-1 front and
    back once per group of 32 levels (the front kernel resamples the pyramid levels itself),
    candidates, windows, replay; with batch_frames == 1 stage 1 is one persistent launch instead. In
    the batched form, per group of batch_frames frames: gray, the count reset, one persistent
    pyramid + stage-1 launch, candidates, windows, replay; leftover frames run per frame. The learned
    gate adds its inference and one mask launch per group of 32 levels to every frame."""
    groups = -(-n_levels // 32)
    gate = (1 + groups) if gated else 0
    per_frame = (5 if batch_frames == 1 else 4 + 2 * groups) + gate
    if batch_frames and batch_frames >= 2:
        full = n_frames // batch_frames
        leftover = (n_frames - full * batch_frames) * (4 + 2 * groups + gate)
        return full * (6 + batch_frames * gate) + leftover
    return n_frames * per_frame


def run_batched_pyramid(dev, args):
    """Scale 1.05, min face 20, no max face (the largest level is an upsampled 1.35x copy): 80+
    pyramid levels of uneven sizes per frame, device-resident frames (rendered on the device by the
    seeded generator) in 8-frame batches, device time from the library's events. Two forms: every
    frame its own captured graph (8 frames in flight), and the batched form (groups of 8 frames one
    graph each, the pyramid and stage 1 of all levels of all 8 frames in one persistent launch fed by
    a device work queue, two groups in flight)."""
    import torch
    import compactcnncascade_b200 as ccnn
    from compactcnncascade_b200 import _capi, autotune
    L = _capi.lib()
    out = {}
    B = args.batched_frames
    for (w, h), nf, lo, hi in BATCHED:
        p = ccnn.default_params()
        p.max_image_width, p.max_image_height = w, h
        p.min_face_height, p.max_face_height, p.scale_factor = 20, 0, 1.05
        p.detect_mode = 1
        p.cuda_device_id = dev
        det = ccnn.FaceDetector()
        if det.Init(p) != 0:
            raise SystemExit(f"detector init failed: {_capi.last_error()}")
        frames = []
        for i in range(B):
            t = torch.empty((h, w, 3), dtype=torch.uint8, device=f"cuda:{dev}")
            ccnn.synth_frame_device(t.data_ptr(), w, h, 700_000 + 1000 * w + i, nf, lo, hi)
            frames.append(t)
        arr = (_capi.Image * B)(*[_capi.Image(w, h, 3, t.data_ptr(), w * 3) for t in frames])
        cap = 1024
        faces = (_capi.Face * (B * cap))()
        nfaces = (ctypes.c_int * B)()
        gms = ctypes.c_float()

        def step():
            if L.ccnn_detect_device_batch(det._h, arr, B, faces, cap, nfaces, ctypes.byref(gms)) < 0:
                raise SystemExit(f"ccnn_detect_device_batch failed: {_capi.last_error()}")
            return gms.value

        res = {}
        # the autotuner's schedule for this workload where it has one (its other knobs also for the
        # batched form)
        tuned = autotune.lookup(p) or {}
        for form, sched in (("per_frame", dict(tuned, frame_slots=tuned.get("frame_slots", B), batch_frames=0)),
                            ("batched", dict(tuned, frame_slots=2 * B, batch_frames=B))):
            autotune.set_schedule(det, sched)
            for _ in range(max(3, args.warmup)):
                step()
            ref_faces = [list(faces[j * cap: j * cap + nfaces[j]]) for j in range(B)]
            steps = max(3, args.steps // 4)
            ms = sum(step() for _ in range(steps))
            if form == "batched":  # the batched form's faces equal the per-frame form's
                res["faces_equal_per_frame"] = all(
                    [(f.x, f.y, f.width, f.height, f.score) for f in faces[j * cap: j * cap + nfaces[j]]] ==
                    [(f.x, f.y, f.width, f.height, f.score) for f in res["_pf_faces"][j]] for j in range(B))
            else:
                res["_pf_faces"] = ref_faces
            n_levels = len(det.levels())
            res[form] = {"frames_per_s": round(steps * B / (ms / 1e3), 1), "steps": steps,
                         "launches_per_8_frames": launches_per_frames(8, n_levels, sched["batch_frames"]),
                         "schedule": autotune.get_schedule(det)}
        res.pop("_pf_faces", None)
        autotune.set_schedule(det, {"frame_slots": B, "batch_frames": 0})
        lat = []
        for i in range(10):
            t0 = time.perf_counter()
            det.DetectDevice(frames[i % B].data_ptr(), w, h, 3, w * 3)
            lat.append((time.perf_counter() - t0) * 1e3)
        res.update({"frames_per_s": max(res["per_frame"]["frames_per_s"], res["batched"]["frames_per_s"]), "levels": n_levels,
                    "faces_per_frame": round(sum(nfaces[j] for j in range(B)) / B, 1),
                    "p50_ms": round(float(np.percentile(lat[2:], 50)), 3), "batch": B})
        out[f"{w}x{h}"] = res
        det.Clear()
    out["note"] = ("seeded frames with 60 face patches 20-600 px, scale 1.05, min face 20, no max face; device-resident frames, "
                   "device time from CUDA events. per_frame: every frame's chain one CUDA graph (stage 1, whose front kernel "
                   "resamples the pyramid levels, in level tables of at most 32 levels a launch), the autotuned frames in flight. "
                   "batched: 8 frames one graph, the pyramid and stage 1 "
                   "of all levels of all 8 frames in one persistent launch fed by a device work queue, two 8-frame groups in flight")
    return out


# ---------------- reference CPU path (test oracle; never the measured product) ----------------

def _ref_worker(args):
    seeds, fast, warmup, runs = args
    from oracle import ref
    import compactcnncascade_b200 as ccnn
    L = ref.load(fast=fast)
    p = ref.params(min_face=MIN_FACE, max_face=MAX_FACE, scale_factor=SCALE_FACTOR)
    L.ref_api_init(ctypes.byref(p))
    out = (ref.RefDet * 65536)()
    frames = [ccnn.synth_frame(W, H, s, N_FACES, MIN_PATCH, MAX_PATCH)[0] for s in seeds]
    # the first colour frame re-initialises the detector (cnn_detector_v3.cpp:2531-2546): warm-up
    for i in range(max(1, warmup)):
        f = frames[i % len(frames)]
        L.ref_api_detect(f.ctypes.data, W, H, 3, W * 3, out, 65536)
    t = time.perf_counter()
    n = 0
    for i in range(runs):
        f = frames[i % len(frames)]
        n += max(0, L.ref_api_detect(f.ctypes.data, W, H, 3, W * 3, out, 65536))
    return time.perf_counter() - t, runs, n


def reference_cpu(runs_per_worker, warmup=1, distinct=2, workers=None, seed0=10_000):
    """The reference's CPU cascade on all host cores: one detector per process (the reference API
    is a per-process singleton), each cycling `distinct` frames of the workload for
    `runs_per_worker` timed detections after `warmup` untimed ones.
    Returns (frames/s, workers, frames, seconds of the slowest worker, fast-build flag)."""
    from oracle import ref
    fast = ref.available(fast=True)
    if not ref.available(fast=fast):
        return None
    workers = workers or os.cpu_count() or 1
    jobs = [([seed0 + w * distinct + i for i in range(distinct)], fast, warmup, runs_per_worker) for w in range(workers)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        res = pool.map(_ref_worker, jobs)
    wall = max(r[0] for r in res)
    nfr = sum(r[1] for r in res)
    return nfr / wall, workers, nfr, wall, fast


# ---------------- clocks ----------------

class ClockSampler:
    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------- work accounting (per frame) ----------------

def algorithmic_work(levels, gw, gh):
    """Per-frame algorithmic work of the two stage-1 kernels: (fp32 ops, bytes).

    fp32 ops count every IEEE multiply, add, compare-free activation step and division as one
    lane operation (the exact arithmetic issues no fused multiply-add):
      front, per pooled L1 pixel: 4 maps x 4 pre-pool positions x (16 mul + 15 add + 5 BN/LReLU)
                                  + 6 neighbour-sum adds
      back, per pooled L2 pixel:  8 maps x 4 positions x (9 mul + 8 add + 5) + 14 sum adds
            per response pixel:   16 L3 maps x (20 mul + 19 add + 5)
                                  + 52 hidden x (4 mul + 4 add + 1 slope + 13 tanh + 2 scale + 2 out)
                                  + 8 output ops
    bytes: front reads the gray samples of each level pixel (4 B per level pixel; it resamples the
    level tiles from the gray frame, no level image is stored) and writes 4 S1 planes (16 B per
    pooled L1 pixel); back reads the S1 planes and writes the response maps (4 B per response pixel)."""
    ops_front = ops_back = 0
    by_front = 0
    by_back = 0
    for (w, h, _s, ow, oh) in levels:
        p1w, p1h = (w - 3) >> 1, (h - 3) >> 1
        p2w, p2h = (p1w - 2) >> 1, (p1h - 2) >> 1
        ops_front += p1w * p1h * (16 * 36 + 6)
        ops_back += p2w * p2h * (32 * 22 + 14) + ow * oh * (16 * 44 + 52 * 26 + 8)
        by_front += 4 * w * h + 16 * p1w * p1h
        by_back += 16 * p1w * p1h + 4 * ow * oh
    return {"stage1_front": (ops_front, by_front), "stage1_back": (ops_back, by_back)}


def dram_traffic():
    """DRAM bytes per launch of each kernel from the committed ncu capture summary
    (profiles/dram_traffic_1080p.txt: `kernel bytes` lines), or {} when absent."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic_1080p.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 2 and not line.startswith("#"):
                    out[parts[0]] = float(parts[1])
    except OSError:
        pass
    return out


def frame_bytes(levels, w, h):
    """Algorithmic bytes of a frame: BGR read, gray write, the gray samples of every level pixel read by
    the stage-1 front kernel, the S1 planes written and read (4 planes of pooled L1 pixels), the
    response maps written and read."""
    s1 = sum(((a[0] - 3) >> 1) * ((a[1] - 3) >> 1) for a in levels)
    return 3 * w * h + 4 * w * h + sum(4 * a[0] * a[1] for a in levels) + 32 * s1 + sum(8 * a[3] * a[4] for a in levels)


def committed_records():
    """Longer measurements recorded once on a B200 and committed under profiles/: the serving sweep
    (`bench.py --serving`) and the learned gate's held-out evaluation (`python -m
    compactcnncascade_b200.gate --eval-only --report ...`). Empty when absent."""
    out = {}
    for key, name in (("serving_sweep", "serving_sweep_mixed_resolutions.json"), ("gate_heldout", "gate_heldout_eval_1080p.json")):
        try:
            with open(os.path.join(ROOT, "profiles", name)) as f:
                out[key] = json.load(f)
        except (OSError, ValueError):
            pass
    return out


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------- main ----------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=128, help="frames per step")
    ap.add_argument("--distinct", type=int, default=24, help="distinct frames cycled (24 x 6.2 MB > L2)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-frames", type=int, default=48,
                    help="timed detections per host core for the CPU baseline (2 distinct frames cycled; about 10 s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--latency-frames", type=int, default=200)
    ap.add_argument("--profile-iters", type=int, default=20)
    ap.add_argument("--serve-frames", type=int, default=2000, help="frames of the serving-loop phase (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="Poisson arrival rate of the serving phase, frames/s")
    ap.add_argument("--no-gate", action="store_true", help="skip the batched+gated phase")
    ap.add_argument("--gate-threshold", type=float, default=None, help="gate probability threshold (default: the weights' own)")
    ap.add_argument("--gate-fallback", type=float, default=0.25, help="ambiguous-cell fraction that falls back to the full scan")
    ap.add_argument("--gate-margin", type=int, default=None, help="gate candidate margin in pixels (default: the weights' own)")
    ap.add_argument("--recall-frames", type=int, default=400,
                    help="further seeded frames the gated phase's box recall is also measured on (0: only the timed frames)")
    ap.add_argument("--batched-frames", type=int, default=8,
                    help="frames per batch of the batched-pyramid phase (3840x2160 and 4800x2400; 0: skip)")
    ap.add_argument("--schedule", default="auto",
                    help="schedule of the main phases: 'auto' (the autotuner's table entry), 'default', or knob=value,... "
                         "(compactcnncascade_b200.autotune.KNOBS) on top of the defaults")
    ap.add_argument("--serving", action="store_true",
                    help="only the serving sweep: 10,000 mixed-resolution frames per offered rate, plain and gated")
    ap.add_argument("--serve-rates", default="500,1000,2000,4000,8000,16000", help="offered rates of the serving sweep, frames/s")
    ap.add_argument("--serve-frames-sweep", type=int, default=10_000, help="frames per offered rate of the serving sweep")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    if args.serving:
        if rank == 0:
            fr = serve_frames(4)
            rates = [float(r) for r in args.serve_rates.split(",")]
            sweep = [run_serving(fr, r, args.serve_frames_sweep, seed=int(r)) for r in rates]
            from compactcnncascade_b200 import gate as gate_mod
            gthr = gate_mod.load_meta().get("operating_threshold", 0.1)
            gmargin = gate_mod.load_meta().get("operating_margin", 16)
            gsweep = [run_serving(fr, r, args.serve_frames_sweep, seed=int(r), gate=(gate_mod.load(), gthr, args.gate_fallback, gmargin))
                      for r in rates]
            print(json.dumps({"metric": "serving loop p50/p99 ms and fps, mixed 640x480/1280x720/1920x1080/3840x2160 at 30/30/30/10 %",
                              "unit": "ms", "data": "synthetic (seeded generator)", "frames_per_rate": args.serve_frames_sweep,
                              "sweep": sweep, "gated_threshold": gthr, "gated_margin_px": gmargin, "sweep_gated": gsweep}), flush=True)
        return

    from compactcnncascade_b200.replicas import rank_seeds
    # frames and the CPU baseline use spawn pools, started before this process touches CUDA
    seeds = rank_seeds(rank, args.distinct)
    frames = _frames(seeds, os.cpu_count() or 4)
    sframes = serve_frames(2) if (rank == 0 and args.serve_frames > 0) else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_cpu(runs_per_worker=args.cpu_frames)

    import torch
    import compactcnncascade_b200 as ccnn
    from compactcnncascade_b200 import _capi

    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)

    p = ccnn.default_params()
    p.max_image_width, p.max_image_height = W, H
    p.min_face_height, p.max_face_height, p.scale_factor = MIN_FACE, MAX_FACE, SCALE_FACTOR
    p.detect_mode = 1
    p.cuda_device_id = dev
    det = ccnn.FaceDetector()
    from compactcnncascade_b200 import autotune
    if args.schedule in ("auto", "default"):
        sched_arg, sched_src = (args.schedule if args.schedule == "auto" else None), None
    else:
        sched_arg = dict((k, int(v)) for k, v in (kv.split("=") for kv in args.schedule.split(",")))
        sched_src = f"command line ({args.schedule})"
    if det.Init(p, schedule=sched_arg) != 0:  # the autotuner's schedule for this workload, when tuned
        raise SystemExit(f"detector init failed: {_capi.last_error()}")
    schedule = autotune.get_schedule(det)
    L = _capi.lib()

    d_frames = [torch.from_numpy(f).to(f"cuda:{dev}") for f in frames]
    h_frames = [torch.from_numpy(f).pin_memory() for f in frames]
    B = args.batch
    cap = 256

    def make_batch(step, dev_side):
        arr = (_capi.Image * B)()
        for j in range(B):
            k = (step * B + j) % len(frames)
            t = d_frames[k] if dev_side else h_frames[k]
            arr[j] = _capi.Image(W, H, 3, t.data_ptr(), W * 3)
        return arr

    faces = (_capi.Face * (B * cap))()
    nf = (ctypes.c_int * B)()
    gms = ctypes.c_float()

    def device_step(step):
        st = L.ccnn_detect_device_batch(det._h, make_batch(step, True), B, faces, cap, nf, ctypes.byref(gms))
        if st < 0:
            raise SystemExit(f"ccnn_detect_device_batch failed: {_capi.last_error()}")
        return gms.value

    def host_step(step):
        st = L.ccnn_detect_batch(det._h, make_batch(step, False), B, faces, cap, nf)
        if st < 0:
            raise SystemExit(f"ccnn_detect_batch failed: {_capi.last_error()}")

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- value: device-resident inputs ----
    for s in range(args.warmup):
        device_step(s)
    barrier()
    # NVTX ranges name the timed regions for profilers (ncu --nvtx --nvtx-include "plain/")
    with ClockSampler(dev) as clk:
        t0 = time.perf_counter()
        gpu_ms = 0.0
        faces_total = 0
        torch.cuda.nvtx.range_push("plain")
        for s in range(args.steps):
            gpu_ms += device_step(args.warmup + s)
            faces_total += sum(nf[j] for j in range(B))
        torch.cuda.nvtx.range_pop()
        barrier()
        wall_dev = time.perf_counter() - t0
    clocks = clk.summary()
    t_dev = gpu_ms / 1e3
    if dist:
        t = torch.tensor([t_dev, wall_dev], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_dev, wall_dev = float(t[0]), float(t[1])
    frames_timed = args.steps * B * world
    value = frames_timed / t_dev

    # ---- e2e: pinned host frames through the public host API ----
    for s in range(args.warmup):
        host_step(s)
    barrier()
    t0 = time.perf_counter()
    for s in range(args.steps):
        host_step(args.warmup + s)
    barrier()
    wall_e2e = time.perf_counter() - t0
    if dist:
        t = torch.tensor([wall_e2e], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall_e2e = float(t[0])
    e2e = frames_timed / wall_e2e

    # ---- single-frame latency (synchronous ccnn_detect, pinned host input) ----
    lat = []
    one = (_capi.Face * cap)()
    n1 = ctypes.c_int()
    for i in range(args.latency_frames):
        t = h_frames[i % len(frames)]
        im = _capi.Image(W, H, 3, t.data_ptr(), W * 3)
        t0 = time.perf_counter()
        L.ccnn_detect(det._h, ctypes.byref(im), one, cap, ctypes.byref(n1))
        lat.append((time.perf_counter() - t0) * 1e3)
    lat = np.array(lat[min(5, len(lat) - 1):])

    # ---- per-kernel profile of the last frame (CUDA events around each kernel) ----
    kms = (ctypes.c_float * (len(KERNELS) + 2))()
    L.ccnn_profile_last_frame(det._h, args.profile_iters, kms, len(KERNELS) + 2)
    kernel_ms = {KERNELS[i]: float(kms[i]) for i in range(len(KERNELS))}
    single_launch_ms = float(kms[len(KERNELS) + 1])
    levels = det.levels()
    cands = det.candidates()
    work = algorithmic_work(levels, W, H)
    # dominant kernel: the grid-wide kernel with the largest device time (the replay/merge kernel
    # is one CTA per frame and overlaps other frames' grid-wide kernels in the slot pipeline)
    dom = max(work, key=lambda k: kernel_ms[k])
    hbm_peak, peak_src = load_peaks()
    ops, by = work[dom]
    ms = kernel_ms[dom]
    achieved_gbs = by / (ms * 1e-3) / 1e9
    # the fp32 ceiling, measured now on this GPU by the library's microbenchmark of the packed IEEE
    # add / product instructions the stage-1 kernels issue (ccnn_measure_fp32_peak)
    peak_ops = ctypes.c_double()
    peak_ms = ctypes.c_float()
    with ClockSampler(dev) as pclk:
        pst = L.ccnn_measure_fp32_peak(2048, 5, ctypes.byref(peak_ops), ctypes.byref(peak_ms))
    if pst != 0:
        raise SystemExit(f"ccnn_measure_fp32_peak failed: {_capi.last_error()}")
    fp32_peak = peak_ops.value / 1e12
    achieved_tops = ops / (ms * 1e-3) / 1e12
    traffic = dram_traffic().get(dom)
    fb_frame = frame_bytes(levels, W, H)
    roofline = {
        "kernel": dom, "bound": "fp32", "achieved": round(achieved_tops, 3), "peak": round(fp32_peak, 3), "unit": "TFLOP/s",
        "frac": round(achieved_tops / fp32_peak, 4),
        "peak_source": ("measured in this run: ccnn_measure_fp32_peak (packed add.rn.f32x2 / fma.rn.f32x2 with a -0 addend, "
                        "eight independent chains a thread, every SM busy), best of 5 launches"),
        "peak_clocks": pclk.summary(),
        "ops_note": ("fp32 lane operations (each IEEE multiply, add and activation step once; the exact arithmetic issues no "
                     "fused multiply-add) per launch / CUDA-event time of the launch"),
        "ops_per_launch": ops, "kernel_ms": round(ms, 4),
        "traffic": traffic, "algorithmic_bytes_per_launch": by,
        "hbm": {"achieved": round(achieved_gbs, 2), "peak": hbm_peak, "unit": "GB/s", "frac": round(achieved_gbs / hbm_peak, 4),
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback 6650 GB/s"},
        "frame_hbm": {"bytes_per_frame": fb_frame, "achieved": round(value / world * fb_frame / 1e9, 2), "unit": "GB/s",
                      "frac": round(value / world * fb_frame / (hbm_peak * 1e9), 5),
                      "note": "whole-frame algorithmic bytes (BGR read, gray write, gray samples of every level pixel, S1 planes and response maps written and read) "
                              "x frames/s"},
        "frame_fp32": {"ops_per_frame": work["stage1_front"][0] + work["stage1_back"][0],
                       "achieved": round(value / world * (work["stage1_front"][0] + work["stage1_back"][0]) / 1e12, 3),
                       "unit": "T lane ops/s",
                       "frac": round(value / world * (work["stage1_front"][0] + work["stage1_back"][0]) / 1e12 / fp32_peak, 4),
                       "note": "the pipeline's stage-1 fp32 lane operations (front + back, per the formula in algorithmic_work) x "
                               "frames/s per GPU against the same measured ceiling: the whole frame stream, not one launch"},
        "single_launch_stage1": ({"ms": round(single_launch_ms, 4),
                                  "achieved": round((work["stage1_front"][0] + work["stage1_back"][0]) / (single_launch_ms * 1e-3) / 1e12, 3),
                                  "frac": round((work["stage1_front"][0] + work["stage1_back"][0]) / (single_launch_ms * 1e-3) / 1e12 / fp32_peak, 4),
                                  "note": "the pyramid and stage 1 of the frame as one persistent launch (the batched form's kernel on one "
                                          "frame): front + back fp32 lane operations / its event time, same ceiling"}
                                 if single_launch_ms > 0 else None),
        "latency_kernel": {"kernel": "replay_merge", "ms": round(kernel_ms["replay_merge"], 4),
                           "note": "one block per frame (sequential reference semantics); it overlaps other frames' kernels in "
                                   "the slot pipeline, so it sets single-frame latency rather than throughput"},
        "kernel_ms_all": {k: round(v, 4) for k, v in kernel_ms.items()},
    }
    fb = fb_frame

    # ---- batched+gated: the same frames with the learned gate in front of stage 1 ----
    gated = None
    from compactcnncascade_b200 import gate as gate_mod
    if not args.no_gate and os.path.exists(gate_mod.WEIGHTS_1080P):
        meta = gate_mod.load_meta()
        thr = args.gate_threshold if args.gate_threshold is not None else meta.get("operating_threshold", 0.1)
        plain_boxes = [det.Detect(f) for f in frames]
        # the autotuner's schedule for the gated workload, when tuned (the plain one otherwise)
        g_sched = autotune.lookup(p, gated=True) if args.schedule == "auto" else None
        if g_sched:
            autotune.set_schedule(det, g_sched)
        g_schedule = dict(autotune.get_schedule(det), source="autotuner table, gated entry" if g_sched else "same as plain")
        det.setGate(gate_mod.load(), thr, args.gate_fallback)
        margin = args.gate_margin if args.gate_margin is not None else meta.get("operating_margin", 16)
        det.setGateMargin(margin)
        hit = tot = 0
        tiles = np.zeros(5)
        for f, ref_boxes in zip(frames, plain_boxes):
            h_, t_ = gate_mod.box_recall(ref_boxes, det.Detect(f))
            hit, tot = hit + h_, tot + t_
            tiles += np.array(det.gateStats())
        for s in range(args.warmup):
            device_step(s)
        barrier()
        with ClockSampler(dev) as gclk:
            g_ms = 0.0
            torch.cuda.nvtx.range_push("gated")
            for s in range(args.steps):
                g_ms += device_step(args.warmup + s)
            torch.cuda.nvtx.range_pop()
            barrier()
        g_wall_e2e = None
        for s in range(args.warmup):
            host_step(s)
        barrier()
        t0 = time.perf_counter()
        for s in range(args.steps):
            host_step(args.warmup + s)
        barrier()
        g_wall_e2e = time.perf_counter() - t0
        g_t = g_ms / 1e3
        if dist:  # the slowest rank sets the job's time, as for `value`
            t = torch.tensor([g_t, g_wall_e2e], device=f"cuda:{dev}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            g_t, g_wall_e2e = float(t[0]), float(t[1])
        g_value = args.steps * B * world / g_t
        g_e2e = args.steps * B * world / g_wall_e2e
        glat = []
        for i in range(args.latency_frames):
            t = h_frames[i % len(frames)]
            im = _capi.Image(W, H, 3, t.data_ptr(), W * 3)
            t0 = time.perf_counter()
            L.ccnn_detect(det._h, ctypes.byref(im), one, cap, ctypes.byref(n1))
            glat.append((time.perf_counter() - t0) * 1e3)
        glat = np.array(glat[min(5, len(glat) - 1):])
        gk = (ctypes.c_float * (len(KERNELS) + 1))()
        L.ccnn_profile_last_frame(det._h, args.profile_iters, gk, len(KERNELS) + 1)
        # recall on a larger sample: further seeded frames (rendered on the device), outside the timing
        extra = None
        if args.recall_frames > 0:
            extra = gate_mod.evaluate(det, range(RECALL_SEED0, RECALL_SEED0 + args.recall_frames), gate_mod.load(), [thr],
                                      args.gate_fallback, margin=margin)[0]
        det.disableGate()
        if g_sched:
            autotune.set_schedule(det, schedule)
        gated = {"value": round(g_value, 2), "unit": "frames/s", "speedup_vs_plain": round(g_value / value, 3),
                 "e2e": round(g_e2e, 2), "e2e_speedup_vs_plain": round(g_e2e / e2e, 3),
                 "p50_ms": round(float(np.percentile(glat, 50)), 3), "p99_ms": round(float(np.percentile(glat, 99)), 3),
                 "box_recall": round((hit + (round(extra["box_recall"] * extra["boxes"]) if extra else 0)) /
                                     max(1, tot + (extra["boxes"] if extra else 0)), 4),
                 "boxes": tot + (extra["boxes"] if extra else 0), "recall_frames": len(frames) + (args.recall_frames if extra else 0),
                 "recall_timed_frames": {"frames": len(frames), "box_recall": round(hit / max(1, tot), 4), "boxes": tot},
                 "recall_sample": ({"frames": args.recall_frames, "seeds": [RECALL_SEED0, RECALL_SEED0 + args.recall_frames],
                                    "box_recall": round(extra["box_recall"], 4), "boxes": extra["boxes"],
                                    "frames_all_boxes": extra["frames_all_boxes"], "back_tiles_run": round(extra["back_tiles_run"], 4)}
                                   if extra else None),
                 "threshold": thr, "margin": margin,
                 "fallback_fraction": args.gate_fallback,
                 "front_tiles_run": round(tiles[0] / max(1, tiles[1]), 4), "back_tiles_run": round(tiles[2] / max(1, tiles[3]), 4),
                 "fallback_frames": int(tiles[4]), "clocks": gclk.summary(), "schedule": g_schedule,
                 "kernel_ms_all": dict({KERNELS[i]: round(float(gk[i]), 4) for i in range(len(KERNELS))},
                                       gate=round(float(gk[len(KERNELS)]), 4)),
                 "weights": {k: meta.get(k) for k in ("train_frames", "epochs", "eval_frames")},
                 "note": "same frames, detector and batch as `value`, with the learned gate (include/ccnn_gate.h) skipping "
                         "stage-1 tiles; box recall = plain-cascade boxes matched by a gated box at IoU >= 0.5, over the timed "
                         "frames and the further seeded sample together (each also given alone); `heldout` is the gate's own "
                         "1,000-frame evaluation"}

    batched = run_batched_pyramid(dev, args) if (rank == 0 and args.batched_frames > 0) else None
    serving = run_serving(sframes, args.serve_rate, args.serve_frames) if sframes else None
    serving_gated = None
    if serving and gated:
        serving_gated = run_serving(sframes, args.serve_rate, args.serve_frames,
                                    gate=(gate_mod.load(), gated["threshold"], args.gate_fallback, gated["margin"]))

    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "frames/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_dev / args.steps * 1e3, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator; no public frames available)",
        "config": {"workload": WORKLOAD, "frames_per_step": B, "distinct_frames": len(frames),
                   "l2": f"inputs larger than L2: {len(frames)} distinct frames x {W * H * 3 / 1e6:.1f} MB cycled",
                   "parallelism": f"replicas x{world}", "levels": len(levels),
                   "schedule": dict(schedule, source=sched_src or ("autotuner table (compactcnncascade_b200/schedules.json)"
                                                                   if (args.schedule == "auto" and autotune.lookup(p)) else "defaults")),
                   "stage1_candidates_last_frame": len(cands), "faces_per_frame": round(faces_total / (args.steps * B), 2)},
        "p50_ms": round(float(np.percentile(lat, 50)), 3),
        "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "hbm_frac_frame_bytes": round(value / world * fb / (hbm_peak * 1e9), 5),
        "clocks": clocks,
        "e2e": {"value": round(e2e, 2), "unit": "frames/s", "h2d_gbs": round(e2e * W * H * 3 / 1e9, 2),
                "bound_note": "host frames cross PCIe: h2d_gbs is the upload rate this throughput implies",
                "h2d_bytes_per_step": B * W * H * 3,
                "d2h_bytes_per_step": B * (4 + 1024 * 20)},
        "gpu_launches": args.steps * launches_per_frames(B, len(levels), schedule.get("batch_frames", 0)),
        "roofline": roofline,
        "wall_value": round(frames_timed / wall_dev, 2),
    }
    if gated:
        line["gated"] = gated
    if batched:
        line["batched_pyramid"] = batched
    rec = committed_records()
    if gated and rec.get("gate_heldout"):
        gated["heldout"] = rec["gate_heldout"]
    if serving:
        line["serving"] = dict(serving, note="serving loop (ccnn_server_*): Poisson arrivals of mixed 640x480/1280x720/"
                                             "1920x1080/3840x2160 frames at 30/30/30/10 %, latency = submit to result")
    if serving and rec.get("serving_sweep"):
        line["serving"]["sweep"] = rec["serving_sweep"]
    if serving_gated:
        line["serving"]["gated"] = dict(serving_gated, note="the same stream with the learned gate on in every resolution "
                                                            "class (weights trained at 1080p; recall measured at 1080p only)")
    if cpu:
        fps, workers, nfr, secs, fast = cpu
        line["cpu_baseline"] = {"value": round(fps, 3), "unit": "frames/s", "cores": workers, "kind": "reference",
                                "sample": f"{nfr} detections of the same workload ({args.cpu_frames} per core over 2 distinct frames, "
                                          f"one process per core), reference plain-C++ cascade "
                                          f"({'-O2 -ffast-math as shipped' if fast else 'strict IEEE build'}), {secs:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    det.Clear()
    if dist:
        dist.destroy_process_group()


def run_reference(args, world, rank):
    """The reference's own CPU cascade on all host cores (rank 0 only): each step is one frame
    per host core; one detector process per core runs W untimed and K timed steps."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"}))
        return
    res = reference_cpu(runs_per_worker=args.steps, warmup=max(1, args.warmup), distinct=2, seed0=20_000)
    v, workers, total_frames, t, fast = res
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)", "config": {"workload": WORKLOAD, "frames_per_step": workers,
                                                               "parallelism": f"{workers} host processes"},
            "cpu_baseline": {"value": round(v, 3), "unit": "frames/s", "cores": workers, "kind": "reference",
                             "sample": f"{total_frames} detections, one frame per host core per step over 2 distinct frames per core, "
                                       f"reference plain-C++ cascade ({'-O2 -ffast-math as shipped' if fast else 'strict IEEE build'}), "
                                       f"{t:.1f} s"},
            "e2e": {"value": round(v, 3), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
