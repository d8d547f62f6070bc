"""Test infrastructure only: ctypes access to the reference's own CPU path.

oracle/_ref/libccnn_ref.so (strict IEEE build) and libccnn_ref_fast.so (the reference's shipped
-O2 -ffast-math flags) are compiled by oracle/Makefile from the unmodified reference sources plus
oracle/ref_harness.cpp. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may use this module; it is the checker, never the measured or shipped path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_STRICT = os.path.join(HERE, "_ref", "libccnn_ref.so")
REF_FAST = os.path.join(HERE, "_ref", "libccnn_ref_fast.so")
REF_LEGACY = os.path.join(HERE, "_ref", "libccnn_ref_legacy.so")
MODELS = os.path.join(HERE, "..", "compactcnncascade_b200", "models")


class RefParams(ctypes.Structure):
    _fields_ = [("max_image_w", ctypes.c_int), ("max_image_h", ctypes.c_int), ("min_face_height", ctypes.c_int),
                ("max_face_height", ctypes.c_int), ("scale_factor", ctypes.c_float), ("min_neighbors", ctypes.c_int),
                ("detect_precision", ctypes.c_int), ("treshold", ctypes.c_float * 3), ("drop_detect", ctypes.c_int),
                ("equalize", ctypes.c_int), ("reflection", ctypes.c_int), ("detect_mode", ctypes.c_int)]


class RefFace(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("score", ctypes.c_float), ("gender", ctypes.c_int), ("smile", ctypes.c_int), ("glasses", ctypes.c_int)]


class RefDet(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("score", ctypes.c_float), ("scale", ctypes.c_float), ("knn", ctypes.c_int), ("num_detect", ctypes.c_int)]


def available(fast=False):
    return os.path.exists(REF_FAST if fast else REF_STRICT)


_libs = {}


def load(fast=False):
    path = REF_FAST if fast else REF_STRICT
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (oracle/Makefile needs the reference sources)")
        L = ctypes.CDLL(path)
        vp, ci, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        L.ref_gray.argtypes = [vp, ci, ci, ci, ci, vp]
        L.ref_resize_f32.argtypes = [vp, ci, ci, ci, vp, ci, ci, ci]
        L.ref_resize_u8.argtypes = [vp, ci, ci, ci, vp, ci, ci, ci]
        L.ref_equalize.argtypes = [vp, ci, ci]
        L.ref_net_forward.argtypes = [ctypes.c_char_p, ci, vp, ci, ci, ci, vp, ci, P(ci), P(ci)]
        L.ref_face_detect.argtypes = [P(RefParams), vp, ci, ci, ci, ci, P(RefDet), ci]
        if hasattr(L, "ref_cnn_detect"):
            from compactcnncascade_b200._capi import CnnAdvancedParam, CnnParam
            L.ref_cnn_detect.argtypes = [P(CnnParam), P(CnnAdvancedParam), vp, ci, ci, ci, ci, P(RefDet), ci, P(RefDet), ci,
                                         P(CnnParam), P(CnnAdvancedParam)]
        L.ref_face_detect_fa.argtypes = [P(RefParams), vp, ci, ci, ci, ci, P(RefFace), ci]
        L.ref_cntk_dump2binary.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_api_init.argtypes = [P(RefParams)]
        L.ref_api_detect.argtypes = [vp, ci, ci, ci, ci, P(RefDet), ci]
        L.ref_detect_steps.argtypes = [P(RefParams), vp, ci, ci, ci, ci,
                                       vp, P(ci), P(ci),
                                       ci, P(ci), vp, vp, vp,
                                       vp, ctypes.c_long,
                                       vp, vp, vp, ctypes.c_long,
                                       P(RefDet), ci, P(ci),
                                       P(RefDet), ci]
        L.ref_sort_by_scale_desc.argtypes = [vp, ci, vp]
        L.ref_merger.argtypes = [P(RefDet), ci, ctypes.c_float, ci, P(RefDet), ci]
        _libs[path] = L
    return _libs[path]


def params(min_face=40, max_face=240, scale_factor=1.15, max_w=1920, max_h=1080, precision=3, thr=(-1.5, -1.25, -1.0),
           min_neighbors=2, drop_detect=1, equalize=1, reflection=1, detect_mode=1):
    return RefParams(max_w, max_h, min_face, max_face, scale_factor, min_neighbors, precision,
                     (ctypes.c_float * 3)(*thr), drop_detect, equalize, reflection, detect_mode)


def gray(img):
    L = load()
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    out = np.empty((h, w), np.float32)
    rc = L.ref_gray(img.ctypes.data, w, h, ch, img.strides[0], out.ctypes.data)
    assert rc == 0
    return out


def resize_f32(src, dw, dh, type_):
    L = load()
    src = np.ascontiguousarray(src, np.float32)
    out = np.empty((dh, dw), np.float32)
    L.ref_resize_f32(src.ctypes.data, src.shape[1], src.shape[0], src.shape[1], out.ctypes.data, dw, dh, type_)
    return out


def net_forward(stage, img, index_output):
    L = load()
    img = np.ascontiguousarray(img, np.float32)
    out = np.empty(img.size, np.float32)
    ow, oh = ctypes.c_int(), ctypes.c_int()
    path = os.path.join(MODELS, f"cnn4face{stage}_cntk.bin").encode()
    rc = L.ref_net_forward(path, index_output, img.ctypes.data, img.shape[1], img.shape[0], img.shape[1], out.ctypes.data,
                           out.size, ctypes.byref(ow), ctypes.byref(oh))
    if rc != 0:
        raise RuntimeError(f"ref_net_forward failed ({rc})")
    return out[: ow.value * oh.value].reshape(oh.value, ow.value)


def face_detect(img, p, fast=False):
    L = load(fast)
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    out = (RefDet * 65536)()
    n = L.ref_face_detect(ctypes.byref(p), img.ctypes.data, w, h, ch, img.strides[0], out, 65536)
    if n < 0:
        raise RuntimeError(f"ref_face_detect failed ({n})")
    return [(d.x, d.y, d.w, d.h, d.score) for d in out[:n]]


def cnn_detect(img, p, ap, prior=()):
    """The reference's own CNNDetector(&param, &advanced_param) + Detect(detections, image) with `prior`
    (tuples x, y, w, h, score, scale, knn, num_detect) already in the vector. `p` / `ap` are
    ccnn_cnn_param / ccnn_cnn_advanced_param structures (the harness shares their layout). Returns
    (detections, param after, advanced param after)."""
    from compactcnncascade_b200._capi import CnnAdvancedParam, CnnParam
    L = load()
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    img = np.ascontiguousarray(img)
    pr = (RefDet * max(1, len(prior)))(*[RefDet(*d) for d in prior])
    out = (RefDet * 65536)()
    pa, apa = CnnParam(), CnnAdvancedParam()
    n = L.ref_cnn_detect(ctypes.byref(p), ctypes.byref(ap), img.ctypes.data, w, h, ch, img.strides[0], pr, len(prior), out, 65536,
                         ctypes.byref(pa), ctypes.byref(apa))
    if n < 0:
        raise RuntimeError(f"ref_cnn_detect failed ({n})")
    return [(d.x, d.y, d.w, d.h, d.score, d.scale, d.knn, d.num_detect) for d in out[:n]], pa, apa


def merger(dets, threshold, delete=False):
    """The reference Merger (cnn_detector_v3.cpp:2814-2936) on a list of (x, y, w, h, score, scale, knn, num_detect)."""
    L = load()
    inp = (RefDet * max(1, len(dets)))(*[RefDet(*d) for d in dets])
    out = (RefDet * max(1, len(dets)))()
    n = L.ref_merger(inp, len(dets), threshold, 1 if delete else 0, out, len(dets))
    return [(d.x, d.y, d.w, d.h, d.score, d.scale, d.knn, d.num_detect) for d in out[:n]]


def face_detect_fa(img, p, fast=False):
    """The reference's public Detect with facial analysis on: (x, y, w, h, score, gender, smile, glasses)."""
    L = load(fast)
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    out = (RefFace * 65536)()
    n = L.ref_face_detect_fa(ctypes.byref(p), img.ctypes.data, w, h, ch, img.strides[0], out, 65536)
    if n < 0:
        raise RuntimeError(f"ref_face_detect_fa failed ({n})")
    return [(d.x, d.y, d.w, d.h, d.score, d.gender, d.smile, d.glasses) for d in out[:n]]


def cntk_dump2binary(binary_file, dump_file):
    """The reference's FaceDetector::CNTKDump2Binary."""
    load().ref_cntk_dump2binary(binary_file.encode(), dump_file.encode())


def detect_steps(img, p, with_levels=True, resp_cap=None):
    """Replay of CNNDetector::Detect capturing gray, levels, response maps, raw and final detections.
    With `resp_cap` (floats for all response maps together, an upper bound) and no level images, the
    reference runs once instead of once more to size its outputs."""
    L = load()
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    img = np.ascontiguousarray(img)
    cap = 1024

    def run(lev_cap, resp_cap):
        r = {"gray": np.empty(h * w, np.float32), "gw": ctypes.c_int(), "gh": ctypes.c_int(), "nl": ctypes.c_int(),
             "scales": np.empty(cap, np.float32), "lw": np.empty(cap, np.int32), "lh": np.empty(cap, np.int32),
             "rw": np.empty(cap, np.int32), "rh": np.empty(cap, np.int32), "nraw": ctypes.c_int(),
             "raw": (RefDet * 400000)(), "fin": (RefDet * 65536)()}
        r["levels"] = np.empty(max(lev_cap, 1), np.float32) if lev_cap else None
        r["resp"] = np.empty(max(resp_cap, 1), np.float32) if resp_cap else None
        nf = L.ref_detect_steps(ctypes.byref(p), img.ctypes.data, w, h, ch, img.strides[0],
                                r["gray"].ctypes.data, ctypes.byref(r["gw"]), ctypes.byref(r["gh"]),
                                cap, ctypes.byref(r["nl"]), r["scales"].ctypes.data, r["lw"].ctypes.data, r["lh"].ctypes.data,
                                r["levels"].ctypes.data if lev_cap else None, lev_cap,
                                r["rw"].ctypes.data, r["rh"].ctypes.data, r["resp"].ctypes.data if resp_cap else None, resp_cap,
                                r["raw"], 400000, ctypes.byref(r["nraw"]), r["fin"], 65536)
        if nf < 0:
            raise RuntimeError(f"ref_detect_steps failed ({nf})")
        r["nf"] = nf
        return r

    if resp_cap is not None and not with_levels:
        r = run(0, int(resp_cap))
        nl = r["nl"].value
        if nl > cap or int(sum(int(r["rw"][i]) * int(r["rh"][i]) for i in range(nl))) > resp_cap:
            raise RuntimeError("ref_detect_steps: response capacity too small")
        return _steps_result(r, nl, with_levels)
    first = run(0, 0)
    nl = first["nl"].value
    lev_cap = int(sum(int(first["lw"][i]) * int(first["lh"][i]) for i in range(nl))) if with_levels else 0
    resp_cap = int(sum(int(first["rw"][i]) * int(first["rh"][i]) for i in range(nl)))
    r = run(lev_cap, resp_cap)
    return _steps_result(r, nl, with_levels)


def _steps_result(r, nl, with_levels):
    res = {"gray": r["gray"][: r["gw"].value * r["gh"].value].reshape(r["gh"].value, r["gw"].value), "levels": [], "resp": []}
    lo = ro = 0
    for i in range(nl):
        W, H = int(r["lw"][i]), int(r["lh"][i])
        lvl = np.array(r["levels"][lo: lo + W * H]).reshape(H, W) if with_levels else None
        res["levels"].append((W, H, float(r["scales"][i]), lvl))
        lo += W * H
        RW, RH = int(r["rw"][i]), int(r["rh"][i])
        res["resp"].append(np.array(r["resp"][ro: ro + RW * RH]).reshape(RH, RW))
        ro += RW * RH
    res["raw"] = [(d.x, d.y, d.w, d.h, d.score, d.scale, d.knn, d.num_detect) for d in r["raw"][: r["nraw"].value]]
    res["final"] = [(d.x, d.y, d.w, d.h, d.score) for d in r["fin"][: r["nf"]]]
    return res


def sort_perm(keys):
    L = load()
    keys = np.ascontiguousarray(keys, np.float32)
    perm = np.empty(len(keys), np.int32)
    L.ref_sort_by_scale_desc(keys.ctypes.data, len(keys), perm.ctypes.data)
    return perm


# ---- legacy model family (format 1.0, the `_new.bin` networks) ----

def legacy_available():
    return os.path.exists(REF_LEGACY)


def legacy_net_forward(model_path, img):
    """Response map of the reference's legacy network (SIMD::ConvNeuralNetwork of
    src/CNNObjectDetector/cnn_simd.cpp, plain-C++ build) on a float32 H x W image, in this process.
    The model is passed as its bytes: the legacy reader cannot open a path (its file stream shadows
    the stream it parses, cnn_simd.cpp:40-60)."""
    if REF_LEGACY not in _libs:
        L = ctypes.CDLL(REF_LEGACY)
        ci, vp, P = ctypes.c_int, ctypes.c_void_p, ctypes.POINTER
        L.ref_net_forward_bytes.argtypes = [ctypes.c_char_p, ci, vp, ci, ci, ci, vp, ci, P(ci), P(ci)]
        _libs[REF_LEGACY] = L
    L = _libs[REF_LEGACY]
    with open(model_path, "rb") as f:
        blob = f.read()
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape
    out = np.zeros(w * h, np.float32)
    ow, oh = ctypes.c_int(), ctypes.c_int()
    r = L.ref_net_forward_bytes(blob, len(blob), a.ctypes.data, w, h, w, out.ctypes.data, out.size, ctypes.byref(ow), ctypes.byref(oh))
    if r != 0:
        raise RuntimeError(f"reference legacy forward failed ({r})")
    return out[: ow.value * oh.value].reshape(oh.value, ow.value)


def legacy_net_forward_isolated(model_path, img):
    """legacy_net_forward in a fresh process. The reference's fully connected 24-map route keeps the
    pointers of the first network that ran it in a function-local static (mulC24_add_tanh call,
    cnn_simd.cpp:806-809), so in one process only the first network instance computes correctly."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(1, maxtasksperchild=1) as pool:
        return pool.apply(legacy_net_forward, (model_path, img))


def _legacy_face_detect_worker(img, pargs):
    L = ctypes.CDLL(REF_LEGACY)
    L.ref_face_detect.argtypes = [ctypes.POINTER(RefParams), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(RefDet), ctypes.c_int]
    p = params(**pargs)
    a = np.ascontiguousarray(img)
    h, w = a.shape[:2]
    ch = 1 if a.ndim == 2 else a.shape[2]
    out = (RefDet * 65536)()
    n = L.ref_face_detect(ctypes.byref(p), a.ctypes.data, w, h, ch, a.strides[0], out, 65536)
    if n < 0:
        raise RuntimeError(f"ref_face_detect (legacy) failed ({n})")
    return [(d.x, d.y, d.w, d.h, d.score) for d in out[:n]]


def legacy_face_detect(img, **pargs):
    """The reference's public FaceDetector::Detect built for the legacy model family (its embedded
    cnn4face{1,2,3}_new.bin), in a fresh process for the reason given at legacy_net_forward_isolated.
    pargs are params() keywords."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(1, maxtasksperchild=1) as pool:
        return pool.apply(_legacy_face_detect_worker, (img, pargs))
