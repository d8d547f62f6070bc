"""Test infrastructure only: ctypes access to oracle/liboracle.so, the CPU restatement of the
detection path (oracle/ccnn_oracle.cpp). Used as the checker by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline fallback; never the measured or shipped path."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
MODELS = os.path.normpath(os.path.join(HERE, "..", "compactcnncascade_b200", "models"))


class OrcParams(ctypes.Structure):
    _fields_ = [("max_image_w", ctypes.c_int), ("max_image_h", ctypes.c_int), ("min_face_height", ctypes.c_int),
                ("max_face_height", ctypes.c_int), ("scale_factor", ctypes.c_float), ("min_neighbors", ctypes.c_int),
                ("detect_precision", ctypes.c_int), ("treshold", ctypes.c_float * 3), ("drop_detect", ctypes.c_int),
                ("equalize", ctypes.c_int), ("reflection", ctypes.c_int), ("detect_mode", ctypes.c_int)]


class OrcDet(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int), ("score", ctypes.c_float),
                ("scale", ctypes.c_float), ("knn", ctypes.c_int), ("num_detect", ctypes.c_int)]


class OrcCand(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int), ("x", ctypes.c_int), ("y", ctypes.c_int), ("score", ctypes.c_float)]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
        L = ctypes.CDLL(LIB)
        vp, ci, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        L.orc_gray.argtypes = [vp, ci, ci, ci, ci, vp]
        L.orc_resize_f32.argtypes = [vp, ci, ci, ci, vp, ci, ci, ci]
        L.orc_equalize.argtypes = [vp, ci, ci]
        L.orc_net_forward.argtypes = [ctypes.c_char_p, ci, vp, ci, ci, ci, vp, ci, P(ci), P(ci)]
        L.orc_detect.argtypes = [P(OrcParams), ctypes.c_char_p, vp, ci, ci, ci, ci, vp, P(ci), P(ci), ci, P(ci), vp, vp, vp, vp,
                                 ctypes.c_long, vp, vp, P(OrcCand), ci, P(ci), P(OrcDet), ci, P(ci), P(OrcDet), ci]
        L.orc_sort_perm.argtypes = [vp, ci, vp]
        _lib = L
    return _lib


def params(min_face=40, max_face=240, scale_factor=1.15, max_w=1920, max_h=1080, precision=3, thr=(-1.5, -1.25, -1.0),
           min_neighbors=2, drop_detect=1, equalize=1, reflection=1, detect_mode=1):
    return OrcParams(max_w, max_h, min_face, max_face, scale_factor, min_neighbors, precision, (ctypes.c_float * 3)(*thr),
                     drop_detect, equalize, reflection, detect_mode)


def gray(img):
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    out = np.empty((h, w), np.float32)
    assert load().orc_gray(img.ctypes.data, w, h, ch, img.strides[0], out.ctypes.data) == 0
    return out


def resize_f32(src, dw, dh, type_):
    src = np.ascontiguousarray(src, np.float32)
    out = np.empty((dh, dw), np.float32)
    load().orc_resize_f32(src.ctypes.data, src.shape[1], src.shape[0], src.shape[1], out.ctypes.data, dw, dh, type_)
    return out


def net_forward(stage, img, index_output):
    img = np.ascontiguousarray(img, np.float32)
    out = np.empty(img.size, np.float32)
    ow, oh = ctypes.c_int(), ctypes.c_int()
    rc = load().orc_net_forward(os.path.join(MODELS, f"cnn4face{stage}_cntk.bin").encode(), index_output, img.ctypes.data,
                                img.shape[1], img.shape[0], img.shape[1], out.ctypes.data, out.size, ctypes.byref(ow),
                                ctypes.byref(oh))
    if rc != 0:
        raise RuntimeError(f"orc_net_forward failed ({rc})")
    return out[: ow.value * oh.value].reshape(oh.value, ow.value)


def detect(img, p=None, **kw):
    """Full detection with intermediates: gray, levels (w, h, scale), response maps, candidates,
    raw detections (reference order) and final boxes."""
    p = p or params(**kw)
    L = load()
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    img = np.ascontiguousarray(img)
    gray_out = np.empty(h * w, np.float32)
    gw, gh = ctypes.c_int(), ctypes.c_int()
    cap = 1024
    nl = ctypes.c_int()
    scales = np.empty(cap, np.float32)
    lw = np.empty(cap, np.int32)
    lh = np.empty(cap, np.int32)
    rw = np.empty(cap, np.int32)
    rh = np.empty(cap, np.int32)
    resp = np.empty(2 * w * h + 1024, np.float32)  # upsampled pyramids hold more response pixels than the frame
    ccap = w * h // 4 + 1024
    cands = (OrcCand * ccap)()
    nc = ctypes.c_int()
    raw = (OrcDet * ccap)()
    nraw = ctypes.c_int()
    fin = (OrcDet * 65536)()
    nf = L.orc_detect(ctypes.byref(p), MODELS.encode(), img.ctypes.data, w, h, ch, img.strides[0], gray_out.ctypes.data,
                      ctypes.byref(gw), ctypes.byref(gh), cap, ctypes.byref(nl), scales.ctypes.data, lw.ctypes.data,
                      lh.ctypes.data, resp.ctypes.data, resp.size, rw.ctypes.data, rh.ctypes.data, cands, ccap,
                      ctypes.byref(nc), raw, ccap, ctypes.byref(nraw), fin, 65536)
    if nf < 0:
        raise RuntimeError(f"orc_detect failed ({nf})")
    out = {"gray": gray_out[: gw.value * gh.value].reshape(gh.value, gw.value), "levels": [], "resp": []}
    ro = 0
    for i in range(nl.value):
        out["levels"].append((int(lw[i]), int(lh[i]), float(scales[i])))
        n = int(rw[i]) * int(rh[i])
        out["resp"].append(np.array(resp[ro: ro + n]).reshape(int(rh[i]), int(rw[i])))
        ro += n
    out["candidates"] = [(c.level, c.x, c.y, c.score) for c in cands[: nc.value]]
    out["raw"] = [(d.x, d.y, d.w, d.h, d.score, d.scale, d.knn, d.num_detect) for d in raw[: nraw.value]]
    out["final"] = [(d.x, d.y, d.w, d.h, d.score) for d in fin[:nf]]
    return out


def sort_perm(keys):
    keys = np.ascontiguousarray(keys, np.float32)
    perm = np.empty(len(keys), np.int32)
    load().orc_sort_perm(keys.ctypes.data, len(keys), perm.ctypes.data)
    return perm
