"""B200-native face-detection cascade (Compact CNN Cascade, arXiv:1508.01292).

`FaceDetector` mirrors the reference's public class CompactCNNLib::FaceDetector
(src/CNNObjectDetector/CompactCNNLibAPI_v2.h:35-190): the same method names, parameter fields and
return conventions (Init/Detect/Clear return 0 or the face count, -1 on error). Every call goes
through the C ABI in include/ccnn.h to hand-written sm_100a kernels; nothing runs on the CPU.
"""
import ctypes

import numpy as np

from . import _capi
from ._capi import CCNNError, Face, Image, Params

__all__ = ["FaceDetector", "FaceServer", "Param", "synth_frame", "synth_frame_device", "CCNNError", "default_params", "pinned_frame"]

Pipeline = {"CPU": 0, "GPU": 1, "GPU_CPU": 2}
DetectMode = {"disable": 0, "sync": 1, "async": 2}
DetectPrecision = {"def": 0, "low": 1, "normal": 2, "high": 3, "ultra": 4}


def default_params():
    """FaceDetector::Param defaults (CompactCNNLibAPI_v2.h:97-161)."""
    p = Params()
    _capi.lib().ccnn_default_params(ctypes.byref(p))
    return p


Param = default_params


def _as_image(img):
    a = np.ascontiguousarray(img) if not img.flags["C_CONTIGUOUS"] else img
    if a.dtype != np.uint8 or a.ndim not in (2, 3):
        raise ValueError("image must be a uint8 HxW or HxWxC array")
    ch = 1 if a.ndim == 2 else a.shape[2]
    im = Image(a.shape[1], a.shape[0], ch, a.ctypes.data, a.strides[0])
    return im, a


class FaceDetector:
    """CompactCNNLib::FaceDetector over the B200 path; one handle per instance (no global singleton)."""

    def __init__(self):
        self._h = None
        self._param = None
        self._models = [None, None, None]

    # ---- lifecycle ----
    def Init(self, param=None, models=None, schedule=None):
        """FaceDetector::Init (CompactCNNLibAPI_v2.cpp:373-407). Returns 0 or -1. `schedule`:
        None (defaults), "auto" (the autotuner's entry for these parameters, when it has one) or a
        dict of schedule knobs (compactcnncascade_b200.autotune.KNOBS)."""
        if self._h is not None:
            self.Clear()
        self._param = param if param is not None else default_params()
        if models is not None:
            self._models = list(models)
        arr = (ctypes.c_char_p * 3)(*[(m.encode() if m else None) for m in self._models])
        h = ctypes.c_void_p()
        st = _capi.lib().ccnn_create(ctypes.byref(self._param), arr, ctypes.byref(h))
        if st != _capi.OK:
            self.last_status = st
            return -1
        self._h = h
        if schedule is not None:
            from . import autotune
            sched = autotune.lookup(self._param) if schedule == "auto" else dict(schedule)
            if sched is not None:
                autotune.set_schedule(self, sched)
        return 0

    def Clear(self):
        if self._h is None:
            return -1
        _capi.lib().ccnn_destroy(self._h)
        self._h = None
        return 0

    def isEmpty(self):
        return self._h is None

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass

    # ---- detection ----
    def Detect(self, img, capacity=4096, attributes=False):
        """FaceDetector::Detect: returns a list of (x, y, width, height, score), with
        (gender, smile, glasses) appended when `attributes` (set by facial analysis, else -1)."""
        if self._h is None:
            raise CCNNError(_capi.ERR_INVALID_ARG, "Detect (detector not initialised)")
        im, _keep = _as_image(img)
        faces = (Face * capacity)()
        n = ctypes.c_int(0)
        st = _capi.lib().ccnn_detect(self._h, ctypes.byref(im), faces, capacity, ctypes.byref(n))
        _capi.check(st, "ccnn_detect")
        if attributes:
            return [(f.x, f.y, f.width, f.height, f.score, f.gender, f.smile, f.glasses) for f in faces[: min(n.value, capacity)]]
        return [(f.x, f.y, f.width, f.height, f.score) for f in faces[: min(n.value, capacity)]]

    def DetectBatch(self, imgs, capacity=4096):
        """Several frames of one size through the pipelined batch entry point."""
        if not imgs:
            return []
        keep = []
        arr = (Image * len(imgs))()
        for i, img in enumerate(imgs):
            im, a = _as_image(img)
            arr[i] = im
            keep.append(a)
        faces = (Face * (capacity * len(imgs)))()
        ns = (ctypes.c_int * len(imgs))()
        st = _capi.lib().ccnn_detect_batch(self._h, arr, len(imgs), faces, capacity, ns)
        _capi.check(st, "ccnn_detect_batch")
        out = []
        for i in range(len(imgs)):
            fs = faces[i * capacity: i * capacity + min(ns[i], capacity)]
            out.append([(f.x, f.y, f.width, f.height, f.score) for f in fs])
        return out

    def DetectDevice(self, data_ptr, width, height, channels, step, stream=None, capacity=4096):
        """Detect on a frame already in device memory (uint8, interleaved, row pitch `step` bytes)."""
        if self._h is None:
            raise CCNNError(_capi.ERR_INVALID_ARG, "DetectDevice (detector not initialised)")
        im = Image(width, height, channels, data_ptr, step)
        faces = (Face * capacity)()
        n = ctypes.c_int(0)
        st = _capi.lib().ccnn_detect_device(self._h, ctypes.byref(im), stream, faces, capacity, ctypes.byref(n))
        _capi.check(st, "ccnn_detect_device")
        return [(f.x, f.y, f.width, f.height, f.score) for f in faces[: min(n.value, capacity)]]

    # ---- learned gate (include/ccnn_gate.h) ----
    def setGate(self, params, threshold=0.5, fallback_fraction=0.25):
        """Skips stage-1 tiles that the gate network (700 fp32 parameters) finds unlikely."""
        p = np.ascontiguousarray(params, np.float32)
        _capi.check(_capi.lib().ccnn_gate_set(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size, float(threshold),
                                              float(fallback_fraction)), "ccnn_gate_set")

    def setGateMargin(self, pixels):
        """Pixels (0-64, default 16) around a candidate's window centre the gate searches for a likely cell."""
        _capi.check(_capi.lib().ccnn_gate_set_margin(self._h, int(pixels)), "ccnn_gate_set_margin")

    def disableGate(self):
        _capi.check(_capi.lib().ccnn_gate_disable(self._h), "ccnn_gate_disable")

    def gateStats(self):
        """(front tiles run, front tiles, back tiles run, back tiles, fell back) of the last frame."""
        v = [ctypes.c_int() for _ in range(5)]
        _capi.check(_capi.lib().ccnn_gate_stats(self._h, *[ctypes.byref(x) for x in v]), "ccnn_gate_stats")
        return tuple(x.value for x in v)

    def gateProbabilities(self):
        """The learned gate's probabilities of the last frame, shape (4, rows // 16, cols // 16)."""
        n = ctypes.c_int()
        _capi.check(_capi.lib().ccnn_gate_probabilities(self._h, None, 0, ctypes.byref(n)), "ccnn_gate_probabilities")
        out = np.empty(n.value, np.float32)
        _capi.check(_capi.lib().ccnn_gate_probabilities(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n.value,
                                                        ctypes.byref(n)), "ccnn_gate_probabilities")
        _, gw, gh, _ = self.grayDevice()
        return out.reshape(4, (gh // 8) // 2, (gw // 8) // 2)

    def grayDevice(self):
        """(device pointer, cols, rows, step in bytes) of the last frame's fp32 gray image."""
        ptr, w, h, step = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        _capi.check(_capi.lib().ccnn_get_gray_device(self._h, ctypes.byref(ptr), ctypes.byref(w), ctypes.byref(h), ctypes.byref(step)),
                    "ccnn_get_gray_device")
        return ptr.value, w.value, h.value, step.value

    # ---- parameters ----
    def getParam(self):
        p = Params()
        _capi.check(_capi.lib().ccnn_get_params(self._h, ctypes.byref(p)), "ccnn_get_params")
        return p

    def setParam(self, param):
        _capi.check(_capi.lib().ccnn_set_params(self._h, ctypes.byref(param)), "ccnn_set_params")

    def getMaxImageSize(self):
        p = self.getParam()
        return (p.max_image_width, p.max_image_height)

    def setMaxImageSize(self, size):
        _capi.check(_capi.lib().ccnn_set_max_image_size(self._h, int(size[0]), int(size[1])), "ccnn_set_max_image_size")

    def getMinObjectHeight(self):
        return self.getParam().min_face_height

    def setMinObjectHeight(self, v):
        _capi.check(_capi.lib().ccnn_set_min_object_height(self._h, int(v)), "ccnn_set_min_object_height")

    def getMaxObjectHeight(self):
        return self.getParam().max_face_height

    def setMaxObjectHeight(self, v):
        _capi.check(_capi.lib().ccnn_set_max_object_height(self._h, int(v)), "ccnn_set_max_object_height")

    def getNumThreads(self):
        return self.getParam().num_threads

    def setNumThreads(self, v):
        _capi.check(_capi.lib().ccnn_set_num_threads(self._h, int(v)), "ccnn_set_num_threads")

    def getGrayImage32F(self):
        """The fp32 gray image of the last frame, copied to a numpy array."""
        w, h = ctypes.c_int(), ctypes.c_int()
        p = self.getParam()
        out = np.empty(p.max_image_width * p.max_image_height, np.float32)
        _capi.check(_capi.lib().ccnn_get_gray_host(self._h, out.ctypes.data, out.size, ctypes.byref(w), ctypes.byref(h)),
                    "ccnn_get_gray_host")
        return out[: w.value * h.value].reshape(h.value, w.value)

    @staticmethod
    def CNTKDump2Binary(binary_file, cntk_model_dump):
        """FaceDetector::CNTKDump2Binary: converts a CNTK text dump into a binary model file
        (".bin" appended when missing). Raises on a malformed dump."""
        _capi.check(_capi.lib().ccnn_cntk_dump_to_binary(binary_file.encode(), cntk_model_dump.encode()), "ccnn_cntk_dump_to_binary")

    # ---- inspection (include/ccnn_inspect.h) ----
    def levels(self):
        L = _capi.lib()
        buf = (_capi.LevelInfo * 512)()
        n = ctypes.c_int()
        _capi.check(L.ccnn_inspect_levels(self._h, buf, 512, ctypes.byref(n)), "ccnn_inspect_levels")
        return [(b.width, b.height, b.scale, b.resp_width, b.resp_height) for b in buf[: n.value]]

    def response_map(self, level):
        info = self.levels()[level]
        out = np.empty(info[3] * info[4], np.float32)
        _capi.check(_capi.lib().ccnn_inspect_response(self._h, level, out.ctypes.data, out.size), "ccnn_inspect_response")
        return out.reshape(info[4], info[3])

    def candidates(self):
        L = _capi.lib()
        n = ctypes.c_int()
        _capi.check(L.ccnn_inspect_candidates(self._h, None, 0, ctypes.byref(n)), "ccnn_inspect_candidates")
        buf = (_capi.CandidateInfo * max(1, n.value))()
        _capi.check(L.ccnn_inspect_candidates(self._h, buf, n.value, ctypes.byref(n)), "ccnn_inspect_candidates")
        return [(c.level, c.x, c.y, c.score, c.accepted, c.check_score, c.knn) for c in buf[: n.value]]

    def raw_detections(self):
        L = _capi.lib()
        n = ctypes.c_int()
        _capi.check(L.ccnn_inspect_raw_detections(self._h, None, 0, ctypes.byref(n)), "ccnn_inspect_raw_detections")
        buf = (_capi.Detection * max(1, n.value))()
        _capi.check(L.ccnn_inspect_raw_detections(self._h, buf, n.value, ctypes.byref(n)), "ccnn_inspect_raw_detections")
        return [(d.x, d.y, d.width, d.height, d.score, d.scale, d.knn, d.num_detect) for d in buf[: n.value]]


class FaceServer:
    """Serving loop over the B200 cascade (include/ccnn_server.h): submit frames of any resolution
    as they arrive, collect each result by ticket. Frames must stay alive (and unmodified) until
    their result has been taken; `pinned_frame` gives page-locked arrays that upload asynchronously."""

    def __init__(self, param=None, models=None, hbm_budget_bytes=0, slots_per_class=0, max_queue=0):
        L = _capi.lib()
        p = param if param is not None else default_params()
        cfg = _capi.ServerConfig(hbm_budget_bytes, slots_per_class, max_queue)
        arr = None
        if models is not None:
            arr = (ctypes.c_char_p * 3)(*[(m.encode() if m else None) for m in models])
        h = ctypes.c_void_p()
        _capi.check(L.ccnn_server_create(ctypes.byref(p), arr, ctypes.byref(cfg), ctypes.byref(h)), "ccnn_server_create")
        self._h = h
        self._frames = {}

    def close(self):
        if self._h:
            _capi.lib().ccnn_server_destroy(self._h)
            self._h = None
            self._frames.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_gate(self, params, threshold=0.5, fallback_fraction=0.25, margin=16):
        """The learned gate (FaceDetector.setGate, setGateMargin) for every resolution class; before the
        first submit."""
        p = np.ascontiguousarray(params, np.float32)
        _capi.check(_capi.lib().ccnn_server_set_gate(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size,
                                                     float(threshold), float(fallback_fraction)), "ccnn_server_set_gate")
        _capi.check(_capi.lib().ccnn_server_set_gate_margin(self._h, int(margin)), "ccnn_server_set_gate_margin")

    def submit(self, img):
        """Queues a uint8 HxW / HxWxC frame; returns its ticket, or None when the queue is full."""
        im, a = _as_image(img)
        t = ctypes.c_longlong()
        st = _capi.lib().ccnn_server_submit(self._h, ctypes.byref(im), ctypes.byref(t))
        if st == _capi.BUSY:
            return None
        _capi.check(st, "ccnn_server_submit")
        self._frames[t.value] = a  # keep the pixels alive until the result is taken
        return t.value

    def _take(self, fn, ticket, capacity):
        faces = (Face * capacity)()
        n = ctypes.c_int()
        lat = ctypes.c_double()
        st = fn(self._h, ticket, faces, capacity, ctypes.byref(n), ctypes.byref(lat))
        if st == _capi.PENDING:
            return None
        self._frames.pop(ticket, None)
        _capi.check(st, "ccnn_server result")
        return [(f.x, f.y, f.width, f.height, f.score) for f in faces[: min(n.value, capacity)]], lat.value

    def wait(self, ticket, capacity=4096):
        """(faces, latency_ms) of a ticket, blocking until the frame is done."""
        return self._take(_capi.lib().ccnn_server_wait, ticket, capacity)

    def poll(self, ticket, capacity=4096):
        """(faces, latency_ms) if the frame is done, else None."""
        return self._take(_capi.lib().ccnn_server_poll, ticket, capacity)

    def stats(self):
        s = _capi.ServerStats()
        _capi.check(_capi.lib().ccnn_server_stats_get(self._h, ctypes.byref(s)), "ccnn_server_stats_get")
        return {k: getattr(s, k) for k, _ in s._fields_}


class _PinnedBuffer:
    """Page-locked host bytes exposed to numpy; freed when the last array using them goes away."""

    def __init__(self, n):
        self._lib = _capi.lib()
        self.ptr = self._lib.ccnn_host_alloc(max(1, n))
        if not self.ptr:
            raise MemoryError("ccnn_host_alloc failed")
        self.__array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (self.ptr, False), "version": 3}

    def __del__(self):
        if getattr(self, "ptr", None):
            self._lib.ccnn_host_free(self.ptr)
            self.ptr = None


def pinned_frame(shape):
    """A uint8 array of `shape` in page-locked host memory."""
    n = int(np.prod(shape))
    return np.asarray(_PinnedBuffer(n)).reshape(shape)


def synth_frame_device(out_ptr, width, height, seed, n_faces, min_face, max_face, channels=3, step=None, stream=None):
    """The same seeded frame as `synth_frame`, rendered on the device into `out_ptr` (device
    memory, row pitch `step` bytes, default width * channels); returns the face patches."""
    faces = (_capi.SynthFace * max(1, n_faces))()
    st = _capi.lib().ccnn_synth_frame_device(out_ptr, width, height, channels, step or width * channels, seed, n_faces, min_face,
                                             max_face, faces, stream)
    _capi.check(st, "ccnn_synth_frame_device")
    return [(f.cx, f.cy, f.w, f.h, f.angle_deg, f.contrast) for f in faces[:n_faces]]


def synth_frame(width, height, seed, n_faces, min_face, max_face, channels=3):
    """Seeded synthetic frame (uint8 HxWxC, BGR order for 3 channels) and its face patches."""
    S = _capi.synth()
    shape = (height, width) if channels == 1 else (height, width, channels)
    img = np.empty(shape, np.uint8)
    faces = (_capi.SynthFace * max(1, n_faces))()
    st = S.ccnn_synth_frame(img.ctypes.data, width, height, channels, width * channels, seed, n_faces, min_face, max_face,
                            faces)
    if st < 0:
        raise ValueError(f"ccnn_synth_frame failed ({st})")
    return img, [(f.cx, f.cy, f.w, f.h, f.angle_deg, f.contrast) for f in faces[:n_faces]]
