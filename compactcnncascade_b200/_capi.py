"""ctypes binding of the C ABI declared in include/ccnn.h, include/ccnn_inspect.h and
include/ccnn_server.h.

The shared library is built in-tree (compactcnncascade_b200/libccnn.so) by
compactcnncascade_b200/build.py. Loading fails loudly when it is missing: there is no
Python or CPU fallback for the detection path.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libccnn.so")
SYNTH_PATH = os.path.join(_HERE, "libccnn_synth.so")

# ccnn_status
OK = 0
TRUNCATED = 1
PENDING = 2
BUSY = 3
ERR_INVALID_ARG = -1
ERR_MODEL = -2
ERR_CONFIG = -3
ERR_CUDA = -4
ERR_OOM = -5
ERR_UNSUPPORTED = -6

EXPORTED = [
    "ccnn_default_params", "ccnn_create", "ccnn_destroy", "ccnn_detect", "ccnn_detect_device",
    "ccnn_detect_batch", "ccnn_get_gray_device", "ccnn_get_gray_host", "ccnn_get_params",
    "ccnn_set_params", "ccnn_set_max_image_size", "ccnn_set_min_object_height",
    "ccnn_set_max_object_height", "ccnn_set_num_threads", "ccnn_last_error", "ccnn_version",
    "ccnn_gray_u8_to_f32", "ccnn_resize_f32", "ccnn_stage1_forward", "ccnn_inspect_levels",
    "ccnn_inspect_response", "ccnn_inspect_candidates", "ccnn_inspect_raw_detections",
    "ccnn_sort_permutation", "ccnn_detect_device_batch", "ccnn_profile_last_frame", "ccnn_plan_levels", "ccnn_stage1_forward_static",
    "ccnn_server_create", "ccnn_server_destroy", "ccnn_server_submit", "ccnn_server_poll", "ccnn_server_wait",
    "ccnn_server_stats_get", "ccnn_host_alloc", "ccnn_host_free", "ccnn_cntk_dump_to_binary",
    "ccnn_check_reciprocal", "ccnn_synth_frame_device", "ccnn_gate_set", "ccnn_gate_disable", "ccnn_gate_stats", "ccnn_gate_probabilities", "ccnn_gate_set_margin",
    "ccnn_gate_labels", "ccnn_gate_features", "ccnn_gate_gradient", "ccnn_gate_train", "ccnn_server_set_gate", "ccnn_server_set_gate_margin",
    "ccnn_legacy_model_info", "ccnn_legacy_net_forward", "ccnn_set_schedule", "ccnn_get_schedule",
    "ccnn_measure_fp32_peak", "ccnn_cnn_default_params", "ccnn_cnn_create", "ccnn_cnn_detect", "ccnn_cnn_nms",
    "ccnn_cnn_get_params", "ccnn_cnn_set_params", "ccnn_set_schedule_ex", "ccnn_get_schedule_ex",
    "ccnn_sort_permutation_device",
]


class Params(ctypes.Structure):
    _fields_ = [
        ("max_image_width", ctypes.c_int), ("max_image_height", ctypes.c_int),
        ("min_face_height", ctypes.c_int), ("max_face_height", ctypes.c_int),
        ("scale_factor", ctypes.c_float), ("min_neighbors", ctypes.c_int),
        ("detect_precision", ctypes.c_int), ("treshold", ctypes.c_float * 3),
        ("drop_detect", ctypes.c_int), ("equalize", ctypes.c_int), ("reflection", ctypes.c_int),
        ("pipeline", ctypes.c_int), ("detect_mode", ctypes.c_int), ("num_threads", ctypes.c_int),
        ("index_output", ctypes.c_int * 3), ("device_info", ctypes.c_int),
        ("cuda_device_id", ctypes.c_int), ("cl_platform_id", ctypes.c_int), ("cl_device_id", ctypes.c_int),
        ("facial_analysis", ctypes.c_int),
    ]


class Face(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("score", ctypes.c_float), ("gender", ctypes.c_int), ("smile", ctypes.c_int),
                ("glasses", ctypes.c_int)]


class Image(ctypes.Structure):
    _fields_ = [("cols", ctypes.c_int), ("rows", ctypes.c_int), ("channels", ctypes.c_int),
                ("data", ctypes.c_void_p), ("step", ctypes.c_size_t)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("slots_per_class", ctypes.c_int), ("max_queue", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("queued", ctypes.c_int), ("in_flight", ctypes.c_int), ("classes", ctypes.c_int),
                ("hbm_bytes", ctypes.c_size_t)]


class LevelInfo(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("scale", ctypes.c_float),
                ("resp_width", ctypes.c_int), ("resp_height", ctypes.c_int)]


class CandidateInfo(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int), ("x", ctypes.c_int), ("y", ctypes.c_int), ("score", ctypes.c_float),
                ("accepted", ctypes.c_int), ("check_score", ctypes.c_float), ("knn", ctypes.c_int)]


class Detection(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("score", ctypes.c_float), ("scale", ctypes.c_float), ("knn", ctypes.c_int),
                ("num_detect", ctypes.c_int)]


class CnnParam(ctypes.Structure):
    """ccnn_cnn_param: CNNDetector::Param (include/ccnn_cnn.h)."""
    _fields_ = [("pipeline", ctypes.c_int), ("max_image_width", ctypes.c_int), ("max_image_height", ctypes.c_int),
                ("min_obj_width", ctypes.c_int), ("min_obj_height", ctypes.c_int), ("max_obj_width", ctypes.c_int),
                ("max_obj_height", ctypes.c_int), ("scale_factor", ctypes.c_float), ("min_neighbors", ctypes.c_int),
                ("num_threads", ctypes.c_int)]


class CnnAdvancedParam(ctypes.Structure):
    """ccnn_cnn_advanced_param: CNNDetector::AdvancedParam (include/ccnn_cnn.h)."""
    _fields_ = [(n, ctypes.c_int) for n in ("detect_mode", "detect_precision", "packet_detection", "gray_image_only",
                                            "facial_analysis", "equalize", "reflection", "type_check")] + \
               [(n, ctypes.c_float) for n in ("treshold_1", "treshold_2", "treshold_3")] + \
               [(n, ctypes.c_int) for n in ("adapt_min_neighbors", "double_check", "drop_detect", "min_num_detect", "device_info",
                                            "cuda_device_id", "cl_platform_id", "cl_device_id", "concurrent_kernels",
                                            "num_cnn_copy", "blur", "img_resize", "uniform_noise", "merger_detect")] + \
               [("index_output", ctypes.c_int * 4)]


class Schedule(ctypes.Structure):
    """ccnn_schedule (include/ccnn_inspect.h)."""
    _fields_ = [("frame_slots", ctypes.c_int), ("window_ctas_per_sm", ctypes.c_int), ("front_blocks_per_sm", ctypes.c_int),
                ("back_blocks_per_sm", ctypes.c_int), ("batch_frames", ctypes.c_int), ("batch_blocks_per_sm", ctypes.c_int)]


class SynthFace(ctypes.Structure):
    _fields_ = [("cx", ctypes.c_int), ("cy", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("angle_deg", ctypes.c_float), ("contrast", ctypes.c_float)]


_lib = None
_synth = None


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; g.build()'` "
                               "(the detector has no fallback without its CUDA library)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        ci = ctypes.c_int
        L.ccnn_default_params.argtypes = [P(Params)]
        L.ccnn_default_params.restype = None
        L.ccnn_create.argtypes = [P(Params), P(ctypes.c_char_p), P(vp)]
        L.ccnn_destroy.argtypes = [vp]
        L.ccnn_detect.argtypes = [vp, P(Image), P(Face), ci, P(ci)]
        L.ccnn_detect_device.argtypes = [vp, P(Image), vp, P(Face), ci, P(ci)]
        L.ccnn_detect_batch.argtypes = [vp, P(Image), ci, P(Face), ci, P(ci)]
        L.ccnn_get_gray_device.argtypes = [vp, P(vp), P(ci), P(ci), P(ctypes.c_size_t)]
        L.ccnn_get_gray_host.argtypes = [vp, vp, ci, P(ci), P(ci)]
        L.ccnn_get_params.argtypes = [vp, P(Params)]
        L.ccnn_set_params.argtypes = [vp, P(Params)]
        L.ccnn_set_max_image_size.argtypes = [vp, ci, ci]
        L.ccnn_set_min_object_height.argtypes = [vp, ci]
        L.ccnn_set_max_object_height.argtypes = [vp, ci]
        L.ccnn_set_num_threads.argtypes = [vp, ci]
        L.ccnn_last_error.restype = ctypes.c_char_p
        L.ccnn_version.restype = ctypes.c_char_p
        L.ccnn_gray_u8_to_f32.argtypes = [vp, ci, ci, ci, ctypes.c_size_t, vp, ctypes.c_size_t, vp]
        L.ccnn_resize_f32.argtypes = [vp, ci, ci, ctypes.c_size_t, vp, ci, ci, ctypes.c_size_t, ci, vp]
        L.ccnn_stage1_forward.argtypes = [vp, vp, ci, ci, ctypes.c_size_t, vp, ci, P(ci), P(ci), vp]
        L.ccnn_measure_fp32_peak.argtypes = [ci, ci, P(ctypes.c_double), P(ctypes.c_float)]
        L.ccnn_cnn_default_params.argtypes = [P(CnnParam), P(CnnAdvancedParam)]
        L.ccnn_cnn_default_params.restype = None
        L.ccnn_cnn_create.argtypes = [P(CnnParam), P(CnnAdvancedParam), P(ctypes.c_char_p), P(vp)]
        L.ccnn_cnn_detect.argtypes = [vp, P(Image), P(Detection), ci, P(Detection), ci, P(ci)]
        L.ccnn_cnn_nms.argtypes = [vp, P(Detection), ci, P(Detection), ci, P(ci)]
        L.ccnn_cnn_get_params.argtypes = [vp, P(CnnParam), P(CnnAdvancedParam)]
        L.ccnn_cnn_set_params.argtypes = [vp, P(CnnParam), P(CnnAdvancedParam)]
        L.ccnn_inspect_levels.argtypes = [vp, P(LevelInfo), ci, P(ci)]
        L.ccnn_inspect_response.argtypes = [vp, ci, vp, ci]
        L.ccnn_inspect_candidates.argtypes = [vp, P(CandidateInfo), ci, P(ci)]
        L.ccnn_inspect_raw_detections.argtypes = [vp, P(Detection), ci, P(ci)]
        L.ccnn_sort_permutation.argtypes = [vp, ci, vp]
        L.ccnn_sort_permutation_device.argtypes = [vp, ci, vp]
        L.ccnn_detect_device_batch.argtypes = [vp, P(Image), ci, P(Face), ci, P(ci), P(ctypes.c_float)]
        L.ccnn_profile_last_frame.argtypes = [vp, ci, P(ctypes.c_float), ci]
        L.ccnn_plan_levels.argtypes = [P(Params), ci, ci, ci, P(LevelInfo), ci, P(ci)]
        L.ccnn_stage1_forward_static.argtypes = [ctypes.c_char_p, vp, ci, ci, ctypes.c_size_t, vp, ci, P(ci), P(ci), vp]
        ll = ctypes.c_longlong
        L.ccnn_server_create.argtypes = [P(Params), P(ctypes.c_char_p), P(ServerConfig), P(vp)]
        L.ccnn_server_destroy.argtypes = [vp]
        L.ccnn_server_submit.argtypes = [vp, P(Image), P(ll)]
        L.ccnn_server_poll.argtypes = [vp, ll, P(Face), ci, P(ci), P(ctypes.c_double)]
        L.ccnn_server_wait.argtypes = [vp, ll, P(Face), ci, P(ci), P(ctypes.c_double)]
        L.ccnn_server_stats_get.argtypes = [vp, P(ServerStats)]
        L.ccnn_host_alloc.argtypes = [ctypes.c_size_t]
        L.ccnn_host_alloc.restype = vp
        L.ccnn_host_free.argtypes = [vp]
        L.ccnn_host_free.restype = None
        L.ccnn_cntk_dump_to_binary.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ccnn_check_reciprocal.argtypes = [P(ctypes.c_longlong), P(ctypes.c_longlong)]
        L.ccnn_synth_frame_device.argtypes = [vp, ci, ci, ci, ctypes.c_size_t, ctypes.c_ulonglong, ci, ci, ci, vp, vp]
        fp = P(ctypes.c_float)
        L.ccnn_gate_set.argtypes = [vp, fp, ci, ctypes.c_float, ctypes.c_float]
        L.ccnn_gate_disable.argtypes = [vp]
        L.ccnn_server_set_gate.argtypes = [vp, fp, ci, ctypes.c_float, ctypes.c_float]
        L.ccnn_server_set_gate_margin.argtypes = [vp, ci]
        L.ccnn_legacy_model_info.argtypes = [ctypes.c_char_p, P(ci), ci]
        L.ccnn_set_schedule.argtypes = [vp, ci, ci]
        L.ccnn_get_schedule.argtypes = [vp, P(ci), P(ci)]
        L.ccnn_set_schedule_ex.argtypes = [vp, P(Schedule)]
        L.ccnn_get_schedule_ex.argtypes = [vp, P(Schedule)]
        L.ccnn_legacy_net_forward.argtypes = [ctypes.c_char_p, vp, ci, ci, ctypes.c_size_t, vp, ci, P(ci), P(ci), vp]
        L.ccnn_gate_stats.argtypes = [vp, P(ci), P(ci), P(ci), P(ci), P(ci)]
        L.ccnn_gate_probabilities.argtypes = [vp, P(ctypes.c_float), ci, P(ci)]
        L.ccnn_gate_set_margin.argtypes = [vp, ci]
        L.ccnn_gate_labels.argtypes = [vp, vp, vp]
        L.ccnn_gate_features.argtypes = [vp, ci, ci, ctypes.c_size_t, vp, vp]
        L.ccnn_gate_gradient.argtypes = [vp, vp, vp, ci, ci, ci, ctypes.c_float, fp, fp]
        L.ccnn_gate_train.argtypes = [fp, vp, vp, ci, ci, ci, ci, ci, ctypes.c_float, ctypes.c_float, fp]
        _lib = L
    return _lib


def synth():
    """The synthetic-frame generator library."""
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError(f"{SYNTH_PATH} is missing: build the package first")
        S = ctypes.CDLL(SYNTH_PATH)
        S.ccnn_synth_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(SynthFace)]
        _synth = S
    return _synth


def last_error():
    return lib().ccnn_last_error().decode(errors="replace")


class CCNNError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        super().__init__(f"{where} failed with status {status}: {last_error()}")


def check(status, where):
    if status < 0:
        raise CCNNError(status, where)
    return status
