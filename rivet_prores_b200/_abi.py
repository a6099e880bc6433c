"""ctypes binding of libprores_b200.so (include/prores_b200.h).

The library is built in-tree (rivet_prores_b200/build.py). Loading fails
loudly if it is missing: there is no CPU fallback behind this package.
"""

from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libprores_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "prores_b200.h")

OK, INVALID, UNSUPPORTED, CONFIG, DEVICE, TIMEOUT = 0, 1, 2, 3, 4, 5

P = ctypes.POINTER


class Frame_(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("bit_depth", ctypes.c_uint32),
        ("chroma", ctypes.c_int32),
        ("interlace", ctypes.c_int32),
        ("aspect_ratio", ctypes.c_uint8),
        ("frame_rate_code", ctypes.c_uint8),
        ("color_primaries", ctypes.c_uint8),
        ("transfer_characteristic", ctypes.c_uint8),
        ("matrix_coefficients", ctypes.c_uint8),
        ("reserved_", ctypes.c_uint8 * 3),
        ("data", P(ctypes.c_uint16)),
        ("data_len", ctypes.c_size_t),
        ("alpha", P(ctypes.c_uint16)),
        ("alpha_len", ctypes.c_size_t),
    ]


class Config_(ctypes.Structure):
    _fields_ = [
        ("profile", ctypes.c_int32),
        ("log2_slice_mbs", ctypes.c_uint32),
        ("alpha", ctypes.c_int32),
        ("has_luma_matrix", ctypes.c_int32),
        ("has_chroma_matrix", ctypes.c_int32),
        ("luma_matrix", ctypes.c_uint8 * 64),
        ("chroma_matrix", ctypes.c_uint8 * 64),
        ("target_frame_bytes", ctypes.c_int64),
        ("encoder_identifier", ctypes.c_uint8 * 4),
        ("threads", ctypes.c_uint32),
    ]


class Buf_(ctypes.Structure):
    _fields_ = [("data", P(ctypes.c_uint8)), ("len", ctypes.c_size_t)]


class Span_(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_size_t), ("len", ctypes.c_size_t)]


class FrameHeader_(ctypes.Structure):
    _fields_ = [
        ("frame_size", ctypes.c_uint32),
        ("header_size", ctypes.c_uint16),
        ("bitstream_version", ctypes.c_uint8),
        ("encoder_identifier", ctypes.c_uint8 * 4),
        ("reserved_", ctypes.c_uint8),
        ("width", ctypes.c_uint16),
        ("height", ctypes.c_uint16),
        ("chroma", ctypes.c_int32),
        ("interlace", ctypes.c_int32),
        ("alpha", ctypes.c_int32),
        ("aspect_ratio", ctypes.c_uint8),
        ("frame_rate_code", ctypes.c_uint8),
        ("color_primaries", ctypes.c_uint8),
        ("transfer_characteristic", ctypes.c_uint8),
        ("matrix_coefficients", ctypes.c_uint8),
        ("reserved2_", ctypes.c_uint8 * 3),
        ("has_luma_matrix", ctypes.c_int32),
        ("has_chroma_matrix", ctypes.c_int32),
        ("luma_matrix", ctypes.c_uint8 * 64),
        ("chroma_matrix", ctypes.c_uint8 * 64),
    ]


class Tuning_(ctypes.Structure):
    _fields_ = [
        ("cost_lane_items_per_sm", ctypes.c_int32),
        ("entropy_warps_per_block", ctypes.c_int32),
        ("entropy_blocks_per_sm", ctypes.c_int32),
        ("entropy_components_per_lane", ctypes.c_int32),
        ("staging_depth", ctypes.c_int32),
        ("decode_fused", ctypes.c_int32),
        ("decode_slot_positions", ctypes.c_int32),
        ("decode_slot_bytes", ctypes.c_int32),
    ]


_lib = None


def declared_functions() -> list[str]:
    """Every function include/prores_b200.h declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(prores_[a-z_0-9]+)\s*\(", text)))


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    # RIVET_PRORES_LIB names another build of the same library (to compare
    # builds side by side); by default the in-tree one.
    path = os.environ.get("RIVET_PRORES_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python rivet_prores_b200/build.py` (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "prores_create": (vp, [ctypes.c_int]),
        "prores_destroy": (None, [vp]),
        "prores_last_error": (ctypes.c_char_p, []),
        "prores_batch_error": (ctypes.c_char_p, [ctypes.c_int]),
        "prores_probe": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32, P(Frame_)]),
        "prores_parse_frame_header": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t, P(FrameHeader_)]),
        "prores_decode": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32, P(Frame_)]),
        "prores_decode_batch": (ctypes.c_int, [vp, P(Buf_), ctypes.c_int, ctypes.c_uint32, P(Frame_),
                                               P(ctypes.c_int)]),
        "prores_frame_free": (None, [P(Frame_)]),
        "prores_config_default": (None, [P(Config_), ctypes.c_int32]),
        "prores_target_frame_bytes": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32]),
        "prores_encode": (ctypes.c_int, [vp, P(Config_), P(Frame_), P(P(ctypes.c_uint8)), P(ctypes.c_size_t)]),
        "prores_encode_batch": (ctypes.c_int, [vp, P(Config_), P(Frame_), ctypes.c_int, P(Buf_), P(ctypes.c_int)]),
        "prores_buffer_free": (None, [vp]),
        "prores_decode_job_create": (ctypes.c_int, [vp, P(Buf_), ctypes.c_int, ctypes.c_uint32, P(vp)]),
        "prores_decode_job_launch": (ctypes.c_int, [vp, vp, ctypes.c_int]),
        "prores_decode_job_upload": (ctypes.c_int, [vp, P(Buf_), ctypes.c_int, vp]),
        "prores_decode_job_fetch": (ctypes.c_int, [vp, vp, P(Frame_), P(ctypes.c_int)]),
        "prores_decode_job_planes": (ctypes.c_int, [vp, ctypes.c_int, P(P(ctypes.c_uint16)),
                                                    P(P(ctypes.c_uint16))]),
        "prores_decode_job_destroy": (None, [vp]),
        "prores_encode_job_create": (ctypes.c_int, [vp, P(Config_), P(Frame_), ctypes.c_int, P(vp)]),
        "prores_encode_job_launch": (ctypes.c_int, [vp, vp, ctypes.c_int]),
        "prores_encode_job_upload": (ctypes.c_int, [vp, P(Frame_), ctypes.c_int, vp]),
        "prores_encode_job_fetch": (ctypes.c_int, [vp, vp, P(Buf_), P(ctypes.c_int)]),
        "prores_encode_job_destroy": (None, [vp]),
        "prores_job_kernel_times": (ctypes.c_int, [vp, ctypes.c_int, P(ctypes.c_char_p), P(ctypes.c_float),
                                                   ctypes.c_int]),
        "prores_tuning_default": (None, [P(Tuning_)]),
        "prores_scan_frames": (ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t, P(Span_), ctypes.c_size_t]),
        "prores_scan_frames_device": (ctypes.c_int, [vp, vp, ctypes.c_size_t, P(Span_), ctypes.c_size_t,
                                                     P(ctypes.c_size_t), vp]),
        "prores_probe_device": (ctypes.c_int, [vp, vp, ctypes.c_size_t, P(Span_), ctypes.c_int, ctypes.c_uint32,
                                               P(Frame_), P(ctypes.c_int)]),
        "prores_decode_device": (ctypes.c_int, [vp, vp, ctypes.c_size_t, P(Span_), ctypes.c_int, ctypes.c_uint32,
                                                P(Frame_), P(ctypes.c_int), vp]),
        "prores_encode_device": (ctypes.c_int, [vp, P(Config_), P(Frame_), ctypes.c_int, P(Buf_), P(ctypes.c_int),
                                                vp]),
        "prores_set_tuning": (ctypes.c_int, [vp, P(Tuning_)]),
        "prores_get_tuning": (ctypes.c_int, [vp, P(Tuning_)]),
        "prores_set_timeout": (ctypes.c_int, [vp, ctypes.c_uint32]),
        "prores_shard_frames": (ctypes.c_int, [P(ctypes.c_uint32), P(ctypes.c_uint32), ctypes.c_int, ctypes.c_int,
                                               P(ctypes.c_int)]),
        "prores_decode_batch_multi": (ctypes.c_int, [P(vp), ctypes.c_int, P(Buf_), ctypes.c_int, ctypes.c_uint32,
                                                     P(Frame_), P(ctypes.c_int)]),
        "prores_encode_batch_multi": (ctypes.c_int, [P(vp), ctypes.c_int, P(Config_), P(Frame_), ctypes.c_int,
                                                     P(Buf_), P(ctypes.c_int)]),
        "prores_get_timeout": (ctypes.c_uint32, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def batch_error(i: int) -> str:
    m = lib().prores_batch_error(i)
    return m.decode("utf-8", "replace") if m else ""


def last_error() -> str:
    m = lib().prores_last_error()
    return m.decode("utf-8", "replace") if m else ""
