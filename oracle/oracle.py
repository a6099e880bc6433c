"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (prores_oracle.cpp) restates the rivet-prores crate's decode and
encode on the CPU. Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module; the product package never does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libprores_oracle.so")

OK, INVALID, UNSUPPORTED, CONFIG = 0, 1, 2, 3
KIND_NAMES = {INVALID: "Invalid", UNSUPPORTED: "Unsupported", CONFIG: "Config"}


class _Frame(ctypes.Structure):
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
        ("pad_", ctypes.c_uint8 * 3),
        ("data", ctypes.POINTER(ctypes.c_uint16)),
        ("data_len", ctypes.c_size_t),
        ("alpha", ctypes.POINTER(ctypes.c_uint16)),
        ("alpha_len", ctypes.c_size_t),
    ]


class _Config(ctypes.Structure):
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


def build() -> str:
    """Compiles the oracle with its Makefile (g++ only; seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        L.ora_decode.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32,
                                 P(_Frame), ctypes.c_char_p, ctypes.c_size_t]
        L.ora_frame_free.argtypes = [P(_Frame)]
        L.ora_encode.argtypes = [P(_Config), P(_Frame), P(P(ctypes.c_uint8)), P(ctypes.c_size_t),
                                 ctypes.c_char_p, ctypes.c_size_t]
        L.ora_free.argtypes = [ctypes.c_void_p]
        L.ora_last_qindices.argtypes = [ctypes.c_int, P(ctypes.c_uint8), ctypes.c_size_t]
        L.ora_last_qindices.restype = ctypes.c_size_t
        L.ora_target_frame_bytes.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
        L.ora_target_frame_bytes.restype = ctypes.c_size_t
        L.ora_slice_sizes.argtypes = [ctypes.c_uint32, ctypes.c_uint32, P(ctypes.c_uint32), ctypes.c_size_t]
        L.ora_slice_sizes.restype = ctypes.c_size_t
        L.ora_codeword.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t]
        L.ora_codeword_len.argtypes = [ctypes.c_int, ctypes.c_uint32]
        L.ora_codeword_len.restype = ctypes.c_uint32
        L.ora_codebook_read.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t, P(ctypes.c_uint32),
                                        P(ctypes.c_uint32)]
        L.ora_alpha_run_code.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t]
        L.ora_alpha_diff_code.argtypes = [ctypes.c_int32, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t]
        L.ora_rescale.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint16]
        L.ora_rescale.restype = ctypes.c_uint16
        L.ora_qscale.argtypes = [ctypes.c_uint32]
        L.ora_qscale.restype = ctypes.c_uint32
        L.ora_scans.argtypes = [P(ctypes.c_uint8), P(ctypes.c_uint8)]
        L.ora_basis.argtypes = [P(ctypes.c_float)]
        L.ora_idct_put.argtypes = [P(ctypes.c_int32), P(ctypes.c_float), ctypes.c_uint32, P(ctypes.c_uint16)]
        L.ora_fdct_load.argtypes = [P(ctypes.c_uint16), ctypes.c_float, P(ctypes.c_float)]
        L.ora_set_simd.argtypes = [ctypes.c_int]
        L.ora_quantise.argtypes = [P(ctypes.c_float), ctypes.c_size_t, P(ctypes.c_float), ctypes.c_float,
                                   P(ctypes.c_int32), P(ctypes.c_uint64)]
        L.ora_encode_coefficients.argtypes = [P(ctypes.c_int32), ctypes.c_size_t, P(ctypes.c_uint8),
                                              ctypes.c_size_t, P(ctypes.c_size_t)]
        L.ora_encode_coefficients.restype = ctypes.c_size_t
        L.ora_decode_coefficients.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_size_t,
                                              P(ctypes.c_int32), ctypes.c_char_p, ctypes.c_size_t]
        L.ora_encode_alpha.argtypes = [P(ctypes.c_uint16), ctypes.c_size_t, ctypes.c_uint32, P(ctypes.c_uint8),
                                       ctypes.c_size_t]
        L.ora_encode_alpha.restype = ctypes.c_size_t
        L.ora_decode_alpha.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_size_t,
                                       ctypes.c_size_t, P(ctypes.c_uint16), P(ctypes.c_size_t)]
        L.ora_test_frame.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint32,
                                     ctypes.c_int32, ctypes.c_uint32, P(ctypes.c_uint16)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


# ------------------------------------------------------------------ frames

def plane_layout(width: int, height: int, chroma: int):
    """(offset, width, height) of Y', Cb, Cr (src/frame.rs:247-266)."""
    cw = (width + 1) // 2 if chroma == 2 else width
    y = (0, width, height)
    cb = (width * height, cw, height)
    cr = (cb[0] + cw * height, cw, height)
    return [y, cb, cr]


@dataclass
class Picture:
    """A frame as the oracle sees it: packed u16 planes plus optional alpha."""

    width: int
    height: int
    bit_depth: int
    chroma: int  # 2 = 4:2:2, 3 = 4:4:4
    interlace: int = 0
    metadata: tuple = (0, 0, 2, 2, 2)
    data: np.ndarray = field(default=None)
    alpha: Optional[np.ndarray] = None

    def plane(self, i: int) -> np.ndarray:
        off, w, h = plane_layout(self.width, self.height, self.chroma)[i]
        return self.data[off:off + w * h].reshape(h, w)


def _to_c_frame(p: Picture, keep: list) -> _Frame:
    f = _Frame()
    f.width, f.height, f.bit_depth = p.width, p.height, p.bit_depth
    f.chroma, f.interlace = p.chroma, p.interlace
    (f.aspect_ratio, f.frame_rate_code, f.color_primaries, f.transfer_characteristic,
     f.matrix_coefficients) = p.metadata
    d = np.ascontiguousarray(p.data, dtype=np.uint16)
    keep.append(d)
    f.data = _ptr(d, ctypes.c_uint16)
    f.data_len = d.size
    if p.alpha is not None:
        a = np.ascontiguousarray(p.alpha, dtype=np.uint16)
        keep.append(a)
        f.alpha = _ptr(a, ctypes.c_uint16)
        f.alpha_len = a.size
    return f


def test_frame(width, height, chroma, bit_depth, grain, seed) -> Picture:
    """The reference tests' picture generator (tests/common/mod.rs:26-80)."""
    total = sum(w * h for _, w, h in plane_layout(width, height, chroma))
    data = np.zeros(total, dtype=np.uint16)
    lib().ora_test_frame(width, height, chroma, bit_depth, grain, seed, _ptr(data, ctypes.c_uint16))
    return Picture(width, height, bit_depth, chroma, 0, (0, 0, 2, 2, 2), data, None)


# ------------------------------------------------------------------ codec

def decode(data: bytes, bit_depth: int = 0, threads: int = 0):
    """(kind, message, Picture or None)."""
    f = _Frame()
    msg = ctypes.create_string_buffer(512)
    k = lib().ora_decode(bytes(data), len(data), bit_depth, threads, ctypes.byref(f), msg, 512)
    if k != OK:
        return k, msg.value.decode("utf-8"), None
    d = np.ctypeslib.as_array(f.data, shape=(f.data_len,)).copy()
    a = np.ctypeslib.as_array(f.alpha, shape=(f.alpha_len,)).copy() if f.alpha_len else None
    p = Picture(f.width, f.height, f.bit_depth, f.chroma, f.interlace,
                (f.aspect_ratio, f.frame_rate_code, f.color_primaries, f.transfer_characteristic,
                 f.matrix_coefficients), d, a)
    lib().ora_frame_free(ctypes.byref(f))
    return OK, "", p


@dataclass
class Config:
    """src/encode.rs:135-174. alpha: 0 none, 1 8-bit, 2 16-bit (default)."""

    profile: int
    log2_slice_mbs: int = 3
    alpha: int = 2
    luma_matrix: Optional[bytes] = None
    chroma_matrix: Optional[bytes] = None
    target_frame_bytes: Optional[int] = None
    encoder_identifier: bytes = b"rivt"
    threads: int = 0


def _to_c_config(c: Config) -> _Config:
    k = _Config()
    k.profile, k.log2_slice_mbs, k.alpha = c.profile, c.log2_slice_mbs, c.alpha
    if c.luma_matrix is not None:
        k.has_luma_matrix = 1
        k.luma_matrix[:] = list(bytes(c.luma_matrix))
    if c.chroma_matrix is not None:
        k.has_chroma_matrix = 1
        k.chroma_matrix[:] = list(bytes(c.chroma_matrix))
    k.target_frame_bytes = -1 if c.target_frame_bytes is None else c.target_frame_bytes
    k.encoder_identifier[:] = list(c.encoder_identifier)
    k.threads = c.threads
    return k


def encode(cfg: Config, pic: Picture):
    """(kind, message, bytes or None)."""
    keep = []
    f = _to_c_frame(pic, keep)
    k = _to_c_config(cfg)
    out = ctypes.POINTER(ctypes.c_uint8)()
    n = ctypes.c_size_t()
    msg = ctypes.create_string_buffer(512)
    r = lib().ora_encode(ctypes.byref(k), ctypes.byref(f), ctypes.byref(out), ctypes.byref(n), msg, 512)
    if r != OK:
        return r, msg.value.decode("utf-8"), None
    b = ctypes.string_at(out, n.value)
    lib().ora_free(out)
    return OK, "", b


def last_qindices(picture: int = 0) -> np.ndarray:
    buf = np.zeros(1 << 20, dtype=np.uint8)
    n = lib().ora_last_qindices(picture, _ptr(buf, ctypes.c_uint8), buf.size)
    return buf[:n].copy()


def target_frame_bytes(profile: int, w: int, h: int) -> int:
    return lib().ora_target_frame_bytes(profile, w, h)


def slice_sizes(width_in_mb: int, log2: int):
    buf = np.zeros(width_in_mb + 8, dtype=np.uint32)
    n = lib().ora_slice_sizes(width_in_mb, log2, _ptr(buf, ctypes.c_uint32), buf.size)
    return [int(x) for x in buf[:n]]


# codebook ids: 0..3 DC (Table 9), 4..19 run (Table 10), 20..28 level (Table 11), 29 first DC
DC_BOOK, RUN_BOOK, LEVEL_BOOK, FIRST_DC_BOOK = 0, 4, 20, 29


def codeword(book: int, n: int) -> str:
    buf = ctypes.create_string_buffer(256)
    lib().ora_codeword(book, n, buf, 256)
    return buf.value.decode()


def codeword_len(book: int, n: int) -> int:
    return lib().ora_codeword_len(book, n)


def codebook_read(book: int, data: bytes):
    v, c = ctypes.c_uint32(), ctypes.c_uint32()
    k = lib().ora_codebook_read(book, bytes(data), len(data), ctypes.byref(v), ctypes.byref(c))
    return k, v.value, c.value


def alpha_run_code(run: int) -> str:
    buf = ctypes.create_string_buffer(64)
    lib().ora_alpha_run_code(run, buf, 64)
    return buf.value.decode()


def alpha_diff_code(d: int, bits: int) -> str:
    buf = ctypes.create_string_buffer(64)
    lib().ora_alpha_diff_code(d, bits, buf, 64)
    return buf.value.decode()


def rescale(bits_in: int, bits_out: int, a: int) -> int:
    return lib().ora_rescale(bits_in, bits_out, a)


def qscale(q: int) -> int:
    return lib().ora_qscale(q)


def scans():
    p = np.zeros(64, np.uint8)
    i = np.zeros(64, np.uint8)
    lib().ora_scans(_ptr(p, ctypes.c_uint8), _ptr(i, ctypes.c_uint8))
    return p, i


def basis() -> np.ndarray:
    b = np.zeros(64, np.float32)
    lib().ora_basis(_ptr(b, ctypes.c_float))
    return b


def set_simd(on: bool) -> None:
    """Runs the dsp kernels (IDCT, FDCT, quantise) in their AVX2 forms (the
    default) or their scalar forms, process-wide; both give the same results."""
    lib().ora_set_simd(1 if on else 0)


def idct_put(coef: np.ndarray, scale: np.ndarray, depth: int) -> np.ndarray:
    c = np.ascontiguousarray(coef, np.int32)
    s = np.ascontiguousarray(scale, np.float32)
    o = np.zeros(64, np.uint16)
    lib().ora_idct_put(_ptr(c, ctypes.c_int32), _ptr(s, ctypes.c_float), depth, _ptr(o, ctypes.c_uint16))
    return o


def fdct_load(pix: np.ndarray, scale: float) -> np.ndarray:
    p = np.ascontiguousarray(pix, np.uint16)
    o = np.zeros(64, np.float32)
    lib().ora_fdct_load(_ptr(p, ctypes.c_uint16), scale, _ptr(o, ctypes.c_float))
    return o


def quantise(f: np.ndarray, n: int, inv: np.ndarray, rounding: float = 0.42):
    f = np.ascontiguousarray(f, np.float32)
    inv = np.ascontiguousarray(inv, np.float32)
    out = np.zeros(64 * n, np.int32)
    mask = np.zeros(n, np.uint64)
    lib().ora_quantise(_ptr(f, ctypes.c_float), n, _ptr(inv, ctypes.c_float), rounding,
                       _ptr(out, ctypes.c_int32), _ptr(mask, ctypes.c_uint64))
    return out, mask


def encode_coefficients(scanned: np.ndarray, n_blocks: int):
    """(bytes, bit count before alignment) for one component in scanned order."""
    s = np.ascontiguousarray(scanned, np.int32)
    cap = 16 * s.size + 64
    out = np.zeros(cap, np.uint8)
    bits = ctypes.c_size_t()
    n = lib().ora_encode_coefficients(_ptr(s, ctypes.c_int32), n_blocks, _ptr(out, ctypes.c_uint8), cap,
                                      ctypes.byref(bits))
    return out[:n].tobytes(), bits.value


def decode_coefficients(data: bytes, n_blocks: int):
    out = np.zeros(64 * n_blocks, np.int32)
    msg = ctypes.create_string_buffer(256)
    k = lib().ora_decode_coefficients(bytes(data), len(data), n_blocks, _ptr(out, ctypes.c_int32), msg, 256)
    return k, msg.value.decode(), out


def encode_alpha(values: np.ndarray, bits: int) -> bytes:
    v = np.ascontiguousarray(values, np.uint16)
    cap = 4 * v.size + 64
    out = np.zeros(cap, np.uint8)
    n = lib().ora_encode_alpha(_ptr(v, ctypes.c_uint16), v.size, bits, _ptr(out, ctypes.c_uint8), cap)
    return out[:n].tobytes()


def decode_alpha(data: bytes, bits: int, count: int, needed: int):
    out = np.zeros(count, np.uint16)
    got = ctypes.c_size_t()
    k = lib().ora_decode_alpha(bytes(data), len(data), bits, count, needed, _ptr(out, ctypes.c_uint16),
                               ctypes.byref(got))
    return k, out[:got.value].copy()
