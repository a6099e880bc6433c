"""B200-native ProRes (SMPTE RDD 36) decode and encode.

A drop-in for the rivet-prores crate's public API (imported there as
`prores`, src/lib.rs:52-56): `Decoder`, `Encoder`, `Config`, `Profile`,
`Frame`, `Plane`, `ChromaFormat`, `Interlace`, `Metadata`, `FrameHeader`,
`AlphaType`, `Error`. Every per-slice step runs in the sm_100a kernels of
libprores_b200.so; decoded planes and encoded bytes are bit-identical to the
crate's. Batched forms (`Decoder.decode_batch`, `Encoder.encode_batch`) put
many frames of any size and format into one launch.
"""

from __future__ import annotations

import ctypes
import enum
import threading
from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _abi
from ._abi import Buf_, Config_, Frame_, FrameHeader_

__all__ = [
    "AlphaType", "ChromaFormat", "Config", "Decoder", "Encoder", "Error", "Frame", "FrameHeader",
    "Interlace", "Metadata", "Plane", "Profile", "Tuning", "context", "scan_frames", "DeviceFrame",
]


# ------------------------------------------------------------------ errors

class Error(Exception):
    """src/error.rs:6-21: Invalid, Unsupported and Config, each with a message;
    Device and Timeout are this library's (a CUDA failure, a wait that ran out).
    Catch a kind as `Error.Invalid`, `Error.Unsupported`, `Error.Config`."""

    kind = "Error"

    def __init__(self, message: str):
        super().__init__(message)
        self.message = message

    def __eq__(self, other):
        return type(self) is type(other) and self.message == other.message

    def __hash__(self):
        return hash((type(self).__name__, self.message))


class _Invalid(Error):
    kind = "Invalid"


class _Unsupported(Error):
    kind = "Unsupported"


class _Config(Error):
    kind = "Config"


class _Device(Error):
    kind = "Device"


class _Timeout(Error):
    kind = "Timeout"


Error.Invalid = _Invalid
Error.Unsupported = _Unsupported
Error.Config = _Config
Error.Device = _Device
Error.Timeout = _Timeout
_KINDS = {_abi.INVALID: _Invalid, _abi.UNSUPPORTED: _Unsupported, _abi.CONFIG: _Config,
          _abi.DEVICE: _Device, _abi.TIMEOUT: _Timeout}


def _error(code: int, message: Optional[str] = None) -> Error:
    return _KINDS.get(code, _Device)(message if message is not None else _abi.last_error())


def _check(code: int):
    if code != _abi.OK:
        raise _error(code)


# ------------------------------------------------------------------ types

class ChromaFormat(enum.Enum):
    """src/frame.rs:8-41."""

    Yuv422 = 2
    Yuv444 = 3

    def subsampling(self):
        return (2, 1) if self is ChromaFormat.Yuv422 else (1, 1)

    def code(self) -> int:
        return self.value

    @staticmethod
    def from_code(code: int) -> Optional["ChromaFormat"]:
        return {2: ChromaFormat.Yuv422, 3: ChromaFormat.Yuv444}.get(code)


class Interlace(enum.Enum):
    """src/frame.rs:47-77: woven output, the top field on the even rows."""

    Progressive = 0
    TopFieldFirst = 1
    BottomFieldFirst = 2

    def code(self) -> int:
        return self.value

    @staticmethod
    def from_code(code: int) -> Optional["Interlace"]:
        return {0: Interlace.Progressive, 1: Interlace.TopFieldFirst, 2: Interlace.BottomFieldFirst}.get(code)


class AlphaType(enum.Enum):
    """src/header.rs:10-40."""

    None_ = 0
    Bits8 = 1
    Bits16 = 2

    def code(self) -> int:
        return self.value

    def bits(self) -> int:
        return {0: 0, 1: 8, 2: 16}[self.value]


_FRAME_RATES = {1: (24000, 1001), 2: (24, 1), 3: (25, 1), 4: (30000, 1001), 5: (30, 1), 6: (50, 1),
                7: (60000, 1001), 8: (60, 1), 9: (100, 1), 10: (120000, 1001), 11: (120, 1)}


@dataclass(frozen=True)
class Metadata:
    """src/frame.rs:83-146: the frame header's descriptive codes."""

    aspect_ratio: int = 0
    frame_rate_code: int = 0
    color_primaries: int = 2
    transfer_characteristic: int = 2
    matrix_coefficients: int = 2

    def frame_rate(self):
        return _FRAME_RATES.get(self.frame_rate_code)

    @staticmethod
    def frame_rate_code_for(numerator: int, denominator: int) -> int:
        for c, (n, d) in _FRAME_RATES.items():
            if n * denominator == numerator * d:
                return c
        return 0


@dataclass(frozen=True)
class Plane:
    """src/frame.rs:148-170: where a plane sits in `Frame.data` (samples)."""

    offset: int
    width: int
    height: int

    def len(self) -> int:
        return self.width * self.height

    def is_empty(self) -> bool:
        return self.len() == 0


def _layout(width: int, height: int, chroma: ChromaFormat) -> List[Plane]:
    cw = -(-width // chroma.subsampling()[0])
    y = Plane(0, width, height)
    cb = Plane(y.len(), cw, height)
    cr = Plane(cb.offset + cb.len(), cw, height)
    return [y, cb, cr]


@dataclass
class Frame:
    """src/frame.rs:179-341: packed u16 planes Y', Cb, Cr and an optional alpha
    plane, values in the low `bit_depth` bits."""

    width: int
    height: int
    bit_depth: int
    chroma: ChromaFormat
    interlace: Interlace = Interlace.Progressive
    metadata: Metadata = field(default_factory=Metadata)
    data: np.ndarray = None
    planes: List[Plane] = None
    alpha: Optional[np.ndarray] = None

    @staticmethod
    def new(width: int, height: int, chroma: ChromaFormat, bit_depth: int) -> "Frame":
        """Mid-grey, no alpha, progressive (src/frame.rs:209-245)."""
        if width == 0 or height == 0 or width > 65535 or height > 65535:
            raise Error.Config(f"invalid ProRes configuration: a frame of {width}×{height} cannot be coded "
                               "(1–65535 each way)")
        if not 8 <= bit_depth <= 16:
            raise Error.Config(f"invalid ProRes configuration: bit depth {bit_depth} is outside 8–16")
        planes = _layout(width, height, chroma)
        total = planes[2].offset + planes[2].len()
        return Frame(width, height, bit_depth, chroma, Interlace.Progressive, Metadata(),
                     np.full(total, 1 << (bit_depth - 1), np.uint16), planes, None)

    def plane(self, i: int) -> np.ndarray:
        p = self.planes[i]
        return self.data[p.offset:p.offset + p.len()]

    plane_mut = plane

    def plane2d(self, i: int) -> np.ndarray:
        p = self.planes[i]
        return self.plane(i).reshape(p.height, p.width)

    def packed(self) -> np.ndarray:
        return self.data

    def to_le_bytes(self) -> bytes:
        return self.data.astype("<u2").tobytes()


@dataclass
class FrameHeader:
    """src/header.rs:43-255: the parsed frame header."""

    frame_size: int
    header_size: int
    bitstream_version: int
    encoder_identifier: bytes
    width: int
    height: int
    chroma: ChromaFormat
    interlace: Interlace
    metadata: Metadata
    alpha: AlphaType
    luma_matrix: Optional[bytes]
    chroma_matrix: Optional[bytes]

    @staticmethod
    def parse(data: bytes) -> "FrameHeader":
        h = FrameHeader_()
        data = bytes(data)
        _check(_abi.lib().prores_parse_frame_header(data, len(data), ctypes.byref(h)))
        return FrameHeader(
            h.frame_size, h.header_size, h.bitstream_version, bytes(h.encoder_identifier), h.width, h.height,
            ChromaFormat(h.chroma), Interlace(h.interlace),
            Metadata(h.aspect_ratio, h.frame_rate_code, h.color_primaries, h.transfer_characteristic,
                     h.matrix_coefficients),
            AlphaType(h.alpha), bytes(h.luma_matrix) if h.has_luma_matrix else None,
            bytes(h.chroma_matrix) if h.has_chroma_matrix else None)

    def picture_count(self) -> int:
        return 1 if self.interlace is Interlace.Progressive else 2

    def _is_top(self, index: int) -> bool:
        return (self.interlace is Interlace.TopFieldFirst) == (index == 0)

    def picture_height(self, index: int) -> int:
        if self.interlace is Interlace.Progressive:
            return self.height
        return (self.height + 1) // 2 if self._is_top(index) else self.height // 2


# ------------------------------------------------------------------ profiles

class Profile(enum.Enum):
    """src/encode.rs:26-118."""

    Proxy = 0
    Lt = 1
    Standard = 2
    Hq = 3
    P4444 = 4
    P4444Xq = 5

    def fourcc(self) -> bytes:
        return [b"apco", b"apcs", b"apcn", b"apch", b"ap4h", b"ap4x"][self.value]

    @staticmethod
    def from_fourcc(code: bytes) -> Optional["Profile"]:
        for p in Profile:
            if p.fourcc() == bytes(code):
                return p
        return None

    def chroma(self) -> ChromaFormat:
        return ChromaFormat.Yuv444 if self.value >= 4 else ChromaFormat.Yuv422

    def reference_bitrate(self) -> int:
        return [45_000_000, 102_000_000, 147_000_000, 220_000_000, 330_000_000, 500_000_000][self.value]

    def target_frame_bytes(self, width: int, height: int) -> int:
        return int(_abi.lib().prores_target_frame_bytes(self.value, width, height))


Profile.ALL = [Profile.Proxy, Profile.Lt, Profile.Standard, Profile.Hq, Profile.P4444, Profile.P4444Xq]


@dataclass
class Config:
    """src/encode.rs:133-193."""

    profile: Profile
    log2_slice_mbs: int = 3
    alpha: AlphaType = AlphaType.Bits16
    luma_matrix: Optional[bytes] = None
    chroma_matrix: Optional[bytes] = None
    target_frame_bytes: Optional[int] = None
    encoder_identifier: bytes = b"rivt"
    threads: int = 0

    @staticmethod
    def new(profile: Profile) -> "Config":
        return Config(profile)

    def _c(self) -> Config_:
        c = Config_()
        c.profile = self.profile.value
        c.log2_slice_mbs = self.log2_slice_mbs
        c.alpha = self.alpha.value
        if self.luma_matrix is not None:
            c.has_luma_matrix = 1
            c.luma_matrix[:] = list(bytes(self.luma_matrix))
        if self.chroma_matrix is not None:
            c.has_chroma_matrix = 1
            c.chroma_matrix[:] = list(bytes(self.chroma_matrix))
        c.target_frame_bytes = -1 if self.target_frame_bytes is None else int(self.target_frame_bytes)
        c.encoder_identifier[:] = list(bytes(self.encoder_identifier)[:4])
        c.threads = self.threads
        return c


# ------------------------------------------------------------------ device

@dataclass
class Tuning:
    """Launch shapes and host pipeline depth (prores_tuning in the C ABI).
    None of them changes an output; `autotune` picks them per GPU."""

    cost_lane_items_per_sm: int = 640
    entropy_warps_per_block: int = 8
    entropy_blocks_per_sm: int = 0
    entropy_components_per_lane: int = 1
    staging_depth: int = 4
    decode_fused: int = 0
    decode_slot_positions: int = 65536
    decode_slot_bytes: int = 1

    def _c(self) -> "_abi.Tuning_":
        t = _abi.Tuning_()
        for k in self.__dataclass_fields__:
            setattr(t, k, int(getattr(self, k)))
        return t

    @staticmethod
    def _from_c(t: "_abi.Tuning_") -> "Tuning":
        return Tuning(**{k: int(getattr(t, k)) for k in Tuning.__dataclass_fields__})


class Context:
    """A device context (workspaces and streams) of libprores_b200. On
    creation it takes the tuning the autotuner cached for this GPU, if any."""

    def __init__(self, device: int = 0):
        self.device = device
        self.handle = _abi.lib().prores_create(device)
        if not self.handle:
            raise Error.Device(_abi.last_error())
        from . import autotune

        cached = autotune.load(device)
        if cached is not None:
            self.set_tuning(cached)

    @property
    def tuning(self) -> Tuning:
        t = _abi.Tuning_()
        _check(_abi.lib().prores_get_tuning(self.handle, ctypes.byref(t)))
        return Tuning._from_c(t)

    def set_tuning(self, tuning: Tuning) -> None:
        t = tuning._c()
        _check(_abi.lib().prores_set_tuning(self.handle, ctypes.byref(t)))

    @property
    def timeout_ms(self) -> int:
        """Bound on every host wait for the device in this context's calls
        (0: none). A call whose wait runs out raises Error.Timeout and leaves
        its device work running; a job stays usable."""
        return int(_abi.lib().prores_get_timeout(self.handle))

    @timeout_ms.setter
    def timeout_ms(self, ms: int) -> None:
        _check(_abi.lib().prores_set_timeout(self.handle, int(ms)))

    def __del__(self):
        h = getattr(self, "handle", None)
        lib = getattr(_abi, "_lib", None) if _abi is not None else None
        if h and lib is not None:
            lib.prores_destroy(h)
            self.handle = None


_contexts = {}
_ctx_lock = threading.Lock()


def context(device: int = 0) -> Context:
    """The process-wide context of `device` (created on first use)."""
    with _ctx_lock:
        if device not in _contexts:
            _contexts[device] = Context(device)
        return _contexts[device]


def _frame_from_c(f: Frame_, data: np.ndarray, alpha: Optional[np.ndarray]) -> Frame:
    chroma = ChromaFormat(f.chroma)
    return Frame(f.width, f.height, f.bit_depth, chroma, Interlace(f.interlace),
                 Metadata(f.aspect_ratio, f.frame_rate_code, f.color_primaries, f.transfer_characteristic,
                          f.matrix_coefficients),
                 data, _layout(f.width, f.height, chroma), alpha)


def _ptr16(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))


class Decoder:
    """src/decode.rs:15-104. Stateless settings; decoding runs on the GPU."""

    def __init__(self, bit_depth: Optional[int] = None, threads: int = 0, device: int = 0):
        self.bit_depth = bit_depth
        self.threads = threads
        self.device = device

    @staticmethod
    def new() -> "Decoder":
        return Decoder()

    @staticmethod
    def with_bit_depth(bit_depth: int) -> "Decoder":
        if not 8 <= bit_depth <= 16:
            raise Error.Config(f"invalid ProRes configuration: output bit depth {bit_depth} is outside 8–16")
        return Decoder(bit_depth)

    def with_threads(self, threads: int) -> "Decoder":
        """Accepted for the crate's API; the output does not depend on it."""
        return replace_decoder(self, threads=threads)

    def decode(self, data: bytes) -> Frame:
        r = self.decode_batch([data])[0]
        if isinstance(r, Error):
            raise r
        return r

    def decode_batch(self, datas: Sequence[bytes], alloc=None, devices: Optional[Sequence[int]] = None
                     ) -> List[Union[Frame, Error]]:
        """Decodes every frame in one batched launch; each entry is a Frame or
        the Error that frame gave. `alloc(n, dtype)`, when given, makes the
        output arrays (for example from a pool of page-locked buffers, which
        the planes then reach by DMA with no host copy). With `devices`, the
        batch is split over those GPUs by macroblock count (one batched call
        each, on host threads of their own) and gathered in input order."""
        L = _abi.lib()
        n = len(datas)
        alloc = alloc or np.empty
        depth = self.bit_depth or 0
        bufs = (Buf_ * max(n, 1))()
        outs = (Frame_ * max(n, 1))()
        status = (ctypes.c_int * max(n, 1))()
        results: List[Union[Frame, Error, None]] = [None] * n
        arrays = [None] * n
        keep = []
        for i, d in enumerate(datas):
            a = _as_u8(d) if len(d) else np.zeros(1, np.uint8)
            keep.append(a)
            bufs[i].data = a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
            bufs[i].len = len(d)
            info = Frame_()
            if L.prores_probe(a.ctypes.data_as(ctypes.c_char_p), len(d), depth, ctypes.byref(info)) == _abi.OK:
                data = alloc(info.data_len, np.uint16)
                alpha = alloc(info.alpha_len, np.uint16) if info.alpha_len else None
                outs[i].data, outs[i].data_len = _ptr16(data), info.data_len
                if alpha is not None:
                    outs[i].alpha, outs[i].alpha_len = _ptr16(alpha), info.alpha_len
                arrays[i] = (data, alpha)
        if devices:
            ctxs = (ctypes.c_void_p * len(devices))(*[context(d).handle for d in devices])
            code = L.prores_decode_batch_multi(ctxs, len(devices), bufs, n, depth, outs, status)
        else:
            code = L.prores_decode_batch(context(self.device).handle, bufs, n, depth, outs, status)
        if code != _abi.OK:
            raise _error(code)
        for i in range(n):
            if status[i] != _abi.OK:
                results[i] = _error(status[i], _abi.batch_error(i))
            else:
                data, alpha = arrays[i]
                results[i] = _frame_from_c(outs[i], data, alpha)
        return results

    def probe_device(self, data, frames, length: Optional[int] = None) -> List[Union["_abi.Frame_", Error]]:
        """Sizes and metadata of frames that lie in device memory (`data`,
        with `frames` as (offset, length) pairs); only their headers are
        read back."""
        n_bytes = int(length if length is not None else data.numel())
        n = len(frames)
        infos = (Frame_ * max(n, 1))()
        status = (ctypes.c_int * max(n, 1))()
        _check(_abi.lib().prores_probe_device(context(self.device).handle, _device_ptr(data), n_bytes,
                                              _spans(frames), n, self.bit_depth or 0, infos, status))
        return [infos[i] if status[i] == _abi.OK else _error(status[i], _abi.batch_error(i)) for i in range(n)]

    def decode_device(self, data, frames, alloc, length: Optional[int] = None, stream=None
                      ) -> List[Union["DeviceFrame", Error]]:
        """Decodes frames that lie in device memory into device buffers that
        `alloc(n_samples)` makes (for example torch int16/uint16 tensors on
        the device); no bitstream or plane crosses to the host."""
        n_bytes = int(length if length is not None else data.numel())
        n = len(frames)
        probes = self.probe_device(data, frames, n_bytes)
        outs = (Frame_ * max(n, 1))()
        status = (ctypes.c_int * max(n, 1))()
        bufs = [None] * n
        for i, info in enumerate(probes):
            if isinstance(info, Error):
                continue
            d = alloc(info.data_len)
            a = alloc(info.alpha_len) if info.alpha_len else None
            bufs[i] = (d, a)
            outs[i].data = ctypes.cast(_device_ptr(d), ctypes.POINTER(ctypes.c_uint16))
            outs[i].data_len = info.data_len
            if a is not None:
                outs[i].alpha = ctypes.cast(_device_ptr(a), ctypes.POINTER(ctypes.c_uint16))
                outs[i].alpha_len = info.alpha_len
        _check(_abi.lib().prores_decode_device(context(self.device).handle, _device_ptr(data), n_bytes,
                                               _spans(frames), n, self.bit_depth or 0, outs, status,
                                               _stream_ptr(stream)))
        res: List[Union[DeviceFrame, Error]] = []
        for i in range(n):
            if status[i] != _abi.OK:
                res.append(_error(status[i], _abi.batch_error(i)))
                continue
            f = outs[i]
            res.append(DeviceFrame(f.width, f.height, f.bit_depth, ChromaFormat(f.chroma), Interlace(f.interlace),
                                   Metadata(f.aspect_ratio, f.frame_rate_code, f.color_primaries,
                                            f.transfer_characteristic, f.matrix_coefficients),
                                   bufs[i][0], bufs[i][1]))
        return res


def scan_frames(data) -> List[tuple]:
    """The (offset, length) of every whole frame in a MOV file or a prefix of
    one, found by its 'icpf' identifier and frame_size without parsing the
    container (the crate's tests/sample.rs:20-38)."""
    a = _as_u8(data) if len(data) else np.zeros(1, np.uint8)
    L = _abi.lib()
    ptr = a.ctypes.data_as(ctypes.c_char_p)
    n = L.prores_scan_frames(ptr, len(data), None, 0)
    spans = (_abi.Span_ * max(n, 1))()
    L.prores_scan_frames(ptr, len(data), spans, n)
    return [(spans[i].offset, spans[i].len) for i in range(n)]


def _device_ptr(x) -> int:
    return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x)


@dataclass
class DeviceFrame:
    """A frame decoded into device memory: the crate's Frame fields, with
    `data` and `alpha` the caller's device buffers (for example torch
    tensors) holding Y'‖Cb‖Cr and the alpha plane."""

    width: int
    height: int
    bit_depth: int
    chroma: "ChromaFormat"
    interlace: "Interlace"
    metadata: "Metadata"
    data: object
    alpha: object = None


def _spans(frames) -> "ctypes.Array":
    arr = (_abi.Span_ * max(len(frames), 1))()
    for i, (off, n) in enumerate(frames):
        arr[i].offset, arr[i].len = int(off), int(n)
    return arr


def scan_frames_device(data, length: Optional[int] = None, stream=None, device: int = 0) -> List[tuple]:
    """scan_frames over bytes in device memory (`data`: a device pointer or
    an object with data_ptr(), such as a torch uint8 tensor)."""
    n_bytes = int(length if length is not None else data.numel())
    ctx = context(device)
    L = _abi.lib()
    cap = 1024
    while True:
        spans = (_abi.Span_ * cap)()
        count = ctypes.c_size_t()
        _check(L.prores_scan_frames_device(ctx.handle, _device_ptr(data), n_bytes, spans, cap, ctypes.byref(count),
                                           _stream_ptr(stream)))
        if count.value <= cap:
            return [(spans[i].offset, spans[i].len) for i in range(count.value)]
        cap = count.value


def replace_decoder(d: Decoder, **kw) -> Decoder:
    return Decoder(kw.get("bit_depth", d.bit_depth), kw.get("threads", d.threads), kw.get("device", d.device))


def _frame_to_c(f: Frame, keep: list) -> Frame_:
    c = Frame_()
    c.width, c.height, c.bit_depth = f.width, f.height, f.bit_depth
    c.chroma = f.chroma.value
    c.interlace = f.interlace.value
    m = f.metadata
    (c.aspect_ratio, c.frame_rate_code, c.color_primaries, c.transfer_characteristic,
     c.matrix_coefficients) = (m.aspect_ratio, m.frame_rate_code, m.color_primaries, m.transfer_characteristic,
                               m.matrix_coefficients)
    d = np.ascontiguousarray(f.data, dtype=np.uint16)
    keep.append(d)
    c.data, c.data_len = _ptr16(d), d.size
    if f.alpha is not None:
        a = np.ascontiguousarray(f.alpha, dtype=np.uint16)
        keep.append(a)
        c.alpha, c.alpha_len = _ptr16(a), a.size
    return c


class Encoder:
    """src/encode.rs:195-287."""

    def __init__(self, config: Config, device: int = 0):
        self._config = config
        self.device = device

    @staticmethod
    def new(config: Config) -> "Encoder":
        return Encoder(config)

    def config(self) -> Config:
        return self._config

    def encode(self, frame: Frame) -> bytes:
        r = self.encode_batch([frame])[0]
        if isinstance(r, Error):
            raise r
        return r

    def encode_batch(self, frames: Sequence[Frame], configs: Optional[Sequence[Config]] = None,
                     devices: Optional[Sequence[int]] = None) -> List[Union[bytes, Error]]:
        """Encodes every frame (each with its own Config, default this
        encoder's) in one batched launch; with `devices`, split over those
        GPUs by macroblock count and gathered in input order."""
        L = _abi.lib()
        n = len(frames)
        configs = list(configs) if configs is not None else [self._config] * n
        keep = []
        cfgs = (Config_ * max(n, 1))()
        ins = (Frame_ * max(n, 1))()
        outs = (Buf_ * max(n, 1))()
        status = (ctypes.c_int * max(n, 1))()
        for i in range(n):
            cfgs[i] = configs[i]._c()
            ins[i] = _frame_to_c(frames[i], keep)
        if devices:
            ctxs = (ctypes.c_void_p * len(devices))(*[context(d).handle for d in devices])
            code = L.prores_encode_batch_multi(ctxs, len(devices), cfgs, ins, n, outs, status)
        else:
            code = L.prores_encode_batch(context(self.device).handle, cfgs, ins, n, outs, status)
        if code != _abi.OK:
            raise _error(code)
        res: List[Union[bytes, Error]] = []
        for i in range(n):
            if status[i] != _abi.OK:
                res.append(_error(status[i], _abi.batch_error(i)))
            else:
                res.append(ctypes.string_at(outs[i].data, outs[i].len))
                L.prores_buffer_free(outs[i].data)
        return res

    def encode_device(self, frames: Sequence["DeviceFrame"], configs: Optional[Sequence[Config]] = None,
                      stream=None) -> List[Union[bytes, Error]]:
        """encode_batch for frames whose planes lie in device memory
        (DeviceFrame: `data`, `alpha` device buffers with data_ptr() and
        numel(), such as torch tensors); the packets come back to the host."""
        L = _abi.lib()
        n = len(frames)
        configs = list(configs) if configs is not None else [self._config] * n
        cfgs = (Config_ * max(n, 1))()
        ins = (Frame_ * max(n, 1))()
        outs = (Buf_ * max(n, 1))()
        status = (ctypes.c_int * max(n, 1))()
        for i, f in enumerate(frames):
            cfgs[i] = configs[i]._c()
            c = ins[i]
            c.width, c.height, c.bit_depth = f.width, f.height, f.bit_depth
            c.chroma, c.interlace = f.chroma.value, f.interlace.value
            m = f.metadata
            (c.aspect_ratio, c.frame_rate_code, c.color_primaries, c.transfer_characteristic,
             c.matrix_coefficients) = (m.aspect_ratio, m.frame_rate_code, m.color_primaries,
                                       m.transfer_characteristic, m.matrix_coefficients)
            c.data = ctypes.cast(_device_ptr(f.data), ctypes.POINTER(ctypes.c_uint16))
            c.data_len = int(f.data.numel())
            if f.alpha is not None:
                c.alpha = ctypes.cast(_device_ptr(f.alpha), ctypes.POINTER(ctypes.c_uint16))
                c.alpha_len = int(f.alpha.numel())
        code = L.prores_encode_device(context(self.device).handle, cfgs, ins, n, outs, status, _stream_ptr(stream))
        if code != _abi.OK:
            raise _error(code)
        res: List[Union[bytes, Error]] = []
        for i in range(n):
            if status[i] != _abi.OK:
                res.append(_error(status[i], _abi.batch_error(i)))
            else:
                res.append(ctypes.string_at(outs[i].data, outs[i].len))
                L.prores_buffer_free(outs[i].data)
        return res


# ------------------------------------------------------------------ resident jobs

def _as_u8(x) -> np.ndarray:
    """A uint8 view of x's bytes (no copy for bytes, bytearray, memoryview
    or arrays)."""
    if isinstance(x, np.ndarray):
        return x if x.dtype == np.uint8 else x.view(np.uint8)
    return np.frombuffer(x, dtype=np.uint8)


def _stream_ptr(stream) -> Optional[int]:
    """A cudaStream_t as an int: accepts None, an int, or any object with a
    `cuda_stream` attribute (torch.cuda.Stream)."""
    if stream is None:
        return None
    return int(getattr(stream, "cuda_stream", stream)) or None


class DecodeJob:
    """A batch of frames kept resident on the device: its bitstreams, slice
    lists and planes stay allocated, so the batch is decoded again with no
    host work (`launch`, optionally as one CUDA-graph launch), new bitstreams
    of the same sizes can be copied in (`upload`) and the planes copied out
    (`fetch`). The building block of batching and serving."""

    def __init__(self, packets: Sequence, bit_depth: Optional[int] = None, device: int = 0):
        self.device = device
        self.n = len(packets)
        self.depth = bit_depth or 0
        self._ctx = context(device)
        self._keep = [_as_u8(p) for p in packets]
        bufs = self._bufs(self._keep)
        h = ctypes.c_void_p()
        _check(_abi.lib().prores_decode_job_create(self._ctx.handle, bufs, self.n, self.depth, ctypes.byref(h)))
        self.handle = h
        self.infos = []
        for p in self._keep:
            info = Frame_()
            ok = _abi.lib().prores_probe(p.ctypes.data_as(ctypes.c_char_p), p.size, self.depth, ctypes.byref(info))
            self.infos.append(info if ok == _abi.OK else None)

    @staticmethod
    def _bufs(arrays):
        bufs = (Buf_ * max(len(arrays), 1))()
        for i, a in enumerate(arrays):
            bufs[i].data = a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
            bufs[i].len = a.size
        return bufs

    def upload(self, packets: Sequence, stream=None):
        arrays = [_as_u8(p) for p in packets]
        self._upload_keep = arrays
        _check(_abi.lib().prores_decode_job_upload(self.handle, self._bufs(arrays), len(arrays), _stream_ptr(stream)))

    def launch(self, stream=None, graph: bool = False):
        _check(_abi.lib().prores_decode_job_launch(self.handle, _stream_ptr(stream), int(graph)))

    def output_arrays(self, alloc=np.empty):
        """Arrays for fetch(): (data, alpha) per frame, made by `alloc(n,
        dtype)` (for example views of pinned memory)."""
        out = []
        for info in self.infos:
            if info is None:
                out.append((None, None))
            else:
                out.append((alloc(info.data_len, np.uint16),
                            alloc(info.alpha_len, np.uint16) if info.alpha_len else None))
        return out

    def fetch(self, stream=None, arrays=None) -> List[Union[Frame, Error]]:
        arrays = arrays if arrays is not None else self.output_arrays()
        outs = (Frame_ * max(self.n, 1))()
        status = (ctypes.c_int * max(self.n, 1))()
        for i, (d, a) in enumerate(arrays):
            if d is not None:
                outs[i].data, outs[i].data_len = _ptr16(d), d.size
            if a is not None:
                outs[i].alpha, outs[i].alpha_len = _ptr16(a), a.size
        _check(_abi.lib().prores_decode_job_fetch(self.handle, _stream_ptr(stream), outs, status))
        res: List[Union[Frame, Error]] = []
        for i in range(self.n):
            if status[i] != _abi.OK:
                res.append(_error(status[i], _abi.batch_error(i)))
            else:
                res.append(_frame_from_c(outs[i], arrays[i][0], arrays[i][1]))
        return res

    def kernel_times(self):
        return _kernel_times(self.handle, 0)

    def close(self):
        if getattr(self, "handle", None):
            _abi.lib().prores_decode_job_destroy(self.handle)
            self.handle = None

    __del__ = close


class EncodeJob:
    """The encode counterpart of DecodeJob: frames, coefficients, rate-control
    tables and the output buffer stay resident; `fetch` returns the packets."""

    def __init__(self, frames: Sequence[Frame], configs: Union[Config, Sequence[Config]], device: int = 0):
        self.device = device
        self.n = len(frames)
        configs = [configs] * self.n if isinstance(configs, Config) else list(configs)
        self._ctx = context(device)
        self._keep = []
        self._cfgs = (Config_ * max(self.n, 1))()
        ins = (Frame_ * max(self.n, 1))()
        for i in range(self.n):
            self._cfgs[i] = configs[i]._c()
            ins[i] = _frame_to_c(frames[i], self._keep)
        h = ctypes.c_void_p()
        _check(_abi.lib().prores_encode_job_create(self._ctx.handle, self._cfgs, ins, self.n, ctypes.byref(h)))
        self.handle = h

    def upload(self, frames: Sequence[Frame], stream=None):
        keep = []
        ins = (Frame_ * max(len(frames), 1))()
        for i, f in enumerate(frames):
            ins[i] = _frame_to_c(f, keep)
        self._upload_keep = keep
        _check(_abi.lib().prores_encode_job_upload(self.handle, ins, len(frames), _stream_ptr(stream)))

    def launch(self, stream=None, graph: bool = False):
        _check(_abi.lib().prores_encode_job_launch(self.handle, _stream_ptr(stream), int(graph)))

    def fetch(self, stream=None, copy: bool = True) -> List[Union[bytes, memoryview, Error]]:
        outs = (Buf_ * max(self.n, 1))()
        status = (ctypes.c_int * max(self.n, 1))()
        _check(_abi.lib().prores_encode_job_fetch(self.handle, _stream_ptr(stream), outs, status))
        res: List[Union[bytes, memoryview, Error]] = []
        for i in range(self.n):
            if status[i] != _abi.OK:
                res.append(_error(status[i], _abi.batch_error(i)))
            elif copy:
                res.append(ctypes.string_at(outs[i].data, outs[i].len))
            else:
                res.append(memoryview((ctypes.c_uint8 * outs[i].len).from_address(
                    ctypes.addressof(outs[i].data.contents))) if outs[i].len else memoryview(b""))
        return res

    def kernel_times(self):
        return _kernel_times(self.handle, 1)

    def close(self):
        if getattr(self, "handle", None):
            _abi.lib().prores_encode_job_destroy(self.handle)
            self.handle = None

    __del__ = close


def _kernel_times(handle, is_encode: int):
    """(name, ms) of each kernel of the job's last launch, when the job was
    made with PRORES_PROFILE_KERNELS=1 in the environment."""
    names = (ctypes.c_char_p * 64)()
    ms = (ctypes.c_float * 64)()
    n = _abi.lib().prores_job_kernel_times(handle, is_encode, names, ms, 64)
    return [(names[i].decode(), float(ms[i])) for i in range(max(n, 0))]
