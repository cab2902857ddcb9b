"""B200-native ProRes RAW decode, linearize and develop.

A drop-in for the hot path of the proresraw_rs crate (src/lib.rs:50-66):
`decode_frame`, `decode_frame_with(Idct.APPLE | Idct.FFMPEG)`,
`decode_frame_reduced(_with)`, `Frame.linearize(_into)` and
`develop`, `develop_with`, `develop_into`, `develop_planar(_into)`, with the
crate's names, argument meaning and error behaviour. The work runs in the
hand-written CUDA kernels of libprr.so behind the C ABI of include/prr.h;
there is no CPU path. Device buffers are torch CUDA tensors (plumbing only);
the `_into` forms also accept host numpy arrays, which are filled by a copy
from the device.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import threading
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib

BLACK_LEVEL = 256  # src/header.rs:7
PREFIX_LEN = 10    # src/decoder.rs:13
FOURCCS = (b"aprn", b"aprh")  # src/lib.rs:68-75


def is_prores_raw_fourcc(fourcc: bytes) -> bool:
    return bytes(fourcc).lower() in FOURCCS


class Idct(enum.IntEnum):
    """src/idct.rs:20-26"""
    APPLE = 0
    FFMPEG = 1


class Scale(enum.IntEnum):
    """src/reduced.rs:25-61; the value is log2 of the factor."""
    HALF = 1
    QUARTER = 2
    EIGHTH = 3

    def factor(self) -> int:
        return 1 << int(self)


class Greens(enum.IntEnum):
    """src/reduced.rs:65-72"""
    FIRST = 0
    AVERAGE = 1


class Stage(enum.IntEnum):
    """src/demosaic.rs:112-123"""
    DEMOSAICED = 0
    WHITE_BALANCED = 1
    REC2020 = 2


class Exposure(enum.IntEnum):
    """src/demosaic.rs:127-133"""
    NORMALIZED = 0
    REFLECTION = 1


class BayerPattern(enum.IntEnum):
    """src/header.rs:20-96 (value = header code)."""
    RGGB = 0
    GRBG = 1
    GBRG = 2
    BGGR = 3

    def red_position(self) -> Tuple[int, int]:
        return {0: (0, 0), 1: (0, 1), 2: (1, 0), 3: (1, 1)}[int(self)]

    def stream_phases(self):
        r, c = self.red_position()
        return [(1 - r, c), (r, 1 - c), (1 - r, 1 - c), (r, c)]

    def color_at(self, row: int, col: int) -> str:
        rr, rc = self.red_position()
        row, col = row & 1, col & 1
        if (row, col) == (rr, rc):
            return "red"
        if (row, col) == (rr ^ 1, rc ^ 1):
            return "blue"
        return "green"


_ERROR_NAMES = {
    _lib.ERR_TRUNCATED: "Truncated",
    _lib.ERR_FRAME_SIZE_MISMATCH: "FrameSizeMismatch",
    _lib.ERR_BAD_QUANT_MATRIX: "BadQuantMatrix",
    _lib.ERR_BAD_CURVE: "BadCurve",
    _lib.ERR_UNEXPECTED_CURVE: "UnexpectedCurve",
    _lib.ERR_BAD_TAG: "BadTag",
    _lib.ERR_HEADER_TOO_SHORT: "HeaderTooShort",
    _lib.ERR_UNSUPPORTED_VERSION: "UnsupportedVersion",
    _lib.ERR_BAD_DIMENSIONS: "BadDimensions",
    _lib.ERR_BAD_ALIGNMENT: "BadAlignment",
    _lib.ERR_TILE_OUT_OF_BOUNDS: "TileOutOfBounds",
    _lib.ERR_BAD_TILE_HEADER: "BadTileHeader",
    _lib.ERR_BUFFER: "Buffer",
    _lib.ERR_CUDA: "Cuda",
    _lib.ERR_TIMEOUT: "Timeout",
    _lib.ERR_INVALID: "Invalid",
    _lib.ERR_NO_MEMORY: "NoMemory",
}


class Error(Exception):
    """The crate's `Error` (src/error.rs:6-63): `kind` names the variant and
    `fields` holds its payload."""

    def __init__(self, code: int, fields: Optional[dict] = None, message: str = ""):
        self.code = code
        self.kind = _ERROR_NAMES.get(code, f"Status{code}")
        self.fields = fields or {}
        super().__init__(message or f"{self.kind} {self.fields}")

    def __eq__(self, other):
        return isinstance(other, Error) and (self.kind, self.fields) == (other.kind, other.fields)

    __hash__ = Exception.__hash__


def _error(code: int, e: Optional[_lib.CError] = None, ctx=None) -> Error:
    f: dict = {}
    if e is not None:
        if code == _lib.ERR_TRUNCATED:
            f = {"what": e.what.decode(), "needed": e.needed, "available": e.available}
        elif code == _lib.ERR_FRAME_SIZE_MISMATCH:
            f = {"declared": e.declared, "actual": e.actual}
        elif code == _lib.ERR_BAD_QUANT_MATRIX:
            f = {"index": e.index, "value": e.value}
        elif code == _lib.ERR_BAD_CURVE:
            f = {"points": list(e.curve)}
        elif code == _lib.ERR_BAD_TAG:
            f = {"tag": bytes(e.tag)}
        elif code in (_lib.ERR_HEADER_TOO_SHORT, _lib.ERR_UNSUPPORTED_VERSION, _lib.ERR_BAD_ALIGNMENT):
            f = {"value": e.value}
        elif code == _lib.ERR_BAD_DIMENSIONS:
            f = {"width": e.width, "height": e.height}
        elif code in (_lib.ERR_TILE_OUT_OF_BOUNDS, _lib.ERR_BAD_TILE_HEADER):
            f = {"tile": e.index}
    msg = ""
    if code == _lib.ERR_CUDA and ctx is not None:
        msg = "CUDA error: " + (_lib.lib().prr_last_error_string(ctx) or b"").decode()
    return Error(code, f, msg)


# ---------------------------------------------------------------------------
# Header


@dataclasses.dataclass
class Curve:
    """src/curve.rs:7-33"""
    points: Tuple[int, ...]

    DEFAULT_POINTS = (0, 512, 1024, 2048, 4096, 8192, 16384, 32768)

    def linearize(self, code: int) -> int:
        seg, frac = code >> 13, code & 0x1FFF
        c0 = self.points[seg]
        c1 = self.points[seg + 1] if seg < 7 else 65536
        return min((c0 * 8192 + ((c1 - c0) & 0xFFFF) * frac + 4096) >> 13, 65535)


@dataclasses.dataclass
class FrameHeader:
    """src/header.rs:112-146"""
    version: int
    vendor: bytes
    width: int
    height: int
    crop: Tuple[int, int, int, int]
    bayer_pattern: BayerPattern
    white_level: int
    wb_red: float
    wb_blue: float
    color_matrix: Tuple[Tuple[float, float, float], ...]
    gain: float
    wb_cct: int
    flags: int
    alignment: int
    quant_matrix: Tuple[int, ...]
    curve: Curve
    _c: _lib.CHeader = dataclasses.field(repr=False, compare=False, default=None)

    def coded_width(self) -> int:
        return (self.width + 15) & ~15

    def coded_height(self) -> int:
        return (self.height + 15) & ~15

    @staticmethod
    def _from_c(h: _lib.CHeader) -> "FrameHeader":
        keep = _lib.CHeader()
        C.memmove(C.byref(keep), C.byref(h), C.sizeof(h))
        m = list(h.color_matrix)
        return FrameHeader(
            version=h.version, vendor=bytes(h.vendor), width=h.width, height=h.height,
            crop=tuple(h.crop), bayer_pattern=BayerPattern(h.bayer_pattern), white_level=h.white_level,
            wb_red=h.wb_red, wb_blue=h.wb_blue, color_matrix=(tuple(m[0:3]), tuple(m[3:6]), tuple(m[6:9])),
            gain=h.gain, wb_cct=h.wb_cct, flags=h.flags, alignment=h.alignment,
            quant_matrix=tuple(h.quant_matrix), curve=Curve(tuple(h.curve)), _c=keep,
        )


def _pkt(packet) -> Tuple[object, int]:
    """(buffer, length) of a bytes-like or numpy packet in host memory: a
    uint8 view of the caller's bytes, not a copy (the library only reads
    them)."""
    if isinstance(packet, np.ndarray):
        a = np.ascontiguousarray(packet, dtype=np.uint8).reshape(-1)
    else:
        a = np.frombuffer(packet, dtype=np.uint8)
    if a.size == 0:
        return np.zeros(1, dtype=np.uint8), 0
    return a, a.size


def _ptr(obj) -> int:
    if isinstance(obj, np.ndarray):
        return obj.ctypes.data
    return C.addressof(obj)


def header_len(packet) -> int:
    """src/decoder.rs:58-73"""
    buf, n = _pkt(packet)
    out, err = C.c_size_t(), _lib.CError()
    rc = _lib.lib().prr_header_len(_ptr(buf), n, C.byref(out), C.byref(err))
    if rc:
        raise _error(rc, err)
    return out.value


def parse_header(packet) -> FrameHeader:
    """src/decoder.rs:45-53"""
    buf, n = _pkt(packet)
    h, err = _lib.CHeader(), _lib.CError()
    rc = _lib.lib().prr_parse_header(_ptr(buf), n, C.byref(h), C.byref(err))
    if rc:
        raise _error(rc, err)
    return FrameHeader._from_c(h)


@dataclasses.dataclass
class ParsedFrame:
    """src/decoder.rs:17-29 (tile payloads are left in the packet)."""
    header: FrameHeader
    ntiles: int
    tiles_per_row: int
    tile_rows: int
    max_qscale: int
    info: _lib.CFrameInfo = dataclasses.field(repr=False, default=None)


def parse_frame(packet) -> ParsedFrame:
    """src/decoder.rs:76-123, on the host."""
    buf, n = _pkt(packet)
    info, mq, err = _lib.CFrameInfo(), C.c_uint8(), _lib.CError()
    rc = _lib.lib().prr_parse_frame(_ptr(buf), n, C.byref(info), C.byref(mq), C.byref(err))
    if rc:
        raise _error(rc, err)
    return ParsedFrame(FrameHeader._from_c(info.header), info.ntiles, info.tiles_per_row, info.tile_rows,
                       mq.value, info)


def frame_info(packet) -> _lib.CFrameInfo:
    """The host half of parse_frame (prefix, header, size-table bounds)."""
    buf, n = _pkt(packet)
    info, err = _lib.CFrameInfo(), _lib.CError()
    rc = _lib.lib().prr_frame_info_parse(_ptr(buf), n, C.byref(info), C.byref(err))
    if rc:
        raise _error(rc, err)
    return info


def frame_quantizer(parsed: ParsedFrame) -> int:
    """src/demosaic.rs:50-52"""
    return parsed.header.quant_matrix[0] * parsed.max_qscale


# ---------------------------------------------------------------------------
# Contexts: one per (device, torch stream), so that the kernels run in
# stream order with the torch tensors they read and write.

_CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy in cuda_runtime_api.h
_ctx_lock = threading.Lock()
_contexts: Dict[Tuple[int, int], C.c_void_p] = {}


def _torch():
    import torch

    return torch


def context(device: Optional[int] = None) -> C.c_void_p:
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError("proresraw_rs_b200 needs a CUDA device (there is no CPU path)")
    dev = torch.cuda.current_device() if device is None else device
    stream = torch.cuda.current_stream(dev).cuda_stream
    # torch's default stream is the legacy NULL stream; a NULL handle would
    # make the library create a stream of its own, so name the legacy
    # stream explicitly (cudaStreamLegacy).
    handle = stream if stream else _CUDA_STREAM_LEGACY
    key = (dev, stream)
    with _ctx_lock:
        ctx = _contexts.get(key)
        if ctx is None:
            ctx = C.c_void_p()
            rc = _lib.lib().prr_ctx_create(dev, C.c_void_p(handle), C.byref(ctx))
            if rc:
                raise _error(rc)
            _contexts[key] = ctx
    return ctx


def kernel_launches() -> int:
    """Kernel launches made through libprr.so so far."""
    return int(_lib.lib().prr_kernel_launches())


def _check(rc: int, err=None, ctx=None):
    if rc:
        raise _error(rc, err, ctx)


def _dptr(t) -> int:
    return t.data_ptr()


# ---------------------------------------------------------------------------
# Decoding


class Frame:
    """A decoded frame (src/decoder.rs:132-217): code values of every sensel
    over the coded size, on the device (`samples`, a torch uint16 tensor)."""

    def __init__(self, header: FrameHeader, samples, skipped_tiles: List[int], max_qscale: int):
        self.header = header
        self.samples = samples
        self.skipped_tiles = skipped_tiles
        self.max_qscale = max_qscale

    def quantizer(self) -> int:
        return self.header.quant_matrix[0] * self.max_qscale

    def width(self) -> int:
        return self.header.width

    def height(self) -> int:
        return self.header.height

    def stride(self) -> int:
        return self.header.coded_width()

    def samples_host(self) -> np.ndarray:
        return self.samples.cpu().numpy().view(np.uint16)

    def linearize(self):
        """Linear values of the visible picture, tightly packed, on the device."""
        torch = _torch()
        out = torch.empty(self.width() * self.height(), dtype=torch.uint16, device=self.samples.device)
        self.linearize_into(out)
        return out

    def linearize_into(self, out) -> None:
        """src/decoder.rs:197-216. `out`: device tensor or host numpy array."""
        n = self.width() * self.height()
        if _numel(out) != n:
            raise Error(_lib.ERR_BUFFER, message="output size")
        torch = _torch()
        dev = out if _is_cuda(out) else torch.empty(n, dtype=torch.uint16, device=self.samples.device)
        ctx = context(self.samples.device.index)
        _check(_lib.lib().prr_linearize(ctx, C.byref(self.header._c), _dptr(self.samples), _dptr(dev), n), ctx=ctx)
        if dev is not out:
            _to_host(dev, out)


def _numel(a) -> int:
    return a.size if isinstance(a, np.ndarray) else a.numel()


def _is_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


def _to_host(dev, out) -> None:
    if isinstance(out, np.ndarray):
        host = dev.cpu().numpy()
        out.reshape(-1)[:] = host.view(out.dtype).reshape(-1)
    else:
        out.copy_(dev.reshape(out.shape))


def _decode_common(packet, reduced: bool, idct=Idct.APPLE, scale=Scale.HALF, greens=Greens.FIRST):
    torch = _torch()
    info = frame_info(packet)
    cw, ch = info.coded_width, info.coded_height
    if reduced:
        n = 3 * (cw >> int(scale)) * (ch >> int(scale))
    else:
        n = cw * ch
    ctx = context()
    out = torch.empty(n, dtype=torch.uint16, device="cuda")
    buf, ln = _pkt(packet)
    skipped = (C.c_uint64 * max(1, info.ntiles))()
    res, err = _lib.CDecodeResult(), _lib.CError()
    res.skipped = skipped
    res.skipped_cap = info.ntiles
    if reduced:
        rc = _lib.lib().prr_decode_reduced(ctx, _ptr(buf), ln, int(scale), int(greens), _dptr(out), n,
                                           C.byref(res), C.byref(err))
    else:
        rc = _lib.lib().prr_decode(ctx, _ptr(buf), ln, int(idct), _dptr(out), n, C.byref(res), C.byref(err))
    _check(rc, err, ctx)
    header = FrameHeader._from_c(res.header)
    skipped_list = [int(skipped[i]) for i in range(min(res.n_skipped, info.ntiles))]
    return header, out, skipped_list, res.max_qscale


def decode_frame(packet) -> Frame:
    """src/decoder.rs:221-223"""
    return decode_frame_with(packet, Idct.APPLE)


def decode_frame_with(packet, idct: Idct) -> Frame:
    """src/decoder.rs:226-267"""
    header, samples, skipped, mq = _decode_common(packet, False, idct=idct)
    return Frame(header, samples, skipped, mq)


class RgbFrame:
    """A reduced-resolution decode (src/reduced.rs:75-132): linear RGB,
    interleaved, over the coded size divided by the scale, on the device."""

    def __init__(self, header, scale, greens, samples, skipped_tiles, max_qscale):
        self.header = header
        self.scale = Scale(scale)
        self.greens = Greens(greens)
        self.samples = samples
        self.skipped_tiles = skipped_tiles
        self.max_qscale = max_qscale

    def width(self) -> int:
        return self.header.width >> int(self.scale)

    def height(self) -> int:
        return self.header.height >> int(self.scale)

    def stride(self) -> int:
        return self.header.coded_width() >> int(self.scale)

    def quantizer(self) -> int:
        return self.header.quant_matrix[0] * self.max_qscale

    def samples_host(self) -> np.ndarray:
        return self.samples.cpu().numpy().view(np.uint16)

    def to_packed(self) -> np.ndarray:
        s = self.samples_host().reshape(-1, self.stride(), 3)
        return s[: self.height(), : self.width(), :].reshape(-1).copy()


def decode_frame_reduced(packet, scale: Scale) -> RgbFrame:
    """src/reduced.rs:142-144"""
    return decode_frame_reduced_with(packet, scale, Greens.FIRST)


def decode_frame_reduced_with(packet, scale: Scale, greens: Greens) -> RgbFrame:
    """src/reduced.rs:147-201"""
    header, samples, skipped, mq = _decode_common(packet, True, scale=scale, greens=greens)
    return RgbFrame(header, scale, greens, samples, skipped, mq)


# ---------------------------------------------------------------------------
# Develop


@dataclasses.dataclass
class DemosaicParams:
    """src/demosaic.rs:57-106"""
    cfa_phase: int
    black: int
    one_over_range: float
    noise: Tuple[float, float, float]
    clip: Tuple[float, float]
    black_over_range: float
    wb: Tuple[float, float]

    @staticmethod
    def new(header: FrameHeader, quantizer: int) -> "DemosaicParams":
        p = _lib.CParams()
        _check(_lib.lib().prr_params_new(C.byref(header._c), quantizer, C.byref(p)))
        return DemosaicParams._from_c(p)

    @staticmethod
    def with_white_balance(header: FrameHeader, quantizer: int, red: float, blue: float) -> "DemosaicParams":
        p = _lib.CParams()
        _check(_lib.lib().prr_params_with_white_balance(C.byref(header._c), quantizer, red, blue, C.byref(p)))
        return DemosaicParams._from_c(p)

    @staticmethod
    def _from_c(p: _lib.CParams) -> "DemosaicParams":
        return DemosaicParams(p.cfa_phase, p.black, p.one_over_range, tuple(p.noise), tuple(p.clip),
                              p.black_over_range, tuple(p.wb))

    def _c(self) -> _lib.CParams:
        p = _lib.CParams()
        p.cfa_phase, p.black, p.one_over_range = self.cfa_phase, self.black, self.one_over_range
        p.noise[:] = list(self.noise)
        p.clip[:] = list(self.clip)
        p.black_over_range = self.black_over_range
        p.wb[:] = list(self.wb)
        return p


def output_matrix(header: FrameHeader, exposure: Exposure = Exposure.NORMALIZED) -> np.ndarray:
    """src/demosaic.rs:138-153"""
    m = np.zeros(9, dtype=np.float32)
    _check(_lib.lib().prr_output_matrix(C.byref(header._c), int(exposure), m.ctypes.data))
    return m


@dataclasses.dataclass
class RgbImage:
    """src/demosaic.rs:158-165; `data` is a device tensor of 3*w*h f32."""
    width: int
    height: int
    data: object


@dataclasses.dataclass
class RgbPlanes:
    """src/demosaic.rs:169-178; `planes` are three device tensors of w*h f32."""
    width: int
    height: int
    planes: List[object]


def develop(frame: Frame, stage: Stage = Stage.WHITE_BALANCED) -> RgbImage:
    """src/demosaic.rs:190-193"""
    return develop_with(frame, DemosaicParams.new(frame.header, frame.quantizer()), stage)


def develop_with(frame: Frame, params: DemosaicParams, stage: Stage) -> RgbImage:
    """src/demosaic.rs:206-215"""
    torch = _torch()
    w, h = frame.width(), frame.height()
    data = torch.empty(3 * w * h, dtype=torch.float32, device=frame.samples.device)
    develop_into(frame, params, stage, data)
    return RgbImage(w, h, data)


def _develop(frame: Frame, params: DemosaicParams, stage: Stage, layout: int, outs: Sequence) -> None:
    torch = _torch()
    w, h = frame.width(), frame.height()
    n = w * h
    want = n if layout == 1 else 3 * n
    for o in outs:
        if _numel(o) != want:
            raise Error(_lib.ERR_BUFFER, message="plane size" if layout == 1 else "output size")
    dev = [o if _is_cuda(o) else torch.empty(want, dtype=torch.float32, device=frame.samples.device) for o in outs]
    ctx = context(frame.samples.device.index)
    ptrs = [_dptr(d) for d in dev] + [None] * (3 - len(dev))
    rc = _lib.lib().prr_develop(ctx, C.byref(frame.header._c), C.byref(params._c()), int(stage),
                                _dptr(frame.samples), layout, ptrs[0], ptrs[1], ptrs[2], want)
    _check(rc, ctx=ctx)
    for d, o in zip(dev, outs):
        if d is not o:
            _to_host(d, o)


def develop_into(frame: Frame, params: DemosaicParams, stage: Stage, out) -> None:
    """src/demosaic.rs:223-227: interleaved RGB into a caller buffer."""
    _develop(frame, params, stage, 0, [out])


def develop_planar(frame: Frame, params: DemosaicParams, stage: Stage) -> RgbPlanes:
    """src/demosaic.rs:232-242"""
    torch = _torch()
    w, h = frame.width(), frame.height()
    planes = [torch.empty(w * h, dtype=torch.float32, device=frame.samples.device) for _ in range(3)]
    develop_planar_into(frame, params, stage, planes)
    return RgbPlanes(w, h, planes)


def develop_planar_into(frame: Frame, params: DemosaicParams, stage: Stage, out: Sequence) -> None:
    """src/demosaic.rs:250-261: three caller planes."""
    if len(out) != 3:
        raise Error(_lib.ERR_BUFFER, message="plane size")
    _develop(frame, params, stage, 1, list(out))


@dataclasses.dataclass
class DevelopConfig:
    """Launch shape of the develop kernel (prr_develop_config): output tile
    32x32 (default), 32x16 or 64x16, and CTAs per SM (0: as many as fit)."""
    tile_w: int = 32
    tile_h: int = 32
    ctas_per_sm: int = 0

    def _c(self) -> _lib.CDevelopConfig:
        return _lib.CDevelopConfig(self.tile_w, self.tile_h, self.ctas_per_sm)

    @staticmethod
    def _from_c(c: _lib.CDevelopConfig) -> "DevelopConfig":
        return DevelopConfig(int(c.tile_w), int(c.tile_h), int(c.ctas_per_sm))


def develop_bucket(width: int, height: int) -> int:
    """The frame-size bucket the develop's launch shape is kept for."""
    return int(_lib.lib().prr_develop_bucket(width, height))


def develop_set_config(bucket: int, cfg: DevelopConfig) -> None:
    """Use `cfg` for the frames of `bucket` (current device and stream)."""
    ctx = context()
    c = cfg._c()
    _check(_lib.lib().prr_develop_set_config(ctx, bucket, C.byref(c)), ctx=ctx)


def develop_get_config(bucket: int) -> DevelopConfig:
    ctx = context()
    c = _lib.CDevelopConfig()
    _check(_lib.lib().prr_develop_get_config(ctx, bucket, C.byref(c)), ctx=ctx)
    return DevelopConfig._from_c(c)


def develop_tune(frame: Frame, params: DemosaicParams, stage: Stage, out: Sequence,
                 reps: int = 3) -> Tuple[DevelopConfig, float]:
    """prr_develop_tune: develop `frame` into the device planes `out` (3
    planes, or one interleaved buffer) with every candidate launch shape;
    the fastest becomes the config of the frame's size bucket. Returns
    (config, median ms)."""
    w, h = frame.width(), frame.height()
    layout = 1 if len(out) == 3 else 0
    want = w * h if layout == 1 else 3 * w * h
    ctx = context(frame.samples.device.index)
    ptrs = [_dptr(o) for o in out] + [None] * (3 - len(out))
    best, ms = _lib.CDevelopConfig(), C.c_float()
    _check(_lib.lib().prr_develop_tune(ctx, C.byref(frame.header._c), C.byref(params._c()), int(stage),
                                       _dptr(frame.samples), layout, ptrs[0], ptrs[1], ptrs[2], want, reps,
                                       C.byref(best), C.byref(ms)), ctx=ctx)
    return DevelopConfig._from_c(best), float(ms.value)


# ---------------------------------------------------------------------------
# Batched decode (prr_batch_* in include/prr.h): many frames of any mix of
# sizes, versions, patterns, qscales and alignments, full or reduced, in one
# persistent kernel. Each job's result is what decode_frame_with or
# decode_frame_reduced_with returns for its packet, or the Error it raises.


@dataclasses.dataclass
class BatchJob:
    packet: object
    scale: Optional[Scale] = None  # None: full resolution
    idct: Idct = Idct.APPLE
    greens: Greens = Greens.FIRST


@dataclasses.dataclass
class BatchConfig:
    """Launch shape of the batch kernel for one bucket of batches: CTAs per
    SM, packet bytes an entropy item stages, graph replay, and the
    component streams each thread decodes in an entropy item (1, 2 or 4:
    items of 64, 128 or 256 tiles, 256 threads a CTA)."""
    ctas_per_sm: int = 0  # 0: as many as fit
    stage_bytes: int = 32 * 1024
    use_graph: bool = True
    streams_per_thread: int = 2

    def _c(self) -> _lib.CBatchConfig:
        return _lib.CBatchConfig(self.ctas_per_sm, self.stage_bytes, 1 if self.use_graph else 0,
                                 self.streams_per_thread)

    @staticmethod
    def _from_c(c: _lib.CBatchConfig) -> "BatchConfig":
        return BatchConfig(int(c.ctas_per_sm), int(c.stage_bytes), bool(c.use_graph),
                           int(c.streams_per_thread) or 2)


class BatchDecoder:
    """A context's batch decoder: submit / wait, per-bucket launch shapes
    and the autotuner that picks them."""

    def __init__(self, device: Optional[int] = None):
        # The context of the device's current stream: decoders made under
        # different streams have contexts (and batch buffers) of their own.
        self.ctx = context(device)
        self._pending = None

    def _prepare(self, jobs: Sequence[BatchJob], outs=None):
        torch = _torch()
        n = len(jobs)
        arr = (_lib.CJob * max(1, n))()
        keep = []
        frames = []
        for i, job in enumerate(jobs):
            buf, ln = _pkt(job.packet)
            keep.append(buf)
            cj = arr[i]
            cj.packet = _ptr(buf)
            cj.len = ln
            cj.scale = _lib.SCALE_FULL if job.scale is None else int(job.scale)
            cj.idct = int(job.idct)
            cj.greens = int(job.greens)
            out = None if outs is None else outs[i]
            ntiles = 1
            if out is None:
                try:
                    info = frame_info(job.packet)
                    ntiles = max(1, info.ntiles)
                    cw, ch = info.coded_width, info.coded_height
                    if job.scale is None:
                        n_out = cw * ch
                    else:
                        n_out = 3 * (cw >> int(job.scale)) * (ch >> int(job.scale))
                    out = torch.empty(max(1, n_out), dtype=torch.uint16, device="cuda")
                except Error:
                    out = torch.empty(1, dtype=torch.uint16, device="cuda")
            else:
                try:
                    ntiles = max(1, frame_info(job.packet).ntiles)
                except Error:
                    pass
            cj.dev_out = _dptr(out)
            cj.out_len = _numel(out)
            skipped = (C.c_uint64 * ntiles)()
            cj.result.skipped = skipped
            cj.result.skipped_cap = ntiles
            keep.append(skipped)
            frames.append((out, skipped))
        return arr, keep, frames

    def _results(self, jobs, arr, frames) -> List[object]:
        results = []
        for i, job in enumerate(jobs):
            cj = arr[i]
            if cj.status:
                results.append(_error(cj.status, cj.error, self.ctx))
                continue
            out, skipped = frames[i]
            header = FrameHeader._from_c(cj.result.header)
            sk = [int(skipped[k]) for k in range(min(int(cj.result.n_skipped), int(cj.result.skipped_cap)))]
            if job.scale is None:
                results.append(Frame(header, out, sk, int(cj.result.max_qscale)))
            else:
                results.append(RgbFrame(header, job.scale, job.greens, out, sk, int(cj.result.max_qscale)))
        return results

    def decode(self, jobs: Sequence[BatchJob], outs=None) -> List[object]:
        """Decode every job; each result is a Frame, an RgbFrame or an Error.
        `outs` optionally gives each job's device output tensor."""
        self.submit(jobs, outs)
        return self.wait()

    def submit(self, jobs: Sequence[BatchJob], outs=None) -> None:
        """prr_batch_submit: parse and stage the batch, queue its upload and
        kernels on the decoder's stream, and return without waiting for
        them; wait() gives the results. One batch at a time per decoder (a
        second submit before wait() raises PRR_ERR_INVALID). Two decoders
        made under two streams pipeline: while one decoder's kernels run,
        the other stages and uploads the next batch."""
        arr, keep, frames = self._prepare(jobs, outs)
        _check(_lib.lib().prr_batch_submit(self.ctx, arr, len(jobs)), ctx=self.ctx)
        self._pending = (list(jobs), arr, keep, frames)

    def wait(self, timeout_ms: int = 0) -> List[object]:
        """prr_batch_wait: block until the submitted batch is decoded (0: no
        time limit) and return its results, as decode() does."""
        if self._pending is None:
            raise _error(_lib.ERR_INVALID)
        jobs, arr, keep, frames = self._pending
        _check(_lib.lib().prr_batch_wait(self.ctx, timeout_ms), ctx=self.ctx)
        self._pending = None
        return self._results(jobs, arr, frames)

    def last_ms(self) -> float:
        """Device time of the last batch's kernels, in milliseconds."""
        ms = C.c_float()
        _check(_lib.lib().prr_batch_last_ms(self.ctx, C.byref(ms)), ctx=self.ctx)
        return float(ms.value)

    def bucket(self, jobs: Sequence[BatchJob]) -> int:
        arr, keep, _ = self._prepare(jobs)
        b = C.c_uint32()
        _check(_lib.lib().prr_batch_bucket(self.ctx, arr, len(jobs), C.byref(b)), ctx=self.ctx)
        return int(b.value)

    def tune(self, jobs: Sequence[BatchJob], reps: int = 3) -> Tuple[BatchConfig, float]:
        """Time each candidate launch shape on this batch; the fastest
        becomes its bucket's config. Returns (config, median ms)."""
        arr, keep, frames = self._prepare(jobs)
        best, ms = _lib.CBatchConfig(), C.c_float()
        _check(_lib.lib().prr_batch_tune(self.ctx, arr, len(jobs), reps, C.byref(best), C.byref(ms)),
               ctx=self.ctx)
        return BatchConfig._from_c(best), float(ms.value)

    def set_config(self, bucket: int, cfg: BatchConfig) -> None:
        c = cfg._c()
        _check(_lib.lib().prr_batch_set_config(self.ctx, bucket, C.byref(c)), ctx=self.ctx)

    def get_config(self, bucket: int) -> BatchConfig:
        c = _lib.CBatchConfig()
        _check(_lib.lib().prr_batch_get_config(self.ctx, bucket, C.byref(c)), ctx=self.ctx)
        return BatchConfig._from_c(c)

    def set_wait_limit(self, microseconds: int) -> None:
        """prr_batch_set_wait_limit: how long a transform segment waits for
        the entropy chunks of its tiles before its frame reports
        PRR_ERR_TIMEOUT (0: the 2 s default)."""
        _check(_lib.lib().prr_batch_set_wait_limit(self.ctx, int(microseconds)), ctx=self.ctx)

    def drop_chunk_for_test(self, chunk: Optional[int]) -> None:
        """prr_batch_drop_chunk_for_test: from the next batch on, entropy
        chunk `chunk` is claimed and abandoned, so that the waits on it run
        out (None: off)."""
        v = 0xFFFFFFFF if chunk is None else int(chunk)
        _check(_lib.lib().prr_batch_drop_chunk_for_test(self.ctx, v), ctx=self.ctx)


def decode_batch(jobs: Sequence[BatchJob]) -> List[object]:
    """Decode a batch of frames on the current device (see BatchDecoder)."""
    return BatchDecoder().decode(jobs)


__all__ = [
    "BLACK_LEVEL", "PREFIX_LEN", "FOURCCS", "is_prores_raw_fourcc", "Idct", "Scale", "Greens", "Stage",
    "Exposure", "BayerPattern", "Error", "Curve", "FrameHeader", "ParsedFrame", "header_len", "parse_header",
    "parse_frame", "frame_info", "frame_quantizer", "context", "kernel_launches", "Frame", "decode_frame",
    "decode_frame_with", "RgbFrame", "decode_frame_reduced", "decode_frame_reduced_with", "DemosaicParams",
    "output_matrix", "RgbImage", "RgbPlanes", "develop", "develop_with", "develop_into", "develop_planar",
    "develop_planar_into", "DevelopConfig", "develop_bucket", "develop_set_config", "develop_get_config",
    "develop_tune", "BatchJob", "BatchConfig", "BatchDecoder", "decode_batch",
]
