"""DNG export of decoded frames (prr_dng_* / prr_lj92_* in include/prr.h),
mirroring the crate's DNG writer (examples/prr2dng: dng.rs, lj92.rs,
tiff.rs, colour.rs).

`write(frame, clip)` gives the bytes of one frame's DNG file: the visible
picture as 16-bit CFA data, as code values with the curve as the
`LinearizationTable` or as linear values, stored as 256-square lossless JPEG
tiles (encoded on the device) or as one uncompressed strip, with the
crate's tags. `lj92_tiles` exposes the device tile encoder alone.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import enum
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import FrameHeader, _check, _dptr, _error, _lib, context


class Samples(enum.IntEnum):
    """dng::Samples (dng.rs:36-43)."""

    CODE_VALUES = _lib.DNG_CODE_VALUES
    LINEAR = _lib.DNG_LINEAR


class Compression(enum.IntEnum):
    """dng::Compression (dng.rs:27-34)."""

    NONE = _lib.DNG_UNCOMPRESSED
    LOSSLESS_JPEG = _lib.DNG_LJ92


TILE = 256  # dng.rs:23-25
SOFTWARE = "proresraw_rs prr2dng 0.1.0"


@dataclasses.dataclass
class ClipInfo:
    """Facts about the clip that every frame's file repeats (dng.rs:46-57)."""

    make: Optional[str] = None
    model: Optional[str] = None
    fps: Optional[Tuple[int, int]] = None
    date_time: Optional[str] = None  # "YYYY:MM:DD HH:MM:SS"
    orientation: int = 1  # EXIF 1..8
    software: str = SOFTWARE

    @staticmethod
    def of_track(track) -> "ClipInfo":
        """As the crate's converter fills it from a movie track
        (examples/prr2dng/main.rs:144-151)."""
        return ClipInfo(
            make=track.text(["com.apple.proapps.manufacturer", "com.apple.quicktime.make"]),
            model=track.text(["com.apple.proapps.modelname", "com.apple.quicktime.model"]),
            fps=track.fps,
            date_time=None if track.creation_time is None else quicktime_date_time(track.creation_time),
            orientation=int(track.orientation),
        )

    def _c(self):
        keep = []

        def enc(s):
            if s is None:
                return None
            b = s.encode("utf-8")
            keep.append(b)
            return b

        c = _lib.CDngClip()
        c.make, c.model, c.date_time, c.software = enc(self.make), enc(self.model), enc(self.date_time), \
            enc(self.software)
        if self.fps is not None:
            c.fps_num, c.fps_den = int(self.fps[0]), int(self.fps[1])
        c.orientation = int(self.orientation)
        return c, keep


@dataclasses.dataclass
class DngColour:
    """DngColour (colour.rs:58-72): the colour tags of a frame header."""

    temperature: float
    illuminant: int
    color_matrix: np.ndarray  # 3x3, XYZ -> camera RGB under the shot illuminant
    forward_matrix: np.ndarray  # 3x3, white-balanced camera RGB -> XYZ (D50)
    as_shot_neutral: np.ndarray
    baseline_exposure: float

    @staticmethod
    def new(header) -> "DngColour":
        c = _lib.CDngColour()
        _check(_lib.lib().prr_dng_colour_of(C.byref(_header_c(header)), C.byref(c)))
        return DngColour(c.temperature, int(c.illuminant), np.array(c.color_matrix).reshape(3, 3),
                         np.array(c.forward_matrix).reshape(3, 3), np.array(c.as_shot_neutral),
                         c.baseline_exposure)


def _header_c(header) -> _lib.CHeader:
    if isinstance(header, _lib.CHeader):
        return header
    if isinstance(header, FrameHeader) and header._c is not None:
        return header._c
    raise TypeError("a FrameHeader from the library (or its CHeader) is needed")


def srational(v: float) -> Tuple[int, int]:
    """Value::srational (tiff.rs:62-79) of one value."""
    n, d = C.c_int32(), C.c_int32()
    _lib.lib().prr_dng_srational(float(v), C.byref(n), C.byref(d))
    return n.value, d.value


def rational(v: float) -> Tuple[int, int]:
    """Value::rational (tiff.rs:81-98) of one value."""
    n, d = C.c_uint32(), C.c_uint32()
    _lib.lib().prr_dng_rational(float(v), C.byref(n), C.byref(d))
    return n.value, d.value


def quicktime_date_time(seconds: int) -> str:
    """dng.rs:211-232: UTC `YYYY:MM:DD HH:MM:SS` of a QuickTime time."""
    buf = C.create_string_buffer(20)
    rc = _lib.lib().prr_dng_date_time(int(seconds), buf)
    if rc:
        raise _error(rc)
    return buf.value.decode("ascii")


def _file_bytes(f) -> bytes:
    L = _lib.lib()
    n = C.c_size_t()
    p = L.prr_dng_data(f, C.byref(n))
    try:
        return C.string_at(p, n.value)
    finally:
        L.prr_dng_free(f)


def write(frame, clip: Optional[ClipInfo] = None, samples: Samples = Samples.CODE_VALUES,
          compression: Compression = Compression.LOSSLESS_JPEG) -> bytes:
    """dng::write (dng.rs:77-111) of a decoded Frame: the DNG file's bytes."""
    clip = clip or ClipInfo()
    c, keep = clip._c()
    ctx = context(frame.samples.device.index)
    f = C.c_void_p()
    _check(_lib.lib().prr_dng_write(ctx, C.byref(_header_c(frame.header)), _dptr(frame.samples), int(samples),
                                    int(compression), C.byref(c), C.byref(f)), ctx=ctx)
    del keep
    return _file_bytes(f)


def write_into(frame, out, clip: Optional[ClipInfo] = None, samples: Samples = Samples.CODE_VALUES,
               compression: Compression = Compression.LOSSLESS_JPEG) -> int:
    """write() into a caller's writable buffer (a pinned host tensor's
    memory takes the device copy fastest); returns the file's length. Raises
    Error (status ERR_BUFFER) when the buffer is too small."""
    clip = clip or ClipInfo()
    c, keep = clip._c()
    ctx = context(frame.samples.device.index)
    if hasattr(out, "data_ptr"):
        ptr, cap = out.data_ptr(), out.numel() * out.element_size()
    else:
        mv = memoryview(out).cast("B")
        cap = mv.nbytes
        ptr = C.addressof((C.c_uint8 * max(1, cap)).from_buffer(mv))
    n = C.c_size_t()
    rc = _lib.lib().prr_dng_write_into(ctx, C.byref(_header_c(frame.header)), _dptr(frame.samples), int(samples),
                                       int(compression), C.byref(c), ptr, cap, C.byref(n))
    del keep
    _check(rc, ctx=ctx)
    return int(n.value)


def assemble(header, chunks: Sequence[bytes], clip: Optional[ClipInfo] = None,
             samples: Samples = Samples.CODE_VALUES, compression: Compression = Compression.LOSSLESS_JPEG) -> bytes:
    """The DNG container alone (host): `chunks` are one strip of the visible
    samples (little-endian u16) or the frame's tiles' streams in order."""
    clip = clip or ClipInfo()
    c, keep = clip._c()
    data = b"".join(chunks)
    offsets = np.zeros(len(chunks) + 1, np.uint64)
    if chunks:
        offsets[1:] = np.cumsum([len(x) for x in chunks])
    buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(data or b"\0")
    f = C.c_void_p()
    _check(_lib.lib().prr_dng_assemble(C.byref(_header_c(header)), C.byref(c), int(samples), int(compression), buf,
                                       offsets.ctypes.data, len(chunks), C.byref(f)))
    del keep
    return _file_bytes(f)


def lj92_tiles(image, width: int, height: int, stride: Optional[int] = None, tile: int = TILE) -> List[bytes]:
    """The lossless JPEG streams of every tile of a device image (a torch
    uint16 tensor, rows `stride` samples apart), encoded on the device:
    lj92::encode(dng::tile(...), tile, tile, 2) for each, in order."""
    ctx = context(image.device.index)
    L = _lib.lib()
    across, down = -(-width // tile), -(-height // tile)
    n = across * down
    offsets = np.zeros(n + 1, np.uint64)
    total = C.c_size_t()
    cap = int(n * L.prr_lj92_tile_bound(tile))
    out = np.empty(max(1, cap), np.uint8)
    _check(L.prr_lj92_encode_host(ctx, _dptr(image), width, height, stride or width, tile, out.ctypes.data, cap,
                                  offsets.ctypes.data, C.byref(total)), ctx=ctx)
    return [out[int(offsets[i]):int(offsets[i + 1])].tobytes() for i in range(n)]
