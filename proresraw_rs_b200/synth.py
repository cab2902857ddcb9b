"""Synthetic ProRes RAW input (ctypes over libprr_synth.so).

Restates the crate's test support (src/synth.rs: Rng, Spec, frame,
random_frame, tile, specs; src/idct.rs:359-459: testgen::Gen and fnv1a) and
adds what the crate lacks: a seeded Bayer mosaic generator, an encoder that
turns a mosaic into a valid frame packet, and a seeded tile corrupter. The
frames of the benchmark configurations are built here.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libprr_synth.so")


class _Spec(C.Structure):
    _fields_ = [
        ("width", C.c_uint16),
        ("height", C.c_uint16),
        ("alignment", C.c_uint8),
        ("pattern", C.c_uint8),
        ("has_quant_matrix", C.c_uint8),
        ("has_curve", C.c_uint8),
        ("quant_matrix", C.c_uint8 * 64),
        ("curve", C.c_uint16 * 8),
        ("vendor", C.c_uint8 * 4),
        ("crop", C.c_uint8 * 4),
        ("white_level", C.c_uint16),
        ("wb", C.c_float * 2),
        ("color_matrix", C.c_float * 9),
        ("gain", C.c_float),
        ("wb_cct", C.c_uint16),
        ("valid_tiles", C.c_uint8),
        ("version", C.c_uint8),
    ]


class _BitOp(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("a", C.c_uint32), ("b", C.c_uint32)]


class _MosaicParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("pattern", C.c_uint8),
        ("seed", C.c_uint64),
        ("sigma", C.c_float),
        ("specular", C.c_float),
        ("amp_lo", C.c_float),
        ("amp_hi", C.c_float),
        ("chan_gain", C.c_float * 3),
        ("white", C.c_uint16),
    ]


class _EncodeParams(C.Structure):
    _fields_ = [
        ("spec", _Spec),
        ("qscale_lo", C.c_uint8),
        ("qscale_hi", C.c_uint8),
        ("qscale_seed", C.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(
                f"{_LIB_PATH} is missing: build it with "
                "`python -m proresraw_rs_b200.build` (or __graft_entry__.build())"
            )
        L = C.CDLL(_LIB_PATH)
        u64p = C.POINTER(C.c_uint64)
        L.prs_rng_new.restype = C.c_uint64
        L.prs_rng_new.argtypes = [C.c_uint64]
        L.prs_rng_next_u32.restype = C.c_uint32
        L.prs_rng_next_u32.argtypes = [u64p]
        L.prs_rng_below.restype = C.c_uint32
        L.prs_rng_below.argtypes = [u64p, C.c_uint32]
        L.prs_spec_new.argtypes = [C.c_uint16, C.c_uint16, C.c_uint8, C.POINTER(_Spec)]
        L.prs_specs.restype = C.c_size_t
        L.prs_specs.argtypes = [u64p, C.POINTER(_Spec), C.c_size_t]
        L.prs_random_frame.restype = C.c_size_t
        L.prs_random_frame.argtypes = [C.POINTER(_Spec), u64p, C.c_void_p, C.c_size_t]
        L.prs_frame_from_tiles.restype = C.c_size_t
        L.prs_frame_from_tiles.argtypes = [C.POINTER(_Spec), C.c_void_p, C.c_void_p, C.c_size_t,
                                           C.c_void_p, C.c_size_t]
        L.prs_bitwrite.restype = C.c_size_t
        L.prs_bitwrite.argtypes = [C.POINTER(_BitOp), C.c_size_t, C.c_void_p, C.c_size_t]
        L.prs_gen_new.restype = C.c_uint64
        L.prs_gen_new.argtypes = [C.c_uint64]
        L.prs_gen_blocks.argtypes = [u64p, C.c_uint64, C.c_size_t, C.c_void_p, C.c_void_p]
        L.prs_fnv1a_u16.restype = C.c_uint64
        L.prs_fnv1a_u16.argtypes = [C.c_uint64, C.c_void_p, C.c_size_t]
        L.prs_mosaic.argtypes = [C.POINTER(_MosaicParams), C.c_void_p, C.c_int]
        L.prs_encode.restype = C.c_size_t
        L.prs_encode.argtypes = [C.POINTER(_EncodeParams), C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        L.prs_corrupt_tiles.restype = C.c_size_t
        L.prs_corrupt_tiles.argtypes = [C.c_void_p, C.c_size_t, C.c_float, C.c_uint64, C.c_void_p,
                                        C.c_size_t]
        _lib = L
    return _lib


RGGB, GRBG, GBRG, BGGR = 0, 1, 2, 3


class Rng:
    """xorshift64* (src/synth.rs:9-29)."""

    def __init__(self, seed: int):
        self.state = C.c_uint64(lib().prs_rng_new(seed & 0xFFFFFFFFFFFFFFFF))

    def next_u32(self) -> int:
        return lib().prs_rng_next_u32(C.byref(self.state))

    def below(self, bound: int) -> int:
        return lib().prs_rng_below(C.byref(self.state), bound)


@dataclasses.dataclass
class Spec:
    """Parameters of a synthetic frame (src/synth.rs:34-89)."""

    width: int
    height: int
    pattern: int = RGGB
    alignment: int = 3
    quant_matrix: Optional[Sequence[int]] = None
    curve: Optional[Sequence[int]] = None
    vendor: bytes = b"test"
    crop: Sequence[int] = (0, 0, 0, 0)
    white_level: int = 0xFDFF + 256
    wb: Sequence[float] = (1.0, 1.0)
    color_matrix: Sequence[float] = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)
    gain: float = 1.0
    wb_cct: int = 5600
    valid_tiles: bool = False
    version: int = 1

    def _c(self) -> _Spec:
        s = _Spec()
        s.width, s.height = self.width, self.height
        s.alignment, s.pattern = self.alignment, self.pattern
        s.has_quant_matrix = self.quant_matrix is not None
        if self.quant_matrix is not None:
            s.quant_matrix[:] = list(self.quant_matrix)
        s.has_curve = self.curve is not None
        if self.curve is not None:
            s.curve[:] = list(self.curve)
        s.vendor[:] = list(self.vendor)
        s.crop[:] = list(self.crop)
        s.white_level = self.white_level
        s.wb[:] = list(self.wb)
        s.color_matrix[:] = list(self.color_matrix)
        s.gain = self.gain
        s.wb_cct = self.wb_cct
        s.valid_tiles = bool(self.valid_tiles)
        s.version = self.version
        return s

    @staticmethod
    def _from_c(s: _Spec) -> "Spec":
        return Spec(
            width=s.width, height=s.height, pattern=s.pattern, alignment=s.alignment,
            quant_matrix=list(s.quant_matrix) if s.has_quant_matrix else None,
            curve=list(s.curve) if s.has_curve else None,
            vendor=bytes(s.vendor), crop=tuple(s.crop), white_level=s.white_level,
            wb=tuple(s.wb), color_matrix=tuple(s.color_matrix), gain=s.gain, wb_cct=s.wb_cct,
            valid_tiles=bool(s.valid_tiles), version=s.version,
        )


def grid_row(width: int, alignment: int):
    """(x, log2_blocks) of each tile of a tile row (src/tile.rs:79-101)."""
    out = []
    column, remaining, log2 = 0, (width + 15) // 16, alignment
    while remaining > 0:
        unit = 1 << log2
        if unit <= remaining:
            out.append((column * 16, log2))
            column += unit
            remaining -= unit
        else:
            log2 -= 1
    return out


def ntiles(width: int, height: int, alignment: int) -> int:
    return len(grid_row(width, alignment)) * ((height + 15) // 16)


def specs(rng: Rng) -> List[Spec]:
    """The 20 varied specs of src/synth.rs:188-221."""
    buf = (_Spec * 32)()
    n = lib().prs_specs(C.byref(rng.state), buf, 32)
    return [Spec._from_c(buf[i]) for i in range(n)]


def random_frame(spec: Spec, rng: Rng) -> bytes:
    """A packet with random tile headers and streams (src/synth.rs:92-94)."""
    s = spec._c()
    cap = 10 + 70 + 64 + 16 + ntiles(spec.width, spec.height, spec.alignment) * (2 + 8 + 4 * 48 * 16)
    out = (C.c_uint8 * cap)()
    n = lib().prs_random_frame(C.byref(s), C.byref(rng.state), out, cap)
    assert n > 0
    return bytes(out[:n])


def frame(spec: Spec, tiles: Sequence[bytes]) -> bytes:
    """frame(spec, payload) with explicit tile payloads (src/synth.rs:99-152)."""
    s = spec._c()
    data = b"".join(tiles)
    lens = (C.c_uint32 * max(1, len(tiles)))(*[len(t) for t in tiles])
    cap = 10 + 70 + 64 + 16 + 2 * len(tiles) + len(data)
    out = (C.c_uint8 * cap)()
    src = C.create_string_buffer(data, max(1, len(data)))
    n = lib().prs_frame_from_tiles(C.byref(s), src, lens, len(tiles), out, cap)
    return bytes(out[:n])


def tile(qscale: int, streams: Sequence[bytes]) -> bytes:
    """An 8-byte tile header and four streams (src/synth.rs:175-184)."""
    t = bytes([8 << 3, qscale])
    for st in streams[:3]:
        t += len(st).to_bytes(2, "big")
    return t + b"".join(streams)


class BitWriter:
    """Codeword writer (the test encoder of src/bits.rs:136-186)."""

    def __init__(self):
        self.ops = []

    def put(self, value: int, n: int):
        while n > 32:
            self.ops.append((1, 32, 0))
            n -= 32
            assert value == 0
        self.ops.append((1, n, value & 0xFFFFFFFF))

    def symbol(self, cb: int, v: int):
        self.ops.append((0, cb, v))

    def finish(self) -> bytes:
        arr = (_BitOp * max(1, len(self.ops)))(*[_BitOp(*o) for o in self.ops])
        cap = 8 * len(self.ops) + 16
        out = (C.c_uint8 * cap)()
        n = lib().prs_bitwrite(arr, len(self.ops), out, cap)
        return bytes(out[:n])


class Gen:
    """testgen::Gen (src/idct.rs:363-442), the IDCT test-block stream."""

    def __init__(self, seed: int):
        self.state = C.c_uint64(lib().prs_gen_new(seed))
        self.index = 0

    def blocks(self, n: int):
        coefs = np.empty((n, 64), dtype=np.int16)
        q = np.empty((n, 64), dtype=np.int16)
        lib().prs_gen_blocks(C.byref(self.state), self.index, n, coefs.ctypes.data, q.ctypes.data)
        self.index += n
        return coefs, q


FNV_OFFSET = 0xCBF29CE484222325


def fnv1a_u16(h: int, values: np.ndarray) -> int:
    v = np.ascontiguousarray(values, dtype=np.uint16)
    return lib().prs_fnv1a_u16(h, v.ctypes.data, v.size)


def mosaic(width: int, height: int, pattern: int = RGGB, seed: int = 0, sigma: float = 8.0,
           specular: float = 0.0, amp=(300.0, 1500.0), chan_gain=(0.55, 1.0, 0.8),
           white: int = 4095, threads: int = 0) -> np.ndarray:
    """Seeded 12-bit Bayer mosaic: three low-frequency cosines, noise, specular clip."""
    p = _MosaicParams()
    p.width, p.height, p.pattern, p.seed = width, height, pattern, seed
    p.sigma, p.specular = sigma, specular
    p.amp_lo, p.amp_hi = amp
    p.chan_gain[:] = list(chan_gain)
    p.white = white
    out = np.empty((height, width), dtype=np.uint16)
    lib().prs_mosaic(C.byref(p), out.ctypes.data, threads)
    return out


def encode(spec: Spec, mosaic_u16: np.ndarray, qscale=15, qscale_seed: int = 0,
           threads: int = 0) -> bytes:
    """Encode a linear mosaic into a frame packet (no counterpart in the crate)."""
    m = np.ascontiguousarray(mosaic_u16, dtype=np.uint16)
    assert m.shape == (spec.height, spec.width)
    ep = _EncodeParams()
    ep.spec = spec._c()
    lo, hi = (qscale, qscale) if isinstance(qscale, int) else qscale
    ep.qscale_lo, ep.qscale_hi, ep.qscale_seed = lo, hi, qscale_seed
    cap = m.size * 2 + (1 << 20)
    out = np.empty(cap, dtype=np.uint8)
    n = lib().prs_encode(C.byref(ep), m.ctypes.data, out.ctypes.data, cap, threads)
    if n > cap:  # larger than the estimate: encode again into a buffer that fits
        out = np.empty(n, dtype=np.uint8)
        n = lib().prs_encode(C.byref(ep), m.ctypes.data, out.ctypes.data, n, threads)
    if n == 0:
        raise RuntimeError("encoder failed: a tile exceeds 65535 bytes")
    return out[:n].tobytes()


def corrupt_tiles(packet: bytes, fraction: float, seed: int):
    """Corrupt about `fraction` of the tiles (seeded); returns (packet, tile indices)."""
    buf = np.frombuffer(packet, dtype=np.uint8).copy()
    n_t = max(16, int(len(packet)))
    idx = np.empty(min(n_t, 1 << 20), dtype=np.uint64)
    n = lib().prs_corrupt_tiles(buf.ctypes.data, buf.size, fraction, seed, idx.ctypes.data, idx.size)
    return buf.tobytes(), [int(i) for i in idx[:n]]


# Sizes of the mixed-batch workload: HD, DCI 4K, 5.8K, 8K.
BATCH_SIZES = ((1920, 1080), (4096, 2160), (5760, 3040), (8192, 4320))


@dataclasses.dataclass
class BatchItem:
    """One frame of a mixed batch: its packet and how it is decoded."""

    packet: bytes
    width: int
    height: int
    version: int
    pattern: int
    qscale: int
    alignment: int
    scale: int   # 0: full resolution, else log2 of the reduction
    greens: int  # reduced: 0 first green, 1 average
    corrupt_tiles: Sequence[int] = ()


def mixed_batch(n: int, seed: int, sizes=BATCH_SIZES, corrupt: float = 0.0, sigma=(4.0, 32.0),
                threads: int = 0) -> List[BatchItem]:
    """A seeded batch of frames of uneven shape: size from `sizes`, bitstream
    version 0 or 1, RGGB or BGGR, qscale uniform in [15, 45], tile alignment
    uniform in [0, 4]; half of them decoded at full resolution, half reduced
    (Half / Quarter / Eighth, first or averaged greens). Mosaics come from
    mosaic() with sigma uniform in `sigma`; `corrupt` is the fraction of tiles
    byte-corrupted per frame."""
    rng = np.random.default_rng(seed)
    items = []
    for i in range(n):
        w, h = sizes[int(rng.integers(len(sizes)))]
        version = int(rng.integers(2))
        pattern = (RGGB, BGGR)[int(rng.integers(2))]
        qscale = int(rng.integers(15, 46))
        alignment = int(rng.integers(5))
        scale = 0 if i % 2 == 0 else int(rng.integers(1, 4))
        greens = int(rng.integers(2)) if scale else 0
        s = float(rng.uniform(*sigma))
        mseed = int(rng.integers(1 << 31))
        m = mosaic(w, h, pattern, seed=mseed, sigma=s, threads=threads)
        spec = Spec(w, h, pattern=pattern, alignment=alignment, white_level=4095, version=version,
                    valid_tiles=True)
        pkt = encode(spec, m, qscale=qscale, qscale_seed=mseed, threads=threads)
        bad: List[int] = []
        if corrupt > 0:
            pkt, bad = corrupt_tiles(pkt, corrupt, seed=mseed)
        items.append(BatchItem(pkt, w, h, version, pattern, qscale, alignment, scale, greens, bad))
    return items
