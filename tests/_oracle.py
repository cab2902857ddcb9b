"""ctypes bindings of the CPU oracle (oracle/build/libprr_oracle.so).

Test infrastructure: the oracle restates the crate's CPU path and is the
checker the CUDA library is compared against. Nothing in the product imports
this module.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "build", "libprr_oracle.so")


class Error(C.Structure):
    _fields_ = [
        ("code", C.c_int32),
        ("what", C.c_char * 32),
        ("needed", C.c_uint64),
        ("available", C.c_uint64),
        ("declared", C.c_uint32),
        ("actual", C.c_uint64),
        ("index", C.c_uint64),
        ("value", C.c_uint32),
        ("width", C.c_uint16),
        ("height", C.c_uint16),
        ("curve", C.c_uint16 * 8),
        ("tag", C.c_uint8 * 4),
    ]


class Header(C.Structure):
    _fields_ = [
        ("version", C.c_uint8),
        ("vendor", C.c_uint8 * 4),
        ("bayer_pattern", C.c_uint8),
        ("width", C.c_uint16),
        ("height", C.c_uint16),
        ("crop", C.c_uint8 * 4),
        ("white_level", C.c_uint16),
        ("wb_cct", C.c_uint16),
        ("flags", C.c_uint16),
        ("alignment", C.c_uint8),
        ("pad0", C.c_uint8),
        ("wb_red", C.c_float),
        ("wb_blue", C.c_float),
        ("color_matrix", C.c_float * 9),
        ("gain", C.c_float),
        ("quant_matrix", C.c_uint8 * 64),
        ("curve", C.c_uint16 * 8),
    ]

    @property
    def coded_width(self):
        return (self.width + 15) & ~15

    @property
    def coded_height(self):
        return (self.height + 15) & ~15


class Params(C.Structure):
    _fields_ = [
        ("cfa_phase", C.c_int32),
        ("black", C.c_int32),
        ("one_over_range", C.c_float),
        ("noise", C.c_float * 3),
        ("clip", C.c_float * 2),
        ("black_over_range", C.c_float),
        ("wb", C.c_float * 2),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, sz = C.c_void_p, C.c_size_t
        L.orc_codeword.argtypes = [C.c_uint32, C.c_uint16, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_read_symbols.restype = C.c_int
        L.orc_read_symbols.argtypes = [vp, sz, sz, vp, sz, vp]
        L.orc_decode_component_reduced.argtypes = [vp, sz, sz, C.c_uint8, C.c_uint8, vp]
        L.orc_dequantize.restype = C.c_int16
        L.orc_dequantize.argtypes = [C.c_int16, C.c_int16]
        for f in ["orc_apple_block", "orc_ffmpeg_block", "orc_apple_block_4x4", "orc_apple_block_2x2"]:
            getattr(L, f).argtypes = [vp, vp, vp]
        L.orc_output_code.restype = C.c_uint16
        L.orc_output_code.argtypes = [C.c_float]
        L.orc_code_value.restype = C.c_uint16
        L.orc_code_value.argtypes = [C.c_int32]
        L.orc_transform_blocks.argtypes = [C.c_int, vp, vp, vp, sz]
        L.orc_curve_linearize.restype = C.c_uint16
        L.orc_curve_linearize.argtypes = [vp, C.c_uint16]
        L.orc_header_len.restype = C.c_int
        L.orc_header_len.argtypes = [vp, sz, C.POINTER(C.c_size_t), C.POINTER(Error)]
        L.orc_parse_header.restype = C.c_int
        L.orc_parse_header.argtypes = [vp, sz, C.POINTER(Header), C.POINTER(Error)]
        L.orc_parse_frame.restype = C.c_int
        L.orc_parse_frame.argtypes = [vp, sz, C.POINTER(Header), C.POINTER(C.c_size_t),
                                      C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), vp, vp,
                                      C.POINTER(C.c_uint8), C.POINTER(Error)]
        L.orc_tile_parse.restype = C.c_int
        L.orc_tile_parse.argtypes = [vp, sz, sz, C.POINTER(C.c_uint8), vp, vp]
        L.orc_grid_row.restype = C.c_size_t
        L.orc_grid_row.argtypes = [sz, sz, C.c_uint8, vp, vp]
        L.orc_decode_frame.restype = C.c_int
        L.orc_decode_frame.argtypes = [vp, sz, C.c_int, vp, sz, vp, sz, C.POINTER(C.c_size_t),
                                       C.POINTER(C.c_uint8), C.POINTER(Header), C.c_int,
                                       C.POINTER(Error)]
        L.orc_decode_frame_reduced.restype = C.c_int
        L.orc_decode_frame_reduced.argtypes = [vp, sz, C.c_int, C.c_int, vp, sz, vp, sz,
                                               C.POINTER(C.c_size_t), C.POINTER(C.c_uint8),
                                               C.POINTER(Header), C.c_int, C.POINTER(Error)]
        L.orc_linearize.restype = C.c_int
        L.orc_linearize.argtypes = [C.POINTER(Header), vp, vp, sz, C.c_int]
        L.orc_params_with_white_balance.argtypes = [C.POINTER(Header), C.c_uint32, C.c_float,
                                                    C.c_float, C.POINTER(Params)]
        L.orc_output_matrix.argtypes = [C.POINTER(Header), C.c_int, vp]
        L.orc_develop.restype = C.c_int
        L.orc_develop.argtypes = [C.POINTER(Header), vp, C.POINTER(Params), C.c_int, C.c_int, vp,
                                  vp, vp, sz, C.c_int]
        L.orc_green_pass.argtypes = [vp, sz, sz, C.POINTER(Params), vp]
        L.orc_chroma_pass.argtypes = [vp, sz, sz, C.POINTER(Params), vp]
        L.orc_apply_matrix.argtypes = [vp, sz, vp, vp]
        L.orc_sg_param_count.restype = sz
        L.orc_sg_pack.restype = C.c_int
        L.orc_sg_pack.argtypes = [C.POINTER(Header), vp, C.POINTER(Params), vp, vp]
        L.orc_sg_forward.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int, vp, vp]
        L.orc_sg_output.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]
        L.orc_sg_loss.restype = C.c_double
        L.orc_sg_loss.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]
        L.orc_sg_backward.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp]
        L.orc_lj92_encode.restype = C.c_int
        L.orc_lj92_encode.argtypes = [vp, sz, sz, sz, vp, sz, C.POINTER(C.c_size_t)]
        L.orc_lj92_huffman.argtypes = [vp, vp, vp, C.POINTER(C.c_int), vp, vp]
        L.orc_dng_tile.restype = C.c_int
        L.orc_dng_tile.argtypes = [vp, sz, sz, sz, sz, sz, sz, vp]
        L.orc_lj92_tiles.restype = C.c_int
        L.orc_lj92_tiles.argtypes = [vp, sz, sz, sz, sz, C.c_int, vp, sz, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data


class OracleError(Exception):
    def __init__(self, err: Error):
        super().__init__(f"oracle error {err.code}")
        self.err = err
        self.code = err.code


def codeword(p: int, cb: int):
    v, n = C.c_uint32(), C.c_uint32()
    lib().orc_codeword(p, cb, C.byref(v), C.byref(n))
    return v.value, n.value


def read_symbols(data: bytes, align: int, cbs):
    buf = np.frombuffer(data + b"\0", dtype=np.uint8)
    cb = np.array(cbs, dtype=np.uint16)
    out = np.zeros(len(cbs), dtype=np.uint32)
    n = lib().orc_read_symbols(_p(buf), len(data), align, _p(cb), len(cbs), _p(out))
    return [int(v) for v in out[:n]]


def decode_component(data: bytes, align: int, log2_blocks: int, log2_coefs: int = 6):
    buf = np.frombuffer(data + b"\0", dtype=np.uint8)
    out = np.zeros(1 << (log2_coefs + log2_blocks), dtype=np.int16)
    lib().orc_decode_component_reduced(_p(buf), len(data), align, log2_blocks, log2_coefs, _p(out))
    return out


def block(kind: str, coefs, q):
    c = np.ascontiguousarray(coefs, dtype=np.int16)
    qq = np.ascontiguousarray(q, dtype=np.int16)
    n = {"apple": 64, "ffmpeg": 64, "4x4": 16, "2x2": 4}[kind]
    out = np.zeros(n, dtype=np.uint16)
    f = {"apple": "orc_apple_block", "ffmpeg": "orc_ffmpeg_block", "4x4": "orc_apple_block_4x4",
         "2x2": "orc_apple_block_2x2"}[kind]
    getattr(lib(), f)(_p(c), _p(qq), _p(out))
    return out


def transform_blocks(idct: int, coefs: np.ndarray, q: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(coefs, dtype=np.int16)
    qq = np.ascontiguousarray(q, dtype=np.int16)
    out = np.empty(c.shape, dtype=np.uint16)
    lib().orc_transform_blocks(idct, _p(c), _p(qq), _p(out), c.shape[0])
    return out


def curve_linearize(curve, code: int) -> int:
    c = np.array(curve, dtype=np.uint16)
    return lib().orc_curve_linearize(_p(c), code)


def _buf(packet: bytes):
    return np.frombuffer(packet + b"\0" * 8, dtype=np.uint8)


def header_len(packet: bytes) -> int:
    n, e = C.c_size_t(), Error()
    b = _buf(packet)
    rc = lib().orc_header_len(_p(b), len(packet), C.byref(n), C.byref(e))
    if rc:
        raise OracleError(e)
    return n.value


def parse_header(packet: bytes) -> Header:
    h, e = Header(), Error()
    b = _buf(packet)
    rc = lib().orc_parse_header(_p(b), len(packet), C.byref(h), C.byref(e))
    if rc:
        raise OracleError(e)
    return h


def parse_frame(packet: bytes):
    """(header, tile offsets, tile lengths, tiles_per_row, rows, max_qscale)."""
    h, e = Header(), Error()
    nt, tpr, rows, mq = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_uint8()
    b = _buf(packet)
    rc = lib().orc_parse_frame(_p(b), len(packet), C.byref(h), C.byref(nt), C.byref(tpr),
                               C.byref(rows), None, None, C.byref(mq), C.byref(e))
    if rc:
        raise OracleError(e)
    off = np.zeros(max(1, nt.value), dtype=np.uint64)
    ln = np.zeros(max(1, nt.value), dtype=np.uint64)
    lib().orc_parse_frame(_p(b), len(packet), C.byref(h), C.byref(nt), C.byref(tpr), C.byref(rows),
                          _p(off), _p(ln), C.byref(mq), C.byref(e))
    return h, off[: nt.value], ln[: nt.value], tpr.value, rows.value, mq.value


class Frame:
    def __init__(self, header, samples, skipped, max_qscale):
        self.header = header
        self.samples = samples
        self.skipped_tiles = skipped
        self.max_qscale = max_qscale

    @property
    def quantizer(self):
        return int(self.header.quant_matrix[0]) * int(self.max_qscale)

    def linearize(self, threads: int = 0) -> np.ndarray:
        h = self.header
        out = np.zeros(h.width * h.height, dtype=np.uint16)
        rc = lib().orc_linearize(C.byref(h), _p(self.samples), _p(out), out.size, threads)
        assert rc == 0
        return out


def decode_frame(packet: bytes, idct: int = 0, threads: int = 0) -> Frame:
    h = parse_header_or_raise(packet)
    cw, ch = h.coded_width, h.coded_height
    samples = np.zeros(cw * ch, dtype=np.uint16)
    nt = _ntiles(h)
    skipped = np.zeros(max(1, nt), dtype=np.uint64)
    ns, mq, hdr, e = C.c_size_t(), C.c_uint8(), Header(), Error()
    b = _buf(packet)
    rc = lib().orc_decode_frame(_p(b), len(packet), idct, _p(samples), samples.size, _p(skipped),
                                skipped.size, C.byref(ns), C.byref(mq), C.byref(hdr), threads,
                                C.byref(e))
    if rc:
        raise OracleError(e)
    return Frame(hdr, samples, [int(i) for i in skipped[: ns.value]], mq.value)


def decode_frame_reduced(packet: bytes, log2_factor: int, greens: int = 0, threads: int = 0):
    h = parse_header_or_raise(packet)
    cw, ch = h.coded_width, h.coded_height
    samples = np.zeros(3 * (cw >> log2_factor) * (ch >> log2_factor), dtype=np.uint16)
    nt = _ntiles(h)
    skipped = np.zeros(max(1, nt), dtype=np.uint64)
    ns, mq, hdr, e = C.c_size_t(), C.c_uint8(), Header(), Error()
    b = _buf(packet)
    rc = lib().orc_decode_frame_reduced(_p(b), len(packet), log2_factor, greens, _p(samples),
                                        samples.size, _p(skipped), skipped.size, C.byref(ns),
                                        C.byref(mq), C.byref(hdr), threads, C.byref(e))
    if rc:
        raise OracleError(e)
    return Frame(hdr, samples, [int(i) for i in skipped[: ns.value]], mq.value)


def parse_header_or_raise(packet: bytes) -> Header:
    try:
        return parse_header(packet)
    except OracleError:
        # Let decode report the error in the crate's order (prefix checks first).
        h = Header()
        h.width = h.height = 16
        return h


def _ntiles(h: Header) -> int:
    rowlen = lib().orc_grid_row(h.width, h.height, h.alignment, None, None)
    return rowlen * ((h.height + 15) // 16)


def params_with_white_balance(h: Header, quantizer: int, red: float, blue: float) -> Params:
    p = Params()
    lib().orc_params_with_white_balance(C.byref(h), quantizer, red, blue, C.byref(p))
    return p


def params_new(h: Header, quantizer: int) -> Params:
    return params_with_white_balance(h, quantizer, h.wb_red, h.wb_blue)


def output_matrix(h: Header, exposure: int = 0) -> np.ndarray:
    m = np.zeros(9, dtype=np.float32)
    lib().orc_output_matrix(C.byref(h), exposure, _p(m))
    return m


def develop(frame: Frame, params: Params, stage: int, planar: bool, threads: int = 0):
    h = frame.header
    n = h.width * h.height
    if planar:
        r, g, b = (np.zeros(n, dtype=np.float32) for _ in range(3))
        rc = lib().orc_develop(C.byref(h), _p(frame.samples), C.byref(params), stage, 1, _p(r),
                               _p(g), _p(b), n, threads)
        assert rc == 0
        return r, g, b
    out = np.zeros(3 * n, dtype=np.float32)
    rc = lib().orc_develop(C.byref(h), _p(frame.samples), C.byref(params), stage, 0, _p(out), None,
                           None, 3 * n, threads)
    assert rc == 0
    return out


def green_pass(linear: np.ndarray, w: int, h: int, p: Params) -> np.ndarray:
    lin = np.ascontiguousarray(linear, dtype=np.uint16)
    out = np.zeros(2 * w * h, dtype=np.float32)
    lib().orc_green_pass(_p(lin), w, h, C.byref(p), _p(out))
    return out


def chroma_pass(green: np.ndarray, w: int, h: int, p: Params) -> np.ndarray:
    g = np.ascontiguousarray(green, dtype=np.float32)
    out = np.zeros(3 * w * h, dtype=np.float32)
    lib().orc_chroma_pass(_p(g), w, h, C.byref(p), _p(out))
    return out


def apply_matrix(rgb: np.ndarray, m: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(rgb, dtype=np.float32)
    mm = np.ascontiguousarray(m, dtype=np.float32)
    out = np.zeros_like(x)
    lib().orc_apply_matrix(_p(x), x.size // 3, _p(mm), _p(out))
    return out


# --- learned demosaic surrogate (sg_oracle.h) ------------------------------------


def sg_param_count() -> int:
    return int(lib().orc_sg_param_count())


def sg_pack(h: Header, samples: np.ndarray, p: Params):
    wq, hq = (h.width + 1) // 2, (h.height + 1) // 2
    in16 = np.zeros((16, hq, wq), dtype=np.float32)
    base = np.zeros((3, hq, wq), dtype=np.float32)
    s = np.ascontiguousarray(samples, dtype=np.uint16)
    assert lib().orc_sg_pack(C.byref(h), _p(s), C.byref(p), _p(in16), _p(base)) == 0
    return in16, base


def sg_forward(in16: np.ndarray, params: np.ndarray, round_bf16: bool = True):
    _, hq, wq = in16.shape
    acts = np.zeros((6, 32, hq, wq), dtype=np.float32)
    head = np.zeros((16, hq, wq), dtype=np.float32)
    a = np.ascontiguousarray(in16, dtype=np.float32)
    pr = np.ascontiguousarray(params, dtype=np.float32)
    lib().orc_sg_forward(_p(a), hq, wq, _p(pr), 1 if round_bf16 else 0, _p(acts), _p(head))
    return acts, head


def sg_output(head, base, width, height, m9=None, cfa=0):
    _, hq, wq = head.shape
    out = np.zeros((3, height, width), dtype=np.float32)
    m = None if m9 is None else np.ascontiguousarray(m9, dtype=np.float32)
    lib().orc_sg_output(_p(np.ascontiguousarray(head)), _p(np.ascontiguousarray(base)), hq, wq, width, height, cfa,
                        None if m is None else _p(m), _p(out[0]), _p(out[1]), _p(out[2]))
    return out


def sg_loss(head, base, target):
    _, hq, wq = head.shape
    _, height, width = target.shape
    dhead = np.zeros_like(head)
    t = np.ascontiguousarray(target, dtype=np.float32)
    loss = lib().orc_sg_loss(_p(np.ascontiguousarray(head)), _p(np.ascontiguousarray(base)), hq, wq, width,
                             height, _p(t[0]), _p(t[1]), _p(t[2]), _p(dhead))
    return float(loss), dhead


def sg_backward(in16, params, acts, dhead):
    _, hq, wq = in16.shape
    dp = np.zeros(sg_param_count(), dtype=np.float32)
    lib().orc_sg_backward(_p(np.ascontiguousarray(in16, dtype=np.float32)), hq, wq,
                          _p(np.ascontiguousarray(params, dtype=np.float32)), _p(np.ascontiguousarray(acts)),
                          _p(np.ascontiguousarray(dhead)), _p(dp))
    return dp


# --- DNG export: lossless JPEG tiles (examples/prr2dng/lj92.rs, dng.rs) -------


def lj92_encode(samples: np.ndarray, width: int, height: int, components: int = 2) -> bytes:
    s = np.ascontiguousarray(samples, dtype=np.uint16).reshape(-1)
    assert s.size == width * height
    cap = C.c_size_t()
    lib().orc_lj92_encode(_p(s), width, height, components, None, 0, C.byref(cap))
    out = np.zeros(max(1, cap.value), dtype=np.uint8)
    n = C.c_size_t()
    assert lib().orc_lj92_encode(_p(s), width, height, components, _p(out), out.size, C.byref(n)) == 0
    return out[:n.value].tobytes()


def lj92_huffman(histogram):
    h = np.asarray(histogram, dtype=np.uint64)
    counts = np.zeros(16, np.uint8)
    values = np.zeros(17, np.uint8)
    codes = np.zeros(17, np.uint16)
    lengths = np.zeros(17, np.uint8)
    nv = C.c_int()
    lib().orc_lj92_huffman(_p(h), _p(counts), _p(values), C.byref(nv), _p(codes), _p(lengths))
    return counts, values[:nv.value], codes, lengths


def dng_tile(values: np.ndarray, width: int, height: int, left: int, top: int, tile: int = 256,
             stride: int = 0) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.uint16).reshape(-1)
    out = np.zeros(tile * tile, np.uint16)
    assert lib().orc_dng_tile(_p(v), width, height, stride or width, left, top, tile, _p(out)) == 0
    return out


def lj92_tiles(values: np.ndarray, width: int, height: int, tile: int = 256, stride: int = 0, threads: int = 0):
    """Every tile's stream, in order, as dng::write encodes them."""
    v = np.ascontiguousarray(values, dtype=np.uint16).reshape(-1)
    across, down = -(-width // tile), -(-height // tile)
    offsets = np.zeros(across * down + 1, np.uint64)
    cap = across * down * (2 * tile * tile * 4 + 128)
    out = np.zeros(cap, np.uint8)
    assert lib().orc_lj92_tiles(_p(v), width, height, stride or width, tile, threads, _p(out), cap, _p(offsets)) == 0
    return [out[int(offsets[i]):int(offsets[i + 1])].tobytes() for i in range(across * down)]
