"""Known-answer tests of frame parsing, decoding, reduced decoding and the
raw conversion, ported from the crate's unit tests: src/curve.rs:36-70,
src/header.rs:307-489, src/tile.rs:156-250, src/decoder.rs:309-427,
src/reduced.rs:276-360, src/demosaic.rs:778-1008, src/synth.rs:223-274.

Header and tile-table parsing run on the host in both implementations, so
those tests cover the library on the CPU as well. Decode and develop tests
run on the oracle here and on the CUDA library under the `gpu` marker.
"""

import struct

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from _impls import GpuImpl, OracleImpl
from proresraw_rs_b200 import synth as S

IMPLS = [pytest.param("oracle", id="oracle"), pytest.param("gpu", id="gpu", marks=pytest.mark.gpu)]


@pytest.fixture
def impl(request):
    return OracleImpl() if request.param == "oracle" else GpuImpl()


# --- src/curve.rs ---------------------------------------------------------------

def test_default_curve_hits_control_points():
    d = P.Curve(P.Curve.DEFAULT_POINTS)
    for i, p in enumerate(P.Curve.DEFAULT_POINTS):
        assert d.linearize(i * 8192) == p == O.curve_linearize(P.Curve.DEFAULT_POINTS, i * 8192)
    assert d.linearize(65535) == 65532 == O.curve_linearize(P.Curve.DEFAULT_POINTS, 65535)


def test_curve_interpolates_and_rounds():
    c = [0, 100, 200, 300, 400, 500, 600, 700]
    assert O.curve_linearize(c, 4096) == 50
    assert O.curve_linearize(c, 8192 + 2048) == 125
    assert O.curve_linearize(c, 57344 + 4096) == (700 + 65536) // 2
    c = [0, 1, 2, 3, 4, 5, 6, 7]
    assert O.curve_linearize(c, 4095) == 0 and O.curve_linearize(c, 4096) == 1
    c = [0, 224, 288, 468, 1162, 3339, 9431, 25377]
    for code in [0, 1, 8191, 8192, 30000, 65535]:
        assert P.Curve(tuple(c)).linearize(code) == O.curve_linearize(c, code)


# --- src/header.rs --------------------------------------------------------------

def body(flags, tail=b""):
    b = bytearray(70)
    b[2:6] = b"test"
    b[6:8] = struct.pack(">H", 64)
    b[8:10] = struct.pack(">H", 32)
    b[10:14] = bytes([1, 2, 3, 4])
    b[14:16] = struct.pack(">H", 3)
    b[16:18] = struct.pack(">H", 0xFDFF)
    b[18:22] = struct.pack(">f", 2.0)
    b[22:26] = struct.pack(">f", 1.5)
    for i in range(9):
        b[26 + 4 * i: 30 + 4 * i] = struct.pack(">f", float(i))
    b[62:66] = struct.pack(">f", 11.8)
    b[66:68] = struct.pack(">H", 5600)
    b[68:70] = struct.pack(">H", flags)
    return bytes(b) + bytes(tail)


def packet_of(b):
    """A frame prefix around a header body (src/decoder.rs:10-13)."""
    p = struct.pack(">I", 10 + len(b)) + b"prrf" + struct.pack(">H", len(b) + 2) + b
    return p


def both_parse(p):
    """Parse with the oracle and with the library's host parser; both must agree."""
    try:
        oh = O.parse_header(p)
        oerr = None
    except O.OracleError as e:
        oh, oerr = None, e.code
    try:
        ph = P.parse_header(p)
        perr = None
    except P.Error as e:
        ph, perr = None, e
    assert (oerr is None) == (perr is None), (oerr, perr)
    if oerr is not None:
        assert perr.code == oerr
        return None, perr
    from _impls import header_fields

    assert header_fields(oh) == header_fields(ph)
    return ph, None


def test_parses_fixed_fields_and_defaults():
    h, _ = both_parse(packet_of(body(0b0110)))
    assert h.version == 0 and h.vendor == b"test" and (h.width, h.height) == (64, 32)
    assert h.crop == (1, 2, 3, 4)
    assert h.bayer_pattern == P.BayerPattern.BGGR
    assert h.white_level == 65279
    assert (h.wb_red, h.wb_blue) == (2.0, 1.5)
    assert h.color_matrix[1][2] == 5.0
    assert h.gain == np.float32(11.8)
    assert h.wb_cct == 5600 and h.alignment == 3
    assert h.quant_matrix == (1,) * 64
    assert h.curve.points == P.Curve.DEFAULT_POINTS


def test_parses_quant_matrix_and_curve():
    tail = bytes([7] * 64) + b"".join(struct.pack(">H", p) for p in [0, 224, 288, 468, 1162, 3339, 9431, 25377])
    b = bytearray(body(0b11_1001, tail))
    b[1] = 1
    h, _ = both_parse(packet_of(bytes(b)))
    assert h.alignment == 4 and h.quant_matrix == (7,) * 64
    assert h.curve.points == (0, 224, 288, 468, 1162, 3339, 9431, 25377)


def test_rejects_bad_input():
    b = bytearray(body(0))
    b[1] = 2
    _, e = both_parse(packet_of(bytes(b)))
    assert e == P.Error(P._lib.ERR_UNSUPPORTED_VERSION, {"value": 2})
    b = bytearray(body(0))
    b[7] = 65
    _, e = both_parse(packet_of(bytes(b)))
    assert e.kind == "BadDimensions"
    _, e = both_parse(packet_of(body(0b1010)))
    assert e == P.Error(P._lib.ERR_BAD_ALIGNMENT, {"value": 5})
    _, e = both_parse(packet_of(body(1, bytes(10))))
    assert e.kind == "Truncated" and e.fields["what"] == "quantization matrix"
    # A header body shorter than its size field says.
    _, e = both_parse(packet_of(body(0))[:-5])
    assert e.kind == "Truncated"


def test_rejects_what_apple_rejects():
    qmat = bytearray([63] * 64)
    qmat[5] = 64
    _, e = both_parse(packet_of(body(1, bytes(qmat))))
    assert e == P.Error(P._lib.ERR_BAD_QUANT_MATRIX, {"index": 5, "value": 64})
    qmat[5] = 0
    _, e = both_parse(packet_of(body(1, bytes(qmat))))
    assert e == P.Error(P._lib.ERR_BAD_QUANT_MATRIX, {"index": 5, "value": 0})

    def curve(points, version):
        b = bytearray(body(0x10, b"".join(struct.pack(">H", p) for p in points)))
        b[1] = version
        return both_parse(packet_of(bytes(b)))

    rising = [0, 512, 1024, 2048, 4096, 8192, 16384, 32768]
    assert curve(rising, 1)[1] is None
    assert curve(rising, 0)[1].kind == "UnexpectedCurve"
    flat = [0, 512, 512, 2048, 4096, 8192, 16384, 32768]
    assert curve(flat, 1)[1] == P.Error(P._lib.ERR_BAD_CURVE, {"points": flat})
    falling = [0, 512, 1024, 2048, 4096, 8192, 16384, 100]
    assert curve(falling, 1)[1] == P.Error(P._lib.ERR_BAD_CURVE, {"points": falling})


def test_bayer_pattern_colours_and_stream_phases():
    B = P.BayerPattern
    grid = lambda p: [p.color_at(0, 0), p.color_at(0, 1), p.color_at(1, 0), p.color_at(1, 1)]
    assert grid(B.RGGB) == ["red", "green", "green", "blue"]
    assert grid(B.GRBG) == ["green", "red", "blue", "green"]
    assert grid(B.GBRG) == ["green", "blue", "red", "green"]
    assert grid(B.BGGR) == ["blue", "green", "green", "red"]
    assert B.RGGB.stream_phases() == [(1, 0), (0, 1), (1, 1), (0, 0)]
    assert B.BGGR.stream_phases() == [(0, 1), (1, 0), (0, 0), (1, 1)]
    assert B.GRBG.stream_phases() == [(1, 1), (0, 0), (1, 0), (0, 1)]
    assert B.GBRG.stream_phases() == [(0, 0), (1, 1), (0, 1), (1, 0)]
    for p in B:
        g0, g1, b, r = p.stream_phases()
        assert [p.color_at(*g0), p.color_at(*g1), p.color_at(*b), p.color_at(*r)] == ["green", "green", "blue", "red"]


def test_coded_dimensions_round_up_to_tiles():
    b = bytearray(body(0))
    b[6:8] = struct.pack(">H", 4264)
    b[8:10] = struct.pack(">H", 2408)
    h, _ = both_parse(packet_of(bytes(b)))
    assert (h.coded_width(), h.coded_height()) == (4272, 2416)


# --- src/tile.rs ----------------------------------------------------------------

def widths(w, h, a):
    return [(16 << l) for _, l in S.grid_row(w, a)]


def oracle_row(w, h, a):
    import ctypes as C

    n = O.lib().orc_grid_row(w, h, a, None, None)
    x = np.zeros(n, dtype=np.uint64)
    l = np.zeros(n, dtype=np.uint8)
    O.lib().orc_grid_row(w, h, a, x.ctypes.data, l.ctypes.data)
    return [(int(a_), int(b_)) for a_, b_ in zip(x, l)]


def test_tile_grid():
    assert oracle_row(5888, 3312, 3) == S.grid_row(5888, 3)
    assert len(S.grid_row(5888, 3)) == 46 and all(w == 128 for w in widths(5888, 3312, 3))
    w = widths(4264, 2408, 3)
    assert len(w) == 35 and all(v == 128 for v in w[:33]) and w[33:] == [32, 16]
    assert S.grid_row(4264, 3)[-1] == (4256, 0)
    assert widths(48, 16, 0) == [16, 16, 16]
    assert widths(4224, 3024, 4) == [256] * 16 + [128]
    for (w_, a_) in [(5760, 4), (4096, 2), (8192, 3), (1920, 1), (600, 4), (2, 0), (65534, 4)]:
        assert oracle_row(w_, 16, a_) == S.grid_row(w_, a_)
    # Frame-level counts agree with the library's host parser.
    for (w_, h_, a_) in [(5760, 3040, 4), (4096, 2160, 2), (8192, 4320, 3), (1920, 1080, 0)]:
        spec = S.Spec(w_, h_, alignment=a_)
        pkt = S.frame(spec, [S.tile(1, [b"\x80"] * 4)] * S.ntiles(w_, h_, a_))
        f = P.parse_frame(pkt)
        assert f.tiles_per_row == len(S.grid_row(w_, a_)) and f.tile_rows == (h_ + 15) // 16


def tile_ok(hdr, qscale, sizes, length):
    d = bytes([hdr << 3, qscale]) + b"".join(struct.pack(">H", s) for s in sizes)
    d = d + bytes([0xAA]) * (length - len(d))
    q = np.zeros(1, dtype=np.uint8)
    import ctypes as C

    qq = C.c_uint8()
    off = np.zeros(4, dtype=np.uint64)
    ln = np.zeros(4, dtype=np.uint64)
    buf = np.frombuffer(d + b"\0", dtype=np.uint8)
    rc = O.lib().orc_tile_parse(buf.ctypes.data, len(d), 0, C.byref(qq), off.ctypes.data, ln.ctypes.data)
    return rc == 0, qq.value, list(off), list(ln)


def test_tile_header_splits_streams_and_rejects():
    ok, q, off, ln = tile_ok(8, 15, [2, 1, 3], 16)
    assert ok and q == 15 and off == [8, 10, 11, 14] and ln == [2, 1, 3, 2]
    assert tile_ok(8, 1, [1, 1, 1], 12)[0]
    assert not tile_ok(7, 1, [1, 1, 1], 12)[0]
    assert not tile_ok(8, 0, [1, 1, 1], 12)[0]
    assert not tile_ok(8, 1, [0, 1, 1], 12)[0]
    assert not tile_ok(8, 1, [1, 0, 1], 12)[0]
    assert not tile_ok(8, 1, [1, 1, 0], 12)[0]
    assert not tile_ok(8, 1, [1, 1, 1], 11)[0]
    assert not tile_ok(8, 1, [9, 0, 0], 10)[0]


# --- src/decoder.rs -------------------------------------------------------------

def frame_16(tiles_table_and_payload):
    b = bytearray(70)
    b[6:8] = struct.pack(">H", 16)
    b[8:10] = struct.pack(">H", 16)
    p = bytearray(struct.pack(">I", 0) + b"prrf" + struct.pack(">H", 72) + bytes(b))
    p += tiles_table_and_payload
    p[0:4] = struct.pack(">I", len(p))
    return bytes(p)


def decode_err(impl, p):
    try:
        impl.decode(p)
    except O.OracleError as e:
        return e.code
    except P.Error as e:
        return e.code
    return None


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_rejects_bad_prefixes(impl):
    assert decode_err(impl, bytes(4)) == P._lib.ERR_TRUNCATED
    p = bytearray(80)
    p[0:4] = struct.pack(">I", 80)
    p[4:8] = b"xxxx"
    assert decode_err(impl, bytes(p)) == P._lib.ERR_BAD_TAG
    p[4:8] = b"prrf"
    p[8:10] = struct.pack(">H", 61)
    assert decode_err(impl, bytes(p)) == P._lib.ERR_HEADER_TOO_SHORT
    p[0:4] = struct.pack(">I", 81)
    assert decode_err(impl, bytes(p)) == P._lib.ERR_FRAME_SIZE_MISMATCH
    for size in (0, 81):
        p[0:4] = struct.pack(">I", size)
        assert decode_err(impl, bytes(p)) == P._lib.ERR_FRAME_SIZE_MISMATCH
    p[0:4] = struct.pack(">I", 20)  # below the packet length: passes the size check
    assert decode_err(impl, bytes(p)) == P._lib.ERR_HEADER_TOO_SHORT


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_empty_tile_decodes_to_mid_grey(impl):
    p = frame_16(struct.pack(">H", 12) + bytes([8 << 3, 1, 0, 1, 0, 1, 0, 1, 0, 0, 0, 0]))
    f, raw = impl.decode(p)
    assert (f.width(), f.height(), f.stride()) == (16, 16, 16)
    assert f.skipped_tiles == []
    assert np.all(f.samples == 32768)
    assert np.all(impl.linearize(raw) == 4096)
    # Empty streams make the tile invalid: it is skipped and its sensels are 0.
    p = frame_16(struct.pack(">H", 8) + bytes([8 << 3, 1, 0, 0, 0, 0, 0, 0]))
    f, _ = impl.decode(p)
    assert f.skipped_tiles == [0]
    assert np.all(f.samples == 0)


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_missing_tile_is_an_error(impl):
    p = frame_16(struct.pack(">H", 40) + bytes(8))
    assert decode_err(impl, p) == P._lib.ERR_TILE_OUT_OF_BOUNDS
    try:
        impl.decode(p)
    except P.Error as e:
        assert e.fields == {"tile": 0}
    except O.OracleError as e:
        assert e.err.index == 0


def test_header_parses_from_the_packet_start():
    rng = S.Rng(13)
    pkt = S.random_frame(S.Spec(48, 32, pattern=S.BGGR), rng)
    n = P.header_len(pkt)
    assert n == O.header_len(pkt) and n < len(pkt)
    from _impls import header_fields

    assert header_fields(P.parse_header(pkt[:n])) == header_fields(P.parse_frame(pkt).header)
    with pytest.raises(P.Error) as e:
        P.parse_header(pkt[: n - 1])
    assert e.value.kind == "Truncated"
    with pytest.raises(P.Error) as e:
        P.header_len(pkt[:9])
    assert e.value.kind == "Truncated"


def test_parse_frame_matches_the_oracle_on_random_frames():
    rng = S.Rng(21)
    for spec in S.specs(rng):
        pkt = S.random_frame(spec, rng)
        oh, off, ln, tpr, rows, mq = O.parse_frame(pkt)
        f = P.parse_frame(pkt)
        assert (f.ntiles, f.tiles_per_row, f.tile_rows, f.max_qscale) == (len(off), tpr, rows, mq)
        assert P.frame_quantizer(f) == oh.quant_matrix[0] * mq


# --- src/synth.rs + src/reduced.rs + decode -------------------------------------

@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_random_frames_decode_without_panicking(impl):
    rng = S.Rng(1)
    for spec in S.specs(rng):
        pkt = S.random_frame(spec, rng)
        f, raw = impl.decode(pkt)
        assert f.width() == spec.width and f.header.bayer_pattern == spec.pattern
        flat = np.count_nonzero(f.samples == 32768)
        assert flat < f.samples.size // 2, "streams decoded to almost nothing"
        impl.linearize(raw)


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_the_header_carries_the_spec_and_valid_tiles_are_never_skipped(impl):
    rng = S.Rng(2)
    spec = S.Spec(48, 32, pattern=S.BGGR, vendor=b"atm0", crop=(16, 8, 4, 2), white_level=4095 + 256,
                  wb=(1.5, 0.75), color_matrix=(0.7, 0.2, 0.1, 0.3, 1.0, -0.3, 0.0, -0.4, 1.5), gain=11.8,
                  wb_cct=5235, valid_tiles=True)
    f, _ = impl.decode(S.random_frame(spec, rng))
    h = f.header if not hasattr(f.header, "_h") else f.header._h
    assert bytes(h.vendor) == b"atm0" and tuple(h.crop) == (16, 8, 4, 2)
    assert h.white_level == 4095 + 256 and (h.wb_red, h.wb_blue) == (1.5, 0.75)
    assert np.float32(h.gain) == np.float32(11.8) and h.wb_cct == 5235
    assert f.skipped_tiles == []


def _linear_of(impl, pkt):
    f, raw = impl.decode(pkt)
    return f, impl.linearize(raw)


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_half_resolution_matches_full_decode(impl):
    rng = S.Rng(7)
    for spec in S.specs(rng):
        spec.valid_tiles = True
        pkt = S.random_frame(spec, rng)
        full, linear = _linear_of(impl, pkt)
        w, h = full.width(), full.height()
        lin = linear.reshape(h, w)
        g, _, b, r = P.BayerPattern(spec.pattern).stream_phases()
        rgb = impl.decode_reduced(pkt, 1, 0)
        stride = full.stride() // 2
        s = rgb.samples.reshape(-1, stride, 3)[: h // 2, : w // 2]
        for c, (pr, pc) in enumerate([r, g, b]):
            assert np.array_equal(s[:, :, c], lin[pr::2, pc::2][: h // 2, : w // 2]), (spec.pattern, c)


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_half_resolution_can_average_the_greens(impl):
    rng = S.Rng(12)
    for spec in S.specs(rng):
        spec.valid_tiles = True
        pkt = S.random_frame(spec, rng)
        full, linear = _linear_of(impl, pkt)
        w, h = full.width(), full.height()
        lin = linear.reshape(h, w).astype(np.uint32)
        g1, g2, b, r = P.BayerPattern(spec.pattern).stream_phases()
        rgb = impl.decode_reduced(pkt, 1, 1)
        s = rgb.samples.reshape(-1, full.stride() // 2, 3)[: h // 2, : w // 2]
        at = lambda ph: lin[ph[0]::2, ph[1]::2][: h // 2, : w // 2]
        assert np.array_equal(s[:, :, 0], at(r))
        assert np.array_equal(s[:, :, 1], (at(g1) + at(g2) + 1) // 2)
        assert np.array_equal(s[:, :, 2], at(b))


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_reduced_sizes_and_skipped_tiles(impl):
    rng = S.Rng(8)
    for spec in S.specs(rng):
        pkt = S.random_frame(spec, rng)
        full, _ = impl.decode(pkt)
        for shift in (1, 2, 3):
            for greens in (0, 1):
                f = 1 << shift
                rgb = impl.decode_reduced(pkt, shift, greens)
                assert rgb.samples.size == 3 * (full.stride() // f) * (((full.height() + 15) & ~15) // f)
                assert rgb.skipped_tiles == full.skipped_tiles
                assert rgb.max_qscale == full.max_qscale


# --- src/demosaic.rs ------------------------------------------------------------

def kat_params(pattern, wb):
    p = O.Params()
    rng_ = 65279 - 256
    p.cfa_phase = pattern
    p.black = 256
    p.one_over_range = np.float32(1.0) / np.float32(rng_)
    p.noise[:] = [1e-6, 1e-9, 5e-9]
    p.clip[:] = [np.float32(1.0) / np.float32(g) for g in wb]
    p.black_over_range = np.float32(256.0) / np.float32(rng_)
    p.wb[:] = list(wb)
    return p


def mosaic_of(pattern, w, h, rgb):
    bp = P.BayerPattern(pattern)
    m = np.zeros((h, w), dtype=np.uint16)
    for y in range(h):
        for x in range(w):
            m[y, x] = rgb[{"red": 0, "green": 1, "blue": 2}[bp.color_at(y, x)]]
    return m.reshape(-1)


def test_flat_field_is_reproduced_exactly():
    w, h = 12, 10
    for pattern in range(4):
        p = kat_params(pattern, [1.0, 1.0])
        lin = mosaic_of(pattern, w, h, [20000] * 3)
        v = np.float32(p.one_over_range) * np.float32(20000 - 256)
        rgb = O.chroma_pass(O.green_pass(lin, w, h, p), w, h, p)
        assert np.all(rgb == v), pattern


def test_colour_field_lands_on_the_right_channels():
    w, h = 16, 14
    for pattern in range(4):
        p = kat_params(pattern, [2.0, 1.5])
        raw = [12000, 30000, 16000]
        rgb = O.chroma_pass(O.green_pass(mosaic_of(pattern, w, h, raw), w, h, p), w, h, p).reshape(-1, 3)
        norm = [np.float32(p.one_over_range) * np.float32(v - 256) for v in raw]
        want = np.array([norm[0] * 2.0, norm[1], norm[2] * 1.5], dtype=np.float32)
        assert np.all(np.abs(rgb - want) < 1e-6), pattern


def test_red_and_blue_clip_where_white_balance_reaches_one():
    w, h = 8, 8
    p = kat_params(0, [2.0, 4.0])
    rgb = O.chroma_pass(O.green_pass(mosaic_of(0, w, h, [60000, 1000, 60000]), w, h, p), w, h, p).reshape(-1, 3)
    assert np.all(rgb[:, 0] == 1.0) and np.all(rgb[:, 2] == 1.0)


def test_noise_parameters_follow_the_quantizer():
    rng = S.Rng(3)
    pkt = S.random_frame(S.Spec(32, 16, valid_tiles=True), rng)
    h = P.parse_frame(pkt).header
    p = P.DemosaicParams.with_white_balance(h, 64, 2.0, 0.0)
    rng_ = 65023.0
    base = 5.0 * 64.0 * 64.0 + 64.0 / 3.0
    assert p.noise[0] == np.float32(base / 150_994_944.0)
    assert p.noise[1] == np.float32(base / (rng_ * rng_ * 256.0))
    assert p.noise[2] == np.float32(64.0 / 3.0 / (rng_ * rng_))
    assert p.clip == (0.5, 1.0) and p.wb == (2.0, 0.0)
    o = O.params_with_white_balance(O.parse_header(pkt), 64, 2.0, 0.0)
    assert (tuple(o.noise), tuple(o.clip), o.one_over_range, o.black_over_range) == (
        p.noise, p.clip, p.one_over_range, p.black_over_range)


def test_output_matrix_combines_gamut_matrix_and_gain():
    rng = S.Rng(4)
    pkt = S.random_frame(S.Spec(32, 16, gain=2.0), rng)
    h = P.parse_frame(pkt).header
    xyz = [1.716651187971268, -0.355670783776393, -0.25336628137366, -0.666684351832489, 1.616481236634939,
           0.015768545813911, 0.017639857445311, -0.042770613257809, 0.942103121235474]
    refl = P.output_matrix(h, P.Exposure.REFLECTION)
    norm = P.output_matrix(h, P.Exposure.NORMALIZED)
    for i in range(9):
        assert refl[i] == np.float32(xyz[i] * 2.0)
        assert norm[i] == np.float32(xyz[i] * 2.0 * 10.0 / 9.0)
    oh = O.parse_header(pkt)
    assert np.array_equal(O.output_matrix(oh, 0), norm) and np.array_equal(O.output_matrix(oh, 1), refl)


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_quantizer_counts_every_tile_qscale_byte(impl):
    rng = S.Rng(6)
    pkt = bytearray(S.random_frame(S.Spec(64, 32, valid_tiles=True, quant_matrix=[3] * 64), rng))
    oh, off, ln, _, _, mq = O.parse_frame(bytes(pkt))
    assert mq == max(pkt[int(o) + 1] for o in off)
    start = int(off[0])
    pkt[start + 1] = 255
    pkt[start + 2:start + 4] = b"\0\0"
    assert P.frame_quantizer(P.parse_frame(bytes(pkt))) == 3 * 255
    f, _ = impl.decode(bytes(pkt))
    assert f.skipped_tiles == [0] and f.quantizer() == 3 * 255
    assert impl.decode_reduced(bytes(pkt), 1, 0).quantizer() == 3 * 255


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_develop_stages(impl):
    rng = S.Rng(9)
    pkt = S.random_frame(S.Spec(48, 32, valid_tiles=True, wb=(2.0, 1.5)), rng)
    f, raw = impl.decode(pkt)
    q = f.quantizer()
    hdr = raw.header
    demosaiced = impl.develop(raw, impl.params(hdr, q), 0, False)
    plain = O.params_with_white_balance(O.parse_header(pkt), q, 1.0, 1.0)
    lin = O.decode_frame(pkt).linearize()
    w, h = f.width(), f.height()
    want = O.chroma_pass(O.green_pass(lin, w, h, plain), w, h, plain)
    assert np.array_equal(demosaiced, want)
    balanced = impl.develop(raw, impl.params(hdr, q), 1, False)
    assert not np.array_equal(demosaiced, balanced)
    rec = impl.develop(raw, impl.params(hdr, q), 2, False)
    m = O.output_matrix(O.parse_header(pkt), 0)
    assert np.array_equal(rec, O.apply_matrix(balanced, m))


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_planar_and_interleaved_outputs_agree(impl):
    rng = S.Rng(10)
    pkt = S.random_frame(S.Spec(80, 80, pattern=S.GRBG, valid_tiles=True, wb=(1.8, 1.3)), rng)
    f, raw = impl.decode(pkt)
    params = impl.params(raw.header, f.quantizer())
    assert f.height() % 32 != 0
    for stage in (0, 1, 2):
        inter = impl.develop(raw, params, stage, False)
        planes = impl.develop(raw, params, stage, True)
        for c in range(3):
            assert np.array_equal(planes[c], inter[c::3]), (stage, c)


@pytest.mark.gpu
def test_planar_output_must_fit_the_frame():
    rng = S.Rng(11)
    f = P.decode_frame(S.random_frame(S.Spec(32, 16), rng))
    params = P.DemosaicParams.new(f.header, f.quantizer())
    r, g, b = np.zeros(32 * 16, np.float32), np.zeros(32 * 16, np.float32), np.zeros(10, np.float32)
    with pytest.raises(P.Error) as e:
        P.develop_planar_into(f, params, P.Stage.WHITE_BALANCED, [r, g, b])
    assert e.value.kind == "Buffer"


@pytest.mark.parametrize("impl", IMPLS, indirect=True)
def test_develop_runs_on_a_decoded_frame(impl):
    rng = S.Rng(5)
    pkt = S.random_frame(S.Spec(48, 32, pattern=S.BGGR, valid_tiles=True), rng)
    f, raw = impl.decode(pkt)
    assert f.quantizer() > 0
    img = impl.develop(raw, impl.params(raw.header, f.quantizer()), 1, False)
    assert img.size == 48 * 32 * 3
    assert np.all(np.isfinite(img)) and np.all(img <= 1.0)


def _error_code(fn, *args):
    try:
        fn(*args)
    except (P.Error, O.OracleError) as e:
        return e.code, getattr(e, "fields", None)
    return 0, None


def test_corrupted_packets_parse_like_the_oracle():
    # Byte changes and truncations in the prefix, the header and the tile
    # size table: the library's host parse (header, grid, size-table walk)
    # gives the oracle's result, the same error or the same frame, and never
    # reads out of bounds.
    import random

    rng = random.Random(3)
    srng = S.Rng(5)
    bases = [S.random_frame(spec, srng) for spec in S.specs(srng)[:6]]
    for trial in range(800):
        pkt = bytearray(rng.choice(bases))
        n = P.header_len(bytes(pkt)) if len(pkt) > 10 else 10
        for _ in range(rng.randrange(1, 4)):
            kind = rng.randrange(3)
            if kind == 0 and len(pkt) > 1:
                # a byte of the prefix, header or size table
                pkt[rng.randrange(min(len(pkt), n + 64))] = rng.randrange(256)
            elif kind == 1 and len(pkt) > 1:
                del pkt[rng.randrange(1, len(pkt)):]
            elif len(pkt) > 12:
                at = rng.randrange(0, min(len(pkt) - 2, n + 64))
                pkt[at:at + 2] = struct.pack(">H", rng.choice([0, 1, 0xFFFF, 0x8000, len(pkt) & 0xFFFF]))
        p = bytes(pkt)
        got_code, got_fields = _error_code(P.parse_frame, p)
        try:
            want = O.parse_frame(p)
            want_code = 0
        except O.OracleError as e:
            want, want_code = None, e.code
        assert got_code == want_code, (trial, got_code, want_code)
        if want_code == 0:
            f = P.parse_frame(p)
            oh, off, ln, tpr, rows, mq = want
            assert (f.ntiles, f.tiles_per_row, f.tile_rows, f.max_qscale) == (len(off), tpr, rows, mq)
        assert _error_code(P.parse_header, p)[0] == _error_code(O.parse_header, p)[0]
