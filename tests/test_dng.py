"""The DNG container (host C++ of libprr.so: the crate's DNG writer,
examples/prr2dng/{dng,tiff,colour}.rs) on the CPU: the reference's own
tests of the TIFF layout, the rationals, the colour tags and the dates,
then the tags of whole files for frame headers of every Bayer pattern, crop
and clip description, with LJ92 tiles from the CPU oracle. No device."""

import struct

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import dng as D
from proresraw_rs_b200 import synth as S

# --- a small TIFF reader ----------------------------------------------------

SIZES = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 10: 8}


def entries(data):
    """{tag: (type, count, raw value bytes, offset or None)} of the first IFD,
    checking the layout rules on the way."""
    assert data[:4] == b"II*\0"
    ifd = struct.unpack_from("<I", data, 4)[0]
    n = struct.unpack_from("<H", data, ifd)[0]
    out, tags = {}, []
    for i in range(n):
        tag, kind, count, value = struct.unpack_from("<HHII", data, ifd + 2 + 12 * i)
        size = SIZES[kind] * count
        if size <= 4:
            raw, at = struct.pack("<I", value)[:size], None
        else:
            assert value % 2 == 0, (tag, value)
            raw, at = data[value:value + size], value
        out[tag] = (kind, count, raw, at)
        tags.append(tag)
    assert tags == sorted(tags)
    assert struct.unpack_from("<I", data, ifd + 2 + 12 * n)[0] == 0  # no further IFD
    return out


def value(e):
    kind, count, raw, _ = e
    if kind == 2:
        assert raw[-1:] == b"\0"
        return raw[:-1].decode()
    fmt = {1: "B", 3: "H", 4: "I", 5: "II", 10: "ii"}[kind]
    v = struct.unpack("<" + fmt * count, raw)
    if kind in (5, 10):
        return [(v[2 * i], v[2 * i + 1]) for i in range(count)]
    return list(v)


def chunks_of(data, e, offsets_tag, counts_tag):
    offs, counts = value(e[offsets_tag]), value(e[counts_tag])
    for o in offs:
        assert o % 2 == 0
    return [data[o:o + c] for o, c in zip(offs, counts)]


# --- frame headers ----------------------------------------------------------


def header_of(width=64, height=32, pattern=S.RGGB, crop=(0, 0, 0, 0), wb=(1.0, 1.0), cct=5600, gain=1.0,
              matrix=(1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0), curve=None, vendor=b"test", white=4095):
    spec = S.Spec(width, height, pattern=pattern, alignment=0, crop=crop, wb=wb, wb_cct=cct, gain=gain,
                  color_matrix=matrix, curve=curve, vendor=vendor, white_level=white, valid_tiles=True)
    return P.parse_header(S.random_frame(spec, S.Rng(1)))


D65, D50 = (0.31271, 0.32902), (0.34567, 0.35850)


def xyz(w):
    x, y = w
    return np.array([x / y, 1.0, (1.0 - x - y) / y])


def white_xy(t):
    # The white of a colour temperature (colour.rs:138-173), for checking.
    if t < 4000:
        u = (0.860117757 + 1.54118254e-4 * t + 1.28641212e-7 * t * t) / (
            1.0 + 8.42420235e-4 * t + 7.08145163e-7 * t * t)
        v = (0.317398726 + 4.22806245e-5 * t + 4.20481691e-8 * t * t) / (
            1.0 - 2.89741816e-5 * t + 1.61456053e-7 * t * t)
        d = 2.0 * u - 8.0 * v + 4.0
        return 3.0 * u / d, 2.0 * v / d
    if t in (6500.0, 6504.0):
        return D65
    if t <= 7000:
        x = -4.6070e9 / t ** 3 + 2.9678e6 / t ** 2 + 0.09911e3 / t + 0.244063
    else:
        x = -2.0064e9 / t ** 3 + 1.9018e6 / t ** 2 + 0.24748e3 / t + 0.237040
    return x, -3.0 * x * x + 2.870 * x - 0.275


def rec709():
    # Linear Rec.709 to XYZ, the last column adjusted so that (1, 1, 1) maps
    # to D65 exactly, as a header matrix does (colour.rs:213-225).
    w = xyz(D65)
    m = np.array([[0.4124, 0.3576, 0.0], [0.2126, 0.7152, 0.0], [0.0193, 0.1192, 0.0]])
    m[:, 2] = w - m[:, 0] - m[:, 1]
    return tuple(float(np.float32(v)) for v in m.reshape(-1))


# --- the reference's tests --------------------------------------------------


def test_rationals_keep_six_decimals():
    assert [D.srational(v) for v in (-0.3556711, 3.560669, 5000.0)] == [
        (-355671, 1_000_000), (3560669, 1_000_000), (500_000_000, 100_000)]
    assert D.rational(0.5) == (500_000, 1_000_000)
    # Large values lose decimals, never the integer part; NaN is 0.
    assert D.srational(-3e9) == (-2147483647 - 1, 1) and D.rational(5e9) == (4294967295, 1)
    assert D.srational(float("nan"))[0] == 0


def test_quicktime_dates():
    assert D.quicktime_date_time(0) == "1904:01:01 00:00:00"
    # 2021-10-23 12:34:56 UTC is Unix time 1634992496.
    assert D.quicktime_date_time(1_634_992_496 + 2_082_844_800) == "2021:10:23 12:34:56"
    assert D.quicktime_date_time(2_082_844_800 - 1) == "1969:12:31 23:59:59"
    # The last second of the year 9999 still fits the 19 characters; the
    # next one's text would be longer than the 20-byte result.
    last = 253_402_300_799 + 2_082_844_800
    assert D.quicktime_date_time(last) == "9999:12:31 23:59:59"
    with pytest.raises(P.Error) as e:
        D.quicktime_date_time(last + 1)
    assert e.value.code == P._lib.ERR_BUFFER


@pytest.mark.parametrize("cct,r,b", [(5235, 1.0, 1.0), (3200, 1.7, 0.6), (5139, 2.419, 1.5486)])
def test_the_shot_white_maps_to_the_as_shot_neutral(cct, r, b):
    c = D.DngColour.new(header_of(wb=(r, b), cct=cct, gain=11.8, matrix=rec709()))
    neutral = c.color_matrix @ xyz(white_xy(float(cct)))
    scaled = neutral / (neutral[1] / c.as_shot_neutral[1])
    assert np.allclose(scaled, c.as_shot_neutral, atol=1e-6, rtol=0), (cct, scaled)
    assert abs(neutral.max() - 1.0) < 1e-12


def test_the_forward_matrix_maps_neutral_to_d50():
    c = D.DngColour.new(header_of(cct=5600, gain=11.8, matrix=rec709()))
    assert np.allclose(c.forward_matrix @ np.ones(3), xyz(D50), atol=2e-4, rtol=0)
    assert abs(c.baseline_exposure - np.log2(np.float32(11.8))) < 1e-6
    assert c.illuminant == 20


def test_at_d65_the_matrix_is_only_inverted():
    c = D.DngColour.new(header_of(cct=0, matrix=rec709()))
    assert c.temperature == 6504.0 and c.illuminant == 21
    m = np.array(rec709()).reshape(3, 3)
    identity = c.color_matrix @ m
    assert np.allclose(identity, identity[0, 0] * np.eye(3), atol=1e-9, rtol=0)


def test_temperatures_are_clamped_and_gains_defaulted():
    assert D.DngColour.new(header_of(cct=500)).temperature == 1000.0
    assert D.DngColour.new(header_of(cct=40000)).temperature == 25000.0
    c = D.DngColour.new(header_of(wb=(0.0, -1.0), gain=0.0))
    assert list(c.as_shot_neutral) == [1.0, 1.0, 1.0] and c.baseline_exposure == 0.0
    assert D.DngColour.new(header_of(cct=2900)).illuminant == 17


# --- whole files --------------------------------------------------------------


def visible(w, h, seed=1):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 4096, w * h, dtype=np.uint16)


@pytest.mark.parametrize("pattern,cfa", [(S.RGGB, [0, 1, 1, 2]), (1, [1, 0, 2, 1]), (2, [1, 2, 0, 1]),
                                         (S.BGGR, [2, 1, 1, 0])])
def test_tags_of_a_file(pattern, cfa):
    w, h = 300, 270
    hdr = header_of(w, h, pattern=pattern, crop=(2, 4, 6, 8), wb=(1.8, 1.4), cct=5139, gain=2.0,
                    matrix=rec709(), curve=[0, 400, 900, 2000, 4100, 8000, 17000, 33000], white=4000)
    img = visible(w, h)
    tiles = O.lj92_tiles(img, w, h)
    clip = D.ClipInfo(make="Sony", model="FX6", fps=(24000, 1001), date_time="2021:10:23 12:34:56", orientation=6)
    data = D.assemble(hdr, tiles, clip)
    e = entries(data)
    v = lambda t: value(e[t])  # noqa: E731
    assert v(254) == [0] and v(256) == [w] and v(257) == [h] and v(258) == [16] and v(259) == [7]
    assert v(262) == [32803] and v(271) == "Sony" and v(272) == "FX6" and v(274) == [6]
    assert v(277) == [1] and v(284) == [1] and v(305) == "proresraw_rs prr2dng 0.1.0"
    assert v(306) == "2021:10:23 12:34:56"
    assert v(322) == [256] and v(323) == [256]
    assert v(33421) == [2, 2] and v(33422) == cfa
    assert v(50706) == [1, 4, 0, 0] and v(50707) == [1, 3, 0, 0]
    assert v(50708) == "Sony FX6 (ProRes RAW)" and v(50710) == [0, 1, 2] and v(50711) == [1]
    lut = [O.curve_linearize(hdr._c.curve, code) for code in range(65536)]
    assert v(50712) == lut
    assert v(50713) == [1, 1] and v(50714) == [256] and v(50717) == [4000]
    assert v(50719) == [2, 6] and v(50720) == [w - 6, h - 14]
    colour = D.DngColour.new(hdr)
    assert v(50721) == [D.srational(x) for x in colour.color_matrix.reshape(-1)]
    assert v(50728) == [D.rational(x) for x in colour.as_shot_neutral]
    assert v(50730) == [D.srational(colour.baseline_exposure)]
    assert v(50778) == [colour.illuminant]
    assert v(50964) == [D.srational(x) for x in colour.forward_matrix.reshape(-1)]
    assert v(51044) == [(24000, 1001)]
    assert sorted(e) == [254, 256, 257, 258, 259, 262, 271, 272, 274, 277, 284, 305, 306, 322, 323, 324, 325,
                         33421, 33422, 50706, 50707, 50708, 50710, 50711, 50712, 50713, 50714, 50717, 50719,
                         50720, 50721, 50728, 50730, 50778, 50964, 51044]
    # The tiles land where the entries say, each padded to an even length.
    assert chunks_of(data, e, 324, 325) == tiles
    last = value(e[324])[-1] + value(e[325])[-1]
    assert len(data) == last + (last & 1)


def test_optional_tags_and_camera_names():
    w, h = 64, 32
    hdr = header_of(w, h, vendor=b"ab\x01c")
    img = visible(w, h)
    strip = img.astype("<u2").tobytes()
    data = D.assemble(hdr, [strip], D.ClipInfo(), D.Samples.LINEAR, D.Compression.NONE)
    e = entries(data)
    # No make, model, date, frame rate or LinearizationTable; no crop when
    # the margins leave nothing; one strip of the visible samples.
    for t in (271, 272, 306, 50712, 51044):
        assert t not in e
    assert value(e[50708]) == "ProRes RAW ab\\x01c"
    assert value(e[259]) == [1] and value(e[278]) == [h] and value(e[274]) == [1]
    assert chunks_of(data, e, 273, 279) == [strip]
    assert value(e[50719]) == [0, 0] and value(e[50720]) == [w, h]
    e2 = entries(D.assemble(header_of(w, h, crop=(40, 30, 0, 0)), [strip], D.ClipInfo(model="X"),
                            D.Samples.LINEAR, D.Compression.NONE))
    assert 50719 not in e2 and 50720 not in e2
    assert value(e2[50708]) == "X (ProRes RAW)"


def test_a_single_tile_offset_fits_in_its_entry():
    w, h = 200, 100
    hdr = header_of(w, h)
    tiles = O.lj92_tiles(visible(w, h), w, h)
    data = D.assemble(hdr, tiles)
    e = entries(data)
    kind, count, raw, at = e[324]
    assert count == 1 and at is None
    off = value(e[324])[0]
    assert data[off:off + len(tiles[0])] == tiles[0]


def test_wrong_chunk_counts_are_refused():
    hdr = header_of(300, 270)
    with pytest.raises(P.Error):
        D.assemble(hdr, [b"x"] * 3)  # needs 2 x 2 tiles
    with pytest.raises(P.Error):
        D.assemble(hdr, [b"x", b"y"], compression=D.Compression.NONE)
