"""Parity of the CUDA library with the CPU oracle on seeded inputs.

Integer and byte outputs (coefficients, code values, linear values,
skipped-tile lists, max_qscale) must be bit-exact. The develop output is
f32; the bar is the crate's own (bit-exact, as the crate's GPU path is with
its host path), checked as exact equality and, as the looser contract,
|gpu - oracle| <= 1e-5 * max(1, |oracle|).
"""

import ctypes as C

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib
from proresraw_rs_b200 import synth as S
from test_kats_stream import _coef_cases, golden_hash, golden_records, wrapped_zero_run_stream

pytestmark = pytest.mark.gpu

DEVELOP_RTOL = 1e-5


def torch():
    import torch as t

    return t


def dev(a):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a)).cuda()


def transform_dev(kind, coefs, q):
    t = torch()
    n = coefs.shape[0]
    per = {0: 64, 1: 64, 2: 16, 3: 4}[kind]
    c, qq = dev(coefs.astype(np.int16)), dev(q.astype(np.int16))
    out = t.empty(n * per, dtype=t.int16, device="cuda")
    ctx = P.context()
    rc = _lib.lib().prr_transform_blocks(ctx, kind, c.data_ptr(), qq.data_ptr(), out.data_ptr(), n)
    assert rc == 0
    t.cuda.synchronize()
    return out.cpu().numpy().view(np.uint16).reshape(n, per)


def test_apple_matches_reference_vectors_gpu():
    c, q, want = golden_records()
    assert np.array_equal(transform_dev(0, c, q), want)


def test_apple_matches_reference_hash_gpu():
    g = S.Gen(0x4A54)
    h = S.FNV_OFFSET
    for _ in range(4):
        c, q = g.blocks(1 << 18)
        h = S.fnv1a_u16(h, transform_dev(0, c, q))
    assert h == golden_hash()


@pytest.mark.parametrize("kind", [1, 2, 3], ids=["ffmpeg", "4x4", "2x2"])
def test_other_transforms_match_the_oracle(kind):
    g = S.Gen(0x5EED + kind)
    c, q = g.blocks(1 << 15)
    name = {1: "ffmpeg", 2: "4x4", 3: "2x2"}[kind]
    per = {1: 64, 2: 16, 3: 4}[kind]
    cc = c[:, :per].copy()
    got = transform_dev(kind, cc, q)
    want = np.stack([O.block(name, cc[i], q[i]) for i in range(0, cc.shape[0], 37)])
    assert np.array_equal(got[::37], want)
    if kind == 1:
        assert np.array_equal(got, O.transform_blocks(1, c, q))


def decode_components_dev(data: bytes, offs, lens, log2_blocks, log2_coefs):
    t = torch()
    buf = np.zeros(P._lib.lib().prr_padded_packet_bytes(len(data)), dtype=np.uint8)
    buf[: len(data)] = np.frombuffer(data, dtype=np.uint8)
    d = dev(buf)
    o, ln = dev(np.array(offs, dtype=np.uint32)), dev(np.array(lens, dtype=np.uint32))
    codes = 1 << (log2_blocks + log2_coefs)
    out = t.empty(len(offs) * codes, dtype=t.int16, device="cuda")
    rc = _lib.lib().prr_decode_components(P.context(), d.data_ptr(), o.data_ptr(), ln.data_ptr(), len(offs),
                                          log2_blocks, log2_coefs, out.data_ptr())
    assert rc == 0
    t.cuda.synchronize()
    return out.cpu().numpy().reshape(len(offs), codes)


@pytest.mark.parametrize("case", _coef_cases(), ids=lambda c: c[0])
def test_coefficient_kats_gpu(case):
    _, data, log2, check = case
    got = decode_components_dev(data, [0], [len(data)], log2, 6)[0]
    assert check(got)
    assert np.array_equal(got, O.decode_component(data, 0, log2))


@pytest.mark.parametrize("log2_coefs", [6, 4, 2])
def test_entropy_decode_matches_the_oracle_on_random_streams(log2_coefs):
    rng = np.random.default_rng(17 + log2_coefs)
    for log2_blocks in range(5):
        n = 512
        lens = rng.integers(0, 48 * (1 << log2_blocks) + 1, n)
        # Bits biased toward zero so over-long codewords and early ends occur.
        data = bytearray()
        offs = []
        for i in range(n):
            offs.append(len(data))
            raw = rng.integers(0, 256, (2, int(lens[i])), dtype=np.uint8)
            data += (raw[0] & raw[1]).tobytes()
            data += bytes(int(rng.integers(0, 4)))  # vary the 4-byte alignment
        data = bytes(data)
        got = decode_components_dev(data, offs, lens.tolist(), log2_blocks, log2_coefs)
        for i in range(n):
            want = O.decode_component(data[offs[i]: offs[i] + int(lens[i])], offs[i] & 3, log2_blocks, log2_coefs)
            assert np.array_equal(got[i], want), (log2_blocks, i)


def decode_components_events_dev(data: bytes, offs, lens, log2_blocks, log2_coefs, staged):
    """prr_decode_components_events: the frame decode's entropy decoder
    (entropy_events) on raw streams. Returns the dense coefficients and the
    per-stream flags (entry count | bit 30 budget ran out | bit 31 wrapped)."""
    t = torch()
    buf = np.zeros(P._lib.lib().prr_padded_packet_bytes(len(data)), dtype=np.uint8)
    buf[: len(data)] = np.frombuffer(data, dtype=np.uint8)
    d = dev(buf)
    o, ln = dev(np.array(offs, dtype=np.uint32)), dev(np.array(lens, dtype=np.uint32))
    codes = 1 << (log2_blocks + log2_coefs)
    lists = t.full((len(offs) * codes,), -1, dtype=t.int32, device="cuda")
    out = t.full((len(offs) * codes,), 0x5A5A, dtype=t.int16, device="cuda")
    flags = t.zeros(len(offs), dtype=t.int32, device="cuda")
    rc = _lib.lib().prr_decode_components_events(P.context(), d.data_ptr(), o.data_ptr(), ln.data_ptr(), len(offs),
                                                 log2_blocks, log2_coefs, int(staged), lists.data_ptr(),
                                                 out.data_ptr(), flags.data_ptr())
    assert rc == 0
    t.cuda.synchronize()
    return out.cpu().numpy().reshape(len(offs), codes), flags.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("staged", [False, True], ids=["global", "staged"])
@pytest.mark.parametrize("case", _coef_cases(), ids=lambda c: c[0])
def test_coefficient_kats_through_the_frame_entropy_decoder(case, staged):
    # The crate's component KATs (src/coefficients.rs:150-229) on the
    # decoder the frame, reduced and batch decodes run.
    _, data, log2, check = case
    got, flags = decode_components_events_dev(data, [0], [len(data)], log2, 6, staged)
    assert flags[0] >> 30 & 1 == 0  # the symbol budget never runs out
    # A wrapped zero run sets bit 31; with fewer entries than coefficients
    # none was dropped, and the in-order replay is the host's result.
    assert not (flags[0] >> 31 and flags[0] & 0x3FFFFFFF == 64 << log2)
    assert check(got[0])
    assert np.array_equal(got[0], O.decode_component(data, 0, log2))


@pytest.mark.parametrize("staged", [False, True], ids=["global", "staged"])
def test_the_frame_entropy_decoder_flags_a_wrapped_zero_run(staged):
    stream = wrapped_zero_run_stream()
    got, flags = decode_components_events_dev(stream, [0], [len(stream)], 0, 6, staged)
    assert flags[0] >> 31 == 1  # the frame decode replays this stream in order
    # Few enough entries that none was dropped: the in-order replay is exact.
    assert flags[0] & 0x3FFFFFFF < 64
    assert np.array_equal(got[0], O.decode_component(stream, 0, 0))


@pytest.mark.parametrize("staged", [False, True], ids=["global", "staged"])
@pytest.mark.parametrize("log2_coefs", [6, 4, 2])
def test_the_frame_entropy_decoder_matches_the_oracle_on_random_streams(log2_coefs, staged):
    rng = np.random.default_rng(170 + log2_coefs)
    for log2_blocks in range(5):
        n = 384
        lens = rng.integers(0, 48 * (1 << log2_blocks) + 1, n)
        data = bytearray()
        offs = []
        for i in range(n):
            offs.append(len(data))
            raw = rng.integers(0, 256, (2, int(lens[i])), dtype=np.uint8)
            data += (raw[0] & raw[1]).tobytes()
            data += bytes(int(rng.integers(0, 4)))  # vary the 4-byte alignment
        data = bytes(data)
        got, flags = decode_components_events_dev(data, offs, lens.tolist(), log2_blocks, log2_coefs, staged)
        codes = 1 << (log2_blocks + log2_coefs)
        for i in range(n):
            assert flags[i] >> 30 & 1 == 0
            if flags[i] >> 31 and flags[i] & 0x3FFFFFFF == codes:
                continue  # entries may have been dropped; the frame decode decodes it again
            want = O.decode_component(data[offs[i]: offs[i] + int(lens[i])], offs[i] & 3, log2_blocks, log2_coefs)
            assert np.array_equal(got[i], want), (log2_blocks, i)


def assert_frames_equal(pkt, idct=0):
    o = O.decode_frame(pkt, idct)
    g = P.decode_frame_with(pkt, P.Idct(idct))
    assert g.skipped_tiles == o.skipped_tiles
    assert g.max_qscale == o.max_qscale
    gs = g.samples_host()
    assert gs.size == o.samples.size
    mism = np.count_nonzero(gs != o.samples)
    assert mism == 0, f"{mism} of {gs.size} samples differ"
    return o, g


@pytest.mark.parametrize("idct", [0, 1], ids=["apple", "ffmpeg"])
@pytest.mark.parametrize("seed", [1, 11, 23, 31])
def test_decode_matches_the_oracle_on_random_frames(idct, seed):
    rng = S.Rng(seed)
    for spec in S.specs(rng):
        assert_frames_equal(S.random_frame(spec, rng), idct)


def test_a_wrapped_zero_run_overwrites_like_the_host():
    stream = wrapped_zero_run_stream()
    spec = S.Spec(16, 16, alignment=0, valid_tiles=True)
    pkt = S.frame(spec, [S.tile(1, [stream] * 4)])
    assert_frames_equal(pkt)


@pytest.mark.parametrize("seed", [23, 29])
def test_reduced_decode_matches_the_oracle(seed):
    rng = S.Rng(seed)
    for spec in S.specs(rng):
        pkt = S.random_frame(spec, rng)
        for shift in (1, 2, 3):
            for greens in (0, 1):
                o = O.decode_frame_reduced(pkt, shift, greens)
                g = P.decode_frame_reduced_with(pkt, P.Scale(shift), P.Greens(greens))
                assert g.skipped_tiles == o.skipped_tiles and g.max_qscale == o.max_qscale
                assert np.array_equal(g.samples_host(), o.samples), (spec.width, spec.height, shift, greens)


def test_linearize_matches_the_oracle():
    rng = S.Rng(41)
    for spec in S.specs(rng):
        pkt = S.random_frame(spec, rng)
        o, g = assert_frames_equal(pkt)
        assert np.array_equal(g.linearize().cpu().numpy().view(np.uint16), o.linearize())
        host = np.zeros(o.header.width * o.header.height, dtype=np.uint16)
        g.linearize_into(host)
        assert np.array_equal(host, o.linearize())


@pytest.mark.parametrize("w,h", [(5760, 64), (4096, 10), (1000, 38), (1002, 10), (18, 2)])
def test_linearize_packed_and_strided_rows(w, h):
    # Packed rows (width a multiple of 16: one flat pass over 16-byte
    # chunks), rows padded to the coded width, ragged row ends; a custom,
    # curve (version 1).
    curve = [0, 224, 288, 468, 1162, 3339, 9431, 25377]
    pkt = encoded(w, h, pattern=1, alignment=1, qscale=20, sigma=30.0, curve=curve, seed=w + h)
    o, g = assert_frames_equal(pkt)
    assert np.array_equal(g.linearize().cpu().numpy().view(np.uint16), o.linearize())


def develop_compare(pkt, stages=(0, 1, 2), wb=None):
    o = O.decode_frame(pkt)
    g = P.decode_frame(pkt)
    q = o.quantizer
    if wb is None:
        op, gp = O.params_new(o.header, q), P.DemosaicParams.new(g.header, g.quantizer())
    else:
        op = O.params_with_white_balance(o.header, q, *wb)
        gp = P.DemosaicParams.with_white_balance(g.header, g.quantizer(), *wb)
    for stage in stages:
        want = O.develop(o, op, stage, planar=True)
        got = P.develop_planar(g, gp, P.Stage(stage))
        for c in range(3):
            gc = got.planes[c].cpu().numpy()
            assert np.all(np.abs(gc - want[c]) <= DEVELOP_RTOL * np.maximum(1.0, np.abs(want[c])))
            diff = np.count_nonzero(gc.view(np.uint32) != want[c].view(np.uint32))
            assert diff == 0, f"stage {stage} channel {c}: {diff} values differ"
        inter = O.develop(o, op, stage, planar=False)
        got_i = P.develop_with(g, gp, P.Stage(stage)).data.cpu().numpy()
        assert np.array_equal(got_i.view(np.uint32), inter.view(np.uint32))


@pytest.mark.parametrize("seed", [3, 9])
def test_develop_matches_the_oracle_on_random_frames(seed):
    rng = S.Rng(seed)
    for spec in S.specs(rng):
        spec.wb = (1.0 + rng.below(1000) / 500.0, 1.0 + rng.below(1000) / 700.0)
        develop_compare(S.random_frame(spec, rng))


def encoded(w, h, pattern=0, alignment=2, qscale=15, sigma=8.0, specular=0.0, version=1, curve=None,
            qmat=None, white=4095, seed=0, wb=(1.9, 1.4)):
    m = S.mosaic(w, h, pattern, seed=seed, sigma=sigma, specular=specular, white=white)
    spec = S.Spec(w, h, pattern=pattern, alignment=alignment, white_level=white, version=version, curve=curve,
                  quant_matrix=qmat, valid_tiles=True, wb=wb)
    return S.encode(spec, m, qscale=qscale, qscale_seed=seed)


@pytest.mark.parametrize("w,h", [(2, 2), (2, 8), (8, 2), (4, 4), (18, 6), (34, 34), (66, 30), (130, 98),
                                 (250, 66), (512, 96)])
def test_develop_edge_sizes(w, h):
    for pattern in range(4):
        develop_compare(encoded(w, h, pattern=pattern, alignment=pattern % 5, seed=w * h + pattern))


@pytest.mark.parametrize("pattern", range(4))
def test_develop_when_paired_sites_take_different_branches(pattern):
    # Interior tiles compute two sites as the two lanes of f32x2 pairs. A
    # dark, noise-dominated mosaic (many estimates fall back to their mean)
    # with clipped highlights makes the two sites of a pair take different
    # branches often; neither lane's result may change.
    m = S.mosaic(320, 200, pattern, seed=70 + pattern, sigma=40.0, specular=0.05, amp=(2.0, 60.0), white=4095)
    spec = S.Spec(320, 200, pattern=pattern, alignment=2, white_level=4095, valid_tiles=True, wb=(2.4, 1.2))
    pkt = S.encode(spec, m, qscale=(15, 45), qscale_seed=pattern)
    develop_compare(pkt)
    develop_compare(pkt, stages=(1, 2), wb=(0.6, 3.5))


def test_encoded_frames_decode_and_develop_like_the_oracle():
    ident = [0, 8192, 16384, 24576, 32768, 40960, 49152, 57344]
    rng = np.random.default_rng(1)
    cases = [
        dict(w=640, h=352, pattern=0, alignment=2, qscale=15, sigma=8.0),
        dict(w=768, h=320, pattern=3, alignment=4, qscale=45, sigma=24.0, specular=0.02, version=0,
             qmat=[int(v) for v in rng.integers(4, 64, 64)]),
        dict(w=720, h=366, pattern=1, alignment=3, qscale=(15, 45), sigma=16.0, curve=ident),
        dict(w=1920, h=1080, pattern=2, alignment=1, qscale=30),
    ]
    for c in cases:
        pkt = encoded(**c)
        assert_frames_equal(pkt, 0)
        assert_frames_equal(pkt, 1)
        develop_compare(pkt)


def test_corrupted_tiles_are_skipped_like_the_oracle():
    pkt = encoded(1024, 512, pattern=3, alignment=4, qscale=45, sigma=24.0, specular=0.02, version=0)
    bad, tiles = S.corrupt_tiles(pkt, 0.2, seed=5)
    assert len(tiles) > 0
    o, g = assert_frames_equal(bad, 0)
    assert len(o.skipped_tiles) > 0
    assert_frames_equal(bad, 1)
    develop_compare(bad, stages=(1,))


def test_widest_frame():
    # 65534 sensels: 4096 tile columns, the largest width the header allows.
    pkt = encoded(65534, 4, alignment=4, qscale=15)
    assert_frames_equal(pkt)
    develop_compare(pkt, stages=(2,))


def test_async_decode_with_a_device_packet_matches():
    t = torch()
    pkt = encoded(1024, 256, alignment=3)
    info = P.frame_info(pkt)
    L = _lib.lib()
    buf = np.zeros(L.prr_padded_packet_bytes(len(pkt)), dtype=np.uint8)
    buf[: len(pkt)] = np.frombuffer(pkt, dtype=np.uint8)
    dpkt = dev(buf)
    out = t.empty(info.coded_width * info.coded_height, dtype=t.uint16, device="cuda")
    status = t.zeros(4, dtype=t.int32, device="cuda")
    skipped = t.zeros(max(1, info.ntiles), dtype=t.int32, device="cuda")
    nscratch = L.prr_decode_scratch_bytes(C.byref(info))
    scratch = t.empty(nscratch, dtype=t.uint8, device="cuda")
    rc = L.prr_decode_async(P.context(), C.byref(info), dpkt.data_ptr(), 0, out.data_ptr(), status.data_ptr(),
                            skipped.data_ptr(), scratch.data_ptr(), nscratch)
    assert rc == 0
    t.cuda.synchronize()
    st = status.cpu().numpy().view(np.uint32)
    o = O.decode_frame(pkt)
    assert st[0] == 0xFFFFFFFF and st[1] == 0 and st[2] == o.max_qscale and st[3] == 0
    assert np.array_equal(out.cpu().numpy().view(np.uint16), o.samples)
    # A scratch buffer that is too small is refused.
    assert L.prr_decode_async(P.context(), C.byref(info), dpkt.data_ptr(), 0, out.data_ptr(), status.data_ptr(),
                              skipped.data_ptr(), scratch.data_ptr(), 4) == _lib.ERR_BUFFER


def test_host_buffer_develop_matches():
    pkt = encoded(512, 256, pattern=3, alignment=4, qscale=45, sigma=24.0)
    o = O.decode_frame(pkt)
    op = O.params_new(o.header, o.quantizer)
    want = O.develop(o, op, 2, planar=True)
    n = o.header.width * o.header.height
    r, g, b = (np.zeros(n, np.float32) for _ in range(3))
    res = _lib.CDecodeResult()
    err = _lib.CError()
    buf = C.create_string_buffer(pkt, len(pkt))
    rc = _lib.lib().prr_decode_develop_host(P.context(), C.addressof(buf), len(pkt), 0, None, 2, 1,
                                            r.ctypes.data, g.ctypes.data, b.ctypes.data, n, C.byref(res),
                                            C.byref(err))
    assert rc == 0
    for c, plane in enumerate((r, g, b)):
        assert np.array_equal(plane.view(np.uint32), want[c].view(np.uint32))


@pytest.mark.parametrize("ctas", [1, 2, 3])
def test_develop_under_an_occupancy_cap_is_unchanged(ctas):
    # prr_develop_set_occupancy reserves shared memory per CTA so that at
    # most `ctas` develop CTAs share an SM; the output stays the oracle's.
    pkt = encoded(700, 300, pattern=3, alignment=4, qscale=45, sigma=24.0, seed=ctas)
    ctx = P.context()
    assert _lib.lib().prr_develop_set_occupancy(ctx, ctas) == 0
    try:
        develop_compare(pkt, stages=(2,))
    finally:
        assert _lib.lib().prr_develop_set_occupancy(ctx, 0) == 0
    assert _lib.lib().prr_develop_set_occupancy(ctx, 17) == _lib.ERR_INVALID


def test_a_c_program_decodes_and_develops_like_the_oracle(tmp_path):
    # tests/c_abi/decode_develop.c: parse, params and prr_decode_develop_host
    # from C, malloc'ed host buffers, no Python or torch in the process.
    import os
    import shutil
    import subprocess

    from proresraw_rs_b200 import _lib

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    prog = str(tmp_path / "decode_develop")
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "c_abi", "decode_develop.c"), "-o", prog, "-L", lib_dir, "-lprr",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    pkt = encoded(640, 352, pattern=3, alignment=4, qscale=45, sigma=24.0, specular=0.02, version=0, seed=77)
    pkt, bad = S.corrupt_tiles(pkt, 0.05, seed=7)
    (tmp_path / "frame.prr").write_bytes(pkt)
    res = subprocess.run([prog, str(tmp_path / "frame.prr"), str(tmp_path / "planes.f32")], check=True,
                         capture_output=True, text=True)
    got = dict(line.split("=", 1) for line in res.stdout.splitlines())
    o = O.decode_frame(pkt)
    assert int(got["max_qscale"]) == o.max_qscale
    assert [int(v) for v in got["skipped"].split(",") if v] == list(o.skipped_tiles)
    want = O.develop(o, O.params_new(o.header, o.quantizer), 2, planar=True)
    planes = np.fromfile(tmp_path / "planes.f32", dtype=np.float32).reshape(3, -1)
    for c in range(3):
        assert np.array_equal(planes[c].view(np.uint32), want[c].view(np.uint32)), c
