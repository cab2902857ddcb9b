"""prr_decode_noalloc: the decode for callers that may not allocate device
memory while they decode (plug-ins handed only their input and output
buffers by a host application that owns the device memory, real-time loops
in which a cudaMalloc would stall the device or fail against an allocator
that reserved the memory up front).

The entry point keeps its one scratch table in a fixed array inside the
library. Its output must equal the regular decode's bit for bit, on two
calls in a row (the second call reuses the array the first one filled), and
the CPU oracle's on the adversarial corpora: the crate's random specs and
random-byte frames, the wrapped zero run, the 5760x3040 hard bitstream.
A call allocates no device memory and leaves the caller's current device
as it found it. This file is named to run last; it also passes alone in a
fresh process.
"""

import ctypes as C

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib
from proresraw_rs_b200 import synth as S
from test_kats_stream import wrapped_zero_run_stream

pytestmark = pytest.mark.gpu


def _frame(w, h, seed, alignment, corrupt):
    m = S.mosaic(w, h, S.BGGR, seed=seed, sigma=24.0, specular=0.02)
    qm = [int(v) for v in np.random.default_rng(seed).integers(4, 64, 64)]
    spec = S.Spec(w, h, pattern=S.BGGR, alignment=alignment, white_level=4095, version=0, valid_tiles=True,
                  quant_matrix=qm)
    pkt = S.encode(spec, m, qscale=45, qscale_seed=seed)
    pkt, _ = S.corrupt_tiles(pkt, corrupt, seed=seed)
    return pkt


def _regular(pkt, idct):
    """The existing entry point (prr_decode_async with caller scratch)."""
    import torch

    L = _lib.lib()
    info = P.frame_info(pkt)
    buf = torch.zeros(L.prr_padded_packet_bytes(len(pkt)), dtype=torch.uint8, device="cuda")
    buf[: len(pkt)].copy_(torch.frombuffer(bytearray(pkt), dtype=torch.uint8))
    out = torch.empty(info.coded_width * info.coded_height, dtype=torch.uint16, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    sk = torch.zeros(max(1, info.ntiles), dtype=torch.int32, device="cuda")
    nscr = L.prr_decode_scratch_bytes(C.byref(info))
    scr = torch.empty(nscr, dtype=torch.uint8, device="cuda")
    assert L.prr_decode_async(P.context(), C.byref(info), buf.data_ptr(), idct, out.data_ptr(), st.data_ptr(),
                              sk.data_ptr(), scr.data_ptr(), nscr) == 0
    torch.cuda.synchronize()
    s = st.cpu().numpy().view(np.uint32)
    return out.cpu().numpy().view(np.uint16), s, sorted(sk.cpu().numpy().view(np.uint32)[: s[1]].tolist()), buf


def _upload(pkt):
    import torch

    buf = torch.zeros(_lib.lib().prr_padded_packet_bytes(len(pkt)), dtype=torch.uint8, device="cuda")
    buf[: len(pkt)].copy_(torch.frombuffer(bytearray(pkt), dtype=torch.uint8))
    return buf


def _noalloc(pkt, idct, dev_packet, info=None):
    import torch

    L = _lib.lib()
    info = P.frame_info(pkt) if info is None else info
    out = torch.empty(info.coded_width * info.coded_height, dtype=torch.uint16, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    sk = torch.zeros(max(1, info.ntiles), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.prr_decode_noalloc(torch.cuda.current_device(), C.c_void_p(stream or 1), C.byref(info),
                              dev_packet.data_ptr(), idct, out.data_ptr(), st.data_ptr(), sk.data_ptr())
    assert rc == 0, L.prr_status_string(rc)
    torch.cuda.synchronize()
    s = st.cpu().numpy().view(np.uint32)
    return out.cpu().numpy().view(np.uint16), s, sorted(sk.cpu().numpy().view(np.uint32)[: s[1]].tolist())


@pytest.mark.parametrize("idct", [0, 1], ids=["apple", "ffmpeg"])
def test_noalloc_decode_equals_the_regular_decode_twice_in_a_row(idct):
    frames = [_frame(1024, 512, 3, 4, 0.05), _frame(640, 360, 4, 2, 0.05)]
    for pkt in frames:  # two calls in a row, the second one on another frame
        want, wst, wsk, dev_packet = _regular(pkt, idct)
        got, gst, gsk = _noalloc(pkt, idct, dev_packet)
        assert np.array_equal(got, want)
        assert list(gst) == list(wst) and gsk == wsk
    # And the same frame twice: the array keeps the last call's table.
    want, wst, wsk, dev_packet = _regular(frames[0], idct)
    for _ in range(2):
        got, gst, gsk = _noalloc(frames[0], idct, dev_packet)
        assert np.array_equal(got, want) and list(gst) == list(wst) and gsk == wsk


def test_noalloc_rejects_frames_beyond_its_scratch():
    import torch

    pkt = _frame(256, 64, 5, 0, 0.0)
    info = P.frame_info(pkt)
    info.ntiles = _lib.NOALLOC_MAX_TILES + 1
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    rc = _lib.lib().prr_decode_noalloc(torch.cuda.current_device(), None, C.byref(info), dummy.data_ptr(), 0,
                                       dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr())
    assert rc == _lib.ERR_SCRATCH_LIMIT


NO_TILE = 0xFFFFFFFF


def _against_the_oracle(pkt, idct):
    """One frame through prr_decode_noalloc, compared with the oracle's
    decode_frame_with: the same error, or the same samples, skipped tiles
    and max_qscale (src/decoder.rs:221-267)."""
    try:
        want = O.decode_frame(pkt, idct)
    except O.OracleError as e:
        want = e
    try:
        info = P.frame_info(pkt)
    except P.Error as e:
        assert isinstance(want, O.OracleError) and want.code == e.code, (e, want)
        return "host error"
    got, st, sk = _noalloc(pkt, idct, _upload(pkt), info)
    assert st[3] == 0, "a bounded device loop gave up"
    if st[0] != NO_TILE:
        assert isinstance(want, O.OracleError) and want.code == _lib.ERR_TILE_OUT_OF_BOUNDS, want
        assert want.err.index == st[0]
        return "tile out of bounds"
    assert not isinstance(want, O.OracleError), f"oracle error {want.code}, the decode succeeded"
    assert sk == want.skipped_tiles and st[2] == want.max_qscale
    assert np.array_equal(got, want.samples), f"{np.count_nonzero(got != want.samples)} samples differ"
    return "decoded"


@pytest.mark.parametrize("idct", [0, 1], ids=["apple", "ffmpeg"])
@pytest.mark.parametrize("seed", [1, 11, 23, 31])
def test_noalloc_matches_the_oracle_on_random_frames(idct, seed):
    # The crate's random specs and random-byte tile payloads
    # (src/synth.rs:154-221): malformed streams, invalid tile headers,
    # tiles past the packet end.
    rng = S.Rng(seed)
    seen = {}
    for spec in S.specs(rng):
        kind = _against_the_oracle(S.random_frame(spec, rng), idct)
        seen[kind] = seen.get(kind, 0) + 1
    assert seen.get("decoded", 0) > 0


@pytest.mark.parametrize("idct", [0, 1], ids=["apple", "ffmpeg"])
def test_noalloc_overwrites_on_a_wrapped_zero_run_like_the_host(idct):
    # A zero run that wraps the scan position back over a stored
    # coefficient: the later store wins (src/coefficients.rs:112-145).
    stream = wrapped_zero_run_stream()
    for w, h in ((16, 16), (64, 32)):
        spec = S.Spec(w, h, alignment=0, valid_tiles=True)
        pkt = S.frame(spec, [S.tile(1, [stream] * 4)] * S.ntiles(w, h, 0))
        assert _against_the_oracle(pkt, idct) == "decoded"


def _frame_5k8():
    # 5760x3040 BGGR, bitstream version 0, alignment 4 with partial edge
    # tiles, qscale 45, quantization matrix uniform in [4, 63], noise sigma
    # 24, 2 % specular white, 0.5 % of tiles corrupted.
    qmat = [int(v) for v in np.random.default_rng(1).integers(4, 64, 64)]
    m = S.mosaic(5760, 3040, S.BGGR, seed=100, sigma=24.0, specular=0.02, white=4095)
    spec = S.Spec(5760, 3040, pattern=S.BGGR, alignment=4, quant_matrix=qmat, white_level=4095, version=0,
                  wb=(1.82, 1.41), valid_tiles=True)
    pkt = S.encode(spec, m, qscale=45, qscale_seed=0)
    pkt, bad = S.corrupt_tiles(pkt, 0.005, seed=1000)
    assert len(bad) > 0
    return pkt


def test_noalloc_matches_the_oracle_on_the_5k8_hard_bitstream():
    pkt = _frame_5k8()
    for idct in (0, 1):
        assert _against_the_oracle(pkt, idct) == "decoded"


def test_noalloc_allocates_no_device_memory():
    import torch

    pkt = _frame(1024, 512, 6, 4, 0.05)
    info = P.frame_info(pkt)
    dev_packet = _upload(pkt)
    want = _noalloc(pkt, 0, dev_packet, info)  # loads the kernels, looks up the array
    torch.cuda.synchronize()
    free0, reserved0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
    L = _lib.lib()
    out = torch.empty(info.coded_width * info.coded_height, dtype=torch.uint16, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    sk = torch.zeros(max(1, info.ntiles), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free1, reserved1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
    stream = torch.cuda.current_stream().cuda_stream
    assert L.prr_decode_noalloc(torch.cuda.current_device(), C.c_void_p(stream or 1), C.byref(info),
                                dev_packet.data_ptr(), 0, out.data_ptr(), st.data_ptr(), sk.data_ptr()) == 0
    torch.cuda.synchronize()
    # The caching allocator may have grown for the output tensors above;
    # the call itself must change neither figure.
    assert torch.cuda.mem_get_info()[0] == free1 and torch.cuda.memory_reserved() == reserved1
    assert reserved1 >= reserved0 and free1 <= free0
    assert np.array_equal(out.cpu().numpy().view(np.uint16), want[0])


def test_noalloc_leaves_the_callers_current_device():
    import torch

    pkt = _frame(256, 64, 7, 0, 0.0)
    info = P.frame_info(pkt)
    L = _lib.lib()
    n = torch.cuda.device_count()
    dev_packet = _upload(pkt)
    out = torch.empty(info.coded_width * info.coded_height, dtype=torch.uint16, device="cuda:0")
    st = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    sk = torch.zeros(max(1, info.ntiles), dtype=torch.int32, device="cuda:0")
    args = (C.byref(info), dev_packet.data_ptr(), 0, out.data_ptr(), st.data_ptr(), sk.data_ptr())
    torch.cuda.synchronize()
    if n > 1:
        # Device 1 current, the decode on device 0: device 1 stays current.
        torch.cuda.set_device(1)
        try:
            assert L.prr_decode_noalloc(0, None, *args) == 0
            assert torch.cuda.current_device() == 1
        finally:
            torch.cuda.set_device(0)
    assert L.prr_decode_noalloc(0, None, *args) == 0
    assert torch.cuda.current_device() == 0
    # A device that does not exist: a CUDA error, and device 0 still current.
    assert L.prr_decode_noalloc(n, None, *args) == _lib.ERR_CUDA
    assert torch.cuda.current_device() == 0
    torch.cuda.synchronize()
