"""prr_decode_noalloc: the decode for callers that may not allocate device
memory while they decode (plug-ins handed only their input and output
buffers by a host application that owns the device memory, real-time loops
in which a cudaMalloc would stall the device or fail against an allocator
that reserved the memory up front).

The entry point keeps its one scratch table in a fixed array inside the
library. Its output must equal the regular decode's bit for bit, on two
calls in a row (the second call reuses the array the first one filled).
This file is named to run last; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib
from proresraw_rs_b200 import synth as S

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


def _noalloc(pkt, idct, dev_packet):
    import torch

    L = _lib.lib()
    info = P.frame_info(pkt)
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
