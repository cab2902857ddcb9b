"""The C-ABI libraries load and export what their headers declare (no GPU
needed: only loading and host-side entry points are exercised)."""

import ctypes as C
import os
import re

import pytest

import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:prr|prs)_\w+)\s*\(", src)))


def test_libprr_exports_every_declared_symbol():
    names = declared("prr.h")
    assert len(names) >= 25
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_libprr_synth_exports_every_declared_symbol():
    names = declared("prr_synth.h")
    lib = C.CDLL(os.path.join(ROOT, "proresraw_rs_b200", "lib", "libprr_synth.so"))
    assert [n for n in names if not hasattr(lib, n)] == []


def test_status_strings_and_padding():
    L = _lib.lib()
    assert L.prr_status_string(0) == b"ok"
    assert L.prr_status_string(-11) == b"tile out of bounds"
    assert L.prr_padded_packet_bytes(1) >= 17
    assert L.prr_padded_packet_bytes(100) % 16 == 0


def test_scratch_size_covers_the_tile_offsets():
    from proresraw_rs_b200 import synth as S

    pkt = S.frame(S.Spec(5760, 64, alignment=4), [S.tile(1, [b"\x80"] * 4)] * S.ntiles(5760, 64, 4))
    info = P.frame_info(pkt)
    assert _lib.lib().prr_decode_scratch_bytes(C.byref(info)) >= 4 * (info.ntiles + 1)


def test_the_library_refuses_to_run_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(RuntimeError):
        P.context()


def test_clip_calls_refuse_a_null_pipeline():
    # Host-side argument checks of the clip pipeline (no device touched).
    L = _lib.lib()
    assert L.prr_clip_start(None, 0, 1, _lib.SCALE_FULL, 0, 0) == _lib.ERR_INVALID
    assert L.prr_clip_queue(None, 0, 1, _lib.SCALE_FULL, 0, 0) == _lib.ERR_INVALID
    assert L.prr_clip_next(None, None) == _lib.ERR_INVALID


def test_noalloc_refuses_device_ordinals_out_of_range_before_any_cuda_call():
    # prr_decode_noalloc checks its arguments before it touches CUDA, so a
    # device ordinal outside [0, 64) is refused even without a device.
    L = _lib.lib()
    info = _lib.CFrameInfo()
    p = C.c_void_p(16)  # never dereferenced: the call returns first
    for device in (-1, 64, 1 << 20):
        assert L.prr_decode_noalloc(device, None, C.byref(info), p, 0, p, p, p) == _lib.ERR_INVALID
    info.ntiles = _lib.NOALLOC_MAX_TILES + 1
    assert L.prr_decode_noalloc(0, None, C.byref(info), p, 0, p, p, p) == _lib.ERR_SCRATCH_LIMIT


def test_develop_buckets_group_frame_sizes_by_power_of_two():
    L = _lib.lib()
    assert L.prr_develop_bucket(5760, 3040) == (13 << 8) | 12
    assert L.prr_develop_bucket(4096, 2160) == (12 << 8) | 12
    assert L.prr_develop_bucket(4097, 2048) == (13 << 8) | 11
    assert L.prr_develop_set_config(None, 0, None) == _lib.ERR_INVALID
