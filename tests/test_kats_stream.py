"""Known-answer tests of the bit reader, codebooks, entropy decoder and
inverse transforms, ported from the crate's unit tests (src/bits.rs:188-269,
src/codebook.rs:112-165, src/coefficients.rs:148-229, src/idct.rs:462-594,
src/gpu.rs:1407-1464) and pinned to its golden data
(tests/data/idct_vectors.bin, tests/data/idct_hash.txt).

Each test runs on the CPU oracle; the `gpu`-marked twins run the same
inputs through the CUDA library's entry points.
"""

import math
import os
import re

import numpy as np
import pytest

import _oracle as O
from proresraw_rs_b200 import synth as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

FIRST_DC, DC_RESET, AC_INITIAL, RN_INITIAL, LN_INITIAL = 0x2BC, 0x064, 0x031, 0x000, 0x042
DC_CB = [0x010, 0x021, 0x032, 0x033, 0x033, 0x033, 0x044, 0x044, 0x044, 0x044, 0x044, 0x044, 0x076]
LN_CB = [0x100, 0x111, 0x222, 0x222, 0x122, 0x122, 0x433, 0x433] + [0x233] * 6 + [0x033]
SCAN = [0, 8, 1, 9, 16, 24, 17, 25, 2, 10, 3, 11, 18, 26, 19, 27, 32, 40, 33, 34, 41, 48, 56, 49, 42,
        35, 43, 50, 57, 58, 51, 59, 4, 12, 5, 6, 13, 20, 28, 21, 14, 7, 15, 22, 29, 36, 44, 37, 30, 23,
        31, 38, 45, 52, 60, 53, 46, 39, 47, 54, 61, 62, 55, 63]


def ac_cb(i):
    runs = [(1, 0x000), (1, 0x211), (2, 0x111), (3, 0x222), (3, 0x122), (8, 0x233), (2, 0x133),
            (22, 0x244), (52, 0x355), (1, 0x166)]
    t = [v for n, v in runs for _ in range(n)]
    return t[min(i, 94)]


def read(data, align, cbs):
    return O.read_symbols(data, align, cbs)


# --- src/bits.rs ---------------------------------------------------------------

def test_rice_codewords():
    assert read(bytes([0b1110_1100]), 0, [0x132, 0x132]) == [0b11, 4 + 0b10]


def test_exp_golomb_codewords():
    assert read(bytes([0b0110_1000]), 0, [0x031]) == [0b01101 + 2 - 8]


def test_round_trips_through_the_test_encoder_at_every_alignment():
    cbs = [0x2BC, 0x064, 0x031, 0x000, 0x433]
    values = [0, 1, 2, 3, 7, 8, 15, 16, 100, 1000, 4095, 65535]
    expected = []
    w = S.BitWriter()
    for cb in cbs:
        for v in values:
            probe = S.BitWriter()
            probe.symbol(cb, v)
            # Only codewords that fit the 32-bit view are valid.
            if _cw_len(cb, v) <= 32:
                w.symbol(cb, v)
                expected.append((cb, v))
    w.put(1, 1)
    data = w.finish()
    for align in range(4):
        got = read(data, align, [cb for cb, _ in expected])
        assert got == [v for _, v in expected], align


def _cw_len(cb, v):
    s, e, r = cb >> 8, (cb >> 4) & 15, cb & 15
    q = v >> r
    if q <= s:
        return q + 1 + r
    m = v - ((s + 1) << r) + (1 << e)
    bits = m.bit_length()
    return s + 1 + (bits - 1 - e) + bits


def test_ends_on_zero_window_and_past_the_end():
    assert read(bytes([0, 0, 0, 0, 0x80]), 0, [0]) == []
    assert read(bytes([0b1000_0000]), 0, [0, 0]) == [0]
    assert read(b"", 3, [0]) == []


def test_overlong_codeword_shifts_wrap():
    p = 1 << 11
    assert O.codeword(p, 0) == ((1 + (p >> 24) - 1) & 0xFFFFFFFF, 40)


# --- src/codebook.rs (the device tables, read from their source) ---------------

def _device_tables():
    src = open(os.path.join(os.path.dirname(__file__), "..", "proresraw_rs_b200", "csrc",
                            "device_common.cuh")).read()
    body = src[src.index("__constant__ CodeTables c_tables"):]
    groups = re.findall(r"\{([^{}]*)\}", body[: body.index("};")])
    return [[int(x, 0) for x in g.replace("\n", " ").split(",") if x.strip()] for g in groups]


def test_codebook_tables_match_the_format():
    ac, rn, ln, dc, scan, scan4, scan2 = _device_tables()[:7]
    assert ac[:95] == [ac_cb(i) for i in range(95)]
    assert (ac[0], ac[9], ac[10], ac[19], ac[20], ac[41], ac[42], ac[93], ac[94]) == (
        0, 0x122, 0x233, 0x133, 0x244, 0x244, 0x355, 0x355, 0x166)
    assert rn == [0x200, 0x100, 0x000, 0x000, 0x211, 0x211, 0x111, 0x111, 0x011, 0x011, 0x021, 0x021, 0x222]\
        + [0x022] * 12 + [0x032, 0x032, 0x044]
    assert ln[:15] == LN_CB
    assert dc[:13] == DC_CB
    assert scan == SCAN and sorted(scan) == list(range(64))
    # The reduced scans are the full scan's leading corners (src/codebook.rs:149-165).
    assert scan4 == [SCAN[n] // 8 * 4 + SCAN[n] % 8 for n in range(16)]
    assert scan2 == [SCAN[n] // 8 * 2 + SCAN[n] % 8 for n in range(4)]
    # Unpacked parameters (src/codebook.rs:116-134).
    assert (FIRST_DC >> 8, (FIRST_DC >> 4) & 15, FIRST_DC & 15) == (2, 11, 12)
    assert (LN_CB[6] >> 8, (LN_CB[6] >> 4) & 15, LN_CB[6] & 15) == (4, 3, 3)


# --- src/coefficients.rs --------------------------------------------------------

def _coef_cases():
    """(name, stream, log2_blocks, check(coefs)) of the crate's coefficient tests."""
    cases = []
    cases.append(("empty", b"", 2, lambda c: np.all(c == 0)))

    w = S.BitWriter()
    w.symbol(FIRST_DC, 5)
    w.symbol(DC_RESET, 3)
    cases.append(("dc_running_sign", w.finish(), 1, lambda c: c[0] == -3 and c[64] == -5))

    w = S.BitWriter()
    w.symbol(FIRST_DC, 0)
    w.symbol(DC_RESET, 1)
    w.symbol(DC_CB[1], 2)
    w.symbol(DC_CB[1], 0)
    w.symbol(DC_CB[0], 2)
    cases.append(("dc_sign_persists", w.finish(), 3,
                  lambda c: [int(c[b * 64]) for b in range(5)] == [0, -1, -2, -2, -1]))

    w = S.BitWriter()
    w.symbol(FIRST_DC, 0)
    w.symbol(LN_INITIAL, 2)
    w.symbol(AC_INITIAL, 0)
    w.put(0, 1)
    w.symbol(ac_cb(0), 2)
    w.put(1, 1)
    w.symbol(RN_INITIAL, 0)
    w.symbol(ac_cb(2), 1)
    w.put(0, 1)
    cases.append(("ac_runs", w.finish(), 0,
                  lambda c: (c[SCAN[1]], c[SCAN[2]], c[SCAN[3]], c[SCAN[4]]) == (1, -3, 0, 2)
                  and np.count_nonzero(c) == 3))

    w = S.BitWriter()
    w.symbol(FIRST_DC, 0)
    w.symbol(DC_RESET, 0)
    w.symbol(LN_INITIAL, 2)
    w.symbol(AC_INITIAL, 4)
    w.put(0, 1)
    w.symbol(ac_cb(4), 6)
    w.put(0, 1)
    cases.append(("interleave", w.finish(), 1, lambda c: c[SCAN[1]] == 5 and c[64 + SCAN[1]] == 7))

    cases.append(("wrapped_zero_run", wrapped_zero_run_stream(), 0, lambda c: c[SCAN[13]] == 2))
    return cases


def wrapped_zero_run_stream():
    """A zero run that wraps the scan position back over a stored
    coefficient (src/gpu.rs:1410-1436): the later store wins."""
    w = S.BitWriter()
    w.symbol(FIRST_DC, 0)
    w.symbol(LN_INITIAL, 1)
    w.symbol(AC_INITIAL, 0)
    w.put(0, 1)
    w.symbol(RN_INITIAL, 10)
    w.symbol(ac_cb(0), 0)
    w.put(0, 1)
    w.symbol(LN_CB[0], 0)
    w.put(0, 16)
    w.put(1, 1)
    w.put(0, 17)
    w.put(0b0100, 4)
    w.put(0xFFFFFFFF, 32)
    return w.finish()


@pytest.mark.parametrize("case", _coef_cases(), ids=lambda c: c[0])
def test_coefficient_kats_oracle(case):
    _, data, log2, check = case
    assert check(O.decode_component(data, 0, log2))


# --- src/idct.rs ----------------------------------------------------------------

def golden_records():
    d = np.fromfile(os.path.join(GOLDEN, "idct_vectors.bin"), dtype=np.uint8).reshape(-1, 384)
    c = d[:, :128].copy().view(np.int16)
    q = d[:, 128:256].copy().view(np.int16)
    want = d[:, 256:].copy().view(np.uint16)
    return c, q, want


def golden_hash():
    return int(open(os.path.join(GOLDEN, "idct_hash.txt")).read().strip(), 16)


def test_apple_matches_reference_vectors_oracle():
    c, q, want = golden_records()
    assert c.shape[0] == 512
    assert np.array_equal(O.transform_blocks(0, c, q), want)


def test_apple_matches_reference_hash_oracle():
    g = S.Gen(0x4A54)
    h = S.FNV_OFFSET
    for _ in range(16):
        c, q = g.blocks(1 << 16)
        h = S.fnv1a_u16(h, O.transform_blocks(0, c, q))
    assert h == golden_hash()


ONES = np.ones(64, dtype=np.int16)


def float_reference(coefs):
    """The orthonormal 2-D IDCT scaled like the integer one (src/idct.rs:469-493)."""
    u = np.arange(8)
    cu = np.where(u == 0, 1 / math.sqrt(2), 1.0)
    basis = np.cos(np.outer(2 * np.arange(8) + 1, u) * math.pi / 16) * cu  # [x, u]
    C = np.asarray(coefs, dtype=np.float64).reshape(8, 8)  # [v, u]
    # out[y][x] = 2 * sum_{v,u} basis[y, v] C[v, u] basis[x, u] + 32768
    return (basis @ C @ basis.T).reshape(-1) * 2.0 + 32768.0


def random_blocks(n):
    seed = 12345
    out = []
    for _ in range(n):
        b = []
        for _ in range(64):
            seed = (seed * 1664525 + 1013904223) & 0xFFFFFFFF
            b.append(((seed >> 16) % 2001) - 1000)
        out.append(b)
    return np.array(out, dtype=np.int16)


def test_dc_only_block_is_flat_oracle():
    for kind in ("apple", "ffmpeg"):
        for dc in [-32768, -5000, -1, 0, 1, 800, 32767]:
            b = np.zeros(64, dtype=np.int16)
            b[0] = dc
            assert np.all(O.block(kind, b, ONES).astype(np.int64) == dc + 32768), (kind, dc)


def test_both_transforms_match_the_float_reference_closely_oracle():
    for b in random_blocks(50):
        want = float_reference(b)
        for kind, tol in (("apple", 3.0), ("ffmpeg", 2.0)):
            got = O.block(kind, b, ONES).astype(np.float64)
            assert np.max(np.abs(got - want)) <= tol, kind


def test_dequantizes_with_saturation_oracle():
    b = np.zeros(64, dtype=np.int16)
    b[0] = 3000
    q = ONES.copy()
    q[0] = 20
    sat = np.zeros(64, dtype=np.int16)
    sat[0] = 32767
    for kind in ("apple", "ffmpeg"):
        assert np.array_equal(O.block(kind, b, q), O.block(kind, sat, ONES))
    assert O.lib().orc_dequantize(-32768, -1) == 32767
    assert O.lib().orc_dequantize(-300, 300) == -32768


def test_code_values_are_centered_and_clamped_oracle():
    cv = O.lib().orc_code_value
    assert [cv(0), cv(-32768), cv(-40000), cv(32767), cv(40000)] == [32768, 0, 0, 65535, 65535]
    oc = O.lib().orc_output_code
    assert [oc(-0.9), oc(32768.5), oc(70000.0), oc(float("nan"))] == [0, 32768, 65535, 65535]
