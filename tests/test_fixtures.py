"""Comparison with FFmpeg's `prores_raw` decoder on real footage, as the
crate's fixture harness does (tests/oracle.rs:1-162).

Fixtures are not part of the repository. Set PRORES_RAW_FIXTURES to a
directory of `NAME.bin` frame packets, each with `NAME.raw` (FFmpeg's
`bayer_rggb16le` output: visible size, linearized, little-endian u16) when
FFmpeg could decode it; the tests are skipped when the variable is unset.
FFmpeg uses its simple IDCT, so the comparison runs Idct::Ffmpeg. Packets
without a `.raw` are only compared across this library's decoders and the
CPU oracle. A self-check of the harness on a synthetic fixture directory
(references written by the oracle) runs without fixtures.
"""

import os

import numpy as np
import pytest

import _oracle as O
from proresraw_rs_b200 import synth as S

FIXTURES = os.environ.get("PRORES_RAW_FIXTURES")
needs_fixtures = pytest.mark.skipif(not FIXTURES, reason="PRORES_RAW_FIXTURES not set")


def packets(d):
    """The `.bin` packets of the fixture directory, sorted."""
    out = sorted(os.path.join(d, n) for n in os.listdir(d) if n.endswith(".bin"))
    assert out, f"no .bin fixtures in {d}"
    return out


def ffmpeg_reference(path):
    raw = os.path.splitext(path)[0] + ".raw"
    if not os.path.exists(raw):
        return None
    return np.frombuffer(open(raw, "rb").read(), dtype="<u2")


def compare_linearized(d, decode_linearized):
    """Every packet with an FFmpeg reference: decode with the FFmpeg
    transform, linearize, compare sensel for sensel. Returns the number of
    packets compared (at least one is required)."""
    compared = 0
    for p in packets(d):
        want = ffmpeg_reference(p)
        if want is None:
            continue
        compared += 1
        got = decode_linearized(open(p, "rb").read())
        assert want.size == got.size, f"{p}: reference size"
        mism = int(np.count_nonzero(got != want))
        assert mism == 0, f"{p}: {mism} sensels differ"
    assert compared > 0, "no fixture has an FFmpeg reference"
    return compared


def oracle_linearized(pkt):
    return O.decode_frame(pkt, 1).linearize()


def gpu_linearized(pkt):
    import proresraw_rs_b200 as P

    f = P.decode_frame_with(pkt, P.Idct.FFMPEG)
    out = np.zeros(f.width() * f.height(), dtype=np.uint16)
    f.linearize_into(out)
    return out


def test_the_harness_on_a_synthetic_fixture_directory(tmp_path):
    # Two packets with references (written here by the oracle's FFmpeg
    # transform) and one without; a planted one-sensel error must be caught.
    for k, (w, h, pat) in enumerate(((256, 96, S.RGGB), (176, 64, S.BGGR), (64, 32, S.RGGB))):
        m = S.mosaic(w, h, pat, seed=40 + k, sigma=12.0)
        spec = S.Spec(w, h, pattern=pat, alignment=2, white_level=4095, version=1, valid_tiles=True)
        pkt = S.encode(spec, m, qscale=20, qscale_seed=k)
        (tmp_path / f"f{k}.bin").write_bytes(pkt)
        if k < 2:
            (tmp_path / f"f{k}.raw").write_bytes(oracle_linearized(pkt).astype("<u2").tobytes())
    assert compare_linearized(str(tmp_path), oracle_linearized) == 2
    ref = np.frombuffer((tmp_path / "f0.raw").read_bytes(), dtype="<u2").copy()
    ref[17] ^= 1
    (tmp_path / "f0.raw").write_bytes(ref.tobytes())
    with pytest.raises(AssertionError, match="1 sensels differ"):
        compare_linearized(str(tmp_path), oracle_linearized)


@needs_fixtures
def test_the_oracle_matches_ffmpeg_linearized_output():
    compare_linearized(FIXTURES, oracle_linearized)


@needs_fixtures
@pytest.mark.gpu
def test_the_gpu_matches_ffmpeg_linearized_output():
    compare_linearized(FIXTURES, gpu_linearized)


@needs_fixtures
@pytest.mark.gpu
def test_the_gpu_decode_matches_the_oracle_on_every_fixture():
    # tests/oracle.rs:69-104: both transforms, every packet.
    import proresraw_rs_b200 as P

    for p in packets(FIXTURES):
        pkt = open(p, "rb").read()
        for idct in (0, 1):
            want = O.decode_frame(pkt, idct)
            got = P.decode_frame_with(pkt, P.Idct(idct))
            assert got.skipped_tiles == want.skipped_tiles and got.max_qscale == want.max_qscale
            mism = int(np.count_nonzero(got.samples_host() != want.samples))
            assert mism == 0, f"{p} idct {idct}: {mism} sensels differ"


@needs_fixtures
@pytest.mark.gpu
def test_the_gpu_develop_matches_the_oracle_on_every_fixture():
    # tests/oracle.rs:106-162: every stage, planar, bit for bit.
    import proresraw_rs_b200 as P

    for p in packets(FIXTURES):
        pkt = open(p, "rb").read()
        o = O.decode_frame(pkt, 0)
        g = P.decode_frame(pkt)
        prm = P.DemosaicParams.new(g.header, g.quantizer())
        for stage in (0, 1, 2):
            want = O.develop(o, O.params_new(o.header, o.quantizer), stage, planar=True)
            got = P.develop_planar(g, prm, P.Stage(stage))
            for c in range(3):
                gc = got.planes[c].cpu().numpy().view(np.uint32)
                mism = int(np.count_nonzero(gc != want[c].view(np.uint32)))
                assert mism == 0, f"{p} stage {stage} plane {c}: {mism} values differ"
