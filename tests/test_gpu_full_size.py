"""Parity at the full sizes of the benchmark configurations, against the
CPU oracle (threaded, well under a second a frame):

- a 4096x2160 RGGB frame (bitstream version 1, tile alignment 2, qscale 15,
  default quantization matrix, identity curve, noise sigma 8): decode
  bit-exact, develop to white-balanced RGB bit-exact;
- the 5760x3040 hard bitstream (BGGR, version 0, alignment 4 with partial
  edge tiles, qscale 45, quantization matrix uniform in [4, 63], noise sigma
  24, 2 % specular white, 0.5 % of tiles corrupted): both transforms
  bit-exact with identical skipped-tile lists, every reduced scale and
  greens mode bit-exact, develop to Rec.2020 bit-exact;
- the 64-frame mixed batch (HD to 8K, both versions and patterns, half
  reduced) in one persistent launch: every frame as the oracle decodes it.
"""

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import synth as S

pytestmark = pytest.mark.gpu

IDENTITY_CURVE = [0, 8192, 16384, 24576, 32768, 40960, 49152, 57344]


@pytest.fixture(scope="module")
def frame_4k():
    m = S.mosaic(4096, 2160, S.RGGB, seed=0, sigma=8.0, white=4095)
    spec = S.Spec(4096, 2160, pattern=S.RGGB, alignment=2, white_level=4095, version=1, curve=IDENTITY_CURVE,
                  valid_tiles=True, wb=(1.9, 1.4))
    return S.encode(spec, m, qscale=15, qscale_seed=0)


@pytest.fixture(scope="module")
def frame_5k8():
    rng = np.random.default_rng(1)
    qmat = [int(v) for v in rng.integers(4, 64, 64)]
    m = S.mosaic(5760, 3040, S.BGGR, seed=100, sigma=24.0, specular=0.02, white=4095)
    spec = S.Spec(5760, 3040, pattern=S.BGGR, alignment=4, quant_matrix=qmat, white_level=4095, version=0,
                  wb=(1.82, 1.41), valid_tiles=True,
                  color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
    pkt = S.encode(spec, m, qscale=45, qscale_seed=0)
    pkt, bad = S.corrupt_tiles(pkt, 0.005, seed=1000)
    assert len(bad) > 0
    return pkt


def decode_equal(pkt, idct):
    o = O.decode_frame(pkt, idct)
    g = P.decode_frame_with(pkt, P.Idct(idct))
    assert g.skipped_tiles == o.skipped_tiles and g.max_qscale == o.max_qscale
    assert np.array_equal(g.samples_host(), o.samples)
    return o, g


def develop_equal(o, g, stage):
    want = O.develop(o, O.params_new(o.header, o.quantizer), stage, planar=True)
    got = P.develop_planar(g, P.DemosaicParams.new(g.header, g.quantizer()), P.Stage(stage))
    for c in range(3):
        assert np.array_equal(got.planes[c].cpu().numpy().view(np.uint32), want[c].view(np.uint32)), c


def test_4k_frame_decodes_and_develops_bit_exact(frame_4k):
    o, g = decode_equal(frame_4k, 0)
    assert o.skipped_tiles == []
    develop_equal(o, g, int(P.Stage.WHITE_BALANCED))


@pytest.mark.parametrize("idct", [0, 1], ids=["apple", "ffmpeg"])
def test_5k8_hard_bitstream_both_transforms(frame_5k8, idct):
    o, g = decode_equal(frame_5k8, idct)
    assert len(o.skipped_tiles) > 0
    if idct == 0:
        develop_equal(o, g, int(P.Stage.REC2020))


def test_5k8_reduced_scales(frame_5k8):
    for shift in (1, 2, 3):
        for greens in (0, 1):
            o = O.decode_frame_reduced(frame_5k8, shift, greens)
            g = P.decode_frame_reduced_with(frame_5k8, P.Scale(shift), P.Greens(greens))
            assert g.skipped_tiles == o.skipped_tiles and g.max_qscale == o.max_qscale
            assert np.array_equal(g.samples_host(), o.samples), (shift, greens)


def test_64_frame_mixed_batch():
    items = S.mixed_batch(64, seed=2)
    jobs = [P.BatchJob(it.packet, None if it.scale == 0 else P.Scale(it.scale), P.Idct.APPLE, P.Greens(it.greens))
            for it in items]
    dec = P.BatchDecoder()
    results = dec.decode(jobs)
    for it, job, got in zip(items, jobs, results):
        if job.scale is None:
            want = O.decode_frame(it.packet, 0)
        else:
            want = O.decode_frame_reduced(it.packet, int(job.scale), int(job.greens))
        assert not isinstance(got, P.Error), got
        assert got.skipped_tiles == want.skipped_tiles and got.max_qscale == want.max_qscale
        assert np.array_equal(got.samples_host(), want.samples), (it.width, it.height, it.scale)
