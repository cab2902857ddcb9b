"""The develop kernel's launch shapes and their autotuner (prr_develop_*):
every output tile shape (32x32, 32x16, 64x16) at every CTA-per-SM cap the
tuner tries must develop bit for bit what the CPU oracle develops -- edge
tiles, interior tiles, both layouts, all three stages -- and the config the
tuner keeps for a frame-size bucket must be one of them and be used."""

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib
from proresraw_rs_b200 import synth as S

pytestmark = pytest.mark.gpu

SHAPES = [(32, 32), (32, 16), (64, 16)]


def frame(w, h, pattern, seed):
    m = S.mosaic(w, h, pattern, seed=seed, sigma=24.0, specular=0.02, white=4095)
    spec = S.Spec(w, h, pattern=pattern, alignment=2, white_level=4095, valid_tiles=True, wb=(1.9, 1.4))
    return S.encode(spec, m, qscale=(15, 45), qscale_seed=seed)


def developed(g, prm, stage, planar):
    if planar:
        return [p.cpu().numpy() for p in P.develop_planar(g, prm, P.Stage(stage)).planes]
    return [P.develop_with(g, prm, P.Stage(stage)).data.cpu().numpy()]


@pytest.mark.parametrize("w,h,pattern", [(1000, 600, 0), (346, 130, 3), (130, 66, 1)])
def test_every_tile_shape_develops_like_the_oracle(w, h, pattern):
    pkt = frame(w, h, pattern, seed=w + pattern)
    o = O.decode_frame(pkt)
    g = P.decode_frame(pkt)
    prm = P.DemosaicParams.new(g.header, g.quantizer())
    op = O.params_new(o.header, o.quantizer)
    bucket = P.develop_bucket(w, h)
    wants = {(stage, planar): O.develop(o, op, stage, planar=planar) for stage in (0, 1, 2) for planar in (True, False)}
    try:
        for tw, th in SHAPES:
            fit = 1024 // (tw * th // 4)
            for cap in sorted({0, max(1, fit // 2), fit - 1}):
                P.develop_set_config(bucket, P.DevelopConfig(tw, th, cap))
                for (stage, planar), want in wants.items():
                    got = developed(g, prm, stage, planar)
                    want = want if planar else [want]
                    for c in range(len(got)):
                        diff = np.count_nonzero(got[c].view(np.uint32) != want[c].reshape(-1).view(np.uint32))
                        assert diff == 0, f"{tw}x{th} cap {cap} stage {stage} planar {planar}: {diff} differ"
    finally:
        P.develop_set_config(bucket, P.DevelopConfig())


def test_the_tuner_keeps_a_candidate_and_the_develop_uses_it():
    import torch

    w, h = 1280, 720
    pkt = frame(w, h, 2, seed=5)
    o = O.decode_frame(pkt)
    g = P.decode_frame(pkt)
    prm = P.DemosaicParams.new(g.header, g.quantizer())
    out = [torch.empty(w * h, dtype=torch.float32, device="cuda") for _ in range(3)]
    cfg, ms = P.develop_tune(g, prm, P.Stage.REC2020, out, reps=2)
    assert (cfg.tile_w, cfg.tile_h) in SHAPES and ms > 0
    assert P.develop_get_config(P.develop_bucket(w, h)) == cfg
    want = O.develop(o, O.params_new(o.header, o.quantizer), 2, planar=True)
    for c in range(3):  # the tuner's last run, and a develop after it
        assert np.array_equal(out[c].cpu().numpy().view(np.uint32), want[c].view(np.uint32))
    got = developed(g, prm, 2, True)
    for c in range(3):
        assert np.array_equal(got[c].view(np.uint32), want[c].view(np.uint32))
    P.develop_set_config(P.develop_bucket(w, h), P.DevelopConfig())


def test_unsupported_shapes_are_refused():
    with pytest.raises(P.Error) as e:
        P.develop_set_config(P.develop_bucket(64, 64), P.DevelopConfig(16, 16, 0))
    assert e.value.code == _lib.ERR_INVALID


@pytest.mark.parametrize("noise", [(0.0, 0.0, 1e-14), (3e-4, 1e-7, 2e-6), (1000.0, 0.0, 1e-6)],
                         ids=["below-the-floor", "ordinary", "large-slope"])
def test_parameters_outside_the_paired_division_range_take_ieee_division(noise):
    # Parameters a caller sets by hand can leave the range in which the
    # develop's paired division and square root are exact (a noise floor
    # below 2^-40, a slope above 256): the develop then divides and takes
    # roots with div.rn / sqrt.rn throughout. Both paths must be the
    # oracle's, on interior and edge tiles, with these parameters.
    import dataclasses

    pkt = frame(700, 300, 0, seed=9)
    o = O.decode_frame(pkt)
    g = P.decode_frame(pkt)
    prm = dataclasses.replace(P.DemosaicParams.new(g.header, g.quantizer()), noise=noise)
    op = O.params_new(o.header, o.quantizer)
    op.noise[:] = list(noise)
    for stage in (0, 2):
        want = O.develop(o, op, stage, planar=True)
        got = P.develop_planar(g, prm, P.Stage(stage))
        for c in range(3):
            diff = np.count_nonzero(got.planes[c].cpu().numpy().view(np.uint32) != want[c].view(np.uint32))
            assert diff == 0, f"stage {stage} plane {c}: {diff} differ"
