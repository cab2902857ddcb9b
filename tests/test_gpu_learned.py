"""The learned develop on the device against its CPU reference (the oracle's
sg_* functions): the tensor-core forward, the f32 backward, the packing and
output stages, the per-tile fallback to the plain develop, and what training
gains over the network-free output (each quad's own colour).

Tolerances: the forward stores bf16 activations, and the device sums its
bf16 products in another order than the CPU, so an activation can round to
the neighbouring bf16 value; the head is checked to 2 % of its largest
magnitude at worst and 1e-3 on average, gradients to 5 % normwise per
layer. Packing, output and fallback are exact."""

import numpy as np
import pytest

import _oracle as O
import proresraw_rs_b200 as P
from proresraw_rs_b200 import learned as Lrn
from proresraw_rs_b200 import synth as S

pytestmark = pytest.mark.gpu

LAYERS = Lrn.LAYERS


def he_params(rng, gain=1.0):
    parts = []
    for ci, co in LAYERS:
        parts.append(rng.standard_normal(co * ci * 9) * gain * np.sqrt(2.0 / (9 * ci)))
        parts.append(rng.uniform(0.02, 0.1, co))
    return np.concatenate(parts).astype(np.float32)


def random_image(rng, hq, wq):
    in16 = np.zeros((16, hq, wq), dtype=np.float32)
    in16[:4] = rng.uniform(0.0, 1.0, (4, hq, wq))
    in16[4] = rng.uniform(0.0, 0.5, (hq, wq))
    # bf16-representable inputs, as the packing stores them
    u = in16.view(np.uint32)
    in16 = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32)
    base = rng.uniform(0.0, 1.0, (3, hq, wq)).astype(np.float32)
    target = rng.uniform(0.0, 1.0, (3, 2 * hq, 2 * wq)).astype(np.float32)
    return in16, base, target


# Shapes: one strip of 128 pixels and one run of rows; three strips (the
# last 4 pixels wide) over runs of a few rows; a last strip of one pixel.
@pytest.mark.parametrize("hq,wq", [(40, 70), (16, 32), (7, 9), (70, 260), (33, 129), (1, 5)])
def test_forward_matches_the_oracle(hq, wq):
    rng = np.random.default_rng(hq * wq)
    in16, base, target = random_image(rng, hq, wq)
    params = he_params(rng)
    head, _, _ = Lrn.gradients(in16, base, target, params)
    _, want = O.sg_forward(in16, params)
    scale = max(1.0, float(np.max(np.abs(want))))
    err = np.abs(head - want)
    assert float(np.max(err)) <= 2e-2 * scale, float(np.max(err))
    assert float(np.mean(err)) <= 1e-3 * scale, float(np.mean(err))


def test_gradients_match_the_oracle():
    rng = np.random.default_rng(11)
    hq, wq = 20, 36
    in16, base, target = random_image(rng, hq, wq)
    params = he_params(rng)
    head, grad, loss = Lrn.gradients(in16, base, target, params)
    acts, ohead = O.sg_forward(in16, params)
    oloss, dhead = O.sg_loss(ohead, base, target)
    ograd = O.sg_backward(in16, params, acts, dhead)
    assert abs(loss - oloss) <= 1e-3 * oloss
    for k, (ws, bs) in enumerate(Lrn.layer_slices()):
        for sl in (ws, bs):
            g, o = grad[sl], ograd[sl]
            if k == len(LAYERS) - 1:  # head channels 12..15 feed nothing
                o = o.reshape(16, -1)[:12] if sl is ws else o[:12]
                g = g.reshape(16, -1)[:12] if sl is ws else g[:12]
            rel = np.linalg.norm(g - o) / max(np.linalg.norm(o), 1e-12)
            assert rel <= 5e-2, (k, rel)


def encoded_frame(w, h, pattern, seed, sigma, qscale, wb=(1.9, 1.4)):
    m = S.mosaic(w, h, pattern, seed=seed, sigma=sigma, white=4095)
    spec = S.Spec(w, h, pattern=pattern, alignment=2, white_level=4095, valid_tiles=True, wb=wb,
                  color_matrix=(0.61, 0.25, 0.10, 0.26, 0.89, -0.15, 0.02, -0.09, 1.17))
    return S.encode(spec, m, qscale=qscale, qscale_seed=seed)


def planes_of(frame, stage, s: Lrn.Surrogate):
    planes, nfb = Lrn.develop_learned(frame, stage, s)
    return np.stack([p.cpu().numpy() for p in planes.planes]), nfb


def plain_of(frame, stage):
    img = P.develop_planar(frame, P.DemosaicParams.new(frame.header, frame.quantizer()), stage)
    return np.stack([p.cpu().numpy() for p in img.planes])


@pytest.mark.parametrize("w,h", [(200, 132), (258, 70), (66, 18)])
@pytest.mark.parametrize("pattern", [0, 1, 2, 3])
def test_packing_is_exact(w, h, pattern):
    # The network input (bf16 channels) and the quad colours, bit for bit.
    pkt = encoded_frame(w, h, pattern, seed=3 + pattern, sigma=14.0, qscale=25)
    frame = P.decode_frame(pkt)
    in16, base = Lrn.pack(frame, P.Stage.REC2020)
    of = O.decode_frame(pkt)
    want_in, want_base = O.sg_pack(of.header, of.samples, O.params_new(of.header, of.quantizer))
    assert np.array_equal(in16.view(np.uint32), want_in.view(np.uint32))
    assert np.array_equal(base.view(np.uint32), want_base.view(np.uint32))


@pytest.mark.parametrize("pattern", [0, 3])
@pytest.mark.parametrize("stage", [P.Stage.WHITE_BALANCED, P.Stage.REC2020])
def test_network_free_output_is_exact(pattern, stage):
    # All parameters zero: the output is each quad's own colour, clipped and
    # (Rec.2020) matrixed -- packing and output bit for bit.
    pkt = encoded_frame(200, 132, pattern, seed=5, sigma=10.0, qscale=20)
    frame = P.decode_frame(pkt)
    s = Lrn.Surrogate(np.zeros(Lrn.param_count(), dtype=np.float32), 0.0, float("inf"))
    got, nfb = planes_of(frame, stage, s)
    assert nfb == 0
    of = O.decode_frame(pkt)
    p = O.params_new(of.header, of.quantizer)
    _, base = O.sg_pack(of.header, of.samples, p)
    head = np.zeros((16,) + base.shape[1:], dtype=np.float32)
    m = O.output_matrix(of.header) if stage == P.Stage.REC2020 else None
    want = O.sg_output(head, base, 200, 132, m, cfa=p.cfa_phase)
    assert np.array_equal(got.reshape(3, 132, 200), want)


# The develop runs layers 0-1, 2-3 and 4-5 as fused pairs (strips of 126
# pixels): its output against the oracle's network and output stage, on
# frames of several strips and both mirrorings of the network frame.
@pytest.mark.parametrize("w,h,pattern", [(560, 300, 0), (506, 138, 3), (66, 40, 1), (66, 18, 2)])
def test_develop_output_matches_the_oracle(w, h, pattern):
    pkt = encoded_frame(w, h, pattern, seed=9, sigma=12.0, qscale=25)
    frame = P.decode_frame(pkt)
    rng = np.random.default_rng(w + h)
    params = he_params(rng, 0.5)
    got, nfb = planes_of(frame, P.Stage.REC2020, Lrn.Surrogate(params, 0.0, float("inf")))
    assert nfb == 0
    of = O.decode_frame(pkt)
    p = O.params_new(of.header, of.quantizer)
    in16, base = O.sg_pack(of.header, of.samples, p)
    _, head = O.sg_forward(in16, params)
    want = O.sg_output(head, base, w, h, O.output_matrix(of.header), cfa=p.cfa_phase)
    scale = max(1.0, float(np.max(np.abs(head))))
    err = np.abs(got.reshape(3, h, w) - want)
    assert float(np.max(err)) <= 4e-2 * scale, float(np.max(err))
    assert float(np.mean(err)) <= 2e-3 * scale, float(np.mean(err))


def test_interleaved_output_is_the_planar_output():
    # prr_develop_learned with PRR_INTERLEAVED (rgb per pixel) against the
    # planar call, on a frame with some fallback tiles.
    import ctypes as C
    import torch
    from proresraw_rs_b200 import _lib, _dptr, context
    pkt = encoded_frame(300, 200, 3, seed=8, sigma=18.0, qscale=30)
    frame = P.decode_frame(pkt)
    rng = np.random.default_rng(8)
    params = he_params(rng, 0.5)
    of = O.decode_frame(pkt)
    noise = O.sg_pack(of.header, of.samples, O.params_new(of.header, of.quantizer))[0][4]
    s = Lrn.Surrogate(params, 0.0, float(np.median(noise)))
    planar, nfb = planes_of(frame, P.Stage.REC2020, s)
    assert nfb > 0
    n = 300 * 200
    out = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    prm = P.DemosaicParams.new(frame.header, frame.quantizer())
    dp = s.device()
    ctx = context()
    m = Lrn._model(s, dp)
    nfb2 = C.c_uint32()
    rc = _lib.lib().prr_develop_learned(ctx, C.byref(frame.header._c), C.byref(prm._c()), int(P.Stage.REC2020),
                                        _dptr(frame.samples), C.byref(m), 0, _dptr(out), None, None, 3 * n,
                                        C.byref(nfb2))
    assert rc == 0
    assert nfb2.value == nfb
    inter = out.cpu().numpy().reshape(n, 3).T
    assert np.array_equal(inter, planar.reshape(3, n))


def test_fallback_tiles_are_the_plain_develop():
    pkt = encoded_frame(256, 160, 0, seed=7, sigma=16.0, qscale=30)
    frame = P.decode_frame(pkt)
    rng = np.random.default_rng(7)
    params = he_params(rng, 0.3)
    params[Lrn.layer_slices()[-1][0]] *= 0.1
    plain = plain_of(frame, P.Stage.REC2020).reshape(3, 160, 256)
    # Range excluding every quad: all 40 tiles fall back, output = plain.
    got, nfb = planes_of(frame, P.Stage.REC2020, Lrn.Surrogate(params, 0.0, 0.0))
    assert nfb == 8 * 5
    assert np.array_equal(got.reshape(3, 160, 256), plain)
    # A range holding some quads: tile by tile, either plain or network.
    net, n0 = planes_of(frame, P.Stage.REC2020, Lrn.Surrogate(params, 0.0, float("inf")))
    assert n0 == 0
    of = O.decode_frame(pkt)
    in16, _ = O.sg_pack(of.header, of.samples, O.params_new(of.header, of.quantizer))
    noise = in16[4]  # RGGB: the network frame is the picture frame
    hi = float(np.median(noise))
    mixed, n1 = planes_of(frame, P.Stage.REC2020, Lrn.Surrogate(params, 0.0, hi))
    assert 0 < n1 < 40
    net, mixed = net.reshape(3, 160, 256), mixed.reshape(3, 160, 256)
    seen = 0
    for ty in range(5):
        for tx in range(8):
            q = noise[ty * 16:(ty + 1) * 16, tx * 16:(tx + 1) * 16]
            ys, xs = slice(ty * 32, (ty + 1) * 32), slice(tx * 32, (tx + 1) * 32)
            want = plain if (q.max() > hi) else net
            seen += int(q.max() > hi)
            assert np.array_equal(mixed[:, ys, xs], want[:, ys, xs]), (ty, tx)
    assert seen == n1


def test_training_gains_over_the_network_free_output():
    # Trained on 8 frames (noise sigma 4..32, qscale 15..45), judged on two
    # noisy held-out frames against the plain develop: the network must beat
    # its own output without the network (each quad's colour) by 3 dB and
    # stay above 45 dB.
    rng = np.random.default_rng(3)
    frames = []
    for k in range(8):
        sigma, q = float(rng.uniform(4, 32)), int(rng.integers(15, 46))
        frames.append(P.decode_frame(encoded_frame(1024, 768, 0, seed=100 + k, sigma=sigma, qscale=q)))
    held = [P.decode_frame(encoded_frame(1024, 768, 3, seed=200 + k, sigma=s, qscale=q))
            for k, (s, q) in enumerate([(20.0, 25), (28.0, 40)])]
    s, hist = Lrn.train_surrogate(frames, crops=2000, batch=32, crop=256, epochs=6, lr=1e-3, seed=1)
    assert hist[-1] < hist[0]
    lo, hi = s.noise_lo, s.noise_hi
    assert 0.0 < lo < hi
    zero = Lrn.Surrogate(np.zeros(Lrn.param_count(), dtype=np.float32), 0.0, float("inf"))
    for f in held:
        plain = plain_of(f, P.Stage.WHITE_BALANCED)
        trained, _ = planes_of(f, P.Stage.WHITE_BALANCED, Lrn.Surrogate(s.params, 0.0, float("inf")))
        base, _ = planes_of(f, P.Stage.WHITE_BALANCED, zero)
        p_t, p_b = Lrn.psnr(trained, plain), Lrn.psnr(base, plain)
        assert p_t >= 45.0 and p_t - p_b >= 3.0, (p_t, p_b)
