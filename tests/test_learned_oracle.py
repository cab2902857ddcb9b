"""The CPU reference of the learned surrogate, pinned on its own: its
backward pass against finite differences of its forward pass (f32 mode), its
parameter layout against the library's count, its packing against the
oracle's linearization and noise model. These run without a GPU."""

import numpy as np
import pytest

import _oracle as O

LAYERS = [(16, 32)] + [(32, 32)] * 5 + [(32, 16)]


def random_params(rng, gain=1.0):
    """He-normal weights (times `gain`), small positive biases."""
    parts = []
    for ci, co in LAYERS:
        parts.append(rng.standard_normal(co * ci * 9) * gain * np.sqrt(2.0 / (9 * ci)))
        parts.append(rng.uniform(0.02, 0.1, co))
    return np.concatenate(parts).astype(np.float32)


def layer_slices():
    out, off = [], 0
    for ci, co in LAYERS:
        nw = co * ci * 9
        out.append((off, off + nw, off + nw + co))
        off += nw + co
    return out


def test_param_count_matches_the_layer_shapes():
    assert O.sg_param_count() == sum(co * ci * 9 + co for ci, co in LAYERS) == 55504


def loss_of(in16, base, target, params):
    _, head = O.sg_forward(in16, params, round_bf16=False)
    loss, _ = O.sg_loss(head, base, target)
    return loss


@pytest.mark.parametrize("seed", [1, 2])
def test_backward_matches_finite_differences(seed):
    rng = np.random.default_rng(seed)
    hq, wq = 5, 6
    in16 = np.zeros((16, hq, wq), dtype=np.float32)
    in16[:5] = rng.uniform(0.0, 1.0, (5, hq, wq))
    base = rng.uniform(0.0, 1.0, (3, hq, wq)).astype(np.float32)
    target = rng.uniform(0.0, 1.0, (3, 2 * hq, 2 * wq)).astype(np.float32)
    params = random_params(rng)
    acts, head = O.sg_forward(in16, params, round_bf16=False)
    _, dhead = O.sg_loss(head, base, target)
    grad = O.sg_backward(in16, params, acts, dhead)
    gscale = float(np.max(np.abs(grad)))
    # Central differences on a sample of parameters of every layer. A step
    # can cross a ReLU kink of the small image, more often the further the
    # layer is from the head: the bar is 1 % at the head, 10 % before it.
    for k, (start, wend, bend) in enumerate(layer_slices()):
        rel = 1e-2 if k == len(LAYERS) - 1 else 1e-1
        idx = list(rng.choice(np.arange(start, wend), 6, replace=False)) + [int(rng.integers(wend, bend))]
        for i in idx:
            h = 1e-2 * max(0.05, abs(float(params[i])))
            p1, p2 = params.copy(), params.copy()
            p1[i] += h
            p2[i] -= h
            fd = (loss_of(in16, base, target, p1) - loss_of(in16, base, target, p2)) / (2 * h)
            assert abs(fd - grad[i]) <= rel * abs(fd) + 5e-3 * gscale, (k, i, fd, grad[i])


def test_bf16_rounding_is_round_to_nearest_even():
    # Activations are stored as bf16: a value exactly between two bf16 values
    # goes to the even one.
    rng = np.random.default_rng(3)
    params = np.zeros(O.sg_param_count(), dtype=np.float32)
    (s0, w0, b0) = layer_slices()[0]
    # Layer 0: output channel c copies input channel 0 (centre tap) + bias.
    for c in range(32):
        params[s0 + (c * 16 + 0) * 9 + 4] = 1.0
    in16 = np.zeros((16, 1, 4), dtype=np.float32)
    vals = np.array([1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, 3.0 + 2 ** -7], dtype=np.float32)
    in16[0, 0, :] = 1.0
    params[w0:b0] = 0.0
    acts, _ = O.sg_forward(in16, params)
    assert np.all(acts[0, :, 0, :] == 1.0)
    # Through a bias: 1 + bias, rounded.
    for v in vals:
        p = params.copy()
        p[w0:b0] = v - 1.0
        acts, _ = O.sg_forward(in16, p)
        got = float(acts[0, 0, 0, 1])
        u = np.float32(v).view(np.uint32)
        want = np.uint32((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).view(np.float32)
        assert got == want, (v, got, want)


def test_pack_follows_the_plain_develop_normalization():
    import proresraw_rs_b200.synth as S

    # RGGB: the network frame is the picture frame.
    w, h = 36, 22
    m = S.mosaic(w, h, S.RGGB, seed=4, sigma=12.0)
    spec = S.Spec(w, h, pattern=S.RGGB, alignment=1, white_level=4095, valid_tiles=True, wb=(1.7, 1.3))
    pkt = S.encode(spec, m, qscale=20)
    f = O.decode_frame(pkt)
    p = O.params_with_white_balance(f.header, f.quantizer, 1.7, 1.3)
    in16, base = O.sg_pack(f.header, f.samples, p)
    lin = f.linearize().reshape(h, w).astype(np.float32)
    nrm = np.float32(p.one_over_range) * (lin - np.float32(p.black))
    rr, rc = p.cfa_phase >> 1, p.cfa_phase & 1
    r = nrm[rr::2, rc::2] * np.float32(1.7)
    gr = nrm[rr::2, 1 - rc::2]
    gb = nrm[1 - rr::2, rc::2]
    b = nrm[1 - rr::2, 1 - rc::2] * np.float32(1.3)
    gm = (gr + gb) * np.float32(0.5)
    assert np.array_equal(base[0], r) and np.array_equal(base[2], b)
    assert np.array_equal(base[1], gm)
    assert np.all(in16[9:] == 0.0)
    four = np.float32(4.0)

    def near(a, want):  # one bf16 rounding
        return np.all(np.abs(a - want) <= np.abs(want) * 2.0 ** -8 + 1e-30)

    assert near(in16[0], (r - gm) * four) and near(in16[3], (b - gm) * four)
    assert near(in16[5], gm)
    pad = np.pad(gm, 1, mode="edge")
    gx = (pad[1:-1, 2:] - pad[1:-1, :-2]) * np.float32(0.5)
    gy = (pad[2:, 1:-1] - pad[:-2, 1:-1]) * np.float32(0.5)
    lap = gm - ((pad[1:-1, 2:] + pad[1:-1, :-2]) + (pad[2:, 1:-1] + pad[:-2, 1:-1])) * np.float32(0.25)
    assert near(in16[6], gx * four) and near(in16[7], gy * four) and near(in16[8], lap * four)
    assert np.all(in16[4] > 0.0)


@pytest.mark.parametrize("pattern", [1, 2, 3])
def test_every_pattern_packs_as_rggb_in_the_network_frame(pattern):
    # A frame and its mirror image with red moved to the top-left: the
    # network sees the same input.
    import proresraw_rs_b200.synth as S

    w, h = 36, 22
    m = S.mosaic(w, h, pattern, seed=9, sigma=12.0)
    rr, rc = pattern >> 1, pattern & 1
    flipped = m[::-1 if rr else 1, ::-1 if rc else 1].copy()
    spec_a = S.Spec(w, h, pattern=pattern, alignment=1, white_level=4095, valid_tiles=True)
    spec_b = S.Spec(w, h, pattern=S.RGGB, alignment=1, white_level=4095, valid_tiles=True)
    # Lossless enough: qscale 1 keeps the codes within the transform's rounding.
    fa = O.decode_frame(S.encode(spec_a, m, qscale=1))
    fb = O.decode_frame(S.encode(spec_b, flipped, qscale=1))
    sa = fa.samples.reshape(-1, (w + 15) // 16 * 16)[:h, :w]
    sb = fb.samples.reshape(-1, (w + 15) // 16 * 16)[:h, :w]
    fb.samples.reshape(-1, (w + 15) // 16 * 16)[:h, :w] = sa[::-1 if rr else 1, ::-1 if rc else 1]
    pa = O.params_new(fa.header, fa.quantizer)
    pb = O.params_new(fb.header, fb.quantizer)
    ia, ba = O.sg_pack(fa.header, fa.samples, pa)
    ib, bb = O.sg_pack(fb.header, fb.samples, pb)
    assert np.array_equal(ia, ib) and np.array_equal(ba, bb)
    assert sb.shape == sa.shape
