"""The develop's paired division and square root (fastdiv.cuh): Markstein's
method on f32x2 pairs must give IEEE round-to-nearest results bit for bit
wherever the develop uses it. Division (|a|, |b| in [2^-100, 2^100],
quotients in [2^-120, 2^120]): every significand pair of [1, 2) x [1, 2)
with the reciprocal's exact scaling over the exponents, random operands
across the range and edge operands, against numpy's IEEE division. Square
root: every float of [2^-60, 2^61) against sqrt.rn."""

import numpy as np
import pytest

import proresraw_rs_b200 as P
from proresraw_rs_b200 import _lib

pytestmark = pytest.mark.gpu


def pairs_dev(a, b):
    import torch

    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    q = torch.empty_like(ta)
    assert _lib.lib().prr_div_rn_pairs(P.context(), ta.data_ptr(), tb.data_ptr(), q.data_ptr(), a.size) == 0
    torch.cuda.synchronize()
    return q.cpu().numpy()


def test_every_significand_pair_divides_like_ieee():
    import torch

    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert _lib.lib().prr_div_rn_check(P.context(), 0, 1 << 23, bad.data_ptr()) == 0
    torch.cuda.synchronize()
    assert int(bad.item()) == 0


def test_random_operands_across_the_range_divide_like_ieee():
    rng = np.random.default_rng(11)
    n = 1 << 22
    ea = rng.integers(-100, 100, n)
    eb = np.clip(ea - rng.integers(-100, 100, n), -100, 99)
    a = (np.ldexp(rng.uniform(1, 2, n), ea) * rng.choice([-1, 1], n)).astype(np.float32)
    b = (np.ldexp(rng.uniform(1, 2, n), eb) * rng.choice([-1, 1], n)).astype(np.float32)
    q = np.abs(np.float64(a) / np.float64(b))
    keep = (q >= 2.0 ** -120) & (q <= 2.0 ** 120)
    a, b = a[keep], b[keep]
    got = pairs_dev(a, b)
    assert np.array_equal(got.view(np.uint32), (a / b).view(np.uint32))


def test_edge_operands():
    # Zero numerators, exact quotients, a = b, powers of two, the largest and
    # smallest significands, quotients at the binade edges.
    one_minus = np.float32(np.nextafter(np.float32(2), np.float32(0)))
    vals = np.array([1.0, 1.5, one_minus, 2.0 ** -100, 2.0 ** 100, 3.0, 1.0 / 3.0, 1e-20, 7e19], dtype=np.float32)
    a, b = np.meshgrid(vals, vals)
    a, b = a.ravel(), b.ravel()
    a = np.concatenate([a, -a, np.zeros(9, np.float32)])
    b = np.concatenate([b, b, vals])
    q = np.abs(np.float64(a) / np.float64(b))
    keep = (a == 0) | ((q >= 2.0 ** -120) & (q <= 2.0 ** 120))
    a, b = a[keep], b[keep]
    got = pairs_dev(a, b)
    assert np.array_equal(got.view(np.uint32), (a / b).view(np.uint32))


def test_every_float_in_the_develops_range_has_the_ieee_square_root():
    # The paired square root (fastdiv.cuh) against sqrt.rn on every float of
    # [2^-60, 2^61), the range the develop's variances lie in with margin.
    import torch

    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert _lib.lib().prr_sqrt_rn_check(P.context(), -60, 60, bad.data_ptr()) == 0
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
