"""The float32 evaluations' square root (a Newton step from the approximate reciprocal square root)
against sqrtf, through the self-test export fb_sqrt_sum_probe."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _roots(lib, L, x):
    import torch
    xs = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    out = torch.empty_like(xs)
    assert lib.fb_sqrt_sum_probe(xs.data_ptr(), out.data_ptr(), xs.numel(), L.stream_handle()) == 0
    want = torch.sqrt(xs)  # IEEE square root, correctly rounded
    torch.cuda.synchronize()
    return out.cpu().numpy(), want.cpu().numpy()


def test_sqrt_sum_is_correctly_rounded():
    """Every float of [1, 4) (two binades: the pattern of every normal input), and a seeded sample of
    every binade from 2^-99 to 2^100: bit-equal to the IEEE root.  0 gives 0, NaN stays NaN, and
    inputs below 1e-30 are within 1e-15 of their root."""
    import field_b200._lib as L
    lib = L.lib()
    lo = np.float32(1.0).view(np.uint32)
    every = (np.arange(1 << 24, dtype=np.uint64) + int(lo)).astype(np.uint32).view(np.float32)
    got, want = _roots(lib, L, every)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    rng = np.random.default_rng(11)
    e = rng.integers(-99, 101, size=1 << 20)
    m = rng.uniform(1.0, 2.0, size=1 << 20)
    x = np.ldexp(m, e).astype(np.float32)
    got, want = _roots(lib, L, x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    special = np.array([0.0, np.nan, 1e-31, 1e-36, 1e-40, 1e-30], np.float32)
    got, want = _roots(lib, L, special)
    assert got[0] == 0.0 and np.isnan(got[1])
    assert np.all(np.abs(got[2:].astype(np.float64) - np.sqrt(special[2:].astype(np.float64))) <= 1e-15)


def test_quotient_within_one_ulp_of_ieee():
    """The 8^3 tiles' quotient (Newton step from the approximate reciprocal) against the IEEE
    quotient on seeded pairs of the magnitudes the sphere's difference form meets (numerators of
    either sign from 2^-40 to 2^4, positive denominators from 2^-30 to 2^4): within one ulp
    everywhere and equal on all but a sliver."""
    import torch
    import field_b200._lib as L
    lib = L.lib()
    rng = np.random.default_rng(12)
    n = 1 << 22
    num = (np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-40, 5, n)) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    den = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-30, 5, n)).astype(np.float32)
    a = torch.from_numpy(num).cuda()
    b = torch.from_numpy(den).cuda()
    out = torch.empty_like(a)
    assert lib.fb_quotient_probe(a.data_ptr(), b.data_ptr(), out.data_ptr(), n, L.stream_handle()) == 0
    want = (a / b).cpu().numpy()
    got = out.cpu().numpy()
    ulps = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1
    assert (ulps != 0).mean() < 1e-4
