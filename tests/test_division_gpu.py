"""The FP64 kernels divide by the 1-D grid metrics through a quotient
corrected from the divisor's reciprocal (lare::div_rcp).  The MHD step's
bitwise parity rests on that quotient being the IEEE one, so it is checked
here against numpy's division on the host, bit for bit, over random operands
across and beyond the range the fast path takes, special values included."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(a, b):
    import torch
    from lare3d_b200 import gpu
    lib = gpu.library()
    f = lib.lare_gpu_check_division
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    out = torch.empty_like(da)
    assert f(da.data_ptr(), db.data_ptr(), a.size, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    with np.errstate(all="ignore"):
        want = a / b
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    bad = np.flatnonzero(got[~nan].view(np.int64) != want[~nan].view(np.int64))
    assert bad.size == 0, f"{bad.size} quotients differ, e.g. {a[~nan][bad[:3]]} / {b[~nan][bad[:3]]}"


def _random(rng, n, elo, ehi):
    m = 1.0 + rng.random(n)
    s = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return s * np.ldexp(m, rng.integers(elo, ehi, n))


def test_quotients_over_the_fast_range():
    rng = np.random.default_rng(11)
    n = 1 << 22
    _check(_random(rng, n, -520, 520), _random(rng, n, -60, 60))
    # differences of nearby values over grid widths, as in the curl and divergence terms
    x = rng.random(n)
    a = (x + rng.random(n) * 1e-6) - x
    b = np.full(n, 1.0 / 256.0) * (1.0 + rng.integers(0, 3, n) * rng.random(n))
    _check(a, b)


def test_quotients_at_the_edges():
    rng = np.random.default_rng(12)
    n = 1 << 20
    _check(_random(rng, n, -1074, 1024), _random(rng, n, -1074, 1024))
    bits = rng.integers(0, 2 ** 63, n, dtype=np.int64) * np.where(rng.random(n) < 0.5, -1, 1)
    a = bits.view(np.float64).copy()
    b = rng.integers(0, 2 ** 63, n, dtype=np.int64).view(np.float64).copy()
    _check(a, b)
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324, 2.2250738585072014e-308,
                        np.ldexp(1.0, -500), np.ldexp(1.0, 500), np.ldexp(1.9999999999999998, 500),
                        np.ldexp(1.0, -501), 1.0, -3.0, 1e300])
    a, b = np.meshgrid(special, special)
    _check(a.ravel().copy(), b.ravel().copy())
    # significands of all ones (the reciprocal sits next to a power of two)
    m = np.nextafter(2.0, 0.0)
    _check(_random(rng, n, -40, 40), np.ldexp(np.full(n, m), rng.integers(-40, 40, n)))


def test_product_engine_reciprocal():
    """The FP64 product engine divides through lare::fast_rcp (hardware
    approximation plus Newton-Raphson steps): within one ulp of 1/b over the
    range it serves."""
    import torch
    from lare3d_b200 import gpu
    f = gpu.library().lare_gpu_check_reciprocal
    f.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    rng = np.random.default_rng(13)
    n = 1 << 22
    b = _random(rng, n, -1000, 1000)
    b[:4] = [1.0, np.nextafter(2.0, 0.0), 2.0 ** -1000, 2.0 ** 1000]
    db = torch.from_numpy(b).cuda()
    out = torch.empty_like(db)
    assert f(db.data_ptr(), n, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    want = 1.0 / b
    ulps = np.abs(got - want) / np.spacing(np.abs(want))
    assert ulps.max() <= 1.0, f"max {ulps.max():.2f} ulp"
