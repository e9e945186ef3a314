"""Device arithmetic of the fast forms checked directly against the
device's correctly rounded operations: the FP64 reciprocal and square root
(the hardware's approximations refined by Newton steps, with no branch;
arguments near the ends of the exponent range scaled first) are within 1
ulp of 1.0 / x and sqrt(x) over random magnitudes from 1e-300 to 1e300,
both signs, the scaled ranges and subnormals, and at 0, inf and NaN; the
default-mode chemistry's table-driven exponential and reciprocal likewise."""
import ctypes

import numpy as np
import pytest

from evora_b200._native import lib

pytestmark = pytest.mark.gpu


def _fast(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(4 * x.size)
    st = lib().evora_selftest_rcp(x.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), x.size)
    assert st == 0
    return out.reshape(4, x.size)


def _rcp(x):
    o = _fast(x)
    return o[0], o[1]


def test_rcp_fast_within_one_ulp(cuda_device):
    rng = np.random.default_rng(5)
    mag = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    x = mag * rng.choice([-1.0, 1.0], mag.size)
    edges = []
    for e in (-1022, -1000, 126, 1000, 1022):   # the scaled ranges' and the normal range's ends
        b = 2.0 ** e
        edges += [b, np.nextafter(b, 0), np.nextafter(b, np.inf), -b]
    far = np.concatenate([10.0 ** rng.uniform(-323, -301, 1 << 12), 10.0 ** rng.uniform(301, 308, 1 << 12)])
    x = np.concatenate([x, far, -far, edges, [1e-300, 1e300, -1e-300, -1e300, 5e-324, 1.7976931348623157e308,
                                              1.0, -1.0, 3.0, 0.1, 1e-38, 1e38, 1e-37, 1e37]])
    fast, div = _rcp(x)
    with np.errstate(over="ignore", divide="ignore"):
        ref = 1.0 / x
    # the device's division is the IEEE correctly rounded quotient
    np.testing.assert_array_equal(div, ref)
    ulp = np.spacing(np.abs(ref))
    with np.errstate(invalid="ignore"):
        ok = (fast == ref) | (np.abs(fast - ref) <= ulp)
    assert np.all(ok), x[~ok][:8]


def test_rcp_fast_specials(cuda_device):
    x = np.array([0.0, -0.0, np.inf, -np.inf, np.nan])
    fast, div = _rcp(x)
    assert fast[0] == np.inf and fast[1] == -np.inf
    assert fast[2] == 0.0 and fast[3] == 0.0 and np.signbit(fast[3])
    assert np.isnan(fast[4])


def test_sqrt_fast_within_one_ulp(cuda_device):
    """The FP64 fast square root (approximate reciprocal square root, two
    Newton steps and one correction, no branch) within 1 ulp of the
    correctly rounded sqrt over random magnitudes from 1e-300 to 1e300, the
    scaled ranges below 2^-1000 and above 2^1000, subnormals, and 0, -0,
    inf, negative and NaN arguments."""
    rng = np.random.default_rng(9)
    x = np.concatenate([10.0 ** rng.uniform(-300, 300, 1 << 20), 10.0 ** rng.uniform(-323, -301, 1 << 12),
                        10.0 ** rng.uniform(301, 308, 1 << 12),
                        [5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, 2.0 ** -1000, 2.0 ** 1000,
                         np.nextafter(2.0 ** -1000, 0), np.nextafter(2.0 ** 1000, np.inf), 1.0, 2.0, 0.25]])
    o = _fast(x)
    fast, ref = o[2], o[3]
    np.testing.assert_array_equal(ref, np.sqrt(x))   # the device's sqrt is correctly rounded
    assert np.all(np.abs(fast - ref) <= np.spacing(ref))
    with np.errstate(invalid="ignore"):
        sp = _fast(np.array([0.0, -0.0, np.inf, -1.0, -np.inf, np.nan]))[2]
    assert sp[0] == 0.0 and not np.signbit(sp[0]) and sp[1] == 0.0 and np.signbit(sp[1]) and sp[2] == np.inf
    assert np.all(np.isnan(sp[3:]))


def _chem_math(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(3 * x.size)
    st = lib().evora_selftest_exp(x.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), x.size)
    assert st == 0
    return out[:x.size], out[x.size:2 * x.size], out[2 * x.size:]


def _exp(x):
    return _chem_math(x)[0]


def test_rcp64_within_one_ulp(cuda_device):
    """The reciprocal of the default mode's chemistry: the hardware's
    approximation is within 2^-16 relative over normal x (measured about
    1e-6; two Newton steps square the error twice, past 2^-64), the refined
    value within 1 ulp of 1.0 / x, and 0, inf, NaN map to inf, 0, NaN."""
    rng = np.random.default_rng(7)
    mag = 10.0 ** rng.uniform(-307, 307, 1 << 20)
    x = np.concatenate([mag * rng.choice([-1.0, 1.0], mag.size), [1.0, -1.0, 3.0, 0.1, 2.2250738585072014e-308,
                                                                  1.7976931348623157e308 / 8, 1e-300, 1e300]])
    _, r, r0 = _chem_math(x)
    ref = 1.0 / x
    assert np.max(np.abs(r0 * x - 1.0)) < 2.0 ** -16
    assert np.all(np.abs(r - ref) <= np.spacing(np.abs(ref)))
    _, r, _ = _chem_math(np.array([0.0, -0.0, np.inf, -np.inf, np.nan]))
    assert r[0] == np.inf and r[1] == -np.inf and r[2] == 0.0 and r[3] == 0.0 and np.isnan(r[4])


def test_table_exp_within_two_ulp(cuda_device):
    """Tang's table-driven exponential of the default mode's chemistry
    against the host's exp (glibc, within 1 ulp of exact): within 2 ulp
    over normal results, within one subnormal step where exp underflows
    gradually (x in [-745.2, -708.4]), 0 below, inf above 709.79, NaN
    through."""
    rng = np.random.default_rng(6)
    x = np.concatenate([rng.uniform(-708.0, 709.0, 1 << 20), rng.uniform(-30.0, 30.0, 1 << 18),
                        rng.uniform(-1e-6, 1e-6, 1 << 12),
                        np.arange(-20000, 20001) * (np.log(2.0) / 64.0),   # the reduction's half-way points
                        [0.0, -0.0, 1.0, -1.0, 709.78, -708.39, 5e-324, -5e-324]])
    y, ref = _exp(x), np.exp(x)
    assert np.all(np.abs(y - ref) <= 2 * np.spacing(ref))
    sub = rng.uniform(-745.2, -708.4, 1 << 14)
    ys, refs = _exp(sub), np.exp(sub)
    assert np.all(np.abs(ys - refs) <= 5e-324)
    with np.errstate(over="ignore"):
        edge = _exp(np.array([-746.0, -800.0, -1e300, -np.inf, 709.8, 710.0, 1e300, np.inf, np.nan]))
    np.testing.assert_array_equal(edge[:4], 0.0)
    np.testing.assert_array_equal(edge[4:8], np.inf)
    assert np.isnan(edge[8])
