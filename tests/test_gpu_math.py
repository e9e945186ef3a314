"""Device arithmetic of the fast forms checked directly against the
device's correctly rounded operations: the FP64 reciprocal (Newton-Raphson
on a single-precision seed, with the division taken outside the seed's
range) is within 1 ulp of 1.0 / x over random magnitudes from 1e-300 to
1e300, both signs, and at the range edges, 0, inf and NaN."""
import ctypes

import numpy as np
import pytest

from evora_b200._native import lib

pytestmark = pytest.mark.gpu


def _rcp(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(2 * x.size)
    st = lib().evora_selftest_rcp(x.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), x.size)
    assert st == 0
    return out[:x.size], out[x.size:]


def test_rcp_fast_within_one_ulp(cuda_device):
    rng = np.random.default_rng(5)
    mag = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    x = mag * rng.choice([-1.0, 1.0], mag.size)
    edges = []
    for e in (-126, 126):
        b = 2.0 ** e
        edges += [b, np.nextafter(b, 0), np.nextafter(b, np.inf), -b]
    x = np.concatenate([x, edges, [1e-300, 1e300, -1e-300, -1e300, 5e-324, 1.7976931348623157e308,
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
