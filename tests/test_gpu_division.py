"""The stencils divide by dx, dy, 24 and per-cell thicknesses with a correctly rounded
division from a precomputed reciprocal (Markstein's correction). This checks it against
the GPU's IEEE division bit for bit on random operands over many magnitudes, exact
quotients, their neighbours, signed zeros and non-finite values."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_division_matches_ieee():
    import pawsim_b200
    lib = pawsim_b200.load_library()
    fn = lib.pawsim_gpu_check_division
    fn.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_size_t, ctypes.c_double,
                   ctypes.POINTER(ctypes.c_longlong)]
    rng = np.random.default_rng(7)
    n = 1 << 22
    mant = rng.uniform(1.0, 2.0, n)
    expo = rng.integers(-200, 200, n)
    x = np.ldexp(mant, expo) * rng.choice([-1.0, 1.0], n)
    # both ends of the range that takes the corrections (binary exponents -899 .. 899)
    edge = np.ldexp(rng.uniform(1.0, 2.0, 4096), rng.integers(-903, -895, 4096))
    edge = np.concatenate([edge, np.ldexp(rng.uniform(1.0, 2.0, 4096), rng.integers(895, 903, 4096))])
    x = np.concatenate([x, edge, -edge, np.ldexp(1.0, np.arange(-905, 905))])
    divisors = [24.0, 3.0, 1953.125, 2000e3 / 128, 4000e3 / 1024, 977.0, 7812.5 * 900.0,
                1000.0 + 1e-3, 3000.0 - 0.7, 0.1, 1.0 / 3.0, 123456.789]
    for d in divisors:
        q = rng.uniform(-1e6, 1e6, 4096)
        exact = q * d
        extra = np.concatenate([exact, np.nextafter(exact, np.inf), np.nextafter(exact, -np.inf),
                                [0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1e300]])
        data = np.ascontiguousarray(np.concatenate([x, extra]))
        bad = ctypes.c_longlong(-1)
        rc = fn(data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), data.size, d, ctypes.byref(bad))
        assert rc == 0, lib.pawsim_gpu_last_error()
        assert bad.value == 0, (d, bad.value)
