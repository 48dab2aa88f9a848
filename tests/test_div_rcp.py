"""The CUDA library divides by the constant zone widths with a correctly
rounded reciprocal and one residual correction (div_rcp in
csrc/hamr_physics.cuh, Markstein's final Newton-Raphson step) instead of a
full division. The result must be the IEEE quotient bit for bit, or the
strict build would drift from the reference. The method uses only binary64
multiply and fused multiply-add, rounded to nearest, which the host computes
exactly as the GPU does; this checks it on the host over seeded operands
spanning the magnitudes of the step (differences of fluxes times a step size
over zone widths), including exact zeros and signed zeros, and over the whole
range 2^-900 <= |a| <= 2^900 where the method is exact; below it (a residual
that turns subnormal) the quotient may be one ulp off, which the last case
records."""
import ctypes

import numpy as np

from oracle import oracle as O


def _check(a, b):
    a = np.ascontiguousarray(a, float)
    b = np.ascontiguousarray(b, float)
    return O.lib().ho_div_rcp_mismatches(a.ctypes.data_as(ctypes.c_void_p), a.size,
                                         b.ctypes.data_as(ctypes.c_void_p), b.size)


def test_div_rcp_matches_ieee_division():
    rng = np.random.default_rng(2026)
    mant = rng.uniform(1.0, 2.0, 400_000)
    a = mant * np.exp2(rng.integers(-200, 200, mant.size)) * rng.choice([-1.0, 1.0], mant.size)
    a[:16] = [0.0, -0.0, 1.0, -1.0, 3.0, 1e-200, -1e-200, 1e200, 0.1, 1 / 3, 2.0 ** -900, -(2.0 ** 900),
              7.0, 1.5, np.nextafter(1.0, 2.0), np.nextafter(2.0, 1.0)]
    # zone widths of the test and benchmark grids and random ones, with
    # all-ones and all-zeros mantissas among them
    b = np.concatenate([[1 / 32, 1 / 48, 1 / 64, 1 / 128, 2 * np.pi / 192, 2 * np.pi / 64, 0.109375,
                         (np.log(1000.0) - np.log(0.9 * (1 + np.sqrt(1 - 0.9375 ** 2)))) / 384,
                         np.nextafter(2.0, 1.0), 1.0, 3.0, 0.1],
                        rng.uniform(1e-4, 1.0, 52)])
    assert _check(a, b) == 0
    # the residual path covers the whole range the guard admits
    wide = np.exp2(rng.uniform(-899.0, 899.0, 200_000)) * rng.choice([-1.0, 1.0], 200_000)
    assert _check(wide, b) == 0
    # outside the range: residuals below the normal range can misround
    tiny = np.array([9.332636185032189e-302, 5.696189077778436e-306])
    assert _check(tiny, np.array([np.nextafter(2.0, 1.0)])) == 2


def test_div_rcp_inversion_divisors():
    """The guarded form (div_rcp_inf, used by the inversion and wherever
    quotients share a divisor) on the inversion's divisors -- adiabatic
    indices and sqrt(-g) over the range of the torus grids (log-uniform from
    1e-4 to 1e7) -- with dividends over the exact range and infinite
    dividends (an overflowed state), which the guard returns as the IEEE
    quotient does; and with infinite and zero divisors."""
    rng = np.random.default_rng(77)
    b = np.concatenate([[13 / 9, 4 / 3, 5 / 3, 1.4, 2.0],
                        np.exp(rng.uniform(np.log(1e-4), np.log(1e7), 120))])
    a = np.exp2(rng.uniform(-899.0, 899.0, 300_000)) * rng.choice([-1.0, 1.0], 300_000)
    a[:6] = [0.0, -0.0, np.inf, -np.inf, 1.0, -1.0]
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    args = (a.ctypes.data_as(ctypes.c_void_p), a.size, b.ctypes.data_as(ctypes.c_void_p), b.size)
    assert O.lib().ho_div_rcp_mismatches_g(*args, 1) == 0
    # without the guard only the infinite dividends differ (NaN for +-inf)
    assert O.lib().ho_div_rcp_mismatches_g(*args, 0) == 2 * b.size
    # infinite and zero divisors (no NaN results here: their bit patterns
    # are not compared)
    a2 = np.ascontiguousarray([1.0, -3.5, 1e-300, 7e300, np.inf, -np.inf])
    for bad in ([np.inf, -np.inf], [0.0, -0.0]):
        aa = a2 if bad[0] == 0.0 else a2[:4]
        b2 = np.ascontiguousarray(bad)
        assert O.lib().ho_div_rcp_mismatches_g(aa.ctypes.data_as(ctypes.c_void_p), aa.size,
                                               b2.ctypes.data_as(ctypes.c_void_p), b2.size, 1) == 0
