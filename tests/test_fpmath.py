"""The shared FP64 atan/log/exp (dba_b200/csrc/fpmath.h) against mpmath: <= 2.5 ulp,
C99 special values; the FP32 atan of the FP32 dendrite kernels: <= 1.5 ulp with a
correctly rounded reciprocal.  Run through the CPU build of the same header."""
import math
import random

import mpmath as mp
import numpy as np
import pytest

from oracle_lib import lib

mp.mp.dps = 40
FN = {0: mp.exp, 1: mp.log, 2: mp.atan}


def ulp_err(which, x):
    y = lib().oracle_fm(which, x)
    t = FN[which](mp.mpf(x))
    tf = float(t)
    if tf == 0.0:
        return abs(y) / 5e-324
    return float(abs(mp.mpf(y) - t) / math.ulp(tf))


@pytest.mark.parametrize("which,lo,hi,logscale", [
    (0, -700, 700, False), (0, -2, 2, False), (1, -700, 700, True), (1, 0.01, 3.0, False),
    (2, -8, 8, False), (2, -1e6, 1e6, False)])
def test_ulp_error(which, lo, hi, logscale):
    rng = random.Random(1000 + which)
    worst = 0.0
    for _ in range(3000):
        x = rng.uniform(lo, hi)
        if logscale:
            x = math.exp(x)
        worst = max(worst, ulp_err(which, x))
    assert worst <= 2.5, worst


def test_special_values():
    L = lib()
    assert L.oracle_fm(0, 0.0) == 1.0
    assert L.oracle_fm(0, 800.0) == math.inf
    assert L.oracle_fm(0, -800.0) == 0.0
    assert math.isnan(L.oracle_fm(0, math.nan))
    assert L.oracle_fm(1, 1.0) == 0.0
    assert L.oracle_fm(1, 0.0) == -math.inf
    assert math.isnan(L.oracle_fm(1, -1.0))
    assert L.oracle_fm(1, math.inf) == math.inf
    assert abs(L.oracle_fm(1, 5e-324) - math.log(5e-324)) < 1e-12
    assert L.oracle_fm(2, 0.0) == 0.0
    assert L.oracle_fm(2, math.inf) == pytest.approx(math.pi / 2, rel=0, abs=1e-16)
    assert L.oracle_fm(2, -math.inf) == pytest.approx(-math.pi / 2, rel=0, abs=1e-16)
    assert L.oracle_fm(2, 1.0) == pytest.approx(math.pi / 4, rel=2e-16)


def test_fp32_atan_ulp_error():
    """dba_atanf on every float of a dense sample of [0, 1] and of (1, 1e7], and on
    random floats over the whole range, in float ulps of the exact value."""
    rng = np.random.default_rng(7)
    xs = np.concatenate([np.linspace(0.0, 1.0, 20001), np.geomspace(1.0, 1e7, 20001),
                         rng.uniform(-40.0, 40.0, 4000),
                         rng.integers(0, 0x7f800000, 4000, dtype=np.uint32).view(np.float32).astype(np.float64)])
    xs = xs.astype(np.float32).astype(np.float64)
    L = lib()
    worst = 0.0
    for x in xs:
        y = L.oracle_fm(3, float(x))
        assert y == float(np.float32(y))
        t = mp.atan(mp.mpf(float(x)))
        tf = np.float32(float(t))
        u = float(np.spacing(np.abs(tf))) if tf != 0 else 1e-45
        worst = max(worst, float(abs(mp.mpf(y) - t)) / u)
    assert worst <= 1.5, worst
    assert L.oracle_fm(3, 0.0) == 0.0
    assert L.oracle_fm(3, math.inf) == float(np.float32(math.pi / 2))
    assert L.oracle_fm(3, -math.inf) == -float(np.float32(math.pi / 2))
    assert math.isnan(L.oracle_fm(3, math.nan))


def test_halving_by_multiplication_rounds_like_division():
    """The FP64 KH formulas write the reference's divisions by 2 as multiplications by
    0.5.  Both are correctly rounded results of the same real number, so the identity
    holds exactly by IEEE rounding; this test checks it on about a million sampled
    doubles plus edge cases (subnormals, extremes, infinities, signed zeros)."""
    rng = np.random.default_rng(11)
    bits = rng.integers(0, 2**64, size=1 << 20, dtype=np.uint64)
    x = bits.view(np.float64)
    x = x[np.isfinite(x)]
    edge = np.array([0.0, -0.0, 5e-324, -5e-324, 2.2250738585072014e-308, 4.450147717014403e-308,
                     1.7976931348623157e308, -1.7976931348623157e308, np.inf, -np.inf, 1.0, 3.0, 1e-300])
    for v in (x, edge, x * 0.37, x * 1e-300):
        with np.errstate(all="ignore"):
            a, b = v / 2.0, v * 0.5
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    nan = np.array([np.nan])
    assert np.isnan(nan / 2.0) and np.isnan(nan * 0.5)
