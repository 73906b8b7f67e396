"""The kernels' own exp / log / pow (csrc/fmath.h), host build, against
correctly rounded values (Python's decimal module at 40 digits) on the
argument ranges the acoustic substep uses, and special values."""
import decimal

import numpy as np
import pytest

from oracle import _math

decimal.getcontext().prec = 40


def _ulps(a, b):
    """|a - b| in units of the last place of b."""
    spacing = np.abs(np.spacing(b))
    return np.abs(a - b) / spacing


def _cr(fn, xs):
    return np.array([float(fn(decimal.Decimal(float(x)))) for x in xs])


@pytest.fixture(scope="module", autouse=True)
def _built():
    _math.build()


def _device(fn, *args):
    with _math.device_math():
        return fn(*args)


@pytest.mark.parametrize("lo,hi", [(-5.0, 5.0), (-700.0, 700.0), (-1e-8, 1e-8), (0.2, 0.4)])
def test_exp(lo, hi):
    xs = np.random.default_rng(1).uniform(lo, hi, 4000)
    got = _device(_math.exp, xs)
    ref = _cr(lambda d: d.exp(), xs)
    assert _ulps(got, ref).max() <= 1.0
    assert np.mean(got != ref) < 0.01


@pytest.mark.parametrize("lo,hi", [(100.0, 1.2e5), (0.5, 2.0), (1e-300, 1e-290), (1.0, 1.0 + 1e-6), (1e-3, 1e3)])
def test_log(lo, hi):
    xs = np.random.default_rng(2).uniform(lo, hi, 4000)
    got = _device(_math.log, xs)
    ref = _cr(lambda d: d.ln(), xs)
    assert _ulps(got, ref).max() <= 1.0
    assert np.mean(got != ref) < 0.01


def test_pow():
    rng = np.random.default_rng(3)
    xs = rng.uniform(10.0, 1.2e5, 4000)
    ys = rng.uniform(0.1, 0.4, 4000)
    got = _device(_math.power, xs, ys)
    ref = np.array([float(decimal.Decimal(float(x)) ** decimal.Decimal(float(y))) for x, y in zip(xs, ys)])
    assert _ulps(got, ref).max() <= 1.0
    assert np.mean(got != ref) < 0.01


def test_special_values():
    with _math.device_math():
        assert _math.exp(0.0) == 1.0
        assert _math.log(1.0) == 0.0
        assert np.isinf(_math.exp(1000.0)) and _math.exp(-1000.0) == 0.0
        assert np.isnan(_math.log(-1.0)) and np.isnan(_math.exp(float("nan")))
        assert np.isinf(_math.log(0.0)) and _math.log(0.0) < 0
        assert abs(_math.log(2.0) - np.log(2.0)) == 0.0
        assert _math.power(0.0, 0.5) == 0.0 and np.isnan(_math.power(-1.0, 0.5))
        sub = np.array([5e-324, 1e-310])
        assert np.all(_ulps(_math.log(sub), _cr(lambda d: d.ln(), sub)) <= 1.0)


def test_numpy_mode_is_numpy():
    xs = np.linspace(0.1, 10.0, 101)
    assert np.array_equal(_math.exp(xs), np.exp(xs))
    assert np.array_equal(_math.log(xs), np.log(xs))
    assert np.array_equal(_math.power(xs, 0.3), np.power(xs, 0.3))
