"""Accuracy of the library's own single-precision elementary functions
(include/hp_math.h), which the MCC kernels and the CPU oracle share so that
both make identical collision decisions.  Checked here against float64 numpy
on the ranges the kernels use: cross-section lookups (log10 of energies
1e-4..1e4 eV, exp of the table tail), scattering angles (sin/cos of 2 pi U,
U in (0, 1]), the ionisation energy split 10 tan(U atan(E/20)) and the
Maxwellian loader (log, pow).  The bound is a few units in the last place
(ulp of the float32 result)."""
import ctypes as C

import numpy as np
import pytest

import oracle

FN = dict(exp=0, log=1, log10=2, pow=3, sin_turns=4, cos_turns=5, tan=6, atan=7)


def call(name, x, y=None):
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, np.float32)
    out = np.empty_like(x)
    fp = C.POINTER(C.c_float)
    oracle.lib().or_math(FN[name], x.ctypes.data_as(fp), y.ctypes.data_as(fp), out.ctypes.data_as(fp), x.size)
    return out


def ulps(got, exact):
    exact32 = exact.astype(np.float32)
    ulp = np.spacing(np.abs(exact32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - exact) / ulp


rng = np.random.default_rng(7)


@pytest.mark.parametrize("name,x,exact,tol", [
    ("exp", rng.uniform(-80, 80, 20000), np.exp, 3),
    ("log", 10 ** rng.uniform(-30, 30, 20000), np.log, 3),
    ("log10", 10 ** rng.uniform(-4, 4, 20000), np.log10, 4),
    ("atan", rng.uniform(-50, 50, 20000), np.arctan, 3),
    ("tan", rng.uniform(0, 1.5, 20000), np.tan, 6),
])
def test_unary(name, x, exact, tol):
    x32 = x.astype(np.float32)
    got = call(name, x32)
    e = exact(x32.astype(np.float64))
    assert ulps(got, e).max() <= tol, name


def test_sincos_turns():
    t = rng.uniform(0, 1, 20000).astype(np.float32)
    s, c = call("sin_turns", t), call("cos_turns", t)
    a = 2 * np.pi * t.astype(np.float64)
    # absolute error against a unit-scale result (the kernels multiply by velocities)
    assert np.abs(s - np.sin(a)).max() < 4e-7
    assert np.abs(c - np.cos(a)).max() < 4e-7


def test_pow():
    b = 10 ** rng.uniform(-3, 3, 20000)
    e = rng.uniform(-2, 2, 20000)
    got = call("pow", b, e)
    exact = np.power(b.astype(np.float32).astype(np.float64), e.astype(np.float32).astype(np.float64))
    # exp(e log b): relative error grows with |e log b| (<= ~14 here)
    assert (np.abs(got / exact - 1)).max() < 2e-6


def test_special_values():
    assert call("exp", np.array([0.0]))[0] == 1.0
    assert call("log", np.array([1.0]))[0] == 0.0
    assert call("atan", np.array([0.0]))[0] == 0.0
    assert np.isnan(call("atan", np.array([np.nan]))[0])
