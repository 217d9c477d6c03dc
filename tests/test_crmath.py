"""The device's FP64 exp/log/pow for the kernel-length iteration
(gizmo_b200/csrc/crmath.cuh) are correctly rounded.

The header is host-compilable: every operation in it is an explicitly rounded
IEEE add/mul/div/fma, so the host build computes the device's bits. The check
is against 60-digit decimal arithmetic (the exact value rounded to nearest),
not against the platform libm, which misrounds a small fraction of inputs.
"""
import ctypes as C
import math
import os
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "..", "gizmo_b200", "csrc", "crmath.cuh")

SRC = r"""
#include "%s"
extern "C" void cr_eval(int f, long n, const double *x, const double *y, double *out) {
  for (long i = 0; i < n; i++)
    out[i] = f == 0 ? gz::cr::exp(x[i]) : f == 1 ? gz::cr::log(x[i]) : gz::cr::pow(x[i], y[i]);
}
// the ~2^-100 evaluations alone (no shorter first attempt)
extern "C" void cr_eval_long(int f, long n, const double *x, const double *y, double *out) {
  using namespace gz::cr;
  for (long i = 0; i < n; i++)
    out[i] = f == 0 ? exp_rounded({x[i], 0.0}) : f == 1 ? round_dd(dd_log(x[i]))
                    : exp_rounded(dd_mul_d(dd_log(x[i]), y[i]));
}
"""


@pytest.fixture(scope="module")
def crlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("crmath")
    src = d / "w.cc"
    src.write_text(SRC % os.path.abspath(HEADER))
    so = d / "libw.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    D = C.POINTER(C.c_double)
    lib.cr_eval.argtypes = [C.c_int, C.c_long, D, D, D]
    lib.cr_eval_long.argtypes = [C.c_int, C.c_long, D, D, D]

    def ev(f, x, y=None, long=False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(x if y is None else y, dtype=np.float64)
        o = np.empty_like(x)
        fn = lib.cr_eval_long if long else lib.cr_eval
        fn(f, len(x), x.ctypes.data_as(D), y.ctypes.data_as(D), o.ctypes.data_as(D))
        return o
    return ev


def _nearest(exact: Decimal, got: float) -> bool:
    """got is the double nearest to exact (ties cannot occur for these functions)."""
    g = Decimal(got)
    lo = Decimal(float(np.nextafter(got, -np.inf)))
    hi = Decimal(float(np.nextafter(got, np.inf)))
    e = abs(g - exact)
    return e <= abs(lo - exact) and e <= abs(hi - exact)


def test_exp_log_pow_correctly_rounded(crlib):
    getcontext().prec = 60
    rng = np.random.default_rng(7)
    n = 3000
    # arguments of the ranges the iteration uses (jump factors, count ratios, h^3, bracket means)
    x = rng.uniform(-4, 4, n)
    for a, r in zip(x, crlib(0, x)):
        assert _nearest(Decimal(float(a)).exp(), float(r)), a
    x = np.exp(rng.uniform(-12, 4, n))
    for a, r in zip(x, crlib(1, x)):
        assert _nearest(Decimal(float(a)).ln(), float(r)), a
    x = 1 + rng.uniform(-0.01, 0.01, n)
    for a, r in zip(x, crlib(1, x)):
        assert _nearest(Decimal(float(a)).ln(), float(r)), a
    x = np.exp(rng.uniform(-12, 2, n))
    for a, r in zip(x, crlib(2, x, np.full(n, 3.0))):
        assert _nearest(Decimal(float(a)) ** 3, float(r)), a
    third = 1.0 / 3.0
    x = np.exp(rng.uniform(-20, 2, n))
    for a, r in zip(x, crlib(2, x, np.full(n, third))):
        assert _nearest((Decimal(float(a)).ln() * Decimal(third)).exp(), float(r)), a


def test_special_values(crlib):
    assert crlib(0, np.array([0.0]))[0] == 1.0
    assert crlib(1, np.array([1.0]))[0] == 0.0
    assert np.isnan(crlib(1, np.array([-1.0]))[0])
    assert crlib(1, np.array([0.0]))[0] == -np.inf
    assert crlib(0, np.array([800.0]))[0] == np.inf
    assert crlib(0, np.array([-800.0]))[0] == 0.0
    assert crlib(2, np.array([2.0]), np.array([-1.0]))[0] == 0.5
    # agreement with the platform libm on ordinary inputs (it misrounds rarely)
    x = np.random.default_rng(3).uniform(-3, 3, 20000)
    ref = np.array([math.exp(v) for v in x])
    assert (crlib(0, x) == ref).mean() > 0.99


def test_short_evaluation_agrees_with_the_long_one(crlib):
    """The shorter first attempt (error bound 2^-70, rounding test) returns
    what the ~2^-100 evaluation returns, on ranges the iteration uses and on
    the whole domain; ~1.5M arguments."""
    rng = np.random.default_rng(23)
    n = 250_000
    xs = [rng.uniform(-708, 708, n), rng.uniform(-4, 4, n), rng.uniform(-1e-3, 1e-3, n),
          np.ldexp(rng.uniform(-1, 1, n), -rng.integers(0, 60, n))]
    for x in xs:
        assert np.array_equal(crlib(0, x), crlib(0, x, long=True))
    ys = [np.exp(rng.uniform(-700, 700, n)), 1 + rng.uniform(-1e-2, 1e-2, n), 1 + rng.uniform(-1e-8, 1e-8, n)]
    for y in ys:
        assert np.array_equal(crlib(1, y), crlib(1, y, long=True))
    z = np.exp(rng.uniform(-60, 60, n))
    for e in (1.0 / 3.0, -1.0 / 3.0, 2.5, 7.25):
        ee = np.full(n, e)
        assert np.array_equal(crlib(2, z, ee), crlib(2, z, ee, long=True)), e


def test_exp_low_range_rounded_once(crlib):
    """Results between 2^-1022 and ~2^-969: rounded before the scaling by 2^m
    (scaling the low part first drops its bits there)."""
    getcontext().prec = 60
    x = np.random.default_rng(29).uniform(-708, -670, 400)
    for f in (lambda a: crlib(0, a), lambda a: crlib(0, a, long=True)):
        for a, r in zip(x, f(x)):
            assert _nearest(Decimal(float(a)).exp(), float(r)), a
