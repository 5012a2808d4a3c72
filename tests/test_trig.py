"""The library's correctly rounded sin/cos (sdf-slam_b200/csrc/trig.cuh,
used by the device WrapAngle of the odometry residual), built for the host
from the same header, against sin and cos evaluated to 60 digits.

The device build of the header uses only explicitly rounded +, -, * and fma,
so it returns the same bits as this host build."""
import ctypes
import math
import os
import subprocess
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def sincos_rn(tmp_path_factory):
    out = tmp_path_factory.mktemp("trig") / "libtrig_host.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++20", "-shared", "-fPIC",
                    "-I", os.path.join(ROOT, "sdf-slam_b200", "csrc"),
                    os.path.join(ROOT, "tests", "trig_host.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.sincos_rn_host.argtypes = [dp, ctypes.c_int, dp, dp]

    def f(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        s = np.empty_like(x)
        c = np.empty_like(x)
        lib.sincos_rn_host(x.ctypes.data_as(dp), len(x), s.ctypes.data_as(dp), c.ctypes.data_as(dp))
        return s, c
    return f


def _hp_sincos(x: float):
    """sin and cos of the double x to ~70 digits (Taylor series after a
    reduction by a 100-digit pi), rounded once to double."""
    getcontext().prec = 90
    pi = Decimal("3.14159265358979323846264338327950288419716939937510582097494459230781640628620899862803482534211706798")
    X = Decimal(Fraction(x).numerator) / Decimal(Fraction(x).denominator)
    k = int((X / (pi / 2)).to_integral_value())
    r = X - k * (pi / 2)
    s, t, n = Decimal(0), r, 1
    while t != 0 and (s == 0 or abs(t) > abs(s) * Decimal(10) ** -80):
        s += t
        t = -t * r * r / ((n + 1) * (n + 2))
        n += 2
    c, t, n = Decimal(0), Decimal(1), 0
    while abs(t) > Decimal(10) ** -80:
        c += t
        t = -t * r * r / ((n + 1) * (n + 2))
        n += 2
    q = k % 4
    sv, cv = [(s, c), (c, -s), (-s, -c), (-c, s)][q]
    return float(Fraction(sv)), float(Fraction(cv))


def test_sincos_is_correctly_rounded(sincos_rn):
    rng = np.random.default_rng(5)
    x = np.concatenate([
        rng.uniform(-math.pi, math.pi, 1500),            # wrapped pose angles
        rng.uniform(-40.0, 40.0, 300),                    # unwrapped sums
        np.ldexp(rng.uniform(0.5, 1.0, 100), rng.integers(-40, -1, 100)),  # small angles
        np.array([math.pi / 4, -math.pi / 4, math.pi / 2, math.pi, 3 * math.pi / 4, 1e-300, 2.5e-8,
                  np.nextafter(math.pi / 4, 1.0), 1e6, -7.0e5, 2.0 ** 29]),
    ])
    s, c = sincos_rn(x)
    bad = []
    for xi, si, ci in zip(x, s, c):
        es, ec = _hp_sincos(float(xi))
        if si != es or ci != ec:
            bad.append((float(xi).hex(), si.hex(), es.hex(), ci.hex(), ec.hex()))
    assert not bad, bad[:5]


def test_sincos_special_values(sincos_rn):
    s, c = sincos_rn(np.array([0.0, -0.0, np.inf, -np.inf, np.nan]))
    assert s[0] == 0.0 and not math.copysign(1.0, s[0]) < 0 and c[0] == 1.0
    assert s[1] == 0.0 and math.copysign(1.0, s[1]) < 0 and c[1] == 1.0
    assert np.all(np.isnan(s[2:])) and np.all(np.isnan(c[2:]))
