"""Host logic of the muffin-tin integral generation, checked on the CPU.

The library's own Gaunt coefficients (azimuthal integral in closed form,
polar integral by an exact Gauss-Legendre rule) and its spline integral
(weights applied on the device) against the oracle's restatements of
gauntyry.f90 and fderiv.f90; no GPU is touched.
"""
import ctypes

import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import abi
from exciting_b200.crystal import radial_mesh_cubic


def _lib():
    return abi.load()


def _gauntyry(l1, l2, l3, m1, m2, m3):
    out = np.zeros(2)
    rc = _lib().exs_gauntyry(l1, l2, l3, m1, m2, m3, out.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0
    return complex(out[0], out[1])


@pytest.mark.parametrize("l1,l3", [(0, 0), (1, 2), (3, 3), (4, 2), (6, 5), (10, 10)])
def test_gauntyry_matches_oracle(l1, l3):
    worst = 0.0
    for l2 in range(0, 9):
        for m1 in range(-l1, l1 + 1):
            for m2 in range(-l2, l2 + 1):
                for m3 in range(-l3, l3 + 1):
                    g = _gauntyry(l1, l2, l3, m1, m2, m3)
                    ref = O.gauntyry(l1, l2, l3, m1, m2, m3)
                    worst = max(worst, abs(g - ref))
    assert worst < 2e-15


def test_gauntyry_selection_rules_exact_zero():
    assert _gauntyry(1, 1, 1, 0, 0, 0) == 0       # odd l1 + l2 + l3
    assert _gauntyry(1, 4, 1, 0, 0, 0) == 0       # triangle
    assert _gauntyry(2, 1, 2, 1, 1, 1) == 0       # |m3 - m1| != |m2|


def _fint(x, f):
    x = np.ascontiguousarray(x, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = ctypes.c_double()
    rc = _lib().exs_fderiv_int(len(x), x.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p),
                               ctypes.byref(out))
    assert rc == 0
    return out.value


@pytest.mark.parametrize("n,rmt", [(4, 2.0), (7, 1.5), (300, 2.1), (513, 2.6)])
def test_spline_integral_matches_oracle(n, rmt):
    rng = np.random.default_rng(n)
    x = radial_mesh_cubic(rmt, n, 1e-5) if n > 10 else np.cumsum(rng.uniform(0.1, 0.3, n))
    for f in (np.exp(-x) * x * x, np.sin(4 * x) * x, rng.standard_normal(n)):
        a, b = _fint(x, f), O.fint(x, f)
        assert abs(a - b) <= 1e-13 * max(1.0, np.abs(f).max() * (x[-1] - x[0]))


def test_fderiv_int_rejects_short_meshes():
    x = np.array([0.0, 1.0, 2.0])
    out = ctypes.c_double()
    rc = _lib().exs_fderiv_int(3, x.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p),
                               ctypes.byref(out))
    assert rc != 0


def test_unit_coupling_coefficients_match_oracle():
    """The closed forms behind exs_rttddft_genpmat's gradient coefficients
    against the oracle's clebgor (Racah formula), l <= 9."""
    out = ctypes.c_double()
    worst = 0.0
    for l2 in range(0, 10):
        for l in (l2 - 1, l2 + 1):
            if l < 0:
                continue
            for m2 in range(-l2, l2 + 1):
                for q in (-1, 0, 1):
                    m = m2 + q
                    if abs(m) > l:
                        continue
                    assert _lib().exs_clebgor_unit(l2, m2, q, l, m, ctypes.byref(out)) == 0
                    worst = max(worst, abs(out.value - O.clebgor(l2, 1, l, m2, q, m)))
    assert worst < 1e-15
