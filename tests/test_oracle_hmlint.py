"""The muffin-tin integral oracle (hmlint = mt_kin + mt_pot) pinned piece by piece.

The reference ships no unit vectors for these routines and has no Fortran
compiler here, so each ingredient is checked against an independent
computation:

* the spline integral (fderiv, m = -1) against closed-form integrals on the
  reference's cubic muffin-tin mesh, and exactly on polynomials;
* Wigner 3j symbols against known values and their orthogonality relation;
* Gaunt coefficients (complex and real-harmonic) against quadrature of
  scipy's spherical harmonics over the sphere;
* hmlint against its defining identities: Hermitian blocks, lm-diagonal
  blocks for a spherical potential, the kinetic radial integral, and an
  explicit quadrature of one non-spherical element.
"""
import math

import numpy as np
import pytest
import scipy.special as sp

import lapw_oracle as O
from exciting_b200 import workloads as W
from exciting_b200.crystal import radial_mesh_cubic

Y00 = 0.28209479177387814347


# ---------------------------------------------------------------- spline integral
def test_fint_polynomials_exact():
    x = radial_mesh_cubic(2.1, 300, 1e-5)
    for p in range(3):
        f = x ** p
        exact = (x[-1] ** (p + 1) - x[0] ** (p + 1)) / (p + 1)
        assert abs(O.fint(x, f) - exact) < 1e-13 * max(1.0, abs(exact))


@pytest.mark.parametrize("rmt", [1.8, 2.1, 2.6])
def test_fint_smooth_functions(rmt):
    x = radial_mesh_cubic(rmt, 300, 1e-5)
    # integral of r^2 e^{-r} from x1 to R
    F = lambda r: -np.exp(-r) * (r * r + 2 * r + 2)
    exact = F(x[-1]) - F(x[0])
    assert abs(O.fint(x, x * x * np.exp(-x)) - exact) < 1e-8
    # integral of sin(3r) r
    G = lambda r: np.sin(3 * r) / 9 - r * np.cos(3 * r) / 3
    # the end conditions of spline.f90 estimate the end curvature from divided
    # differences: the error is set by the 0.02 Bohr spacing at the sphere edge
    assert abs(O.fint(x, x * np.sin(3 * x)) - (G(x[-1]) - G(x[0]))) < 1e-6


def test_fint_uneven_short_mesh():
    rng = np.random.default_rng(3)
    x = np.cumsum(rng.uniform(0.05, 0.2, 9))
    f = 1.0 + 2.0 * x - 0.5 * x * x
    exact = lambda r: r + r * r - r ** 3 / 6
    assert abs(O.fint(x, f) - (exact(x[-1]) - exact(x[0]))) < 1e-12


# ---------------------------------------------------------------- Wigner 3j and Gaunt
def test_wigner3j_known_values():
    assert abs(O.wigner3j(0, 0, 0, 0, 0, 0) - 1.0) < 1e-15
    assert abs(O.wigner3j(1, 1, 0, 0, 0, 0) + 1 / math.sqrt(3)) < 1e-15
    assert abs(O.wigner3j(1, 1, 2, 0, 0, 0) - math.sqrt(2 / 15)) < 1e-15
    assert abs(O.wigner3j(2, 2, 2, 0, 0, 0) + math.sqrt(2 / 35)) < 1e-15
    assert abs(O.wigner3j(1, 1, 1, 1, -1, 0) - 1 / math.sqrt(6)) < 1e-15
    assert O.wigner3j(1, 1, 3, 0, 0, 0) == 0.0     # triangle rule
    assert O.wigner3j(2, 1, 1, 1, 1, 0) == 0.0     # m1 + m2 + m3 != 0


@pytest.mark.parametrize("j1,j2", [(1, 1), (2, 1), (3, 2), (4, 4)])
def test_wigner3j_orthogonality(j1, j2):
    for j3 in range(abs(j1 - j2), j1 + j2 + 1):
        for j3p in range(abs(j1 - j2), j1 + j2 + 1):
            for m3 in range(-min(j3, j3p), min(j3, j3p) + 1):
                s = sum(O.wigner3j(j1, j2, j3, m1, m2, m3) * O.wigner3j(j1, j2, j3p, m1, m2, m3)
                        for m1 in range(-j1, j1 + 1) for m2 in range(-j2, j2 + 1))
                want = (1.0 / (2 * j3 + 1)) if j3 == j3p else 0.0
                assert abs(s - want) < 1e-14


def _sphere_quadrature(n=24):
    xg, wg = np.polynomial.legendre.leggauss(n)
    theta = np.arccos(xg)
    phi = np.arange(2 * n) * (math.pi / n)
    T, P = np.meshgrid(theta, phi, indexing="ij")
    w = np.outer(wg, np.full(2 * n, math.pi / n))
    return T, P, w


def _ylm(l, m, T, P):
    return sp.sph_harm_y(l, m, T, P)


def _rlm(l, m, T, P):
    """Real harmonics of src/src_lib/genrlm.f90."""
    y = _ylm(l, m, T, P)
    if m < 0:
        return math.sqrt(2.0) * y.imag
    if m == 0:
        return y.real
    return math.sqrt(2.0) * y.real


def test_gaunt_vs_quadrature():
    T, P, w = _sphere_quadrature()
    for l1 in range(4):
        for l2 in range(4):
            for l3 in range(4):
                for m1 in range(-l1, l1 + 1):
                    for m2 in range(-l2, l2 + 1):
                        m3 = m1 - m2
                        if abs(m3) > l3:
                            continue
                        q = np.sum(w * np.conj(_ylm(l1, m1, T, P)) * _ylm(l2, m2, T, P) * _ylm(l3, m3, T, P))
                        assert abs(O.gaunt(l1, l2, l3, m1, m2, m3) - q.real) < 1e-13
                        assert abs(q.imag) < 1e-13


def test_gauntyry_vs_quadrature():
    T, P, w = _sphere_quadrature()
    for l1 in range(4):
        for l2 in range(5):
            for l3 in range(4):
                for m1 in range(-l1, l1 + 1):
                    for m2 in range(-l2, l2 + 1):
                        for m3 in range(-l3, l3 + 1):
                            q = np.sum(w * np.conj(_ylm(l1, m1, T, P)) * _rlm(l2, m2, T, P) * _ylm(l3, m3, T, P))
                            assert abs(O.gauntyry(l1, l2, l3, m1, m2, m3) - q) < 1e-13


# ---------------------------------------------------------------- hmlint
@pytest.fixture(scope="module")
def fcc_hmlint():
    s = W.si_fcc("text")
    rad = W.mt_radial(s, lmaxvr=6)
    return s, rad, O.hmlint(s, rad)


def test_mt_radial_continues_the_tails():
    s = W.si_fcc()
    rad = W.mt_radial(s)
    for ias in range(s.natmtot):
        is_ = s.crystal.atom_species[ias]
        for l in range(s.basis.lmaxapw + 1):
            for io in range(s.basis.apword[is_][l]):
                tail = rad.apwfr[-s.np_tail:, 0, io, l, ias]
                assert np.allclose(tail, s.apwfr_tail[:, io, l, ias], rtol=1e-13, atol=0)
    # du/dr by central differences
    r = rad.spr[:, 0]
    u = rad.apwfr[:, 0, 0, 2, 0]
    du = rad.apwfr[:, 1, 0, 2, 0]
    i = 200
    fd = (u[i + 1] - u[i - 1]) / (r[i + 1] - r[i - 1])
    assert abs(fd - du[i]) < 1e-4 * abs(du[i]) + 1e-8


def test_hmlint_hermitian(fcc_hmlint):
    s, rad, (aa, loa, lolo) = fcc_hmlint
    for ias in range(s.natmtot):
        scale = np.abs(aa[:, :, ias]).max()
        assert np.abs(aa[:, :, ias] - aa[:, :, ias].conj().T).max() < 1e-14 * scale
        assert np.abs(lolo[:, :, ias] - lolo[:, :, ias].conj().T).max() < 1e-14 * scale


def _apw_rows(basis, is_):
    return list(basis.apw_rows(is_))


def _lo_rows(basis, is_):
    rows = []
    for ilo, l in enumerate(basis.lorbl[is_]):
        for m in range(-l, l + 1):
            rows.append((l, m, ilo))
    return rows


def test_hmlint_spherical_potential_is_lm_diagonal():
    s = W.si_fcc("text")
    rad = W.mt_radial(s, lmaxvr=4)
    rad.veffmt[1:] = 0.0
    aa, loa, lolo = O.hmlint(s, rad)
    b = s.basis
    is_ = s.crystal.atom_species[0]
    rows = _apw_rows(b, is_)
    lrows = _lo_rows(b, is_)
    r = rad.spr[:, is_]
    for i, (l1, m1, io1) in enumerate(rows):
        for j, (l3, m3, io2) in enumerate(rows):
            if (l1, m1) != (l3, m3):
                assert aa[i, j, 0] == 0.0
    for i, (l1, m1, _ilo) in enumerate(lrows):
        for j, (l3, m3, _io) in enumerate(rows):
            if (l1, m1) != (l3, m3):
                assert loa[i, j, 0] == 0.0
    # one diagonal element from its definition:
    # 1/2 int (u'^2 + l(l+1) u^2/r^2) r^2 + int u^2 r^2 V_00 Y00
    l, io = 2, 1
    i = rows.index((l, 0, io))
    u, du = rad.apwfr[:, 0, io, l, 0], rad.apwfr[:, 1, io, l, 0]
    kin = O.fint(r, 0.5 * du * du * r * r + 0.5 * l * (l + 1) * u * u)
    pot = O.fint(r, u * u * r * r * rad.veffmt[0, :, 0]) * Y00
    assert abs(aa[i, i, 0] - (kin + pot)) < 1e-12 * abs(kin + pot)


def test_hmlint_nonspherical_element_by_quadrature(fcc_hmlint):
    """aa(f1, f3) = int conj(Y_l1m1) Y_l3m3 u1 u3 sum_lm2 R_lm2 V_lm2 r^2 (+ kinetic)
    evaluated as one angular quadrature of the full potential."""
    s, rad, (aa, loa, lolo) = fcc_hmlint
    b = s.basis
    is_ = s.crystal.atom_species[1]
    rows = _apw_rows(b, is_)
    r = rad.spr[:, is_]
    T, P, w = _sphere_quadrature(16)
    lmaxvr = rad.lmaxvr
    R = np.array([_rlm(l2, m2, T, P) for l2 in range(lmaxvr + 1) for m2 in range(-l2, l2 + 1)])
    for (l1, m1, io1), (l3, m3, io3) in [((1, 0, 0), (2, 1, 1)), ((2, -1, 1), (3, 2, 0)), ((0, 0, 0), (4, -3, 1))]:
        i, j = rows.index((l1, m1, io1)), rows.index((l3, m3, io3))
        ang = np.array([np.sum(w * np.conj(_ylm(l1, m1, T, P)) * Rk * _ylm(l3, m3, T, P)) for Rk in R])
        u1 = rad.apwfr[:, 0, io1, l1, 1]
        u3 = rad.apwfr[:, 0, io3, l3, 1]
        radial = np.array([O.fint(r, u1 * u3 * r * r * rad.veffmt[k, :, 1]) for k in range(R.shape[0])])
        want = np.sum(ang * radial)
        assert abs(aa[i, j, 1] - want) < 1e-12 * max(1.0, abs(want))


def test_hmlint_relativistic_mass_enters_kinetic_only():
    s0 = W.si_fcc("text")
    s1 = W.si_fcc("text", relativity="zora")
    rad = W.mt_radial(s0, lmaxvr=2)
    aa0, _, _ = O.hmlint(s0, rad)
    aa1, _, _ = O.hmlint(s1, rad)
    d = aa1 - aa0
    assert np.abs(d).max() > 1e-6                   # rmtable = 1/(1 - a V_00 Y00) differs from 1
    rows = _apw_rows(s0.basis, s0.crystal.atom_species[0])
    for i, (l1, m1, _a) in enumerate(rows):
        for j, (l3, m3, _b) in enumerate(rows):
            if (l1, m1) != (l3, m3):
                assert d[i, j, 0] == 0.0


# ---------------------------------------------------------------- olprad
def test_olprad_definitions():
    s = W.si_fcc("text", relativity="iora*")
    rad = W.mt_radial(s, lmaxvr=2)
    oalo, ololo, h1aa, h1loa, h1lolo = O.olprad(s, rad)
    b = s.basis
    r = rad.spr[:, 0]
    A2 = 0.5 * (1.0 / 137.03599911) ** 2
    rm = 1.0 / (1.0 - A2 * rad.veffmt[0, :, 1] * Y00)
    for ilo, l in enumerate(b.lorbl[0]):
        v = rad.lofr[:, 0, ilo, 1]
        for io in range(b.apword[0][l]):
            u = rad.apwfr[:, 0, io, l, 1]
            assert abs(oalo[io, ilo, 1] - O.fint(r, u * v * r * r)) < 1e-15
        for ilo2, l2 in enumerate(b.lorbl[0]):
            if l2 != l:
                assert ololo[ilo, ilo2, 1] == 0.0 and h1lolo[ilo, ilo2, 1] == 0.0
    # one lo per l in this basis: ololo is diagonal and positive
    assert np.all(np.diag(ololo[:, :, 1]) > 0)
    # h1aa(io1, io2, l) = a int (u1' u2' + l(l+1) u1 u2 / r^2) rm^2 r^2 / 2
    l = 3
    u1, u2 = rad.apwfr[:, 0, 0, l, 1], rad.apwfr[:, 0, 1, l, 1]
    d1, d2 = rad.apwfr[:, 1, 0, l, 1], rad.apwfr[:, 1, 1, l, 1]
    want = O.fint(r, A2 * (0.5 * d1 * d2 * rm * rm + 0.5 * l * (l + 1) * u1 * u2 * rm * rm / (r * r)) * r * r)
    assert abs(h1aa[0, 1, l, 1] - want) < 1e-14 * abs(want) + 1e-20
    assert abs(h1aa[0, 1, l, 1] - h1aa[1, 0, l, 1]) < 1e-14 * abs(want) + 1e-20


def test_olprad_without_iora_has_no_h1():
    s = W.si_fcc("shipped")
    rad = W.mt_radial(s)
    oalo, ololo, h1aa, h1loa, h1lolo = O.olprad(s, rad)
    assert h1aa is None and h1loa is None and h1lolo is None
    assert np.abs(oalo).max() > 0 and np.abs(ololo).max() > 0
