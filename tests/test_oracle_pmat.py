"""The oracle's momentum matrix elements (pmatrad, gradzfmtr, clebgor,
genpmatbasisik) pinned against independent computations on the CPU:

* Clebsch-Gordan coefficients: known values and orthonormality;
* the spline derivative (fderiv, m = 1): exact on quadratics, close on a
  smooth function on the muffin-tin mesh;
* gradzfmtr: sum_lm2 gfmt(lm2, r, j) Y_lm2 equals the Cartesian gradient of
  f(r) Y_lm by central finite differences (x and z directly; the y entry
  carries a factor -i, which genpmatbasisik's -i on x and z makes uniform);
* genpmatbasisik: the APW block of the oracle equals conj(A) R A^T built
  independently from pmatrad's integrals.
"""
import math

import numpy as np
import pytest
import scipy.special as sp

import lapw_oracle as O
from exciting_b200 import workloads as W
from exciting_b200.crystal import radial_mesh_cubic


def test_clebgor_values_and_orthonormality():
    assert abs(O.clebgor(1, 1, 2, 0, 0, 0) - math.sqrt(2.0 / 3.0)) < 1e-15
    assert abs(O.clebgor(1, 1, 0, 1, -1, 0) - 1.0 / math.sqrt(3.0)) < 1e-15
    assert abs(O.clebgor(2, 1, 3, 2, 1, 3) - 1.0) < 1e-15
    for j1, j2 in [(2, 1), (3, 1), (4, 2)]:
        for J in range(abs(j1 - j2), j1 + j2 + 1):
            for Jp in range(abs(j1 - j2), j1 + j2 + 1):
                for M in range(-min(J, Jp), min(J, Jp) + 1):
                    s = sum(O.clebgor(j1, j2, J, m1, M - m1, M) * O.clebgor(j1, j2, Jp, m1, M - m1, M)
                            for m1 in range(-j1, j1 + 1) if abs(M - m1) <= j2)
                    assert abs(s - (1.0 if J == Jp else 0.0)) < 1e-14


def test_spline_derivative():
    rng = np.random.default_rng(1)
    x = np.cumsum(rng.uniform(0.05, 0.2, 12))
    assert np.max(np.abs(O.fderiv1(x, 3 * x * x - x + 2) - (6 * x - 1))) < 1e-11
    r = radial_mesh_cubic(2.1, 300, 1e-5)
    g = O.fderiv1(r, r ** 2 * np.exp(-r))
    want = (2 * r - r * r) * np.exp(-r)
    assert np.max(np.abs(g - want)[5:-5]) < 1e-5


@pytest.mark.parametrize("l,m", [(0, 0), (1, -1), (2, 1), (3, -2), (3, 3)])
def test_gradzfmtr_is_the_gradient(l, m):
    from lapw_oracle import lib, _p
    lmax = l + 1
    nr = 600
    r = radial_mesh_cubic(2.5, nr, 1e-5)
    f = lambda x: x ** (l + 1) * np.exp(-x)
    ir = 400
    x0 = r[ir]
    th, ph = 0.7, 0.4
    g = O.gradzfmtr(lmax, r, l, m, f(r))
    y = np.array([sp.sph_harm_y(l2, m2, th, ph) for l2 in range(lmax + 1) for m2 in range(-l2, l2 + 1)])
    grad = np.array([np.sum(g[:, ir, j] * y) for j in range(3)])
    # finite differences of f(r) Y_lm in Cartesian coordinates
    p0 = x0 * np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])

    def F(p):
        rr = np.linalg.norm(p)
        return f(rr) * sp.sph_harm_y(l, m, math.acos(p[2] / rr), math.atan2(p[1], p[0]))

    h = 1e-5
    fd = np.array([(F(p0 + h * e) - F(p0 - h * e)) / (2 * h) for e in np.eye(3)])
    assert abs(grad[0] - fd[0]) < 2e-5
    assert abs(1j * grad[1] - fd[1]) < 2e-5
    assert abs(grad[2] - fd[2]) < 2e-5


def test_genpmatbasisik_apw_block_is_conj_a_r_at():
    s = W.si_fcc("shipped")
    rad = W.mt_radial(s, lmaxvr=2)
    rip = O.pmatrad(s, rad)
    gk = s.gkset(s.kpoints[3])
    apwalm, _ = O.match(s, gk)
    pm = O.genpmatbasisik(s, gk, apwalm, rip)
    ng = gk.ngp
    b = s.basis
    ref = np.zeros((ng, ng), dtype=complex)
    for ias in range(s.natmtot):
        cols = O._apw_cols(b, 0)
        A = np.stack([apwalm[:ng, io, lm, ias] for io, lm in cols], axis=1)
        R = np.array([[rip[0][a, b1, c, d, ias, 2] for c, d in cols] for a, b1 in cols])
        ref += np.conj(A) @ R @ A.T
    # pm's z component: -i times the MT part, plus the interstitial term
    gv = s.gv
    iv = gv.ivg[:, gk.igpig - 1]
    ig = gv.ivgig_lookup((iv[:, :, None] - iv[:, None, :]).reshape(3, -1)).reshape(ng, ng) - 1
    ist = gk.vgpc[2][None, :] * np.asarray(s.cfunig)[ig]
    assert np.max(np.abs(pm[:ng, :ng, 2] - (-1j * ref + ist))) < 1e-12 * np.abs(ref).max()
