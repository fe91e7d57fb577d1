"""The CPU oracle pinned against independent references and its own identities.

* special functions against scipy (an independent implementation);
* match: the matching conditions D_l A = b hold (match.f90 header);
* H and O Hermitian, O positive definite;
* the IBS force (forcek) equals minus the derivative of
  sum_j w occ_j c_j^H (H - eps_j O) c_j with respect to the atomic position,
  by central finite differences of the oracle's own H and O.
"""
import numpy as np
import pytest
import scipy.linalg as sl
import scipy.special as sp

import lapw_oracle as O
from exciting_b200 import workloads as W
from exciting_b200.crystal import Crystal, gencfun


@pytest.mark.parametrize("x", [0.0, 1e-9, 1e-3, 0.3, 1.0, 2.5, 7.9, 10.5, 15.0, 40.0])
def test_sbessel_vs_scipy(x):
    jl = O.sbessel(12, x)
    ref = sp.spherical_jn(np.arange(13), x)
    scale = np.maximum(np.abs(ref), 1e-300)
    small = np.abs(ref) > 1e-280
    assert np.max(np.abs(jl - ref)[small] / scale[small]) < 1e-12


@pytest.mark.parametrize("x", [1e-4, 0.3, 0.99, 1.01, 3.0, 8.0])
def test_sbesseldm_first_derivative_vs_scipy(x):
    d = O.sbesseldm(1, 10, x)
    ref = sp.spherical_jn(np.arange(11), x, derivative=True)
    assert np.max(np.abs(d - ref)) < 1e-13


@pytest.mark.parametrize("x", [0.5, 2.0, 6.0])
def test_sbesseldm_second_derivative_by_recurrence(x):
    # j_l'' = j_{l-1}' - (l+1)/x j_l' + (l+1)/x^2 j_l
    d2 = O.sbesseldm(2, 9, x)
    n = np.arange(10)
    j = sp.spherical_jn(np.arange(11), x)
    dj = sp.spherical_jn(np.arange(11), x, derivative=True)
    ref = np.empty(10)
    ref[0] = -dj[1]
    ref[1:] = dj[:-2][: 9] - (n[1:] + 1) / x * dj[1:10] + (n[1:] + 1) / x ** 2 * j[1:10]
    assert np.max(np.abs(d2 - ref)) < 1e-12


@pytest.mark.parametrize("tp", [(0.0, 0.0), (0.7, 2.1), (np.pi / 2, 4.0), (3.0, 5.9)])
def test_genylm_vs_scipy(tp):
    y = O.genylm(10, tp)
    for l in range(11):
        for m in range(-l, l + 1):
            assert abs(y[l * (l + 1) + m] - sp.sph_harm_y(l, m, tp[0], tp[1])) < 1e-13


def test_polynom_derivatives():
    xa = np.array([1.9, 1.97, 2.03, 2.1])
    ya = 3.0 - xa + 0.5 * xa ** 2 - 0.25 * xa ** 3
    x = 2.1
    assert abs(O.polynom(0, xa, ya, x) - (3 - x + 0.5 * x * x - 0.25 * x ** 3)) < 1e-13
    assert abs(O.polynom(1, xa, ya, x) - (-1 + x - 0.75 * x * x)) < 1e-11
    assert abs(O.polynom(2, xa, ya, x) - (1 - 1.5 * x)) < 1e-8


@pytest.mark.parametrize("variant", ["shipped", "text"])
def test_match_solves_matching_conditions(variant):
    s = W.si_fcc(variant)
    gk = s.gkset(s.kpoints[4])
    a, nsing = O.match(s, gk)
    assert nsing == 0
    b = s.basis
    fpso = 4 * np.pi / np.sqrt(s.crystal.omega)
    sf = np.exp(1j * (gk.vgpc.T @ s.crystal.atposc))
    for ias in range(s.natmtot):
        for l in (0, 1, 3, 8):
            n = b.apword[0][l]
            d = np.array([[O.polynom(i, s.spr_tail[:, 0], s.apwfr_tail[:, j, l, ias], s.rmt[0])
                           for j in range(n)] for i in range(n)])
            for igp in (0, 7, gk.ngp - 1):
                djl = [O.sbesseldm(i, 8, gk.gpc[igp] * s.rmt[0])[l] * gk.gpc[igp] ** i for i in range(n)]
                y = O.genylm(8, gk.tpgpc[:, igp])
                for m in (-l, 0, l):
                    lm = l * (l + 1) + m
                    rhs = np.array(djl) * fpso * 1j ** l * sf[igp, ias] * np.conj(y[lm])
                    lhs = d @ a[igp, :n, lm, ias]
                    assert np.allclose(lhs, rhs, rtol=1e-12, atol=1e-14 * np.abs(rhs).max())


@pytest.mark.parametrize("rel", ["none", "zora", "iora*"])
def test_oracle_h_o_hermitian_and_o_definite(rel):
    s = W.si_fcc("text", relativity=rel)
    gk = s.gkset(s.kpoints[3])
    h, o = O.hamiltonandoverlapsetup(s, gk)
    assert h.shape == (gk.ngp + s.basis.nlotot,) * 2
    off = ~np.eye(h.shape[0], dtype=bool)
    assert np.array_equal(h[off], h.conj().T[off])            # copy_UL: exact mirror
    assert np.array_equal(o[off], o.conj().T[off])
    assert np.linalg.eigvalsh(o).min() > 0


def _energy(s, gk, c, eps, occ, wk):
    h, o = O.hamiltonandoverlapsetup(s, gk)
    return wk * sum(occ[j] * np.real(np.vdot(c[:, j], (h - eps[j] * o) @ c[:, j])) for j in range(c.shape[1]))


def _moved(s, ias, x, dx):
    """The same system with atom ias moved by dx along x (cfunig follows)."""
    import copy
    t = copy.copy(s)
    pos = s.crystal.atposl.copy()
    pos[:, ias] += np.linalg.solve(s.crystal.avec, np.eye(3)[x] * dx)
    t.crystal = Crystal(s.crystal.avec, s.crystal.species_rmt, s.crystal.atom_species, pos)
    t.cfunig = np.asfortranarray(gencfun(s.gv, s.crystal.species_rmt, s.crystal.atom_species,
                                         t.crystal.atposc, s.crystal.omega))
    return t


@pytest.mark.slow
def test_forcek_is_minus_energy_derivative():
    s = W.si_fcc("shipped", relativity="none")
    gk = s.gkset(s.kpoints[4])
    nmat = s.nmat(gk)
    rng = np.random.default_rng(3)
    nst = 12
    c, _ = np.linalg.qr(rng.standard_normal((nmat, nst)) + 1j * rng.standard_normal((nmat, nst)))
    eps = rng.uniform(-0.5, 0.5, nst)
    occ = np.full(nst, 2.0)
    wk = 0.375
    f = O.forcek(s, gk, c, eps, occ, wk)
    h = 1e-5
    for ias in range(s.natmtot):
        for x in range(3):
            ep = _energy(_moved(s, ias, x, +h), gk, c, eps, occ, wk)
            em = _energy(_moved(s, ias, x, -h), gk, c, eps, occ, wk)
            fd = -(ep - em) / (2 * h)
            assert abs(f[x, ias] - fd) < 1e-6 * max(1.0, abs(fd)), (ias, x, f[x, ias], fd)


def test_eigenvalues_of_oracle_system_are_finite():
    s = W.si_fcc("shipped")
    gk = s.gkset(s.kpoints[0])
    h, o = O.hamiltonandoverlapsetup(s, gk)
    w = sl.eigh(h, o, eigvals_only=True)
    assert np.all(np.isfinite(w))


def test_apw_block_equals_full_setup_block():
    """The sub-set oracle used at full sizes agrees with the full oracle."""
    from exciting_b200 import workloads as W
    s = W.si_fcc("shipped")
    gk = s.gkset(s.kpoints[2])
    h, o = O.hamiltonandoverlapsetup(s, gk)
    idx = np.sort(np.random.default_rng(0).choice(gk.ngp, 37, replace=False))
    hb, ob = O.apw_block(s, gk, idx)
    assert np.allclose(hb, h[np.ix_(idx, idx)], rtol=0, atol=1e-12 * np.abs(h).max())
    assert np.allclose(ob, o[np.ix_(idx, idx)], rtol=0, atol=1e-12 * np.abs(o).max())
