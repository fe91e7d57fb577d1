"""GPU IBS force (exs_forcek) and adjoint (exs_adjoint) through the C-ABI.

* exs_forcek against the oracle's literal restatement of forcek.f90 (the
  explicit dlh/dlo matrices and zgemm projections): |dF| <= 1e-10 Ha/bohr.
* exs_adjoint: dL/dtau = -F_IBS; dL/dV(G) and dL/dh_a against exact
  differences of L = sum_n w_n c_n^H (H - eps_n O) c_n computed from the
  GPU's own H and O (L is linear in V and h_a); dL/dtau against central
  finite differences with step 1e-5 Bohr, within 1e-6 Ha/bohr.
"""
import ctypes

import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W
from exciting_b200.crystal import Crystal, ffacg_species, gencfun

pytestmark = pytest.mark.gpu

TOL_F = 1e-10


def _setup(s, **kw):
    from exciting_b200.fvsystem import Setup
    return Setup(s, **kw)


def _states(nmat, nst, seed=3):
    rng = np.random.default_rng(seed)
    c, _ = np.linalg.qr(rng.standard_normal((nmat, nst)) + 1j * rng.standard_normal((nmat, nst)))
    eps = rng.uniform(-0.5, 0.5, nst)
    occ = np.full(nst, 2.0)
    return np.asfortranarray(c), eps, occ


@pytest.mark.parametrize("variant,rel,ik", [("shipped", "none", 4), ("text", "none", 1), ("text", "zora", 6),
                                            ("text", "iora*", 2)])
def test_forcek_vs_oracle(variant, rel, ik):
    s = W.si_fcc(variant, relativity=rel)
    st = _setup(s)
    gk = s.gkset(s.kpoints[ik])
    nmat = s.nmat(gk)
    c, eps, occ = _states(nmat, 16)
    wk = float(W.FCC_IRREDUCIBLE_4x4x4_WEIGHTS[ik])
    f_ref = O.forcek(s, gk, c, eps, occ, wk)
    f0 = np.full((3, s.natmtot), 0.25, order="F")            # forcek accumulates
    f = st.forcek(gk, c, eps, occ, wk, forceibs=f0.copy(order="F")) - f0
    assert np.max(np.abs(f - f_ref)) <= TOL_F, (f, f_ref)


def test_forcek_cube8_one_kpoint():
    s = W.si_cube8()
    st = _setup(s)
    gk = s.gkset(s.kpoints[7])
    c, eps, occ = _states(s.nmat(gk), 24, seed=5)
    f_ref = O.forcek(s, gk, c, eps, occ, 1.0 / 27)
    f = st.forcek(gk, c, eps, occ, 1.0 / 27)
    assert np.max(np.abs(f - f_ref)) <= TOL_F


def _adjoint(st, s, gk, c, w, eps):
    lib = st.lib
    ig, vg = st._gk_arrays(gk)
    ff = np.asfortranarray(np.stack([ffacg_species(s.gv.gc[: s.gv.ngvec], r, s.crystal.omega) for r in s.rmt], 1))
    vgc = np.asfortranarray(s.gv.vgc[:, : s.gv.ngvec])
    dtau = np.zeros((3, s.natmtot), order="F")
    dv = np.zeros(s.gv.ngvec, dtype=np.complex128)
    dh = np.zeros((st.maxaa, st.maxaa, s.natmtot), dtype=np.complex128, order="F")
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    c = np.asfortranarray(c)
    rc = lib.exs_adjoint(st.ctx, gk.ngp, p(ig), p(vg), c.shape[1], p(c), c.shape[0], p(np.ascontiguousarray(w)),
                         p(np.ascontiguousarray(eps)), p(ff), p(vgc), p(dtau), p(dv), p(dh))
    assert rc >= 0, lib.exs_last_error(st.ctx)
    return dtau, dv, dh


def _lfun(h, o, c, w, eps):
    return sum(w[j] * np.real(np.vdot(c[:, j], (h - eps[j] * o) @ c[:, j])) for j in range(c.shape[1]))


def test_adjoint_potential_and_mt_gradients_exact_differences():
    s = W.si_fcc("text")
    st = _setup(s)
    gk = s.gkset(s.kpoints[3])
    c, eps, _ = _states(s.nmat(gk), 10)
    w = np.linspace(0.5, 2.0, 10)
    dtau, dv, dh = _adjoint(st, s, gk, c, w, eps)
    h0, o0 = st.hamiltonandoverlapsetup(gk)
    L0 = _lfun(h0, o0, c, w, eps)
    # V(G): perturb a (G, -G) pair keeping V(-G) = conj V(G)
    gv = s.gv
    for ig in (1, 5, 40):
        mig = int(gv.ivgig_lookup(-gv.ivg[:, ig:ig + 1])[0]) - 1
        d = 1e-3 * (0.7 + 0.3j)
        s2 = W.si_fcc("text")
        s2.veffig = s.veffig.copy()
        s2.veffig[ig] += d
        s2.veffig[mig] += np.conj(d)
        st.set_scf_inputs(s2)
        h1, o1 = st.hamiltonandoverlapsetup(gk)
        dl = _lfun(h1, o1, c, w, eps) - L0
        pred = np.real(dv[ig] * d + dv[mig] * np.conj(d))
        assert abs(dl - pred) <= 1e-9 * max(1.0, abs(dl)), (ig, dl, pred)
    st.set_scf_inputs(s)
    # h_a: a Hermitian perturbation of one (f, f') pair of atom 1
    for (f1, f2) in ((0, 0), (3, 17), (40, 41)):
        s2 = W.si_fcc("text")
        d = 1e-3 * (0.2 - 0.9j) if f1 != f2 else 1e-3
        s2.mt_aa = s.mt_aa.copy(order="F")
        s2.mt_aa[f1, f2, 1] += d
        if f1 != f2:
            s2.mt_aa[f2, f1, 1] += np.conj(d)
        st.set_scf_inputs(s2)
        h1, o1 = st.hamiltonandoverlapsetup(gk)
        dl = _lfun(h1, o1, c, w, eps) - L0
        pred = np.real(dh[f1, f2, 1] * d + (dh[f2, f1, 1] * np.conj(d) if f1 != f2 else 0.0))
        assert abs(dl - pred) <= 1e-9 * max(1.0, abs(dl)), ((f1, f2), dl, pred)
    st.set_scf_inputs(s)


def _moved(s, ias, x, dx):
    import copy
    t = copy.copy(s)
    pos = s.crystal.atposl.copy()
    pos[:, ias] += np.linalg.solve(s.crystal.avec, np.eye(3)[x] * dx)
    t.crystal = Crystal(s.crystal.avec, s.crystal.species_rmt, s.crystal.atom_species, pos)
    t.cfunig = np.asfortranarray(gencfun(s.gv, s.crystal.species_rmt, s.crystal.atom_species,
                                         t.crystal.atposc, s.crystal.omega))
    return t


def test_adjoint_positions_central_differences():
    s = W.si_fcc("shipped")
    st = _setup(s)
    gk = s.gkset(s.kpoints[5])
    c, eps, _ = _states(s.nmat(gk), 12, seed=9)
    w = np.full(12, 2.0)
    dtau, _, _ = _adjoint(st, s, gk, c, w, eps)
    h = 1e-5
    for ias in range(s.natmtot):
        for x in range(3):
            lp = _lfun(*_setup(_moved(s, ias, x, +h)).hamiltonandoverlapsetup(gk), c, w, eps)
            lm = _lfun(*_setup(_moved(s, ias, x, -h)).hamiltonandoverlapsetup(gk), c, w, eps)
            fd = (lp - lm) / (2 * h)
            assert abs(dtau[x, ias] - fd) <= 1e-6, (ias, x, dtau[x, ias], fd)
