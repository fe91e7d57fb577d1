"""The adjoint of the setup (exs_adjoint) on the benchmark's force-check recipe.

Recipe (the adjoint/force configuration): 40 seeded random orthonormal
complex vectors c_n of length nmat (QR of a Gaussian, seed 3), occupations
w_n = 2 and eps_n uniform in [-0.5, 0.5] Ha, so that
dL/dH = sum_n w_n c_n c_n^H and dL/dO = -sum_n w_n eps_n c_n c_n^H, i.e.
L = sum_n w_n c_n^H (H - eps_n O) c_n.  Checks:

* dL/dtau against central finite differences of L (step 1e-5 Bohr) within
  1e-6 Ha/bohr, on the 2-atom cell (2 x 3 gradients) and on the 8-atom cell
  (8 x 3 gradients), L from the GPU's own H and O;
* dL/dtau = -F_IBS against the oracle's literal restatement of forcek.f90
  (the explicit dlh/dlo matrices, src/forcek.f90:262-383) with the same
  states, 1e-10 Ha/bohr;
* the adjoint wrapped in a torch.autograd.Function (here, in the test
  harness only): L.backward() gives the positions' gradient, which must equal
  exs_adjoint's and the finite differences of the wrapped forward.
"""
import copy
import ctypes

import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W
from exciting_b200.crystal import Crystal, ffacg_species, gencfun

pytestmark = pytest.mark.gpu

NST = 40
STEP = 1e-5        # Bohr
TOL_FD = 1e-6      # Ha/bohr
TOL_F = 1e-10


def recipe(nmat, seed=3):
    """40 orthonormal complex vectors (QR of a Gaussian), w = 2, eps ~ U[-0.5, 0.5]."""
    rng = np.random.default_rng(seed)
    c, _ = np.linalg.qr(rng.standard_normal((nmat, NST)) + 1j * rng.standard_normal((nmat, NST)))
    eps = rng.uniform(-0.5, 0.5, NST)
    return np.asfortranarray(c), np.full(NST, 2.0), eps


def setup(s):
    from exciting_b200.fvsystem import Setup
    return Setup(s)


def adjoint(st, s, gk, c, w, eps):
    ig, vg = st._gk_arrays(gk)
    ff = np.asfortranarray(np.stack([ffacg_species(s.gv.gc[: s.gv.ngvec], r, s.crystal.omega) for r in s.rmt], 1))
    vgc = np.asfortranarray(s.gv.vgc[:, : s.gv.ngvec])
    dtau = np.zeros((3, s.natmtot), order="F")
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    rc = st.lib.exs_adjoint(st.ctx, gk.ngp, p(ig), p(vg), c.shape[1], p(c), c.shape[0], p(np.ascontiguousarray(w)),
                            p(np.ascontiguousarray(eps)), p(ff), p(vgc), p(dtau), None, None)
    assert rc >= 0, st.lib.exs_last_error(st.ctx)
    return dtau


def lfun(h, o, c, w, eps):
    return sum(w[j] * np.real(np.vdot(c[:, j], (h - eps[j] * o) @ c[:, j])) for j in range(c.shape[1]))


def moved(s, pos_cart):
    """The system with atoms at the Cartesian positions pos_cart (3, natmtot):
    the structure factors follow from the positions, the step function is
    rebuilt (gencfun); the MT integrals and V(G) stay as they are."""
    t = copy.copy(s)
    atposl = np.linalg.solve(s.crystal.avec, pos_cart)
    t.crystal = Crystal(s.crystal.avec, s.crystal.species_rmt, s.crystal.atom_species, atposl)
    t.cfunig = np.asfortranarray(gencfun(s.gv, s.crystal.species_rmt, s.crystal.atom_species,
                                         t.crystal.atposc, s.crystal.omega))
    return t


def l_at(s, gk, pos_cart, c, w, eps):
    st = setup(moved(s, pos_cart))
    h, o = st.hamiltonandoverlapsetup(gk)
    st.close()
    return lfun(h, o, c, w, eps)


def central_differences(s, gk, c, w, eps):
    pos = np.array(s.crystal.atposc, dtype=np.float64)
    fd = np.zeros_like(pos)
    for ias in range(s.natmtot):
        for x in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[x, ias] += STEP
            pm[x, ias] -= STEP
            fd[x, ias] = (l_at(s, gk, pp, c, w, eps) - l_at(s, gk, pm, c, w, eps)) / (2 * STEP)
    return fd


@pytest.mark.parametrize("cell,ik", [("fcc2", 5), ("cube8", 0)])
def test_adjoint_positions_central_differences(cell, ik):
    s = W.si_fcc("text") if cell == "fcc2" else W.si_cube8()
    gk = s.gkset(s.kpoints[ik])
    c, w, eps = recipe(s.nmat(gk))
    st = setup(s)
    dtau = adjoint(st, s, gk, c, w, eps)
    st.close()
    fd = central_differences(s, gk, c, w, eps)
    assert np.max(np.abs(dtau - fd)) <= TOL_FD, np.max(np.abs(dtau - fd))


def test_adjoint_is_minus_the_reference_forcek():
    """dL/dtau = -F_IBS with the forcek weights w_n = wkpt occ_n (wkpt = 1)."""
    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[2])
    c, w, eps = recipe(s.nmat(gk))
    st = setup(s)
    dtau = adjoint(st, s, gk, c, w, eps)
    st.close()
    f_ref = O.forcek(s, gk, c, eps, w, 1.0)
    assert np.max(np.abs(dtau + f_ref)) <= TOL_F


def test_adjoint_autograd_function():
    import torch

    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[5])
    c, w, eps = recipe(s.nmat(gk))

    class SetupLoss(torch.autograd.Function):
        """L(tau) = sum_n w_n c_n^H (H(tau) - eps_n O(tau)) c_n through the
        device setup; its backward is the device adjoint dL/dtau."""

        @staticmethod
        def forward(ctx, tau):
            pos = tau.detach().cpu().numpy().reshape(3, s.natmtot, order="F")
            sm = moved(s, pos)
            st = setup(sm)
            h, o = st.hamiltonandoverlapsetup(gk)
            g = adjoint(st, sm, gk, c, w, eps)
            st.close()
            ctx.save_for_backward(torch.from_numpy(g.reshape(-1, order="F").copy()))
            return torch.tensor(lfun(h, o, c, w, eps), dtype=torch.float64)

        @staticmethod
        def backward(ctx, gl):
            (g,) = ctx.saved_tensors
            return gl * g

    pos0 = np.array(s.crystal.atposc, dtype=np.float64)
    tau = torch.tensor(pos0.reshape(-1, order="F"), dtype=torch.float64, requires_grad=True)
    loss = SetupLoss.apply(tau)
    loss.backward()
    grad = tau.grad.numpy().reshape(3, s.natmtot, order="F")
    st = setup(s)
    direct = adjoint(st, s, gk, c, w, eps)
    st.close()
    # the same quantity up to the forward's rebuilt positions (lattice coordinates from Cartesian
    # ones) and the order of the scatter's atomic additions
    assert np.max(np.abs(grad - direct)) <= TOL_F
    # finite differences through the wrapped forward
    for ias, x in ((0, 0), (1, 2)):
        e = np.zeros(3 * s.natmtot)
        e[x + 3 * ias] = STEP
        lp = float(SetupLoss.apply(torch.tensor(pos0.reshape(-1, order="F") + e)))
        lm = float(SetupLoss.apply(torch.tensor(pos0.reshape(-1, order="F") - e)))
        assert abs((lp - lm) / (2 * STEP) - grad[x, ias]) <= TOL_FD
