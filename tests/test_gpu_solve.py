"""Device eigen-solve after the setup (exs_setup_and_solve_batched): the
lowest nstfv eigenpairs of H x = e O x, as solvewithlapack's zhegvx range
IL = 1 .. IU = nstfv, against LAPACK on the oracle's H and O.
Bars: eigenvalues within an absolute 1e-8 Ha, residual
||H x - e O x|| <= 1e-9 ||H||, O-orthonormal vectors to 1e-10 plus what the
setup's own error allows: the vectors are orthonormal in the O the solver
was given, which differs from the oracle's by up to 1e-12 ||O|| (the setup
bar), so |x^H O_ref x - 1| may reach 1e-12 ||O||_2 ||x||^2."""
import numpy as np
import pytest
import scipy.linalg as sl

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _check(s, gks, ev, vec, nstfv):
    for k, gk in enumerate(gks):
        hr, orf = O.hamiltonandoverlapsetup(s, gk)
        n = hr.shape[0]
        wr = sl.eigh(hr, orf, eigvals_only=True, subset_by_index=[0, nstfv - 1])
        w = ev[:, k]
        assert np.max(np.abs(w - wr)) <= 1e-8, np.max(np.abs(w - wr))
        x = vec[:n, :, k]
        res = hr @ x - (orf @ x) * w[None, :]
        assert np.linalg.norm(res) <= 1e-9 * np.linalg.norm(hr) * np.sqrt(nstfv)
        g = x.conj().T @ orf @ x
        tol = 1e-10 + 1e-12 * np.linalg.norm(orf, 2) * np.max(np.sum(np.abs(x) ** 2, axis=0))
        assert np.max(np.abs(g - np.eye(nstfv))) <= tol


@pytest.mark.parametrize("variant", ["shipped", "text"])
def test_setup_and_solve_si_fcc(variant):
    from exciting_b200.fvsystem import Setup
    s = W.si_fcc(variant)
    gks = s.gksets()
    st = Setup(s, max_batch=len(gks))
    ev, vec = st.setup_and_solve(gks, 16)
    _check(s, gks, ev, vec, 16)


def test_setup_and_solve_cube8_split_precision():
    """The modular split precision (the benchmark's mode) with the default plan."""
    from exciting_b200.fvsystem import Setup
    s = W.si_cube8()
    gks = s.gksets()[:3]
    st = Setup(s, max_batch=3)
    st.set_precision("ozaki_mod", 0)
    ev, vec = st.setup_and_solve(gks, 40)
    _check(s, gks, ev, vec, 40)
