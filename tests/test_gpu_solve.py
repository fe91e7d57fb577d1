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


def test_solve_values_only_matches_the_vector_solve():
    """exs_solve_batched_device with evecfv = NULL (values only, the form used
    for nmat of tens of thousands) gives the eigenvalues of the vector solve."""
    import ctypes

    import torch

    from exciting_b200.fvsystem import Setup
    s = W.si_fcc("text")
    gks = s.gksets()[:2]
    st = Setup(s, max_batch=2)
    ev_ref, _ = st.setup_and_solve(gks, 12)
    nmat = [g.ngp + st.nlotot for g in gks]
    ig = np.zeros((2, st.ngkmax), dtype=np.int32)
    vg = np.zeros((2, st.ngkmax, 3))
    for k, g in enumerate(gks):
        ig[k, : g.ngp] = g.igpig
        vg[k, : g.ngp] = g.vgpc.T
    d_ig, d_vg = torch.from_numpy(ig).cuda(), torch.from_numpy(vg).cuda()
    d_h = [torch.zeros(2 * m * m, dtype=torch.float64, device="cuda") for m in nmat]
    d_o = [torch.zeros(2 * m * m, dtype=torch.float64, device="cuda") for m in nmat]
    st.setup_batched_device([g.ngp for g in gks], d_ig.data_ptr(), d_vg.data_ptr(), [t.data_ptr() for t in d_h],
                            [t.data_ptr() for t in d_o])
    st.synchronize()
    ev = torch.zeros(12 * 2, dtype=torch.float64, device="cuda")
    hp = (ctypes.c_void_p * 2)(*[t.data_ptr() for t in d_h])
    op = (ctypes.c_void_p * 2)(*[t.data_ptr() for t in d_o])
    st._check(st.lib.exs_solve_batched_device(st.ctx, 2, (ctypes.c_int * 2)(*nmat), hp, op, 12,
                                              ctypes.c_void_p(ev.data_ptr()), None, 0))
    w = ev.cpu().numpy().reshape(2, 12).T
    assert np.max(np.abs(w - ev_ref)) <= 1e-10
    st.close()
