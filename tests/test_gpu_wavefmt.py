"""Muffin-tin wavefunction coefficients (exs_wavefmt), the consumer of the
matching coefficients that rhovalk.f90:119-142 and gendmatmt.f90 call after
match, against the oracle's restatement of src/wavefmt.f90 for every atom
and state, through the C-ABI.

Tolerance: max |d wfmt| <= 1e-12 max |wfmt| per case.  The G sums run in
another order (one ZGEMM) and the reference skips constants below 1e-14
(wavefmt_add), so the results agree to FP64 rounding, not bit for bit.
"""
import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _states(nmat, nst, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((nmat, nst)) + 1j * rng.standard_normal((nmat, nst)))


def _check(s, ik, lrstp, lmax, nst=5, seed=7):
    from exciting_b200.fvsystem import Setup
    rad = W.mt_radial(s)
    gk = s.gkset(s.kpoints[ik])
    st = Setup(s)
    apwalm, _ = st.match(gk)
    ev = _states(s.nmat(gk), nst, seed)
    ld = (lmax + 1) ** 2 + 3                     # a leading dimension above (lmax+1)^2: padding rows stay zero
    got = st.wavefmt(gk, apwalm, ev, rad, lrstp=lrstp, lmax=lmax, ld=ld)
    st.close()
    scale = 0.0
    worst = 0.0
    for ias in range(s.natmtot):
        for j in range(nst):
            ref = O.wavefmt(s, rad, lrstp, lmax, ias, gk.ngp, apwalm, ev[:, j], ld)
            nr = ref.shape[1]
            worst = max(worst, np.abs(got[:, :nr, ias, j] - ref).max())
            scale = max(scale, np.abs(ref).max())
            assert np.all(got[:, nr:, ias, j] == 0)
    assert worst <= TOL * scale, worst / scale


@pytest.mark.parametrize("variant,ik,lrstp,lmax", [("shipped", 0, 1, 8), ("shipped", 3, 2, 4), ("text", 5, 1, 2)])
def test_wavefmt_vs_oracle_fcc(variant, ik, lrstp, lmax):
    _check(W.si_fcc(variant), ik, lrstp, lmax)


def test_wavefmt_vs_oracle_cube8():
    """8 atoms, lmaxapw 10, 3 lo per l <= 2 (lo rows through idxlo)."""
    _check(W.si_cube8(), 1, 3, 10, nst=3)


def test_wavefmt_argument_errors():
    from exciting_b200.abi import ExsError
    from exciting_b200.fvsystem import Setup
    s = W.si_fcc("shipped")
    rad = W.mt_radial(s)
    gk = s.gkset(s.kpoints[0])
    st = Setup(s)
    apwalm, _ = st.match(gk)
    ev = _states(s.nmat(gk), 2, 1)
    with pytest.raises(ExsError):                 # lmax > lmaxapw: the reference stops
        st.wavefmt(gk, apwalm, ev, rad, lmax=s.basis.lmaxapw + 1)
    with pytest.raises(ExsError):                 # ld below (lmax + 1)^2
        st.wavefmt(gk, apwalm, ev, rad, lmax=4, ld=20)
    with pytest.raises(ExsError):
        st.wavefmt(gk, apwalm, ev, rad, lrstp=0)
    st.close()
