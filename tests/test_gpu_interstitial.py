"""Stand-alone interstitial gather (exs_hmlistln / exs_olpistln) against the
oracle's restatement of hmlistln.f90 / olpistln.f90: both ADD to the upper
triangle of an existing za and leave the lower triangle alone.  Integer
indexing (ivgig lookup) must pick the same G - G' everywhere; the values
agree to rounding (1e-14 of max|za|)."""
import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _za(n, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))


@pytest.mark.parametrize("variant,rel", [("text", "none"), ("shipped", "zora"), ("text", "iora*")])
def test_hmlistln_olpistln_vs_oracle(variant, rel):
    from exciting_b200.fvsystem import Setup
    s = W.si_fcc(variant, relativity=rel)
    st = Setup(s)
    for ik in (0, 4):
        gk = s.gkset(s.kpoints[ik])
        n = s.nmat(gk)
        h0, o0 = _za(n, ik), _za(n, 100 + ik)
        h, o = h0.copy(order="F"), o0.copy(order="F")
        st.hmlistln(gk, h)
        st.olpistln(gk, o)
        hr, orf = h0.copy(order="F"), o0.copy(order="F")
        O._interstitial(s, gk, hr, None)
        O._interstitial(s, gk, None, orf)
        for got, ref, base in ((h, hr, h0), (o, orf, o0)):
            assert np.max(np.abs(got - ref)) <= 1e-14 * np.abs(ref).max()
            low = np.tril(np.ones((n, n), dtype=bool), -1)
            assert np.array_equal(got[low], base[low])            # lower triangle untouched
            assert not np.array_equal(got[: gk.ngp, : gk.ngp], base[: gk.ngp, : gk.ngp])


def test_device_form_both_blocks():
    import torch
    from exciting_b200.fvsystem import Setup
    s = W.si_cube8()
    st = Setup(s)
    gk = s.gkset(s.kpoints[5])
    n = s.nmat(gk)
    h0, o0 = _za(n, 7), _za(n, 8)
    hr, orf = h0.copy(order="F"), o0.copy(order="F")
    O._interstitial(s, gk, hr, None)
    O._interstitial(s, gk, None, orf)
    ig, vg = st._gk_arrays(gk)
    d_ig = torch.from_numpy(ig).cuda()
    d_vg = torch.from_numpy(np.ascontiguousarray(vg.T)).cuda()
    d_h = torch.from_numpy(h0.T.copy().view(np.float64)).cuda()       # column-major complex as rows of the transpose
    d_o = torch.from_numpy(o0.T.copy().view(np.float64)).cuda()
    st.interstitial_device(3, gk.ngp, d_ig.data_ptr(), d_vg.data_ptr(), d_h.data_ptr(), d_o.data_ptr(), n)
    st.synchronize()
    h = d_h.cpu().numpy().view(np.complex128).T
    o = d_o.cpu().numpy().view(np.complex128).T
    assert np.max(np.abs(h - hr)) <= 1e-14 * np.abs(hr).max()
    assert np.max(np.abs(o - orf)) <= 1e-14 * np.abs(orf).max()
