"""GPU parity of the H/O setup against the FP64 CPU oracle, through the C-ABI.

Tolerances: ||dH||_F/||H||_F <= 1e-12 and ||dO||_F/||O||_F <= 1e-12 (FP64
path), eigenvalues of H x = e O x within 1e-8 Ha, matching coefficients within
1e-12 of max|A|.  The APW-APW off-diagonal mirror must be exact (copy_UL).
"""
import numpy as np
import pytest
import scipy.linalg as sl

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FRO = 1e-12
TOL_EIG = 1e-8


def rel_fro(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _setup(sys_, **kw):
    from exciting_b200.fvsystem import Setup
    return Setup(sys_, **kw)


def _check_pair(h, o, hr, orf, eig=True):
    assert rel_fro(h, hr) <= TOL_FRO, rel_fro(h, hr)
    assert rel_fro(o, orf) <= TOL_FRO, rel_fro(o, orf)
    off = ~np.eye(h.shape[0], dtype=bool)
    assert np.array_equal(h[off], h.conj().T[off])
    assert np.array_equal(o[off], o.conj().T[off])
    if eig:
        w = sl.eigh(h, o, eigvals_only=True)
        wr = sl.eigh(hr, orf, eigvals_only=True)
        assert np.max(np.abs(w - wr)) <= TOL_EIG


@pytest.mark.parametrize("variant", ["shipped", "text"])
def test_match_vs_oracle(variant):
    s = W.si_fcc(variant)
    st = _setup(s)
    for ik in (0, 4, 7):
        gk = s.gkset(s.kpoints[ik])
        a, rc = st.match(gk)
        ar, _ = O.match(s, gk, ngkmax=st.ngkmax)
        assert rc == 0
        scale = np.abs(ar).max()
        assert np.abs(a[: gk.ngp] - ar[: gk.ngp]).max() <= 1e-12 * scale


def test_match_cube8_lmax10():
    s = W.si_cube8()
    st = _setup(s)
    gk = s.gkset(s.kpoints[5])
    a, _ = st.match(gk)
    ar, _ = O.match(s, gk, ngkmax=st.ngkmax)
    assert np.abs(a[: gk.ngp] - ar[: gk.ngp]).max() <= 1e-12 * np.abs(ar).max()


@pytest.mark.parametrize("variant", ["shipped", "text"])
def test_setup_all_kpoints_vs_oracle(variant):
    s = W.si_fcc(variant)
    st = _setup(s)
    for gk in s.gksets():
        h, o = st.hamiltonandoverlapsetup(gk)
        hr, orf = O.hamiltonandoverlapsetup(s, gk)
        _check_pair(h, o, hr, orf)


@pytest.mark.parametrize("rel", ["zora", "iora*"])
def test_setup_relativity_vs_oracle(rel):
    s = W.si_fcc("text", relativity=rel)
    st = _setup(s)
    for ik in (1, 6):
        gk = s.gkset(s.kpoints[ik])
        h, o = st.hamiltonandoverlapsetup(gk)
        hr, orf = O.hamiltonandoverlapsetup(s, gk)
        _check_pair(h, o, hr, orf)


def test_setup_with_caller_apwalm():
    s = W.si_fcc("shipped")
    st = _setup(s)
    gk = s.gkset(s.kpoints[2])
    ar, _ = O.match(s, gk, ngkmax=st.ngkmax)
    h, o = st.hamiltonandoverlapsetup(gk, apwalm=ar)
    hr, orf = O.hamiltonandoverlapsetup(s, gk, apwalm=ar)
    _check_pair(h, o, hr, orf)


def test_batched_cube8_all_kpoints():
    s = W.si_cube8()
    gks = s.gksets()
    st = _setup(s, max_batch=len(gks))
    out = st.setup_batched(gks)
    for ik in (0, 13, 26):
        hr, orf = O.hamiltonandoverlapsetup(s, gks[ik])
        _check_pair(out[ik][0], out[ik][1], hr, orf, eig=(ik == 13))
    for h, o in out:
        off = ~np.eye(h.shape[0], dtype=bool)
        assert np.array_equal(h[off], h.conj().T[off])


def test_batched_in_chunks_matches_single_calls():
    s = W.si_fcc("text")
    gks = s.gksets()
    st = _setup(s, max_batch=3)                    # 8 k-points in chunks of 3
    out = st.setup_batched(gks)
    for ik, gk in enumerate(gks):
        h, o = st.hamiltonandoverlapsetup(gk)
        assert rel_fro(out[ik][0], h) <= 1e-14 and rel_fro(out[ik][1], o) <= 1e-14


def test_errors_are_reported():
    import ctypes
    s = W.si_fcc("shipped")
    st = _setup(s)
    n = st.ngkmax + 1
    ig = np.ones(n, dtype=np.int32)
    vg = np.zeros((3, n), order="F")
    h = np.zeros((n + st.nlotot, n + st.nlotot), dtype=np.complex128, order="F")
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    # ngp above ngkmax -> EXS_ERR_SIZE
    assert st.lib.exs_hamiltonandoverlapsetup(st.ctx, n, None, p(ig), p(vg), p(h), p(h)) == -3
    # an igpig entry outside 1..ngrtot -> EXS_ERR_INDEX
    ig[3] = s.gv.ngrtot + 5
    assert st.lib.exs_hamiltonandoverlapsetup(st.ctx, n - 1, None, p(ig), p(vg), p(h), p(h)) == -4
    # null output
    assert st.lib.exs_hamiltonandoverlapsetup(st.ctx, 4, None, p(ig), p(vg), None, p(h)) == -1


def test_singular_matching_system_warns_and_keeps_rhs():
    s = W.si_fcc("text")
    s.apwfr_tail[:, 1, 3, 0] = 0.0          # u_2 = 0 for l = 3, atom 1: D_3 exactly singular
    st = _setup(s)
    gk = s.gkset(s.kpoints[3])
    a, rc = st.match(gk)
    ar, nsing = O.match(s, gk, ngkmax=st.ngkmax)
    assert nsing > 0 and rc == 1
    assert np.abs(a[: gk.ngp] - ar[: gk.ngp]).max() <= 1e-12 * np.abs(ar).max()


def test_host_copy_modes_identical():
    """Direct, packed and upper-part transfers of H/O (pinned and pageable outputs) give the same bits."""
    import torch
    s = W.si_cube8()
    gks = s.gksets()[:9]
    st = _setup(s, max_batch=9)
    outs = {}
    for mode in ("direct", "packed", "auto"):
        st.set_host_copy_mode(mode)
        outs[mode] = st.setup_batched(gks)
    for k in range(9):
        for w in range(2):
            assert np.array_equal(outs["direct"][k][w], outs["packed"][k][w])
            assert np.array_equal(outs["direct"][k][w], outs["auto"][k][w])
    hr, orf = O.hamiltonandoverlapsetup(s, gks[4])
    _check_pair(outs["packed"][4][0], outs["packed"][4][1], hr, orf, eig=False)
    # pinned outputs through the packed path
    nmat = [g.ngp + st.nlotot for g in gks]
    pin = [(torch.empty((m, m), dtype=torch.complex128).pin_memory(),
            torch.empty((m, m), dtype=torch.complex128).pin_memory()) for m in nmat]
    for mode in ("packed", "upper"):
        st.set_host_copy_mode(mode)
        for a, b in pin:
            a.fill_(float("nan"))
            b.fill_(float("nan"))
        got = st.setup_batched(gks, out=[(a.numpy().T, b.numpy().T) for a, b in pin])
        for k in range(9):
            assert np.array_equal(got[k][0], outs["direct"][k][0]), mode
            assert np.array_equal(got[k][1], outs["direct"][k][1]), mode
    # the upper-part transfer into pageable memory as well
    st.set_host_copy_mode("upper")
    up = st.setup_batched(gks)
    for k in range(9):
        for w in range(2):
            assert np.array_equal(up[k][w], outs["direct"][k][w])
