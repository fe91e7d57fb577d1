"""GPU parity of the real-time TDDFT Hamiltonian update (UpdateHam's k-loop,
src/src_xs/src_rttddft/rttddft_hamiltonianoverlap.f90:40-106) against the
oracle, through the C-ABI.

Tolerance: ||d ham||_F / ||ham||_F <= 1e-12 (the setup's bar; the combination
itself is element-wise FP64).  pmat: seeded Hermitian matrices, the vector
potential of the order of a laser pulse's (|A|/c ~ 1e-2).
"""
import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _setup(s, **kw):
    from exciting_b200.fvsystem import Setup
    return Setup(s, **kw)


def _pmat(n, seed):
    rng = np.random.default_rng(seed)
    p = np.zeros((n, n, 3), dtype=np.complex128, order="F")
    for i in range(3):
        z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        p[:, :, i] = 0.5 * (z + z.conj().T)
    return p


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("variant,relativity", [("shipped", "none"), ("text", "iora*")])
def test_updateham_vs_oracle(variant, relativity):
    s = W.si_fcc(variant, relativity=relativity)
    gks = s.gksets()[:3]
    st = _setup(s, max_batch=len(gks))
    pm = [_pmat(g.ngp + st.nlotot, 10 + k) for k, g in enumerate(gks)]
    st.rttddft_set_pmat(pm)
    atot = np.array([1.3, -0.4, 0.8])
    ham, ovl = st.rttddft_updateham(gks, atot, calculate_overlap=True)
    for k, g in enumerate(gks):
        hr, orf = O.rttddft_updateham(s, g, atot, pm[k])
        assert rel(ham[k], hr) <= 1e-12, rel(ham[k], hr)
        assert rel(ovl[k], orf) <= 1e-12, rel(ovl[k], orf)


def test_updateham_with_a_kept_overlap():
    """calculate_overlap = 0: the given overlap enters the sum, and is not overwritten."""
    s = W.si_fcc("shipped")
    gks = s.gksets()[3:5]
    st = _setup(s, max_batch=len(gks))
    pm = [_pmat(g.ngp + st.nlotot, 20 + k) for k, g in enumerate(gks)]
    st.rttddft_set_pmat(pm)
    atot = np.array([0.0, 2.0, -1.0])
    rng = np.random.default_rng(3)
    kept = []
    for g in gks:
        n = g.ngp + st.nlotot
        z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        kept.append(np.asfortranarray(z + z.conj().T))
    ham, ovl = st.rttddft_updateham(gks, atot, calculate_overlap=False, overlap=kept)
    for k, g in enumerate(gks):
        hr, _ = O.rttddft_updateham(s, g, atot, pm[k], overlap=kept[k])
        assert rel(ham[k], hr) <= 1e-12
        assert np.array_equal(ovl[k], kept[k])


def test_zero_field_gives_the_groundstate_hamiltonian():
    s = W.si_fcc("text")
    gks = s.gksets()[:2]
    st = _setup(s, max_batch=len(gks))
    st.rttddft_set_pmat([_pmat(g.ngp + st.nlotot, k) for k, g in enumerate(gks)])
    ham, ovl = st.rttddft_updateham(gks, np.zeros(3))
    ref = st.setup_batched(gks)
    for k in range(len(gks)):
        assert np.array_equal(ham[k], ref[k][0]) and np.array_equal(ovl[k], ref[k][1])


def test_device_entry_equals_host_entry():
    import torch
    s = W.si_fcc("shipped")
    gks = s.gksets()[:2]
    st = _setup(s, max_batch=len(gks))
    pm = [_pmat(g.ngp + st.nlotot, 30 + k) for k, g in enumerate(gks)]
    st.rttddft_set_pmat(pm)
    atot = np.array([0.7, 0.1, -2.2])
    ham, ovl = st.rttddft_updateham(gks, atot)
    ngp, ig, vg = st._k_arrays(gks)
    d_ig = torch.from_numpy(ig.ravel(order="F")).cuda()
    d_vg = torch.from_numpy(vg.ravel(order="F")).cuda()
    d_p = [torch.from_numpy(np.asfortranarray(p).ravel(order="F").view(np.float64)).cuda() for p in pm]
    nm = [g.ngp + st.nlotot for g in gks]
    d_h = [torch.zeros(2 * n * n, dtype=torch.float64, device="cuda") for n in nm]
    d_o = [torch.zeros(2 * n * n, dtype=torch.float64, device="cuda") for n in nm]
    torch.cuda.synchronize()
    st.rttddft_updateham_device(ngp, d_ig.data_ptr(), d_vg.data_ptr(), atot, True, [p.data_ptr() for p in d_p],
                                [h.data_ptr() for h in d_h], [o.data_ptr() for o in d_o])
    st.synchronize()
    for k, n in enumerate(nm):
        h = d_h[k].cpu().numpy().view(np.complex128).reshape(n, n, order="F")
        o = d_o[k].cpu().numpy().view(np.complex128).reshape(n, n, order="F")
        assert np.array_equal(h, ham[k]) and np.array_equal(o, ovl[k])


@pytest.mark.parametrize("variant", ["shipped", "text", "two_species"])
def test_genpmat_vs_oracle(variant):
    """Momentum matrices on the device (exs_rttddft_genpmat) against the
    oracle's pmatrad + genpmatbasisik, same matching coefficients; the
    two-species cell has different bases per species, lmaxmat < lmaxapw and
    radial meshes of 300 and 250 points."""
    if variant == "two_species":
        s = W.sic_two_species()
        rad = W.mt_radial(s, lmaxvr=2, nrmt=[300, 250])
    else:
        s = W.si_fcc(variant)
        rad = W.mt_radial(s, lmaxvr=2)
    gks = s.gksets()[:2]
    st = _setup(s, max_batch=len(gks))
    al = [st.match(g)[0] for g in gks]
    pm = st.rttddft_genpmat(gks, al, rad)
    rip = O.pmatrad(s, rad)
    for k, g in enumerate(gks):
        ref = O.genpmatbasisik(s, g, al[k], rip)
        for j in range(3):
            assert rel(pm[k][:, :, j], ref[:, :, j]) <= 1e-12, (k, j, rel(pm[k][:, :, j], ref[:, :, j]))
    # the registered matrices drive the update
    atot = np.array([0.4, -1.1, 0.9])
    ham, _ = st.rttddft_updateham(gks, atot)
    for k, g in enumerate(gks):
        hr, _ = O.rttddft_updateham(s, g, atot, O.genpmatbasisik(s, g, al[k], rip))
        assert rel(ham[k], hr) <= 1e-12


def test_rttddft_argument_errors():
    """The update without registered momentum matrices, a batch above
    max_batch and mismatched sizes are rejected; the context stays usable."""
    from exciting_b200.abi import ExsError
    s = W.si_fcc("shipped")
    gks = s.gksets()[:3]
    st = _setup(s, max_batch=2)
    with pytest.raises(ExsError):
        st.rttddft_updateham(gks[:2], np.zeros(3))           # nothing registered yet
    with pytest.raises(ExsError):
        st.rttddft_set_pmat([_pmat(g.ngp + st.nlotot, 0) for g in gks])   # 3 > max_batch
    st.rttddft_set_pmat([_pmat(g.ngp + st.nlotot, 0) for g in gks[:2]])
    with pytest.raises(ExsError):
        st.rttddft_updateham([gks[1], gks[0]], np.zeros(3))  # nmat differs from the registered one
    ham, _ = st.rttddft_updateham(gks[:2], np.zeros(3))
    ref = st.setup_batched(gks[:2])
    assert np.array_equal(ham[0], ref[0][0])
