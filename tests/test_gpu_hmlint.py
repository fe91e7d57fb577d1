"""GPU parity of the muffin-tin integral generation (exs_hmlint) against the
oracle's restatement of hmlint = mt_kin + mt_pot, through the C-ABI.

Tolerance: max |d aa| <= 1e-12 max |aa| (likewise loa, lolo with the scale
of aa): the device applies the spline integral as a weight vector and sums
in another order than one fderiv call per product, so results agree to FP64
rounding, not bit for bit.  The integrals the call installs must then drive
the setup exactly as the same arrays uploaded by exs_set_scf_inputs.
"""
import copy

import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _setup(s, **kw):
    from exciting_b200.fvsystem import Setup
    return Setup(s, **kw)


def _check(got, ref):
    aa, loa, lolo = got
    ar, lr, llr = ref
    scale = np.abs(ar).max()
    assert np.abs(aa - ar).max() <= TOL * scale, np.abs(aa - ar).max() / scale
    assert np.abs(loa - lr).max() <= TOL * scale, np.abs(loa - lr).max() / scale
    assert np.abs(lolo - llr).max() <= TOL * scale, np.abs(lolo - llr).max() / scale


@pytest.mark.parametrize("variant,relativity,lmaxvr", [("shipped", "none", 8), ("text", "zora", 6),
                                                       ("text", "none", 0)])
def test_hmlint_vs_oracle_fcc(variant, relativity, lmaxvr):
    s = W.si_fcc(variant, relativity=relativity)
    rad = W.mt_radial(s, lmaxvr=lmaxvr)
    st = _setup(s)
    _check(st.hmlint(rad), O.hmlint(s, rad))


def test_hmlint_vs_oracle_two_species_ragged_meshes():
    """Different bases per species, lmaxmat < lmaxapw, nrmt 300 / 250 padded to 320."""
    s = W.sic_two_species()
    rad = W.mt_radial(s, nrmt=[300, 250], nrmtmax=320)
    st = _setup(s)
    _check(st.hmlint(rad), O.hmlint(s, rad))
    # a new mesh and a new lmaxvr on the same context rebuild weights and Gaunt list
    rad2 = W.mt_radial(s, nrmt=[280, 310], lmaxvr=4, seed=5)
    _check(st.hmlint(rad2), O.hmlint(s, rad2))


@pytest.mark.slow
def test_hmlint_vs_oracle_cube8():
    s = W.si_cube8()
    rad = W.mt_radial(s)
    st = _setup(s)
    _check(st.hmlint(rad), O.hmlint(s, rad))


def test_hmlint_device_entry_equals_host_entry():
    import torch
    s = W.si_fcc("text")
    rad = W.mt_radial(s)
    st = _setup(s)
    ref = st.hmlint(rad)
    dev = {k: torch.from_numpy(np.asfortranarray(getattr(rad, k)).ravel(order="F")).cuda()
           for k in ("apwfr", "lofr", "veffmt")}
    torch.cuda.synchronize()                     # the copies ran on torch's stream
    st.hmlint_device(rad, dev["apwfr"].data_ptr(), dev["lofr"].data_ptr(), dev["veffmt"].data_ptr())
    st.synchronize()
    # read back what the device call installed through a host call with outputs
    # on a second context fed the device result as uploaded integrals
    s2 = copy.copy(s)
    s2.mt_aa, s2.mt_loa, s2.mt_lolo = ref
    gks = s.gksets()[:2]
    st.set_scf_inputs(keep_mt=True)
    h1 = st.setup_batched(gks)
    st.set_scf_inputs(s2)
    h2 = st.setup_batched(gks)
    for (a, b), (c, d) in zip(h1, h2):
        assert np.array_equal(a, c) and np.array_equal(b, d)


@pytest.mark.parametrize("precision", ["fp64", "ozaki", "ozaki_mod"])
def test_installed_integrals_drive_the_setup(precision):
    """hmlint + set_scf_inputs(keep_mt) gives bit-identical H and O to
    uploading the same integrals, in both arithmetic modes (the split-precision
    slices of h_a are refreshed by the call)."""
    s = W.si_fcc("shipped")
    rad = W.mt_radial(s)
    st = _setup(s)
    st.set_precision(precision, 0 if precision == "ozaki_mod" else 7)
    aa, loa, lolo = st.hmlint(rad)
    st.set_scf_inputs(keep_mt=True)
    gks = s.gksets()[:3]
    got = st.setup_batched(gks)
    s2 = copy.copy(s)
    s2.mt_aa, s2.mt_loa, s2.mt_lolo = aa, loa, lolo
    st.set_scf_inputs(s2)
    ref = st.setup_batched(gks)
    for (h, o), (hr, orf) in zip(got, ref):
        assert np.array_equal(h, hr) and np.array_equal(o, orf)
    # and the setup with these integrals matches the oracle's setup
    ho = O.hamiltonandoverlapsetup(s2, gks[0])
    h, o = got[0]
    tol = 1e-12                                  # the bar of both arithmetic modes
    assert np.linalg.norm(h - ho[0]) / np.linalg.norm(ho[0]) <= tol
    assert np.linalg.norm(o - ho[1]) / np.linalg.norm(ho[1]) <= tol


def test_keep_mt_without_hmlint_is_an_error():
    from exciting_b200.abi import ExsError
    s = W.si_fcc("text")
    st = _setup(s)
    with pytest.raises(ExsError):
        st.set_scf_inputs(keep_mt=True)


# ---------------------------------------------------------------- olprad
def _check_olp(got, ref):
    for g, r in zip(got, ref):
        if r is None:
            assert g is None
            continue
        scale = max(np.abs(r).max(), 1e-300)
        assert np.abs(g - r).max() <= TOL * scale, np.abs(g - r).max() / scale


@pytest.mark.parametrize("make", [lambda: W.si_fcc("shipped"), lambda: W.si_fcc("text", relativity="iora*"),
                                  lambda: W.sic_two_species(relativity="iora*")])
def test_olprad_vs_oracle(make):
    s = make()
    rad = W.mt_radial(s, nrmt=[300] * s.crystal.nspecies)
    st = _setup(s)
    _check_olp(st.olprad(rad), O.olprad(s, rad))


def test_generated_integrals_drive_the_iora_setup():
    """olprad + hmlint installed, then set_scf_inputs(keep_mt, keep_olp): H and
    O equal those from uploading the same arrays, and the oracle's setup."""
    s = W.si_fcc("text", relativity="iora*")
    rad = W.mt_radial(s)
    st = _setup(s)
    oalo, ololo, h1aa, h1loa, h1lolo = st.olprad(rad)
    aa, loa, lolo = st.hmlint(rad)
    st.set_scf_inputs(keep_mt=True, keep_olp=True)
    gks = s.gksets()[:2]
    got = st.setup_batched(gks)
    s2 = copy.copy(s)
    s2.mt_aa, s2.mt_loa, s2.mt_lolo = aa, loa, lolo
    s2.oalo, s2.ololo, s2.h1aa, s2.h1loa, s2.h1lolo = oalo, ololo, h1aa, h1loa, h1lolo
    st.set_scf_inputs(s2)
    ref = st.setup_batched(gks)
    for (h, o), (hr, orf) in zip(got, ref):
        assert np.array_equal(h, hr) and np.array_equal(o, orf)
    ho = O.hamiltonandoverlapsetup(s2, gks[1])
    h, o = got[1]
    assert np.linalg.norm(h - ho[0]) / np.linalg.norm(ho[0]) <= 1e-12
    assert np.linalg.norm(o - ho[1]) / np.linalg.norm(ho[1]) <= 1e-12


def test_keep_olp_without_olprad_is_an_error():
    from exciting_b200.abi import ExsError
    s = W.si_fcc("shipped")
    st = _setup(s)
    with pytest.raises(ExsError):
        st.set_scf_inputs(keep_olp=True)


def test_hmlint_argument_errors():
    """Sizes outside the documented ranges are rejected with EXS_ERR_SIZE and
    leave the context usable."""
    from exciting_b200.abi import ExsError
    s = W.si_fcc("text")
    st = _setup(s)
    rad = W.mt_radial(s, lmaxvr=2)
    bad = copy.copy(rad)
    bad.nrmt = np.array([rad.nrmtmax + 1], dtype=np.int32)
    with pytest.raises(ExsError) as e:
        st.hmlint(bad)
    assert e.value.code == -3 or "nrmt" in str(e.value)
    bad = copy.copy(rad)
    bad.lmaxvr = -1
    with pytest.raises(ExsError):
        st.olprad(bad)
    _check(st.hmlint(rad), O.hmlint(s, rad))                 # still works afterwards
