"""The reference's files around the device path (exciting_b200.fileio).

* eigenpairs of the device solve written as EVECFV.OUT / EVALFV.OUT /
  EIGVAL.OUT records and read back unchanged;
* a STATE.OUT carrying the system's potential drives the setup to the same
  H and O as the system itself.
"""
import numpy as np
import pytest

from exciting_b200 import fileio as F
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _setup(s, **kw):
    from exciting_b200.fvsystem import Setup
    return Setup(s, **kw)


def test_solve_outputs_to_reference_files(tmp_path):
    s = W.si_fcc("shipped")
    gks = s.gksets()[:3]
    st = _setup(s, max_batch=len(gks))
    nstfv = 10
    ev, vec = st.setup_and_solve(gks, nstfv)
    nmatmax = vec.shape[0]
    for ik, g in enumerate(gks):
        F.put_evecfv(tmp_path / "EVECFV.OUT", ik + 1, s.kpoints[ik], vec[:, :, ik])
        F.put_evalfv(tmp_path / "EVALFV.OUT", ik + 1, s.kpoints[ik], ev[:, ik])
    for ik in range(len(gks)):
        vkl, e = F.get_evecfv(tmp_path / "EVECFV.OUT", ik + 1, nmatmax, nstfv)
        assert np.array_equal(vkl, s.kpoints[ik]) and np.array_equal(e[:, :, 0], vec[:, :, ik])
        _, v = F.get_evalfv(tmp_path / "EVALFV.OUT", ik + 1, nstfv)
        assert np.array_equal(v[:, 0], ev[:, ik])
    occ = np.where(np.arange(nstfv)[:, None] < 4, 2.0, 0.0) * np.ones((1, len(gks)))
    F.write_eigval(tmp_path / "EIGVAL.OUT", s.kpoints[: len(gks)], ev, occ)
    vkl, e2, o2 = F.read_eigval(tmp_path / "EIGVAL.OUT")
    assert np.max(np.abs(e2 - ev)) <= 5e-10 * max(1.0, np.abs(ev).max())     # G18.10: 10 significant digits


def test_state_file_drives_the_setup(tmp_path):
    s = W.si_fcc("text")
    gks = s.gksets()[:2]
    ref = _setup(s, max_batch=2).setup_batched(gks)
    z = np.zeros((1, 1, s.natmtot), order="F")
    ngr = int(np.prod(s.gv.ngrid)) if hasattr(s.gv, "ngrid") else 1
    st = F.ExcitingState(version=(11, 0, 0), githash="0" * 40, spinpol=False, nspecies=1, lmmaxvr=1, nrmtmax=1,
                         natoms=[2], nrmt=[1], spr=[np.array([2.1])], ngrid=(ngr, 1, 1), ngvec=s.gv.ngvec, ndmag=0,
                         nspinor=1, ldapu=0, lmmaxlu=0, rhomt=z, rhoir=np.zeros(ngr), vclmt=z, vclir=np.zeros(ngr),
                         vxcmt=z, vxcir=np.zeros(ngr), veffmt=z, veffir=np.zeros(ngr),
                         veffig=np.asarray(s.veffig, dtype=np.complex128))
    F.write_state(tmp_path / "STATE.OUT", st)
    s2, _ = F.state_inputs(F.read_state(tmp_path / "STATE.OUT"), s)
    got = _setup(s2, max_batch=2).setup_batched(gks)
    for (h, o), (hr, orf) in zip(got, ref):
        assert np.array_equal(h, hr) and np.array_equal(o, orf)
