"""The reference's file formats around the setup (exciting_b200.fileio), on the CPU.

* EIGVAL.OUT: the writer reproduces the reference's own test-farm files
  byte for byte (tests/golden/eigval_fixtures.json, made by
  tests/golden/make_eigval_golden.py);
* sequential unformatted records: gfortran's markers, split records;
* STATE.OUT: an image packed by hand from src/writestate.f90's record list
  is read back, and write/read round trips (spin-polarised, LDA+U, a file
  older than the git-hash header);
* EVECFV.OUT / EVALFV.OUT: record lengths and random access by k-point;
* DEBUGHO dumps: list-directed text with repeat counts and D exponents,
  full and packed storage;
* a state drives the setup inputs (veffig, veffmt) of a matching system.
"""
import io
import json
import os
import struct

import numpy as np
import pytest

from exciting_b200 import fileio as F
from exciting_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "eigval_fixtures.json")


# ---------------------------------------------------------------- EIGVAL.OUT
def test_eigval_writer_reproduces_reference_files(tmp_path):
    fixtures = json.load(open(GOLDEN))
    assert len(fixtures) >= 20
    for case, text in fixtures.items():
        src = tmp_path / f"{case}.in"
        src.write_text(text)
        vkl, ev, oc = F.read_eigval(src)
        dst = tmp_path / f"{case}.out"
        F.write_eigval(dst, vkl, ev, oc)
        assert dst.read_text() == text, case


@pytest.mark.parametrize("x,s", [
    (0.0, "   0.000000000    "), (-0.2497444452, " -0.2497444452    "), (2.0, "   2.000000000    "),
    (0.04504004372, "  0.4504004372E-01"), (-0.004504004372, " -0.4504004372E-02"),
    (12345.678901234, "   12345.67890    "), (0.099999999996, "  0.1000000000    "),
    (1.5e10, "  0.1500000000E+11"), (9999999999.4, "   9999999999.    "),
])
def test_fortran_g18_10(x, s):
    assert F.fortran_g(x) == s


# ---------------------------------------------------------------- records
def test_records_round_trip_and_split():
    buf = io.BytesIO()
    payloads = [b"", b"abc", bytes(range(200)) * 3]
    for p in payloads:
        F.write_record(buf, p, max_sub=7)
    buf.seek(0)
    for p in payloads:
        assert F.read_record(buf) == p
    assert F.read_record(buf) is None


def test_split_record_markers_follow_gfortran():
    buf = io.BytesIO()
    F.write_record(buf, b"0123456789", max_sub=4)      # 4 + 4 + 2
    raw = buf.getvalue()
    want = (struct.pack("<i", -4) + b"0123" + struct.pack("<i", 4) +
            struct.pack("<i", -4) + b"4567" + struct.pack("<i", -4) +
            struct.pack("<i", 2) + b"89" + struct.pack("<i", -2))
    assert raw == want


# ---------------------------------------------------------------- STATE.OUT
def _tiny_state(spin=False, ldapu=0, version=(11, 0, 1)):
    rng = np.random.default_rng(0)
    lmmaxvr, nrmtmax, natoms, nrmt = 4, 6, [1, 2], [5, 6]
    nat, ngrid, ngvec, ndmag = 3, (2, 3, 2), 7, 1 if spin else 0
    ngrtot = 12
    mt = (lmmaxvr, nrmtmax, nat)
    r = lambda *s: np.asfortranarray(rng.standard_normal(s))
    st = F.ExcitingState(
        version=version, githash="f" * 40 if version > F.REFVERSION_GITSTATE else "", spinpol=spin, nspecies=2,
        lmmaxvr=lmmaxvr, nrmtmax=nrmtmax, natoms=natoms, nrmt=nrmt,
        spr=[np.linspace(1e-5, 2.0, 5), np.linspace(1e-5, 1.6, 6)], ngrid=ngrid, ngvec=ngvec, ndmag=ndmag,
        nspinor=2 if spin else 1, ldapu=ldapu, lmmaxlu=9 if ldapu else 0,
        rhomt=r(*mt), rhoir=r(ngrtot), vclmt=r(*mt), vclir=r(ngrtot), vxcmt=r(*mt), vxcir=r(ngrtot),
        veffmt=r(*mt), veffir=r(ngrtot), veffig=r(ngvec) + 1j * r(ngvec))
    if spin:
        st.magmt, st.magir = r(*mt, ndmag), r(ngrtot, ndmag)
        st.bxcmt, st.bxcir = r(*mt, ndmag), r(ngrtot, ndmag)
    if ldapu:
        ns = st.nspinor
        st.vmatlu = np.asfortranarray(r(9, 9, ns, ns, nat) + 1j * r(9, 9, ns, ns, nat))
    return st


def _assert_state_equal(a, b):
    for k in ("version", "githash", "spinpol", "nspecies", "lmmaxvr", "nrmtmax", "natoms", "nrmt", "ngrid",
              "ngvec", "ndmag", "ldapu", "lmmaxlu"):
        assert getattr(a, k) == getattr(b, k), k
    for x, y in zip(a.spr, b.spr):
        assert np.array_equal(x, y)
    for k in ("rhomt", "rhoir", "vclmt", "vclir", "vxcmt", "vxcir", "veffmt", "veffir", "veffig", "magmt",
              "magir", "bxcmt", "bxcir", "vmatlu"):
        x, y = getattr(a, k), getattr(b, k)
        assert (x is None and y is None) or np.array_equal(x, y), k


@pytest.mark.parametrize("spin,ldapu,version", [(False, 0, (11, 0, 1)), (True, 2, (11, 0, 1)),
                                                (False, 0, (10, 2, 0))])
def test_state_round_trip(tmp_path, spin, ldapu, version):
    st = _tiny_state(spin, ldapu, version)
    p = tmp_path / "STATE.OUT"
    F.write_state(p, st)
    _assert_state_equal(F.read_state(p), st)


def test_state_reader_on_a_hand_packed_image(tmp_path):
    """Records packed with struct from writestate.f90:9-35, not by write_state."""
    def rec(b):
        return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))
    i4 = lambda *v: struct.pack("<%di" % len(v), *v)
    f8 = lambda a: np.asarray(a, dtype="<f8").tobytes()
    lm, nr = 4, 3
    mt = np.arange(lm * nr, dtype=float).reshape((lm, nr, 1), order="F")
    ir = np.array([1.0, 2.0])
    vig = np.array([1 + 2j, 3 - 4j], dtype="<c16")
    img = (rec(i4(12, 0, 0) + b"x" * 40) + rec(i4(0)) + rec(i4(1)) + rec(i4(lm)) + rec(i4(nr)) +
           rec(i4(1)) + rec(i4(nr)) + rec(f8([0.1, 0.5, 1.0])) + rec(i4(1, 2, 1)) + rec(i4(2)) + rec(i4(0)) +
           rec(i4(1)) + rec(i4(0)) + rec(i4(0)) +
           rec(f8(mt.ravel(order="F")) + f8(ir)) * 3 +
           rec(f8(2 * mt.ravel(order="F")) + f8(2 * ir) + vig.tobytes()))
    p = tmp_path / "STATE.OUT"
    p.write_bytes(img)
    st = F.read_state(p)
    assert st.version == (12, 0, 0) and st.githash == "x" * 40 and not st.spinpol
    assert st.natoms == [1] and st.nrmt == [nr] and np.array_equal(st.spr[0], [0.1, 0.5, 1.0])
    assert st.ngrid == (1, 2, 1) and st.ngvec == 2 and st.ldapu == 0
    assert np.array_equal(st.rhomt, mt) and np.array_equal(st.veffmt, 2 * mt)
    assert np.array_equal(st.veffig, vig)


def test_state_drives_the_setup_inputs(tmp_path):
    s = W.si_fcc("text")
    rad = W.mt_radial(s, lmaxvr=4)
    st = _tiny_state()
    st.nspecies, st.natoms, st.nrmt = 1, [2], [int(rad.nrmt[0])]
    st.nrmtmax, st.lmmaxvr = rad.nrmtmax, 25
    st.spr = [rad.spr[:, 0].copy()]
    st.ngvec = s.gv.ngvec
    st.veffig = np.asfortranarray(np.arange(st.ngvec) * (1 + 0.5j))
    st.veffmt = np.asfortranarray(np.random.default_rng(1).standard_normal((25, rad.nrmtmax, 2)))
    for k in ("rhomt", "vclmt", "vxcmt"):
        setattr(st, k, st.veffmt.copy(order="F"))
    p = tmp_path / "STATE.OUT"
    F.write_state(p, st)
    s2, rad2 = F.state_inputs(F.read_state(p), s, rad)
    assert np.array_equal(s2.veffig, st.veffig) and s2.mt_aa is s.mt_aa
    assert rad2.lmaxvr == 4 and np.array_equal(rad2.veffmt, st.veffmt)
    assert np.array_equal(rad2.apwfr, rad.apwfr)
    st.ngvec, st.veffig = 5, st.veffig[:5]
    with pytest.raises(ValueError):
        F.state_inputs(st, s, rad)


# ---------------------------------------------------------------- EVECFV / EVALFV
def test_evecfv_evalfv_records(tmp_path):
    rng = np.random.default_rng(2)
    nmatmax, nstfv = 9, 4
    ev = {ik: np.asfortranarray(rng.standard_normal((nmatmax, nstfv)) + 1j * rng.standard_normal((nmatmax, nstfv)))
          for ik in (3, 1, 2)}
    vals = {ik: rng.standard_normal(nstfv) for ik in ev}
    pv, pe = tmp_path / "EVECFV.OUT", tmp_path / "EVALFV.OUT"
    for ik in ev:                                      # out of order, as MPI ranks write them
        F.put_evecfv(pv, ik, [0.1 * ik, 0, 0.5], ev[ik])
        F.put_evalfv(pe, ik, [0.1 * ik, 0, 0.5], vals[ik])
    assert os.path.getsize(pv) == 3 * F.evecfv_recl(nmatmax, nstfv) == 3 * (36 + 16 * nmatmax * nstfv)
    assert os.path.getsize(pe) == 3 * F.evalfv_recl(nstfv) == 3 * (32 + 8 * nstfv)
    for ik in ev:
        vkl, e = F.get_evecfv(pv, ik, nmatmax, nstfv)
        assert np.array_equal(vkl, [0.1 * ik, 0, 0.5]) and np.array_equal(e[:, :, 0], ev[ik])
        vkl, v = F.get_evalfv(pe, ik, nstfv)
        assert np.array_equal(v[:, 0], vals[ik])
    with pytest.raises(ValueError):
        F.get_evecfv(pv, 1, nmatmax - 1, nstfv + 1)


# ---------------------------------------------------------------- DEBUGHO dumps
@pytest.mark.parametrize("packed", [False, True])
def test_debugho_round_trip(tmp_path, packed):
    rng = np.random.default_rng(4)
    n = 7
    z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    z = z + z.conj().T
    F.write_debugho(str(tmp_path / "H"), z, packed=packed)
    assert np.array_equal(F.read_debugho(str(tmp_path / "H"), n, packed=packed), z)


def test_list_directed_reader(tmp_path):
    p = tmp_path / "x.OUT"
    p.write_text("   1.0000000000000000       3*0.0000000000000000     \n -2.5D-03, 4.0E+02\n")
    assert np.array_equal(F.read_list_directed(p), [1.0, 0.0, 0.0, 0.0, -2.5e-3, 400.0])
