"""The reference's files on either side of the setup, read and written on the host.

* ``STATE.OUT`` (``src/writestate.f90``, ``src/readstate.f90``): the converged
  density and potentials, Fortran sequential unformatted.  Its ``veffig`` and
  ``veffmt`` are the setup's interstitial potential and the potential of the
  muffin-tin integral generation, so a state written by the reference can
  drive the library (``state_inputs``).
* ``EVECFV.OUT`` / ``EVALFV.OUT`` (``src/putevecfv.f90``,
  ``src/putevalfv.f90``): first-variational eigenpairs, direct-access
  unformatted records, one per k-point.
* ``EIGVAL.OUT`` (``src/writeeval.f90``): eigenvalues and occupancies as text
  with the Fortran edit descriptors I6 and G18.10.
* ``H.real.OUT``, ``H.imag.OUT``, ``O.*`` (``HermitianMatrixToFiles``,
  ``src/src_eigensystem/modfvsystem.f90:512-538``, written when the
  reference is built with -DDEBUGHO): list-directed real and imaginary parts
  of ``za`` in column-major order.

Sequential unformatted files use gfortran's layout: every record framed by
4-byte little-endian length markers; a record longer than 2**31 - 9 bytes is
split into subrecords whose leading marker is negative when more follow and
whose trailing marker is negative when it continues an earlier one.
"""
from __future__ import annotations

import math
import os
import re
import struct
from dataclasses import dataclass
from typing import Optional

import numpy as np

MAX_SUBRECORD = 2147483639    # gfortran's largest subrecord payload


# ------------------------------------------------------------------ sequential records
def write_record(f, payload: bytes, max_sub: int = MAX_SUBRECORD):
    """One sequential unformatted record (split into subrecords if needed)."""
    n = len(payload)
    if n == 0:
        f.write(struct.pack("<ii", 0, 0))
        return
    pos, first = 0, True
    while pos < n:
        m = min(max_sub, n - pos)
        more = pos + m < n
        f.write(struct.pack("<i", -m if more else m))
        f.write(payload[pos:pos + m])
        f.write(struct.pack("<i", -m if not first else m))
        pos += m
        first = False


def read_record(f) -> Optional[bytes]:
    """The next record's payload, or None at the end of the file."""
    out = []
    while True:
        head = f.read(4)
        if not head:
            if out:
                raise ValueError("file ends inside a split record")
            return None
        (n,) = struct.unpack("<i", head)
        m = abs(n)
        data = f.read(m)
        tail = f.read(4)
        if len(data) != m or len(tail) != 4 or abs(struct.unpack("<i", tail)[0]) != m:
            raise ValueError("damaged record markers")
        out.append(data)
        if n >= 0:
            return b"".join(out)


class _Cursor:
    """Reads consecutive items out of one record's payload."""

    def __init__(self, payload: bytes):
        self.b, self.pos = payload, 0

    def take(self, dtype, count=1):
        dt = np.dtype(dtype).newbyteorder("<")
        n = dt.itemsize * count
        if self.pos + n > len(self.b):
            raise ValueError("record shorter than its declared contents")
        a = np.frombuffer(self.b, dtype=dt, count=count, offset=self.pos)
        self.pos += n
        return a

    def done(self):
        return self.pos == len(self.b)


def _ints(*v):
    return np.asarray(v, dtype="<i4").tobytes()


# ------------------------------------------------------------------ STATE.OUT
@dataclass
class ExcitingState:
    """The contents of STATE.OUT (src/writestate.f90:8-41), arrays in the
    reference's shapes and Fortran order."""
    version: tuple                     # (3,) ints
    githash: str                       # 40 characters ('' for files older than 10.4.14)
    spinpol: bool
    nspecies: int
    lmmaxvr: int
    nrmtmax: int
    natoms: list                       # per species
    nrmt: list                         # per species
    spr: list                          # per species, (nrmt,) radial mesh
    ngrid: tuple
    ngvec: int
    ndmag: int
    nspinor: int
    ldapu: int
    lmmaxlu: int
    rhomt: np.ndarray                  # (lmmaxvr, nrmtmax, natmtot)
    rhoir: np.ndarray                  # (ngrtot,)
    vclmt: np.ndarray
    vclir: np.ndarray
    vxcmt: np.ndarray
    vxcir: np.ndarray
    veffmt: np.ndarray
    veffir: np.ndarray
    veffig: np.ndarray                 # (ngvec,) complex
    magmt: Optional[np.ndarray] = None  # (lmmaxvr, nrmtmax, natmtot, ndmag)
    magir: Optional[np.ndarray] = None  # (ngrtot, ndmag)
    bxcmt: Optional[np.ndarray] = None
    bxcir: Optional[np.ndarray] = None
    vmatlu: Optional[np.ndarray] = None  # (lmmaxlu, lmmaxlu, nspinor, nspinor, natmtot) complex

    @property
    def natmtot(self) -> int:
        return int(sum(self.natoms))

    @property
    def ngrtot(self) -> int:
        return int(np.prod(self.ngrid))


REFVERSION_GITSTATE = (10, 4, 14)   # src/mod_misc.F90:33
REFVERSION_LDAPU = (0, 9, 131)      # src/readstate.f90:189-190


def _version_gt(a, b):
    return tuple(a) > tuple(b)


def write_state(path, st: ExcitingState):
    """STATE.OUT as src/writestate.f90 writes it."""
    with open(path, "wb") as f:
        head = _ints(*st.version)
        if _version_gt(st.version, REFVERSION_GITSTATE):
            head += st.githash.ljust(40)[:40].encode("ascii")
        write_record(f, head)
        write_record(f, _ints(1 if st.spinpol else 0))
        write_record(f, _ints(st.nspecies))
        write_record(f, _ints(st.lmmaxvr))
        write_record(f, _ints(st.nrmtmax))
        for is_ in range(st.nspecies):
            write_record(f, _ints(st.natoms[is_]))
            write_record(f, _ints(st.nrmt[is_]))
            write_record(f, np.asarray(st.spr[is_][: st.nrmt[is_]], dtype="<f8").tobytes())
        write_record(f, _ints(*st.ngrid))
        write_record(f, _ints(st.ngvec))
        write_record(f, _ints(st.ndmag))
        if _version_gt(st.version, REFVERSION_LDAPU):
            write_record(f, _ints(st.nspinor))
            write_record(f, _ints(st.ldapu))
            write_record(f, _ints(st.lmmaxlu))

        def fb(a, dt="<f8"):
            return np.asfortranarray(a, dtype=dt).tobytes(order="F")

        write_record(f, fb(st.rhomt) + fb(st.rhoir))
        write_record(f, fb(st.vclmt) + fb(st.vclir))
        write_record(f, fb(st.vxcmt) + fb(st.vxcir))
        write_record(f, fb(st.veffmt) + fb(st.veffir) + fb(st.veffig, "<c16"))
        if st.spinpol:
            write_record(f, fb(st.magmt) + fb(st.magir))
            write_record(f, fb(st.bxcmt) + fb(st.bxcir))
        if st.ldapu != 0:
            write_record(f, fb(st.vmatlu, "<c16"))


def read_state(path) -> ExcitingState:
    """STATE.OUT in the order of src/readstate.f90:60-240 (the file's own
    sizes; no interpolation onto another mesh)."""
    with open(path, "rb") as f:
        def rec():
            r = read_record(f)
            if r is None:
                raise ValueError("STATE.OUT ends early")
            return _Cursor(r)

        c = rec()
        version = tuple(int(v) for v in c.take("i4", 3))
        githash = ""
        if _version_gt(version, REFVERSION_GITSTATE) and not c.done():
            githash = bytes(c.take("u1", 40)).decode("ascii", "replace")
        spinpol = bool(rec().take("i4")[0])
        nspecies = int(rec().take("i4")[0])
        lmmaxvr = int(rec().take("i4")[0])
        nrmtmax = int(rec().take("i4")[0])
        natoms, nrmt, spr = [], [], []
        for _ in range(nspecies):
            natoms.append(int(rec().take("i4")[0]))
            nrmt.append(int(rec().take("i4")[0]))
            spr.append(rec().take("f8", nrmt[-1]).copy())
        ngrid = tuple(int(v) for v in rec().take("i4", 3))
        ngvec = int(rec().take("i4")[0])
        ndmag = int(rec().take("i4")[0])
        if _version_gt(version, REFVERSION_LDAPU):
            nspinor = int(rec().take("i4")[0])
            ldapu = int(rec().take("i4")[0])
            lmmaxlu = int(rec().take("i4")[0])
        else:
            nspinor, ldapu, lmmaxlu = 1, 0, 0
        nat = sum(natoms)
        ngrtot = int(np.prod(ngrid))
        mt = (lmmaxvr, nrmtmax, nat)

        def arr(cur, shape, dt="f8"):
            n = int(np.prod(shape))
            return cur.take(dt, n).reshape(shape, order="F").copy(order="F")

        c = rec(); rhomt, rhoir = arr(c, mt), arr(c, (ngrtot,))
        c = rec(); vclmt, vclir = arr(c, mt), arr(c, (ngrtot,))
        c = rec(); vxcmt, vxcir = arr(c, mt), arr(c, (ngrtot,))
        c = rec(); veffmt, veffir, veffig = arr(c, mt), arr(c, (ngrtot,)), arr(c, (ngvec,), "c16")
        magmt = magir = bxcmt = bxcir = vmatlu = None
        if spinpol:
            c = rec(); magmt, magir = arr(c, mt + (ndmag,)), arr(c, (ngrtot, ndmag))
            c = rec(); bxcmt, bxcir = arr(c, mt + (ndmag,)), arr(c, (ngrtot, ndmag))
        if ldapu != 0:
            c = rec(); vmatlu = arr(c, (lmmaxlu, lmmaxlu, nspinor, nspinor, nat), "c16")
    return ExcitingState(version=version, githash=githash, spinpol=spinpol, nspecies=nspecies, lmmaxvr=lmmaxvr,
                         nrmtmax=nrmtmax, natoms=natoms, nrmt=nrmt, spr=spr, ngrid=ngrid, ngvec=ngvec, ndmag=ndmag,
                         nspinor=nspinor, ldapu=ldapu, lmmaxlu=lmmaxlu, rhomt=rhomt, rhoir=rhoir, vclmt=vclmt,
                         vclir=vclir, vxcmt=vxcmt, vxcir=vxcir, veffmt=veffmt, veffir=veffir, veffig=veffig,
                         magmt=magmt, magir=magir, bxcmt=bxcmt, bxcir=bxcir, vmatlu=vmatlu)


def state_inputs(st: ExcitingState, sys, rad=None):
    """The setup inputs a state provides: ``sys`` with ``veffig`` replaced by
    the state's (the interstitial potential of hmlistln), and, when ``rad``
    (system.MtRadial with the caller's radial functions) is given, ``rad`` with
    the state's ``veffmt`` and radial meshes for hmlint.  The state must come
    from the same crystal and cutoffs (species, atoms, ngvec), as readstate
    requires (src/readstate.f90:82-131)."""
    import copy
    if st.nspecies != sys.crystal.nspecies:
        raise ValueError("differing nspecies")
    for is_ in range(st.nspecies):
        if st.natoms[is_] != sum(1 for s in sys.crystal.atom_species if s == is_):
            raise ValueError(f"differing natoms for species {is_}")
    if st.ngvec != sys.gv.ngvec:
        raise ValueError(f"differing ngvec: state {st.ngvec}, system {sys.gv.ngvec}")
    out = copy.copy(sys)
    out.veffig = np.asfortranarray(st.veffig, dtype=np.complex128)
    if rad is None:
        return out, None
    lmaxvr = int(round(math.sqrt(st.lmmaxvr))) - 1
    if (lmaxvr + 1) ** 2 != st.lmmaxvr:
        raise ValueError("lmmaxvr is not a square")
    if rad.nrmtmax != st.nrmtmax or any(int(a) != b for a, b in zip(rad.nrmt, st.nrmt)):
        raise ValueError("the radial functions are on other meshes than the state")
    r2 = copy.copy(rad)
    r2.lmaxvr = lmaxvr
    r2.veffmt = np.asfortranarray(st.veffmt, dtype=np.float64)
    r2.spr = np.zeros((st.nrmtmax, st.nspecies), order="F")
    for is_ in range(st.nspecies):
        r2.spr[: st.nrmt[is_], is_] = st.spr[is_]
    return out, r2


# ------------------------------------------------------------------ EVECFV / EVALFV
def evecfv_recl(nmatmax, nstfv, nspnfv=1):
    """Record length in bytes of EVECFV.OUT: vkl(3), nmatmax, nstfv, nspnfv,
    evecfv(nmatmax, nstfv, nspnfv) (src/putevecfv.f90:10-11)."""
    return 3 * 8 + 3 * 4 + 16 * nmatmax * nstfv * nspnfv


def evalfv_recl(nstfv, nspnfv=1):
    return 3 * 8 + 2 * 4 + 8 * nstfv * nspnfv


def _put_direct(path, ik, recl, payload):
    assert len(payload) == recl
    mode = "r+b" if os.path.exists(path) else "w+b"
    with open(path, mode) as f:
        f.seek((ik - 1) * recl)
        f.write(payload)


def put_evecfv(path, ik, vkl, evecfv):
    """Record ik (1-based) of EVECFV.OUT; evecfv (nmatmax, nstfv[, nspnfv])."""
    e = np.asarray(evecfv, dtype=np.complex128)
    if e.ndim == 2:
        e = e[:, :, None]
    nmatmax, nstfv, nspnfv = e.shape
    payload = (np.asarray(vkl, dtype="<f8").tobytes() + _ints(nmatmax, nstfv, nspnfv)
               + np.asfortranarray(e, dtype="<c16").tobytes(order="F"))
    _put_direct(path, ik, evecfv_recl(nmatmax, nstfv, nspnfv), payload)


def get_evecfv(path, ik, nmatmax, nstfv, nspnfv=1):
    """(vkl, evecfv (nmatmax, nstfv, nspnfv)) of record ik; the sizes stored in
    the record must match (src/getevecfv.f90 checks them)."""
    recl = evecfv_recl(nmatmax, nstfv, nspnfv)
    with open(path, "rb") as f:
        f.seek((ik - 1) * recl)
        c = _Cursor(f.read(recl))
    vkl = c.take("f8", 3).copy()
    sizes = tuple(int(v) for v in c.take("i4", 3))
    if sizes != (nmatmax, nstfv, nspnfv):
        raise ValueError(f"EVECFV record sizes {sizes} differ from {(nmatmax, nstfv, nspnfv)}")
    e = c.take("c16", nmatmax * nstfv * nspnfv).reshape((nmatmax, nstfv, nspnfv), order="F").copy(order="F")
    return vkl, e


def put_evalfv(path, ik, vkl, evalfv):
    v = np.asarray(evalfv, dtype=np.float64)
    if v.ndim == 1:
        v = v[:, None]
    nstfv, nspnfv = v.shape
    payload = (np.asarray(vkl, dtype="<f8").tobytes() + _ints(nstfv, nspnfv)
               + np.asfortranarray(v, dtype="<f8").tobytes(order="F"))
    _put_direct(path, ik, evalfv_recl(nstfv, nspnfv), payload)


def get_evalfv(path, ik, nstfv, nspnfv=1):
    recl = evalfv_recl(nstfv, nspnfv)
    with open(path, "rb") as f:
        f.seek((ik - 1) * recl)
        c = _Cursor(f.read(recl))
    vkl = c.take("f8", 3).copy()
    sizes = tuple(int(v) for v in c.take("i4", 2))
    if sizes != (nstfv, nspnfv):
        raise ValueError(f"EVALFV record sizes {sizes} differ from {(nstfv, nspnfv)}")
    return vkl, c.take("f8", nstfv * nspnfv).reshape((nstfv, nspnfv), order="F").copy(order="F")


# ------------------------------------------------------------------ EIGVAL.OUT (text)
def fortran_g(x: float, w: int = 18, d: int = 10) -> str:
    """The Fortran edit descriptor Gw.d (exponent width 2) for a real value:
    F editing with d - k decimals and 4 trailing blanks when the value,
    rounded to d significant digits, lies in [0.1, 10**d) (k digits before
    the point), otherwise Ew.d; zero prints as F with d - 1 decimals."""
    if x == 0.0 or not math.isfinite(x):
        if x == 0.0:
            s = f"{0.0:.{d - 1}f}"
            if math.copysign(1.0, x) < 0:
                s = "-" + s
            return s.rjust(w - 4) + " " * 4
        return ("NaN" if math.isnan(x) else ("-Infinity" if x < 0 else "Infinity")).rjust(w)
    mant, exp = f"{abs(x):.{d - 1}e}".split("e")
    e10 = int(exp)                       # rounded value = mant * 10**e10, 1 <= mant < 10
    sign = "-" if x < 0 else ""
    if -1 <= e10 < d:                    # 0.1 <= rounded < 10**d: F editing
        k = e10 + 1
        s = sign + f"{abs(x):.{d - k}f}" + ("." if d == k else "")   # F editing always prints the point
        return s.rjust(w - 4) + " " * 4
    digits = mant.replace(".", "")
    e = e10 + 1
    s = f"{sign}0.{digits}E{'-' if e < 0 else '+'}{abs(e):02d}"
    return s.rjust(w)


def write_eigval(path, vkl, evalsv, occsv):
    """EIGVAL.OUT as src/writeeval.f90:8-31 writes it: vkl (nkpt, 3), evalsv and
    occsv (nstsv, nkpt)."""
    vkl = np.asarray(vkl, dtype=np.float64)
    ev = np.asarray(evalsv, dtype=np.float64)
    oc = np.asarray(occsv, dtype=np.float64)
    nstsv, nkpt = ev.shape
    lines = [f"{nkpt:6d} : nkpt", f"{nstsv:6d} : nstsv"]
    for ik in range(nkpt):
        lines.append(" ")
        lines.append(f"{ik + 1:6d}" + "".join(fortran_g(v) for v in vkl[ik]) + " : k-point, vkl")
        lines.append(" (state, eigenvalue and occupancy below)")
        for ist in range(nstsv):
            lines.append(f"{ist + 1:6d}" + fortran_g(ev[ist, ik]) + fortran_g(oc[ist, ik]))
        lines.append(" ")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_eigval(path):
    """(vkl (nkpt, 3), evalsv (nstsv, nkpt), occsv (nstsv, nkpt)) of an EIGVAL.OUT."""
    lines = open(path).read().splitlines()
    nkpt = int(lines[0].split(":")[0])
    nstsv = int(lines[1].split(":")[0])
    vkl = np.zeros((nkpt, 3))
    ev = np.zeros((nstsv, nkpt))
    oc = np.zeros((nstsv, nkpt))
    i = 2
    for ik in range(nkpt):
        while ": k-point" not in lines[i]:
            i += 1
        f = lines[i].split(":")[0].split()
        vkl[ik] = [float(v) for v in f[1:4]]
        i += 2
        for ist in range(nstsv):
            f = lines[i].split()
            ev[ist, ik], oc[ist, ik] = float(f[1]), float(f[2])
            i += 1
    return vkl, ev, oc


# ------------------------------------------------------------------ DEBUGHO dumps (text)
_REPEAT = re.compile(r"^(\d+)\*(.*)$")


def read_list_directed(path) -> np.ndarray:
    """The real values of a list-directed Fortran file (blank, comma or
    newline separated; r*value repeat counts; D or E exponents)."""
    vals = []
    for tok in open(path).read().replace(",", " ").split():
        m = _REPEAT.match(tok)
        if m:
            vals.extend([float(m.group(2).replace("D", "E").replace("d", "e"))] * int(m.group(1)))
        else:
            vals.append(float(tok.replace("D", "E").replace("d", "e")))
    return np.array(vals, dtype=np.float64)


def write_list_directed(path, values):
    """Real values one per line, 17 significant digits (what a list-directed
    READ takes back exactly)."""
    with open(path, "w") as f:
        for v in np.asarray(values, dtype=np.float64).ravel(order="F"):
            f.write(f" {v: .16E}\n")


def write_debugho(prefix, za, packed=False):
    """prefix.real.OUT / prefix.imag.OUT (or .packed.*) of a matrix, as
    HermitianMatrixToFiles writes them (column-major za; packed: the upper
    triangle column by column, zap)."""
    z = np.asarray(za, dtype=np.complex128)
    if packed:
        n = z.shape[0]
        z = np.concatenate([z[: j + 1, j] for j in range(n)])
        tag = ".packed"
    else:
        z = np.asfortranarray(z).ravel(order="F")
        tag = ""
    write_list_directed(f"{prefix}{tag}.real.OUT", z.real)
    write_list_directed(f"{prefix}{tag}.imag.OUT", z.imag)


def read_debugho(prefix, n, packed=False):
    """The (n, n) complex matrix of a HermitianMatrixToFiles dump (packed:
    the full Hermitian matrix rebuilt from the upper triangle)."""
    tag = ".packed" if packed else ""
    re_ = read_list_directed(f"{prefix}{tag}.real.OUT")
    im = read_list_directed(f"{prefix}{tag}.imag.OUT")
    z = re_ + 1j * im
    if not packed:
        if z.size != n * n:
            raise ValueError(f"{z.size} values for a {n} x {n} matrix")
        return z.reshape((n, n), order="F")
    if z.size != n * (n + 1) // 2:
        raise ValueError(f"{z.size} values for a packed {n} x {n} matrix")
    out = np.zeros((n, n), dtype=np.complex128, order="F")
    pos = 0
    for j in range(n):
        out[: j + 1, j] = z[pos: pos + j + 1]
        pos += j + 1
    iu = np.triu_indices(n, 1)
    out[iu[1], iu[0]] = np.conj(out[iu])
    return out
