"""ORACLE -- test infrastructure only.

FP64 CPU restatement of the reference's per-k-point H/O setup and IBS force,
used as the checker by the tests, by the smoke check and by the benchmark's
CPU-baseline leg.  Never imported by the library itself.

* ``match``                    -- src/match.f90:83-191 (C: oracle_lapw.c)
* ``hamiltonsetup``            -- src/src_eigensystem/hamiltonsetup.f90:53-176
* ``overlapsetup``             -- src/src_eigensystem/overlapsetup.f90:47-166
* ``hamiltonandoverlapsetup``  -- both of the above, then copy_UL, on zeroed
                                  matrices as ``newsystem`` leaves them
                                  (src/src_eigensystem/modfvsystem.f90:48-101)
* ``forcek``                   -- src/forcek.f90:83-390 (no second variation:
                                  ``tevecsv`` false, spin-unpolarised)
* ``wavefmt``                  -- src/wavefmt.f90:82-174 (one state and atom)

The zgemm calls go to numpy (OpenBLAS); the scalar loops are in C.
Parity against the reference itself is not pinned for H, O or the IBS force
(no Fortran compiler exists here and the reference ships no H/O dump); the
pieces that do have reference data (G-vector counts, per-k matrix sizes) and
the special functions (checked against scipy) are pinned in the tests.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile oracle/liboracle.so (make in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        i, d = ctypes.c_int, ctypes.c_double
        L.orc_sbessel.argtypes = [i, d, P]
        L.orc_sbessel.restype = i
        L.orc_sbesseldm.argtypes = [i, i, d, P]
        L.orc_sbesseldm.restype = i
        L.orc_genylm.argtypes = [i, P, P]
        L.orc_genylm.restype = i
        L.orc_polynom.argtypes = [i, i, P, P, P, d]
        L.orc_polynom.restype = d
        L.orc_match.argtypes = [i, i, P, P, P, i, P, i, i, P, P, d, i, P, P, P]
        L.orc_match.restype = i
        L.orc_hmlistln_olpistln.argtypes = [i, P, P, i, P, P, P, i, P, P, P, P, i, P, P]
        L.orc_hmlistln_olpistln.restype = None
        L.orc_copy_ul.argtypes = [i, i, P]
        L.orc_copy_ul.restype = None
        L.orc_fint.argtypes = [i, P, P]
        L.orc_fint.restype = d
        L.orc_wigner3j.argtypes = [i] * 6
        L.orc_wigner3j.restype = d
        L.orc_gaunt.argtypes = [i] * 6
        L.orc_gaunt.restype = d
        L.orc_gauntyry_re_im.argtypes = [i] * 6 + [P]
        L.orc_gauntyry_re_im.restype = None
        L.orc_hmlint.argtypes = [i, P, i, i, i, i, P, i, P, P, i, P, P, P, P, P, i, i, i, P, P, P]
        L.orc_hmlint.restype = None
        L.orc_olprad.argtypes = [i, P, i, i, i, i, P, i, P, P, i, P, P, P, P, P, i, i, P, P, P, P, P]
        L.orc_olprad.restype = None
        L.orc_clebgor.argtypes = [i] * 6
        L.orc_clebgor.restype = d
        L.orc_fderiv1.argtypes = [i, P, P, P]
        L.orc_fderiv1.restype = None
        L.orc_gradzfmtr.argtypes = [i, i, P, i, i, i, i, P, P]
        L.orc_gradzfmtr.restype = None
        L.orc_pmatrad.argtypes = [i, P, i, i, P, i, P, P, i, i, P, P, P, P, P, P, P, P]
        L.orc_pmatrad.restype = None
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


# ---------------------------------------------------------------- special functions
def sbessel(lmax, x):
    out = np.zeros(lmax + 1)
    if lib().orc_sbessel(lmax, float(x), _p(out)) != 0:
        raise ValueError("sbessel: argument out of range")
    return out


def sbesseldm(m, lmax, x):
    out = np.zeros(lmax + 1)
    if lib().orc_sbesseldm(m, lmax, float(x), _p(out)) != 0:
        raise ValueError("sbesseldm: argument out of range")
    return out


def genylm(lmax, tp):
    out = np.zeros((lmax + 1) ** 2, dtype=np.complex128)
    tp = np.ascontiguousarray(tp, dtype=np.float64)
    if lib().orc_genylm(lmax, _p(tp), _p(out)) != 0:
        raise ValueError("genylm: lmax out of range")
    return out


def polynom(m, xa, ya, x):
    xa = np.ascontiguousarray(xa, dtype=np.float64)
    ya = np.ascontiguousarray(ya, dtype=np.float64)
    c = np.zeros(len(xa))
    return lib().orc_polynom(m, len(xa), _p(xa), _p(ya), _p(c), float(x))


# ---------------------------------------------------------------- match
def match(sys, gk, ngkmax=None):
    """apwalm(ngkmax, apwordmax, lmmaxapw, natmtot) for one G+k set."""
    from exciting_b200.crystal import gensfacgp
    b = sys.basis
    ngkmax = ngkmax or gk.ngp
    gpc = np.zeros(ngkmax); gpc[: gk.ngp] = gk.gpc
    tpgpc = np.zeros((2, ngkmax), order="F"); tpgpc[:, : gk.ngp] = gk.tpgpc
    sf = np.zeros((ngkmax, sys.natmtot), dtype=np.complex128, order="F")
    sf[: gk.ngp] = gensfacgp(gk.vgpc, sys.crystal.atposc)
    apword = _f(np.array(b.apword).T, np.int32)       # (lmaxapw+1, nspecies)
    species = np.asarray(b.atom_species, dtype=np.int32)
    apwalm = np.zeros((ngkmax, b.apwordmax, b.lmmaxapw, sys.natmtot), dtype=np.complex128, order="F")
    nsing = lib().orc_match(gk.ngp, ngkmax, _p(gpc), _p(tpgpc), _p(sf), sys.natmtot, _p(species),
                            b.lmaxapw, b.apwordmax, _p(apword), _p(_f(sys.rmt, np.float64)),
                            sys.crystal.omega, sys.np_tail, _p(_f(sys.spr_tail, np.float64)),
                            _p(_f(sys.apwfr_tail, np.float64)), _p(apwalm))
    return apwalm, nsing


def _apwi(sys, apwalm, ngp, ias):
    """apwi(maxaa, ngp): rows (l, m, io), l <= lmaxmat (hamiltonsetup.f90:59-71)."""
    b = sys.basis
    is_ = b.atom_species[ias]
    apwi = np.zeros((b.maxaa, ngp), dtype=np.complex128)
    f = 0
    for l in range(b.lmaxmat + 1):
        for m in range(-l, l + 1):
            lm = l * (l + 1) + m
            for io in range(b.apword[is_][l]):
                apwi[f] = apwalm[:ngp, io, lm, ias]
                f += 1
    return apwi


def _lo_range(sys, ngp, ias):
    b = sys.basis
    is_ = b.atom_species[ias]
    off = b.lo_offset(ias)
    return ngp + off, ngp + off + b.losize[is_]


# ---------------------------------------------------------------- hamiltonsetup
def hamiltonsetup(sys, gk, apwalm, h):
    """H += MT (APW-APW, APW-lo, lo-lo) + interstitial upper triangle."""
    b = sys.basis
    ngp = gk.ngp
    for ias in range(sys.natmtot):
        is_ = b.atom_species[ias]
        apwi = _apwi(sys, apwalm, ngp, ias)
        zm = sys.mt_aa[:, :, ias] @ apwi                       # hamiltonsetup.f90:75-88
        h[:ngp, :ngp] += apwi.conj().T @ zm                    # :90-103
        if b.lorbl[is_]:
            j1, j3 = _lo_range(sys, ngp, ias)
            n = j3 - j1
            h[j1:j3, :ngp] += sys.mt_loa[:n, :, ias] @ apwi     # :131-145
            h[:ngp, j1:j3] = np.conj(h[j1:j3, :ngp]).T          # :147-149
            h[j1:j3, j1:j3] += sys.mt_lolo[:n, :n, ias]         # :154-161
    _interstitial(sys, gk, h, None)                            # hmlistln


# ---------------------------------------------------------------- overlapsetup
def overlapsetup(sys, gk, apwalm, o):
    """O += MT (APW-APW with the optional h1aa, APW-lo, lo-lo) + interstitial."""
    b = sys.basis
    ngp = gk.ngp
    for ias in range(sys.natmtot):
        is_ = b.atom_species[ias]
        apwi = _apwi(sys, apwalm, ngp, ias)
        apwi2 = apwi.conj().T                                   # (ngp, maxaa), conj
        zm = np.zeros((ngp, b.maxaa), dtype=np.complex128)      # overlapsetup.f90:72-87
        f = 0
        for l in range(b.lmaxmat + 1):
            for m in range(-l, l + 1):
                n_io = b.apword[is_][l]
                for io2 in range(n_io):
                    if sys.h1aa is not None:
                        for io1 in range(n_io):
                            zm[:, f + io2] += sys.h1aa[io1, io2, l, ias] * apwi2[:, f + io1]
                    zm[:, f + io2] += apwi2[:, f + io2]
                f += n_io
        o[:ngp, :ngp] += apwi.conj().T @ zm.conj().T            # zgemm('C','C') :88-101
        if b.lorbl[is_]:
            for ilo, l in enumerate(b.lorbl[is_]):              # :111-127
                lm1, lm2 = l * (l + 1) - l, l * (l + 1) + l
                j1 = ngp + int(b.idxlo[lm1, ilo, ias]) - 1
                j2 = ngp + int(b.idxlo[lm2, ilo, ias]) - 1
                for io in range(b.apword[is_][l]):
                    w = sys.oalo[io, ilo, ias] + (0.0 if sys.h1loa is None else sys.h1loa[io, ilo, ias])
                    o[:ngp, j1:j2 + 1] += np.conj(apwalm[:ngp, io, lm1:lm2 + 1, ias] * w)
                o[j1:j2 + 1, :ngp] = np.conj(o[:ngp, j1:j2 + 1]).T
            for ilo1, l in enumerate(b.lorbl[is_]):              # :131-146
                for ilo2, l2 in enumerate(b.lorbl[is_]):
                    if l2 != l:
                        continue
                    lm1 = l * (l + 1) - l
                    j1 = ngp + int(b.idxlo[lm1, ilo1, ias]) - 1
                    j2 = ngp + int(b.idxlo[lm1, ilo2, ias]) - 1
                    w = sys.ololo[ilo1, ilo2, ias] + (0.0 if sys.h1lolo is None else sys.h1lolo[ilo1, ilo2, ias])
                    for mm in range(2 * l + 1):
                        o[j1 + mm, j2 + mm] += w
    _interstitial(sys, gk, None, o)                            # olpistln


def _interstitial(sys, gk, h, o):
    gv = sys.gv
    ld = (h if h is not None else o).shape[0]
    ivg = _f(gv.ivg, np.int32)
    ivgig = np.asfortranarray(gv.ivgig, dtype=np.int32)
    intgv = _f(gv.intgv, np.int32)
    vgpc = _f(gk.vgpc, np.float64)
    igpig = _f(gk.igpig, np.int32)
    kinw = _f(sys.kinetic_weight, np.complex128)
    m2 = None if sys.m2effig is None else _f(sys.m2effig, np.complex128)
    lib().orc_hmlistln_olpistln(gk.ngp, _p(igpig), _p(vgpc), ld, _p(ivg), _p(ivgig), _p(intgv),
                                gv.ngvec, _p(sys.veffig), _p(kinw), _p(sys.cfunig), _p(m2),
                                int(sys.h1on), _p(h), _p(o))


def hamiltonandoverlapsetup(sys, gk, apwalm=None):
    """Full Hermitian H and O (nmat x nmat, Fortran order) for one k-point."""
    if apwalm is None:
        apwalm, _ = match(sys, gk)
    nmat = sys.nmat(gk)
    h = np.zeros((nmat, nmat), dtype=np.complex128, order="F")
    o = np.zeros((nmat, nmat), dtype=np.complex128, order="F")
    hamiltonsetup(sys, gk, apwalm, h)
    overlapsetup(sys, gk, apwalm, o)
    lib().orc_copy_ul(nmat, nmat, _p(h))                       # hamiltonoverlapocopy_UL
    lib().orc_copy_ul(nmat, nmat, _p(o))
    return h, o


def apw_block(sys, gk, idx):
    """H and O restricted to the APW rows/columns ``idx`` (0-based G+k indices).

    Every APW-APW element H(i, j) depends only on G_i + k and G_j + k (the
    matching coefficients of the two columns, hamiltonsetup.f90:75-103, and
    the interstitial term of G_i - G_j, hmlistln.f90:61-86), so the block is
    the APW-APW block of the same setup over the G+k subset ``idx``.  This
    checks single entries of H/O at sizes where the full oracle would not
    finish."""
    from dataclasses import replace
    idx = np.asarray(idx)
    sub = replace(gk, ngp=len(idx), igpig=np.ascontiguousarray(gk.igpig[idx]),
                  vgpc=np.ascontiguousarray(gk.vgpc[:, idx]), gpc=np.ascontiguousarray(gk.gpc[idx]),
                  tpgpc=np.ascontiguousarray(gk.tpgpc[:, idx]))
    h, o = hamiltonandoverlapsetup(sys, sub)
    n = len(idx)
    return h[:n, :n], o[:n, :n]


# ---------------------------------------------------------------- forcek (IBS)
def forcek(sys, gk, evecfv, evalfv, occsv, wkpt, apwalm=None):
    """IBS force contribution of one k-point, forceibs(3, natmtot) (src/forcek.f90).

    ``evecfv`` (nmat, nstfv), ``evalfv`` (nstfv), ``occsv`` (nstfv).
    """
    from exciting_b200.crystal import ffacg_species
    b = sys.basis
    gv = sys.gv
    ngp = gk.ngp
    nmat = sys.nmat(gk)
    if apwalm is None:
        apwalm, _ = match(sys, gk)
    evecfv = np.asarray(evecfv)[:nmat]
    evecfv2 = evecfv * np.asarray(evalfv)[None, :]             # forcek.f90:76-80
    # ijgij with the modulo wrap into the FFT box, and dpij (forcek.f90:93-100)
    ivg_k = gv.ivg[:, gk.igpig - 1]
    iv = ivg_k[:, :, None] - ivg_k[:, None, :]
    lo = gv.intgv[:, 0][:, None, None]
    ng = gv.ngrid[:, None, None]
    iv = np.mod(iv - lo, ng) + lo
    ijgij = gv.ivgig_lookup(iv) - 1                           # 0-based
    dpij = 0.5 * (gk.vgpc.T @ gk.vgpc)
    ffacg = [ffacg_species(gv.gc[: gv.ngvec], r, sys.crystal.omega) for r in sys.rmt]
    forceibs = np.zeros((3, sys.natmtot))
    for ias in range(sys.natmtot):
        is_ = b.atom_species[ias]
        h = np.zeros((nmat, nmat), dtype=np.complex128)
        o = np.zeros((nmat, nmat), dtype=np.complex128)
        apwi = _apwi(sys, apwalm, ngp, ias)
        h[:ngp, :ngp] += apwi.conj().T @ (sys.mt_aa[:, :, ias] @ apwi)      # :139-166
        if b.lorbl[is_]:
            j1, j3 = _lo_range(sys, ngp, ias)
            n = j3 - j1
            h[j1:j3, :ngp] += sys.mt_loa[:n, :, ias] @ apwi                  # :174-190
            h[:ngp, j1:j3] = np.conj(h[j1:j3, :ngp]).T
        if sys.relativity != "iora*":
            o[:ngp, :ngp] += apwi.conj().T @ apwi                           # :196-210
        else:
            tmp = np.zeros((nmat, nmat), dtype=np.complex128, order="F")
            overlapsetup_atom_aa(sys, apwalm, ngp, ias, tmp)
            o[:ngp, :ngp] += tmp[:ngp, :ngp]
        if b.lorbl[is_]:
            for ilo, l in enumerate(b.lorbl[is_]):                           # :246-259
                lm1, lm2 = l * (l + 1) - l, l * (l + 1) + l
                j1 = ngp + int(b.idxlo[lm1, ilo, ias]) - 1
                j2 = ngp + int(b.idxlo[lm2, ilo, ias]) - 1
                for io in range(b.apword[is_][l]):
                    w = sys.oalo[io, ilo, ias] + (0.0 if sys.h1loa is None else sys.h1loa[io, ilo, ias])
                    o[:ngp, j1:j2 + 1] += np.conj(apwalm[:ngp, io, lm1:lm2 + 1, ias] * w)
                o[j1:j2 + 1, :ngp] = np.conj(o[:ngp, j1:j2 + 1]).T
        t = gv.vgc[:, ijgij]                                  # (3, ngp, ngp)
        at = sys.crystal.atposc[:, ias]
        sfac = np.exp(1j * (gv.vgc[:, ijgij].transpose(1, 2, 0) @ at))
        zt1 = -ffacg[is_][ijgij] * np.conj(sfac)
        for l in range(3):                                     # :262-287
            dlh = np.zeros((nmat, nmat), dtype=np.complex128)
            dlo = np.zeros((nmat, nmat), dtype=np.complex128)
            t1 = t[l]
            dlh[:ngp, :ngp] = (dpij * zt1 + h[:ngp, :ngp]) * t1 * 1j
            dlo[:ngp, :ngp] = -(zt1 + o[:ngp, :ngp]) * t1 * 1j
            tk = gk.vgpc[l][:, None]
            dlh[:ngp, ngp:] = h[:ngp, ngp:] * tk * 1j
            dlh[ngp:, :ngp] = np.conj(dlh[:ngp, ngp:]).T
            dlo[:ngp, ngp:] = -o[:ngp, ngp:] * tk * 1j
            dlo[ngp:, :ngp] = np.conj(dlo[:ngp, ngp:]).T
            zm = dlh @ evecfv + dlo @ evecfv2                  # :295-322
            ffv_diag = np.einsum("ij,ij->j", evecfv.conj(), zm)  # diag of evecfv^H zm, :323-337
            forceibs[l, ias] += wkpt * float(np.sum(np.asarray(occsv) * ffv_diag.real))  # :373-383
    return forceibs


def overlapsetup_atom_aa(sys, apwalm, ngp, ias, o):
    """APW-APW overlap of one atom with the IORA h1aa term (overlapsetup.f90:72-101)."""
    b = sys.basis
    is_ = b.atom_species[ias]
    apwi = _apwi(sys, apwalm, ngp, ias)
    apwi2 = apwi.conj().T
    zm = np.zeros((ngp, b.maxaa), dtype=np.complex128)
    f = 0
    for l in range(b.lmaxmat + 1):
        for m in range(-l, l + 1):
            n_io = b.apword[is_][l]
            for io2 in range(n_io):
                if sys.h1aa is not None:
                    for io1 in range(n_io):
                        zm[:, f + io2] += sys.h1aa[io1, io2, l, ias] * apwi2[:, f + io1]
                zm[:, f + io2] += apwi2[:, f + io2]
            f += n_io
    o[:ngp, :ngp] += apwi.conj().T @ zm.conj().T


# ---------------------------------------------------------------- muffin-tin wavefunction
def _wavefmt_add(wf, a, b, fr):
    """src/wavefmt.f90:126-174: wf += (a + i b) fr with the reference's skips
    of constants below 1e-14 in magnitude."""
    eps = 1e-14
    if abs(b) < eps:
        if abs(a) < eps:
            return
        wf.real += a * fr
    elif abs(a) < eps:
        wf.imag += b * fr
    else:
        wf.real += a * fr
        wf.imag += b * fr


def wavefmt(sys, rad, lrstp, lmax, ias, ngp, apwalm, evecfv, ld):
    """wfmt(ld, nr) of one state and atom: src/wavefmt.f90:82-123 (APW part
    with zdotu over G, then the local orbitals of l <= lmax)."""
    b = sys.basis
    is_ = b.atom_species[ias]
    if lmax > b.lmaxapw:
        raise ValueError("lmax > lmaxapw")
    nrmt = int(rad.nrmt[is_])
    rs = np.arange(0, nrmt, lrstp)                       # ir = 1, 1 + lrstp, ... (0-based points)
    nr = len(rs)
    wf = np.zeros((ld, nr), dtype=np.complex128)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            lm = l * (l + 1) + m
            for io in range(b.apword[is_][l]):
                zt1 = np.sum(evecfv[:ngp] * apwalm[:ngp, io, lm, ias])
                _wavefmt_add(wf[lm], zt1.real, zt1.imag, rad.apwfr[rs, 0, io, l, ias])
    for ilo, l in enumerate(b.lorbl[is_]):
        if l <= lmax:
            for m in range(-l, l + 1):
                lm = l * (l + 1) + m
                i = ngp + int(b.idxlo[lm, ilo, ias]) - 1
                _wavefmt_add(wf[lm], evecfv[i].real, evecfv[i].imag, rad.lofr[rs, 0, ilo, ias])
    return wf


# ---------------------------------------------------------------- muffin-tin integrals
def fint(x, f):
    """Integral of the cubic spline through (x_i, f_i) from x_1 to x_n
    (src/src_lib/fderiv.f90 with m = -1, gr(nr))."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    return lib().orc_fint(len(x), _p(x), _p(f))


def wigner3j(j1, j2, j3, m1, m2, m3):
    """src/src_lib/wigner3j.f90."""
    return lib().orc_wigner3j(j1, j2, j3, m1, m2, m3)


def gaunt(l1, l2, l3, m1, m2, m3):
    """src/src_lib/gaunt.f90: integral of conj(Y_l1m1) Y_l2m2 Y_l3m3."""
    return lib().orc_gaunt(l1, l2, l3, m1, m2, m3)


def gauntyry(l1, l2, l3, m1, m2, m3):
    """src/src_lib/gauntyry.f90: integral of conj(Y_l1m1) R_l2m2 Y_l3m3."""
    out = np.zeros(2)
    lib().orc_gauntyry_re_im(l1, l2, l3, m1, m2, m3, _p(out))
    return complex(out[0], out[1])


def hmlint(sys, rad):
    """mt_hscf%main after hmlint = mt_kin + mt_pot on zeroed arrays
    (src/src_eigensystem/hmlint.f90:53-55, mt_kin.f90:98-225,
    mt_pot.f90:113-306).  Returns (aa, loa, lolo) in the reference's
    (maxaa, maxaa, natmtot), (maxnlo, maxaa, natmtot), (maxnlo, maxnlo,
    natmtot) layouts."""
    b, cr = sys.basis, sys.crystal
    nat, nsp = cr.natmtot, cr.nspecies
    maxaa, maxnlo = b.maxaa, max(b.maxnlo, 1)
    aa = np.zeros((maxaa, maxaa, nat), dtype=np.complex128, order="F")
    loa = np.zeros((maxnlo, maxaa, nat), dtype=np.complex128, order="F")
    lolo = np.zeros((maxnlo, maxnlo, nat), dtype=np.complex128, order="F")
    species = np.asarray(cr.atom_species, dtype=np.int32)
    apword = _f(np.array(b.apword, dtype=np.int32).T, np.int32)           # (lmaxapw+1, nsp)
    nlorb = np.array([len(x) for x in b.lorbl], dtype=np.int32)
    lorbl = np.zeros((b.nlomax, nsp), dtype=np.int32, order="F")
    for is_ in range(nsp):
        lorbl[:len(b.lorbl[is_]), is_] = b.lorbl[is_]
    nrmt = np.asarray(rad.nrmt, dtype=np.int32)
    spr, apwfr = _f(rad.spr, np.float64), _f(rad.apwfr, np.float64)
    lofr, veffmt = _f(rad.lofr, np.float64), _f(rad.veffmt, np.float64)
    lib().orc_hmlint(nat, _p(species), b.lmaxapw, b.lmaxmat, rad.lmaxvr, b.apwordmax, _p(apword),
                     b.nlomax, _p(nlorb), _p(lorbl), rad.nrmtmax, _p(nrmt), _p(spr), _p(apwfr),
                     _p(lofr), _p(veffmt), 0 if sys.relativity == "none" else 1, maxaa, maxnlo,
                     _p(aa), _p(loa), _p(lolo))
    return aa, loa, lolo


def _radial_args(sys, rad):
    b, cr = sys.basis, sys.crystal
    nsp = cr.nspecies
    species = np.asarray(cr.atom_species, dtype=np.int32)
    apword = _f(np.array(b.apword, dtype=np.int32).T, np.int32)
    nlorb = np.array([len(x) for x in b.lorbl], dtype=np.int32)
    lorbl = np.zeros((b.nlomax, nsp), dtype=np.int32, order="F")
    for is_ in range(nsp):
        lorbl[:len(b.lorbl[is_]), is_] = b.lorbl[is_]
    return [species, apword, nlorb, lorbl, np.asarray(rad.nrmt, dtype=np.int32), _f(rad.spr, np.float64),
            _f(rad.apwfr, np.float64), _f(rad.lofr, np.float64), _f(rad.veffmt, np.float64)]


def olprad(sys, rad):
    """src/src_eigensystem/olprad.f90 on zeroed arrays: (oalo, ololo, h1aa,
    h1loa, h1lolo); the h1 arrays are None unless the relativity is iora*."""
    b, cr = sys.basis, sys.crystal
    nat = cr.natmtot
    A = _radial_args(sys, rad)
    oalo = np.zeros((b.apwordmax, b.nlomax, nat), order="F")
    ololo = np.zeros((b.nlomax, b.nlomax, nat), order="F")
    iora = sys.relativity == "iora*"
    h1aa = np.zeros((b.apwordmax, b.apwordmax, b.lmaxapw + 1, nat), order="F")
    h1loa = np.zeros((b.apwordmax, b.nlomax, nat), order="F")
    h1lolo = np.zeros((b.nlomax, b.nlomax, nat), order="F")
    lib().orc_olprad(nat, _p(A[0]), b.lmaxapw, b.lmaxmat, rad.lmaxvr, b.apwordmax, _p(A[1]), b.nlomax,
                     _p(A[2]), _p(A[3]), rad.nrmtmax, _p(A[4]), _p(A[5]), _p(A[6]), _p(A[7]), _p(A[8]),
                     0 if sys.relativity == "none" else 1, 1 if iora else 0,
                     _p(oalo), _p(ololo), _p(h1aa), _p(h1loa), _p(h1lolo))
    if not iora:
        h1aa = h1loa = h1lolo = None
    return oalo, ololo, h1aa, h1loa, h1lolo


# speed of light in atomic units (src/constants/physical_constants.f90:41-50)
C_AU = 299792458.0 * 2.418884326509e-17 / 0.52917721067e-10


def rttddft_updateham(sys, gk, atot, pmat, overlap=None):
    """One k-point of UpdateHam (src/src_xs/src_rttddft/rttddft_hamiltonianoverlap.f90:40-106).

    H and O are its hamsetup/overlapsetup (:108-330), which build the same
    blocks as the ground-state hamiltonsetup/overlapsetup; the module's
    interstitial loop mirrors each updated (i, j), i <= j, to (j, i) by
    conjugation (:156-185), which agrees with the ground-state mirror to
    rounding.  Then ham_time = H + (|A|^2/2c^2) O + sum_i (A_i/c) P_i (:95-100),
    with O the new overlap, or ``overlap`` when the call skips it.
    Returns (ham_time, O)."""
    h, o = hamiltonandoverlapsetup(sys, gk)
    if overlap is not None:
        o = np.asarray(overlap)
    a = np.asarray(atot, dtype=np.float64)
    fact = float(np.dot(a, a)) / (2.0 * C_AU ** 2)
    ham = h + fact * o
    for i in range(3):
        ham = ham + (a[i] / C_AU) * pmat[:, :, i]
    return ham, o


# ---------------------------------------------------------------- momentum matrix elements
def clebgor(j1, j2, j3, m1, m2, m3):
    """src/src_lib/clebgor.f90: <j1 m1; j2 m2 | j3 m3>."""
    return lib().orc_clebgor(j1, j2, j3, m1, m2, m3)


def fderiv1(x, f):
    """src/src_lib/fderiv.f90 with m = 1: the spline's first derivative at the points."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    g = np.zeros_like(f)
    lib().orc_fderiv1(len(x), _p(x), _p(f), _p(g))
    return g


def gradzfmtr(lmax, r, l1, m1, fmt):
    """src/src_xs/gradzfmtr.F90: gfmt(lmmax, nr, 3), the gradient of
    fmt(r) Y_l1m1 expanded in Y_lm2 (x, y, z; the y entry is -i d/dy)."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    f = np.ascontiguousarray(fmt, dtype=np.float64)
    lmmax = (lmax + 1) ** 2
    g = np.zeros((lmmax, len(r), 3), order="F")
    lib().orc_gradzfmtr(lmax, len(r), _p(r), l1, m1, lmmax, len(r), _p(f), _p(g))
    return g


def pmatrad(sys, rad):
    """src/src_xs/pmatrad.F90: the radial-angular integrals <phi_1 | d/dx_j | phi_2>
    of the APW and local-orbital functions (ripaa, ripalo, riploa, riplolo,
    shapes as src/src_xs/src_rttddft/rttddft_pmat.f90:29-39 allocates them;
    the m index of a local orbital stored at m + lolmax)."""
    b, cr = sys.basis, sys.crystal
    nat = cr.natmtot
    A = _radial_args(sys, rad)
    lmmax = (b.lmaxapw + 1) ** 2
    nm = 2 * b.lolmax + 1
    ao, nlo = b.apwordmax, b.nlomax
    ripaa = np.zeros((ao, lmmax, ao, lmmax, nat, 3), order="F")
    ripalo = np.zeros((ao, lmmax, nlo, nm, nat, 3), order="F")
    riploa = np.zeros((nlo, nm, ao, lmmax, nat, 3), order="F")
    riplolo = np.zeros((nlo, nm, nlo, nm, nat, 3), order="F")
    lib().orc_pmatrad(nat, _p(A[0]), b.lmaxapw, ao, _p(A[1]), nlo, _p(A[2]), _p(A[3]), b.lolmax, rad.nrmtmax,
                      _p(A[4]), _p(A[5]), _p(A[6]), _p(A[7]), _p(ripaa), _p(ripalo), _p(riploa), _p(riplolo))
    return ripaa, ripalo, riploa, riplolo


def _apw_cols(basis, is_):
    """(io, lm) of the APW functions of a species, l <= lmaxapw, in the order
    l, m, io of genpmatbasisik's loops."""
    out = []
    for l in range(basis.lmaxapw + 1):
        for m in range(-l, l + 1):
            for io in range(basis.apword[is_][l]):
                out.append((io, l * (l + 1) + m))
    return out


def genpmatbasisik(sys, gk, apwalm, rip):
    """pmat(nmat, nmat, 3) of one k-point, src/src_xs/src_rttddft/rttddft_pmat.f90:66-188:
    per atom and direction the APW block conj(A) R A^T (zoutpr, :85-104), the
    APW-lo columns, the lo-APW rows and the lo-lo block (:105-166); -i times
    the x and z components (:170-171); then (k+G_j)_x Theta(G_i - G_j) on the
    whole G+k block (:173-184)."""
    ripaa, ripalo, riploa, riplolo = rip
    b, cr = sys.basis, sys.crystal
    ng = gk.ngp
    nmat = sys.nmat(gk)
    lol = b.lolmax
    pm = np.zeros((nmat, nmat, 3), dtype=np.complex128, order="F")
    for ias in range(cr.natmtot):
        is_ = cr.atom_species[ias]
        cols = _apw_cols(b, is_)
        Am = np.stack([apwalm[:ng, io, lm, ias] for io, lm in cols], axis=1)        # (ng, F)
        for j in range(3):
            R = np.array([[ripaa[io1, lm1, io2, lm2, ias, j] for io2, lm2 in cols] for io1, lm1 in cols])
            pm[:ng, :ng, j] += np.conj(Am) @ (R @ Am.T)
        for ilo, l2 in enumerate(b.lorbl[is_]):
            for m2 in range(-l2, l2 + 1):
                c = ng + b.idxlo[l2 * (l2 + 1) + m2, ilo, ias] - 1
                for j in range(3):
                    rl = np.array([ripalo[io, lm, ilo, m2 + lol, ias, j] for io, lm in cols])
                    pm[:ng, c, j] += np.conj(Am) @ rl
                    rla = np.array([riploa[ilo, m2 + lol, io, lm, ias, j] for io, lm in cols])
                    pm[c, :ng, j] += Am @ rla
        for i1, l1 in enumerate(b.lorbl[is_]):
            for m1 in range(-l1, l1 + 1):
                r1 = ng + b.idxlo[l1 * (l1 + 1) + m1, i1, ias] - 1
                for i2, l2 in enumerate(b.lorbl[is_]):
                    for m2 in range(-l2, l2 + 1):
                        r2 = ng + b.idxlo[l2 * (l2 + 1) + m2, i2, ias] - 1
                        for j in range(3):
                            pm[r1, r2, j] = riplolo[i1, m1 + lol, i2, m2 + lol, ias, j]
    pm[:, :, 0] *= -1j
    pm[:, :, 2] *= -1j
    gv = sys.gv
    iv = gv.ivg[:, gk.igpig - 1]                          # (3, ng)
    diff = iv[:, :, None] - iv[:, None, :]                # (3, ng_i, ng_j)
    ig = gv.ivgig_lookup(diff.reshape(3, -1)).reshape(ng, ng) - 1
    th = np.asarray(sys.cfunig)[ig]
    for j in range(3):
        pm[:ng, :ng, j] += gk.vgpc[j][None, :] * th
    return pm
