"""Host-side mirror of the reference's per-k-point H/O setup interface.

``Setup`` owns one library context for one ``LapwSystem`` and exposes the
reference's calls with the reference's argument meaning:

* ``match(gk)``                        -- call match(ngp, gpc, tpgpc, sfacgp, apwalm)
* ``hamiltonandoverlapsetup(gk, apwalm=None)``
                                        -- call hamiltonandoverlapsetup(system, ngp,
                                           apwalm, igpig, vgpc) on newsystem's
                                           zeroed matrices, then copy_UL
* ``setup_batched(gks)``               -- the k-loop of one SCF iteration
* ``forcek(gk, evecfv, evalfv, occsv, wkpt)``
                                        -- the IBS part of call forcek(ik, ffacg)

Everything is computed by libexciting_b200.so on the GPU; errors of the
library raise ``ExsError``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from .crystal import ffacg_species, gensfacgp
from .system import RELATIVITY, LapwSystem

_keep = []


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


class Setup:
    def __init__(self, sys: LapwSystem, *, ngkmax: int | None = None, max_batch: int = 1):
        self.sys = sys
        self.lib = abi.load()
        b = sys.basis
        gv = sys.gv
        gks = sys.gksets() if (ngkmax is None and sys.kpoints is not None) else None
        self.ngkmax = int(ngkmax if ngkmax is not None else max(g.ngp for g in gks))
        nsp = b.nspecies
        nlomax = max(b.nlomax, 1)
        self._arrays = dict(
            atom_species=_f(b.atom_species, np.int32),
            apword=_f(np.array(b.apword).T, np.int32),
            nlorb=_f([len(x) for x in b.lorbl], np.int32),
            lorbl=_f(np.array([list(x) + [0] * (nlomax - len(x)) for x in b.lorbl]).T.reshape(nlomax, nsp), np.int32),
            rmt=_f(sys.rmt, np.float64),
            atposc=_f(sys.crystal.atposc, np.float64),
            bvec=_f(sys.crystal.bvec, np.float64),
            intgv=_f(gv.intgv, np.int32),
            ivg=_f(gv.ivg, np.int32),
            ivgig=np.asfortranarray(gv.ivgig, dtype=np.int32),
        )
        A = self._arrays
        cfg = abi.exs_config()
        cfg.natmtot = sys.natmtot
        cfg.nspecies = nsp
        cfg.atom_species = A["atom_species"].ctypes.data
        cfg.lmaxapw = b.lmaxapw
        cfg.lmaxmat = b.lmaxmat
        cfg.apwordmax = b.apwordmax
        cfg.apword = A["apword"].ctypes.data
        cfg.nlomax = nlomax
        cfg.nlorb = A["nlorb"].ctypes.data
        cfg.lorbl = A["lorbl"].ctypes.data
        cfg.rmt = A["rmt"].ctypes.data
        cfg.omega = sys.crystal.omega
        cfg.atposc = A["atposc"].ctypes.data
        cfg.bvec = A["bvec"].ctypes.data
        cfg.ngkmax = self.ngkmax
        cfg.ngrtot = gv.ngrtot
        cfg.ngvec = gv.ngvec
        cfg.intgv = A["intgv"].ctypes.data
        cfg.ivg = A["ivg"].ctypes.data
        cfg.ivgig = A["ivgig"].ctypes.data
        cfg.relativity = RELATIVITY[sys.relativity]
        cfg.np_tail = sys.np_tail
        cfg.max_batch = max_batch
        self.max_batch = max_batch
        ctx = ctypes.c_void_p()
        rc = self.lib.exs_ctx_create(ctypes.byref(cfg), ctypes.byref(ctx))
        if rc != 0:
            raise abi.ExsError(rc, "exs_ctx_create failed")
        self.ctx = ctx
        sizes = (ctypes.c_int * 3)()
        self.lib.exs_ctx_sizes(ctx, ctypes.byref(sizes, 0), ctypes.byref(sizes, 4), ctypes.byref(sizes, 8))
        self.maxaa, self.maxnlo, self.nlotot = int(sizes[0]), int(sizes[1]), int(sizes[2])
        self.set_scf_inputs()

    # ------------------------------------------------------------------
    def _check(self, rc):
        return abi.check(self.lib, self.ctx, rc)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.exs_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_scf_inputs(self, sys: LapwSystem | None = None, *, keep_mt: bool = False, keep_olp: bool = False):
        """Upload the per-SCF inputs; keep_mt keeps the muffin-tin integrals
        that :meth:`hmlint` left on the device instead of sys.mt_*, keep_olp
        the overlap integrals of :meth:`olprad` instead of sys.oalo, ololo, h1*."""
        s = sys or self.sys
        keep = dict(
            mt_aa=None if keep_mt else _f(s.mt_aa, np.complex128),
            mt_loa=None if keep_mt else _f(s.mt_loa, np.complex128),
            mt_lolo=None if keep_mt else _f(s.mt_lolo, np.complex128), oalo=_f(s.oalo, np.float64),
            ololo=_f(s.ololo, np.float64), veffig=_f(s.veffig, np.complex128),
            cfunig=_f(s.cfunig, np.complex128), spr_tail=_f(s.spr_tail, np.float64),
            apwfr_tail=_f(s.apwfr_tail, np.float64),
            meffig=None if s.meffig is None else _f(s.meffig, np.complex128),
            m2effig=None if s.m2effig is None else _f(s.m2effig, np.complex128),
            h1aa=None if s.h1aa is None else _f(s.h1aa, np.float64),
            h1loa=None if s.h1loa is None else _f(s.h1loa, np.float64),
            h1lolo=None if s.h1lolo is None else _f(s.h1lolo, np.float64),
        )
        if keep_olp:
            for k in ("oalo", "ololo", "h1aa", "h1loa", "h1lolo"):
                keep[k] = None
        inp = abi.exs_scf_inputs()
        for k, v in keep.items():
            setattr(inp, k, None if v is None else v.ctypes.data)
        self._check(self.lib.exs_set_scf_inputs(self.ctx, ctypes.byref(inp)))

    def _mt_radial(self, rad, apwfr, lofr, veffmt):
        keep = dict(nrmt=np.ascontiguousarray(rad.nrmt, dtype=np.int32), spr=_f(rad.spr, np.float64))
        r = abi.exs_mt_radial()
        r.lmaxvr, r.nrmtmax = int(rad.lmaxvr), int(rad.nrmtmax)
        r.nrmt, r.spr = keep["nrmt"].ctypes.data, keep["spr"].ctypes.data
        r.apwfr, r.lofr, r.veffmt = apwfr, lofr, veffmt
        return r, keep

    def hmlint(self, rad, *, outputs: bool = True):
        """Muffin-tin integrals (aa, loa, lolo) of the radial inputs ``rad``
        (system.MtRadial), installed on the device as this context's h_a;
        returned in the reference's layouts when ``outputs``."""
        b, nat = self.sys.basis, self.sys.natmtot
        maxaa, maxnlo = b.maxaa, max(b.maxnlo, 1)
        apwfr, lofr, veffmt = _f(rad.apwfr, np.float64), _f(rad.lofr, np.float64), _f(rad.veffmt, np.float64)
        r, keep = self._mt_radial(rad, apwfr.ctypes.data, lofr.ctypes.data if lofr.size else None,
                                  veffmt.ctypes.data)
        aa = loa = lolo = None
        if outputs:
            aa = np.zeros((maxaa, maxaa, nat), dtype=np.complex128, order="F")
            loa = np.zeros((maxnlo, maxaa, nat), dtype=np.complex128, order="F")
            lolo = np.zeros((maxnlo, maxnlo, nat), dtype=np.complex128, order="F")
        self._check(self.lib.exs_hmlint(self.ctx, ctypes.byref(r), _ptr(aa), _ptr(loa), _ptr(lolo)))
        return aa, loa, lolo

    def wavefmt(self, gk, apwalm, evecfv, rad, *, lrstp: int = 1, lmax: int | None = None, ld: int | None = None):
        """Muffin-tin wavefunction coefficients wfmt(ld, nrc, natmtot, nst)
        of the states evecfv(nmat, nst) at the G+k set ``gk``, from the
        matching coefficients ``apwalm`` (as match returns them) and the
        radial functions of ``rad`` (system.MtRadial): src/wavefmt.f90 for
        every atom and state."""
        b = self.sys.basis
        lmax = b.lmaxapw if lmax is None else lmax
        ld = (lmax + 1) ** 2 if ld is None else ld
        ev = np.asfortranarray(evecfv, dtype=np.complex128)
        nst = ev.shape[1]
        alm = np.zeros((self.ngkmax, b.apwordmax, b.lmmaxapw, self.sys.natmtot), dtype=np.complex128, order="F")
        alm[: apwalm.shape[0]] = apwalm[: self.ngkmax]
        apwfr, lofr = _f(rad.apwfr, np.float64), _f(rad.lofr, np.float64)
        r, keep = self._mt_radial(rad, apwfr.ctypes.data, lofr.ctypes.data if lofr.size else None, None)
        nrc = (int(rad.nrmtmax) - 1) // lrstp + 1 if lrstp >= 1 else 1      # lrstp < 1: the library's error
        out = np.zeros((ld, nrc, self.sys.natmtot, nst), dtype=np.complex128, order="F")
        self._check(self.lib.exs_wavefmt(self.ctx, gk.ngp, _ptr(alm), nst, _ptr(ev), ev.shape[0], lrstp, lmax,
                                         ctypes.byref(r), ld, _ptr(out)))
        return out

    def olprad(self, rad, *, outputs: bool = True):
        """Overlap radial integrals (oalo, ololo, h1aa, h1loa, h1lolo) of ``rad``,
        installed on the device; the h1 arrays are None unless relativity is iora*."""
        b, nat = self.sys.basis, self.sys.natmtot
        nlo = max(b.nlomax, 1)
        apwfr, lofr, veffmt = _f(rad.apwfr, np.float64), _f(rad.lofr, np.float64), _f(rad.veffmt, np.float64)
        r, keep = self._mt_radial(rad, apwfr.ctypes.data, lofr.ctypes.data if lofr.size else None,
                                  veffmt.ctypes.data)
        iora = self.sys.relativity == "iora*"
        out = [None] * 5
        if outputs:
            out = [np.zeros((b.apwordmax, nlo, nat), order="F"), np.zeros((nlo, nlo, nat), order="F"),
                   np.zeros((b.apwordmax, b.apwordmax, b.lmaxapw + 1, nat), order="F") if iora else None,
                   np.zeros((b.apwordmax, nlo, nat), order="F") if iora else None,
                   np.zeros((nlo, nlo, nat), order="F") if iora else None]
        self._check(self.lib.exs_olprad(self.ctx, ctypes.byref(r), *[_ptr(a) for a in out]))
        return tuple(out)

    def olprad_device(self, rad, apwfr_ptr: int, lofr_ptr: int | None, veffmt_ptr: int):
        """exs_olprad_device: inputs already on the device; enqueued, no outputs."""
        r, keep = self._mt_radial(rad, apwfr_ptr, lofr_ptr, veffmt_ptr)
        return self._check(self.lib.exs_olprad_device(self.ctx, ctypes.byref(r)))

    def hmlint_device(self, rad, apwfr_ptr: int, lofr_ptr: int | None, veffmt_ptr: int):
        """exs_hmlint_device: radial functions and potential already on the
        device (their layouts as in system.MtRadial); enqueued, no outputs."""
        r, keep = self._mt_radial(rad, apwfr_ptr, lofr_ptr, veffmt_ptr)
        return self._check(self.lib.exs_hmlint_device(self.ctx, ctypes.byref(r)))

    def set_precision(self, mode: str = "fp64", slices: int = 7):
        """fp64; ozaki (``slices`` int8 slices); ozaki_mod (``slices`` moduli, 0 = automatic)."""
        m = {"fp64": 0, "ozaki": 1, "ozaki_mod": 2}[mode]
        self._check(self.lib.exs_set_precision(self.ctx, m, slices))

    # ------------------------------------------------------------------
    def set_wait_limit(self, cycles: int = 0):
        """Limit (SM cycles) of the split-precision kernels' pipeline waits; 0 = the default (~1 s)."""
        self._check(self.lib.exs_set_wait_limit(self.ctx, int(cycles)))

    def match(self, gk):
        """apwalm(ngkmax, apwordmax, lmmaxapw, natmtot) from the reference's match inputs."""
        b = self.sys.basis
        n = self.ngkmax
        gpc = np.zeros(n); gpc[: gk.ngp] = gk.gpc
        tpgpc = np.zeros((2, n), order="F"); tpgpc[:, : gk.ngp] = gk.tpgpc
        sf = np.zeros((n, self.sys.natmtot), dtype=np.complex128, order="F")
        sf[: gk.ngp] = gensfacgp(gk.vgpc, self.sys.crystal.atposc)
        apwalm = np.zeros((n, b.apwordmax, b.lmmaxapw, self.sys.natmtot), dtype=np.complex128, order="F")
        rc = self._check(self.lib.exs_match(self.ctx, gk.ngp, _ptr(gpc), _ptr(tpgpc), _ptr(sf), _ptr(apwalm)))
        return apwalm, rc

    def _gk_arrays(self, gk):
        ig = np.zeros(self.ngkmax, dtype=np.int32); ig[: gk.ngp] = gk.igpig
        vg = np.zeros((3, self.ngkmax), order="F"); vg[:, : gk.ngp] = gk.vgpc
        return ig, vg

    def hamiltonandoverlapsetup(self, gk, apwalm=None):
        nmat = gk.ngp + self.nlotot
        h = np.empty((nmat, nmat), dtype=np.complex128, order="F")
        o = np.empty((nmat, nmat), dtype=np.complex128, order="F")
        ig, vg = self._gk_arrays(gk)
        a = None if apwalm is None else _f(apwalm, np.complex128)
        self._check(self.lib.exs_hamiltonandoverlapsetup(self.ctx, gk.ngp, _ptr(a), _ptr(ig), _ptr(vg),
                                                         _ptr(h), _ptr(o)))
        return h, o

    def setup_batched(self, gks, out=None):
        """H and O of every k-point in gks; out = optional list of (h, o) host arrays."""
        nk = len(gks)
        ngp = np.array([g.ngp for g in gks], dtype=np.int32)
        ig = np.zeros((self.ngkmax, nk), dtype=np.int32, order="F")
        vg = np.zeros((3, self.ngkmax, nk), order="F")
        for k, g in enumerate(gks):
            ig[: g.ngp, k] = g.igpig
            vg[:, : g.ngp, k] = g.vgpc
        if out is None:
            out = []
            for g in gks:
                nmat = g.ngp + self.nlotot
                out.append((np.empty((nmat, nmat), dtype=np.complex128, order="F"),
                            np.empty((nmat, nmat), dtype=np.complex128, order="F")))
        hp = (ctypes.c_void_p * nk)(*[o[0].ctypes.data for o in out])
        op = (ctypes.c_void_p * nk)(*[o[1].ctypes.data for o in out])
        self._check(self.lib.exs_setup_batched(self.ctx, nk, _ptr(ngp), _ptr(ig), _ptr(vg), hp, op))
        return out

    def setup_and_solve(self, gks, nstfv):
        """Lowest nstfv eigenpairs of H x = e O x for every k-point in gks (H, O stay on the device).

        Returns (evalfv (nstfv, nk), evecfv (ldv, nstfv, nk)), ldv = nmatmax, Fortran order."""
        nk = len(gks)
        ngp = np.array([g.ngp for g in gks], dtype=np.int32)
        ig = np.zeros((self.ngkmax, nk), dtype=np.int32, order="F")
        vg = np.zeros((3, self.ngkmax, nk), order="F")
        for k, g in enumerate(gks):
            ig[: g.ngp, k] = g.igpig
            vg[:, : g.ngp, k] = g.vgpc
        ldv = self.ngkmax + self.nlotot
        ev = np.zeros((nstfv, nk), order="F")
        vec = np.zeros((ldv, nstfv, nk), dtype=np.complex128, order="F")
        self._check(self.lib.exs_setup_and_solve_batched(self.ctx, nk, _ptr(ngp), _ptr(ig), _ptr(vg), int(nstfv),
                                                         _ptr(ev), _ptr(vec), ldv))
        return ev, vec

    def _k_arrays(self, gks):
        nk = len(gks)
        ngp = np.array([g.ngp for g in gks], dtype=np.int32)
        ig = np.zeros((self.ngkmax, nk), dtype=np.int32, order="F")
        vg = np.zeros((3, self.ngkmax, nk), order="F")
        for k, g in enumerate(gks):
            ig[: g.ngp, k] = g.igpig
            vg[:, : g.ngp, k] = g.vgpc
        return ngp, ig, vg

    def rttddft_set_pmat(self, pmats):
        """Register the momentum matrix elements, one (nmat, nmat, 3) complex
        array per k-point (exs_rttddft_set_pmat)."""
        ps = [np.asfortranarray(p, dtype=np.complex128) for p in pmats]
        nmat = np.array([p.shape[0] for p in ps], dtype=np.int32)
        ld = int(max(nmat)) if len(ps) else 1
        blocks = []
        for p in ps:
            b = np.zeros((ld, ld, 3), dtype=np.complex128, order="F")
            b[: p.shape[0], : p.shape[1], :] = p
            blocks.append(b)
        ptrs = (ctypes.c_void_p * len(blocks))(*[b.ctypes.data for b in blocks])
        self._check(self.lib.exs_rttddft_set_pmat(self.ctx, len(blocks), _ptr(nmat), ptrs, ld))

    def rttddft_genpmat(self, gks, apwalms, rad, *, outputs: bool = True):
        """Momentum matrices of the k-points in gks on the device
        (exs_rttddft_genpmat), registered for rttddft_updateham; apwalms: one
        (ngkmax, apwordmax, lmmaxapw, natmtot) array per k-point (as match
        returns them).  Returns the (nmat, nmat, 3) arrays when ``outputs``."""
        nk = len(gks)
        ngp, ig, vg = self._k_arrays(gks)
        al = [np.asfortranarray(a, dtype=np.complex128) for a in apwalms]
        apwfr, lofr = _f(rad.apwfr, np.float64), _f(rad.lofr, np.float64)
        r, keep = self._mt_radial(rad, apwfr.ctypes.data, lofr.ctypes.data if lofr.size else None, None)
        nmat = [g.ngp + self.nlotot for g in gks]
        ld = max(nmat)
        outs = [np.zeros((ld, ld, 3), dtype=np.complex128, order="F") for _ in gks] if outputs else None
        ap = (ctypes.c_void_p * nk)(*[a.ctypes.data for a in al])
        op = (ctypes.c_void_p * nk)(*[o.ctypes.data for o in outs]) if outputs else None
        self._check(self.lib.exs_rttddft_genpmat(self.ctx, nk, _ptr(ngp), _ptr(ig), _ptr(vg), ap, ctypes.byref(r),
                                                 op, ld))
        if not outputs:
            return None
        return [o[: n, : n, :] for o, n in zip(outs, nmat)]

    def rttddft_updateham(self, gks, atot, calculate_overlap=True, overlap=None):
        """UpdateHam's k-loop: returns (ham_time, overlap) lists of (nmat, nmat)
        arrays; with calculate_overlap False, ``overlap`` (one array per
        k-point) is the overlap that enters the sum."""
        nk = len(gks)
        ngp, ig, vg = self._k_arrays(gks)
        nmat = [g.ngp + self.nlotot for g in gks]
        ld = max(nmat)
        ham = [np.zeros((ld, ld), dtype=np.complex128, order="F") for _ in gks]
        ovl = [np.zeros((ld, ld), dtype=np.complex128, order="F") for _ in gks]
        if not calculate_overlap:
            for k, o in enumerate(overlap):
                ovl[k][: nmat[k], : nmat[k]] = o
        at = np.ascontiguousarray(atot, dtype=np.float64)
        hp = (ctypes.c_void_p * nk)(*[h.ctypes.data for h in ham])
        op = (ctypes.c_void_p * nk)(*[o.ctypes.data for o in ovl])
        self._check(self.lib.exs_rttddft_updateham(self.ctx, nk, _ptr(ngp), _ptr(ig), _ptr(vg), _ptr(at),
                                                   1 if calculate_overlap else 0, hp, op, ld))
        return ([h[: n, : n] for h, n in zip(ham, nmat)], [o[: n, : n] for o, n in zip(ovl, nmat)])

    def rttddft_updateham_device(self, ngp, igpig_dev_ptr, vgpc_dev_ptr, atot, calculate_overlap, p_ptrs, h_ptrs,
                                 o_ptrs):
        nk = len(ngp)
        ngp = np.asarray(ngp, dtype=np.int32)
        at = np.ascontiguousarray(atot, dtype=np.float64)
        pp = (ctypes.c_void_p * nk)(*p_ptrs)
        hp = (ctypes.c_void_p * nk)(*h_ptrs)
        op = (ctypes.c_void_p * nk)(*o_ptrs)
        return self._check(self.lib.exs_rttddft_updateham_device(
            self.ctx, nk, _ptr(ngp), ctypes.c_void_p(igpig_dev_ptr), ctypes.c_void_p(vgpc_dev_ptr), _ptr(at),
            1 if calculate_overlap else 0, pp, hp, op))

    def setup_batched_device(self, ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs):
        """Device-resident batched setup: pointers are device addresses (ints)."""
        nk = len(ngp)
        ngp = np.asarray(ngp, dtype=np.int32)
        hp = (ctypes.c_void_p * nk)(*h_ptrs)
        op = (ctypes.c_void_p * nk)(*o_ptrs)
        return self._check(self.lib.exs_setup_batched_device(self.ctx, nk, _ptr(ngp), ctypes.c_void_p(igpig_dev_ptr),
                                                             ctypes.c_void_p(vgpc_dev_ptr), hp, op))

    def _device_batch_args(self, ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs):
        nk = len(ngp)
        ngp = np.asarray(ngp, dtype=np.int32)
        hp = (ctypes.c_void_p * nk)(*h_ptrs)
        op = (ctypes.c_void_p * nk)(*o_ptrs)
        return (nk, ngp, hp, op), (self.ctx, nk, _ptr(ngp), ctypes.c_void_p(igpig_dev_ptr),
                                   ctypes.c_void_p(vgpc_dev_ptr), hp, op)

    def autotune(self, ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs) -> int:
        """Time every kernel configuration of the active precision on this batch
        (device pointers as for setup_batched_device) and keep the fastest."""
        keep, args = self._device_batch_args(ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs)
        choice = ctypes.c_int(-1)
        self._check(self.lib.exs_autotune(*args, ctypes.byref(choice)))
        return choice.value

    def hmlistln(self, gk, h):
        """Add the interstitial H term to the upper triangle of h (Fortran-ordered, in place)."""
        assert h.flags.f_contiguous and h.dtype == np.complex128
        ig, vg = self._gk_arrays(gk)
        return self._check(self.lib.exs_hmlistln(self.ctx, gk.ngp, _ptr(ig), _ptr(vg), _ptr(h), h.shape[0]))

    def olpistln(self, gk, o):
        """Add the interstitial O term to the upper triangle of o (Fortran-ordered, in place)."""
        assert o.flags.f_contiguous and o.dtype == np.complex128
        ig, vg = self._gk_arrays(gk)
        return self._check(self.lib.exs_olpistln(self.ctx, gk.ngp, _ptr(ig), _ptr(vg), _ptr(o), o.shape[0]))

    def interstitial_device(self, which, ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptr, o_ptr, ld):
        """Device form (which: 1 H, 2 O, 3 both); asynchronous on the context's stream."""
        return self._check(self.lib.exs_interstitial_device(
            self.ctx, int(which), int(ngp), ctypes.c_void_p(igpig_dev_ptr), ctypes.c_void_p(vgpc_dev_ptr),
            ctypes.c_void_p(h_ptr) if h_ptr else None, ctypes.c_void_p(o_ptr) if o_ptr else None, int(ld)))

    def interstitial_batched_device(self, which, ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs, ld):
        """All k-points of a batch in one launch (device pointers as for setup_batched_device)."""
        nk = len(ngp)
        ngp = np.asarray(ngp, dtype=np.int32)
        ld = np.asarray(ld, dtype=np.int32)
        hp = (ctypes.c_void_p * nk)(*h_ptrs)
        op = (ctypes.c_void_p * nk)(*o_ptrs)
        return self._check(self.lib.exs_interstitial_batched_device(
            self.ctx, int(which), nk, _ptr(ngp), ctypes.c_void_p(igpig_dev_ptr), ctypes.c_void_p(vgpc_dev_ptr),
            hp, op, _ptr(ld)))

    def set_kernel_config(self, cfg: int):
        """Force a split-precision kernel configuration (0 .. EXS_OZ_NCONFIG-1)."""
        return self._check(self.lib.exs_set_kernel_config(self.ctx, int(cfg)))

    def graph(self, ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs) -> "SetupGraph":
        """Capture the batched device setup of these buffers into a CUDA graph."""
        keep, args = self._device_batch_args(ngp, igpig_dev_ptr, vgpc_dev_ptr, h_ptrs, o_ptrs)
        g = ctypes.c_void_p()
        self._check(self.lib.exs_graph_create(*args, ctypes.byref(g)))
        return SetupGraph(self, g)

    COPY_MODES = {"auto": 0, "direct": 1, "packed": 2, "upper": 3}

    def set_host_copy_mode(self, mode: str):
        """How the host-pointer calls bring H and O back: "auto", "direct", "packed" or "upper"."""
        return self._check(self.lib.exs_set_host_copy_mode(self.ctx, self.COPY_MODES[mode]))

    def set_stream(self, stream_ptr: int | None):
        """Run on a caller-owned cudaStream_t (its integer handle); None = own stream."""
        return self._check(self.lib.exs_set_stream(self.ctx, None if not stream_ptr else ctypes.c_void_p(stream_ptr)))

    def synchronize(self):
        return self._check(self.lib.exs_synchronize(self.ctx))

    def last_timings(self):
        """Device ms of the last setup's phases (match, h_a A, MT + interstitial,
        lo blocks, total) and of the last RT-TDDFT combination."""
        t = np.zeros(6)
        self.lib.exs_last_timings(self.ctx, _ptr(t), 6)
        return t

    def forcek(self, gk, evecfv, evalfv, occsv, wkpt, forceibs=None):
        """IBS force of one k-point accumulated into forceibs(3, natmtot)."""
        s = self.sys
        ig, vg = self._gk_arrays(gk)
        ev = _f(evecfv, np.complex128)
        ffacg = _f(np.stack([ffacg_species(s.gv.gc[: s.gv.ngvec], r, s.crystal.omega) for r in s.rmt], axis=1),
                   np.float64)
        vgc = _f(s.gv.vgc[:, : s.gv.ngvec], np.float64)
        f = np.zeros((3, s.natmtot), order="F") if forceibs is None else forceibs
        self._check(self.lib.exs_forcek(self.ctx, gk.ngp, _ptr(ig), _ptr(vg), ev.shape[1], _ptr(ev), ev.shape[0],
                                        _ptr(_f(evalfv, np.float64)), _ptr(_f(occsv, np.float64)), float(wkpt),
                                        _ptr(ffacg), _ptr(vgc), _ptr(f)))
        return f


    def _force_inputs(self):
        """ffacg(ngvec, nspecies) and vgc(3, ngvec): fixed for the crystal,
        computed once (the reference's genffacg runs once per run too)."""
        if getattr(self, "_fk_inputs", None) is None:
            s = self.sys
            ffacg = _f(np.stack([ffacg_species(s.gv.gc[: s.gv.ngvec], r, s.crystal.omega) for r in s.rmt], axis=1),
                       np.float64)
            self._fk_inputs = (ffacg, _f(s.gv.vgc[:, : s.gv.ngvec], np.float64))
        return self._fk_inputs

    def adjoint(self, gk, c, w, eps, *, dveffig: bool = False, dh: bool = False, out=None):
        """Adjoint of the setup for L = sum_n w_n c_n^H (H - eps_n O) c_n
        (exs_adjoint): (dL/dtau (3, natmtot), dL/dV (ngvec) or None,
        dL/dh_a (maxaa, maxaa, natmtot) or None).  ``out``: a tuple of such
        arrays (as an earlier call returned them) to write into instead of
        new ones."""
        s = self.sys
        ig, vg = self._gk_arrays(gk)
        cv = _f(c, np.complex128)
        ffacg, vgc = self._force_inputs()
        if out is not None:
            dtau, dv, dhv = out
        else:
            dtau = np.zeros((3, s.natmtot), order="F")
            dv = np.zeros(s.gv.ngvec, dtype=np.complex128) if dveffig else None
            dhv = np.zeros((self.maxaa, self.maxaa, s.natmtot), dtype=np.complex128, order="F") if dh else None
        self._check(self.lib.exs_adjoint(self.ctx, gk.ngp, _ptr(ig), _ptr(vg), cv.shape[1], _ptr(cv), cv.shape[0],
                                         _ptr(_f(w, np.float64)), _ptr(_f(eps, np.float64)), _ptr(ffacg),
                                         _ptr(vgc), _ptr(dtau), None if dv is None else _ptr(dv),
                                         None if dhv is None else _ptr(dhv)))
        return dtau, dv, dhv


class SetupGraph:
    """A captured batched setup (exs_graph_*): launch() replays it on the
    (first) context's stream; synchronize() waits and reports device errors."""

    def __init__(self, setup: Setup, handle, others=()):
        self.setup = setup
        self.handle = handle
        self.others = list(others)          # further contexts of a multi-context graph

    def launch(self):
        return self.setup._check(self.setup.lib.exs_graph_launch(self.handle))

    def synchronize(self):
        return self.setup._check(self.setup.lib.exs_graph_synchronize(self.handle))

    def close(self):
        if self.handle:
            self.setup.lib.exs_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ozaki_moduli(n: int, K: int, kx: int):
    """The modular plan of exs_set_precision(EXS_PREC_OZAKI_MOD, n) for contraction
    length K and per-atom windows of kx rows: (moduli, CRT constants, b, bx, h)."""
    lib = abi.load()
    n_out, b, bx, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    p = np.zeros(16, dtype=np.int32)
    c = np.zeros(16, dtype=np.uint64)
    rc = lib.exs_ozaki_moduli(int(n), int(K), int(kx), ctypes.byref(n_out), _ptr(p), _ptr(c), ctypes.byref(b),
                              ctypes.byref(bx), ctypes.byref(h))
    if rc != 0:
        raise abi.ExsError(rc, "no modular plan for n=%d K=%d kx=%d" % (n, K, kx))
    m = n_out.value
    return [int(x) for x in p[:m]], [int(x) for x in c[:m]], b.value, bx.value, h.value


def multi_graph(setups, batches) -> SetupGraph:
    """One CUDA graph over several contexts (exs_graph_create_multi).

    ``batches[i]`` = (ngp list, igpig device pointer, vgpc device pointer,
    h device pointers, o device pointers) for ``setups[i]``, as for
    ``Setup.setup_batched_device``."""
    n = len(setups)
    P = ctypes.c_void_p
    keep = []
    ctxs = (P * n)(*[s.ctx for s in setups])
    nk = np.array([len(b[0]) for b in batches], dtype=np.int32)
    ngp_arrs = [np.asarray(b[0], dtype=np.int32) for b in batches]
    keep += ngp_arrs
    ngp_p = (P * n)(*[a.ctypes.data for a in ngp_arrs])
    ig_p = (P * n)(*[b[1] for b in batches])
    vg_p = (P * n)(*[b[2] for b in batches])
    harr = [(P * len(b[3]))(*b[3]) for b in batches]
    oarr = [(P * len(b[4]))(*b[4]) for b in batches]
    keep += harr + oarr
    h_p = (P * n)(*[ctypes.addressof(a) for a in harr])
    o_p = (P * n)(*[ctypes.addressof(a) for a in oarr])
    g = P()
    lib = setups[0].lib
    rc = lib.exs_graph_create_multi(n, ctxs, _ptr(nk), ngp_p, ig_p, vg_p, h_p, o_p, ctypes.byref(g))
    if rc < 0:
        for s in setups:
            err = lib.exs_last_error(s.ctx)
            if err:
                raise abi.ExsError(rc, err.decode())
        raise abi.ExsError(rc, "exs_graph_create_multi failed")
    return SetupGraph(setups[0], g, setups[1:])
