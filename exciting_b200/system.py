"""Inputs of the per-k-point H/O setup, gathered in one container.

``LapwSystem`` holds what the reference keeps in module globals and hands to
``match``/``hamiltonsetup``/``overlapsetup``/``forcek``:

* per run:            lattice, atoms, basis (apword, lo), G-vector tables
                      (``ivg``, ``ivgig``, ``intgv``, ``vgc``, ``ngvec``)
* per SCF iteration:  MT integrals ``mt_hscf%main%{aa,loa,lolo}``
                      (src/mod_eigensystem.F90:43-60), ``oalo``, ``ololo``,
                      the optional IORA terms ``h1aa``/``h1loa``/``h1lolo``,
                      ``veffig``, ``cfunig``, ``meffig``/``m2effig`` and the
                      tails of the APW radial functions used by ``match``
* per k-point:        the G+k set (``GkSet``)

Array shapes follow the reference's Fortran declarations and every array is
kept Fortran-ordered so that it can be handed to the C-ABI as is.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from .basis import Basis
from .crystal import Crystal, GVectors, GkSet, gengpvec

RELATIVITY = {"none": 0, "zora": 1, "iora*": 2}


def farr(a, dtype):
    """Fortran-ordered copy of a with the given dtype."""
    return np.asfortranarray(np.asarray(a, dtype=dtype))


@dataclass
class LapwSystem:
    crystal: Crystal
    basis: Basis
    gv: GVectors
    gmaxvr: float
    rgkmax: float
    gkmax: float
    relativity: str                   # "none" | "zora" | "iora*"
    np_tail: int                      # max(apwordmax+1, 4) (match.f90:87)
    spr_tail: np.ndarray              # (np, nspecies)
    apwfr_tail: np.ndarray            # (np, apwordmax, lmaxapw+1, natmtot)
    rmt: np.ndarray                   # (nspecies,)
    mt_aa: np.ndarray                 # (maxaa, maxaa, natmtot) complex
    mt_loa: np.ndarray                # (maxnlo, maxaa, natmtot) complex
    mt_lolo: np.ndarray               # (maxnlo, maxnlo, natmtot) complex
    oalo: np.ndarray                  # (apwordmax, nlomax, natmtot) real
    ololo: np.ndarray                 # (nlomax, nlomax, natmtot) real
    veffig: np.ndarray                # (ngvec,) complex
    cfunig: np.ndarray                # (ngrtot,) complex
    meffig: Optional[np.ndarray] = None    # (ngvec,) complex, relativity != none
    m2effig: Optional[np.ndarray] = None   # (ngvec,) complex, iora*
    h1aa: Optional[np.ndarray] = None      # (apwordmax, apwordmax, lmaxapw+1, natmtot) real
    h1loa: Optional[np.ndarray] = None     # (apwordmax, nlomax, natmtot) real
    h1lolo: Optional[np.ndarray] = None    # (nlomax, nlomax, natmtot) real
    kpoints: Optional[np.ndarray] = None   # (nkpt, 3) lattice coordinates
    name: str = ""

    # --- derived sizes ---------------------------------------------------
    @property
    def natmtot(self) -> int:
        return self.crystal.natmtot

    @property
    def kinetic_weight(self) -> np.ndarray:
        """Table multiplying (k+G).(k+G')/2 in H_I: meffig unless relativity is
        "none", then cfunig (src/src_eigensystem/hmlistln.f90:61-86)."""
        if self.relativity == "none":
            return self.cfunig[: self.gv.ngvec]
        return self.meffig

    @property
    def h1on(self) -> bool:
        return self.relativity == "iora*"

    def gkset(self, vpl) -> GkSet:
        return gengpvec(vpl, self.crystal.bvec, self.gv, self.gkmax)

    def gksets(self):
        return [self.gkset(v) for v in self.kpoints]

    def ngkmax(self, gks=None) -> int:
        gks = gks if gks is not None else self.gksets()
        return max(g.ngp for g in gks)

    def nmat(self, gk: GkSet) -> int:
        """nmat = ngk + nlotot (src/init1.f90:474)."""
        return gk.ngp + self.basis.nlotot


@dataclass
class MtRadial:
    """Inputs of the muffin-tin integral generation ``hmlint``
    (src/src_eigensystem/hmlint.f90:52-55): full radial functions on the
    muffin-tin meshes and the effective potential in real spherical
    harmonics, as the reference keeps them in ``apwfr``, ``lofr``,
    ``veffmt`` and ``spr``."""
    lmaxvr: int                       # potential expanded to l <= lmaxvr
    nrmt: np.ndarray                  # (nspecies,) int32, radial points per species
    spr: np.ndarray                   # (nrmtmax, nspecies)
    apwfr: np.ndarray                 # (nrmtmax, 2, apwordmax, lmaxapw+1, natmtot): u, du/dr
    lofr: np.ndarray                  # (nrmtmax, 2, nlomax, natmtot): v, dv/dr
    veffmt: np.ndarray                # (lmmaxvr, nrmtmax, natmtot)

    @property
    def nrmtmax(self) -> int:
        return self.spr.shape[0]

    @property
    def lmmaxvr(self) -> int:
        return (self.lmaxvr + 1) ** 2
