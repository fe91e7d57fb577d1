"""Crystal, G-vector and G+k tables: the host-side producers of the H/O setup inputs.

These mirror the reference's initialisation routines that build the per-run
tables the H/O setup consumes.  They are host code (run once per run or once
per k-point list), not the device hot path:

* ``gridsize``   -- src/gridsize.f90:13-52 (FFT box ``ngrid``, ``intgv``)
* ``nfftifc``    -- src/nfftifc.f90:13-40  (next 2,3,5-smooth size)
* ``gengvec``    -- src/gengvec.f90:13-123 (``ivg``, ``ivgig``, ``vgc``, ``gc``, ``ngvec``)
* ``gengpvec``   -- src/gengpvec.f90:13-97 (G+k set in ``ivg`` order)
* ``sphcrd``     -- src/src_lib/sphcrd.f90:13-58
* ``gensfacgp``  -- src/gensfacgp.f90:10-49
* ``gencfun``    -- src/gencfun.f90:13-120 (``cfunig``, the characteristic function)
* ``genffacg``   -- src/genffacg.f90:9-35
* ``genrmesh``   -- src/genrmesh.f90 (the default "cubic" muffin-tin mesh)
* ``gkmax``      -- src/init1.f90:333-339 (rgkmax / rmt of the smallest sphere)

All arrays follow the reference's Fortran layout when handed to the C-ABI
(column-major); in numpy they are held with the Fortran index order, e.g.
``ivg`` has shape (3, ngrtot) and ``vgpc`` (3, ngp).

G-vector numbering: the reference sorts the box by |G| with a heapsort
(src/sorting.f90 ``sort_index_1d``), which is not stable, so the order of
G-vectors of equal length follows from the heapsort's steps and from the last
bits of each computed length.  Both are reproduced: the lengths with the
reference's operation order (``reciplat`` for bvec, then the same sums and
square root, no fused multiply-add), the order with the library's
``exs_sort_index_1d``, the heapsort of src/sorting.f90:74-117 step for step.
``ivg``, ``ivgig``, ``igpig`` and with them the place of every H/O element
are then the reference's (given a reference build without fused
multiply-add contraction in gengvec).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

FOURPI = 4.0 * math.pi
TWOPI = 2.0 * math.pi


def nfftifc(n: int) -> int:
    """Smallest n' >= n whose only prime factors are 2, 3 and 5 (src/nfftifc.f90:13-40)."""
    if n <= 0:
        raise ValueError(f"nfftifc: n <= 0 : {n}")
    while True:
        i = n
        for p in (2, 3, 5):
            while i % p == 0:
                i //= p
        if i == 1:
            return n
        n += 1


def reciplat(avec: np.ndarray):
    """bvec and omega as src/reciplat.f90:33-53 computes them: b1 = a2 x a3,
    b2 = a3 x a1, b3 = a1 x a2 (r3cross), t1 = a1 . b1, omega = |t1|, then
    bvec = (twopi / t1) bvec, in the same floating-point order."""
    a = [avec[:, j].astype(np.float64) for j in range(3)]

    def cross(x, y):
        return [x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]]

    b = [cross(a[1], a[2]), cross(a[2], a[0]), cross(a[0], a[1])]
    t1 = float(a[0][0] * b[0][0] + a[0][1] * b[0][1] + a[0][2] * b[0][2])
    f = TWOPI / t1
    bvec = np.array([[f * b[j][i] for j in range(3)] for i in range(3)], dtype=np.float64)
    return bvec, abs(t1)


def reciprocal(avec: np.ndarray) -> np.ndarray:
    """Reciprocal lattice vectors bvec(:, j) with a_i . b_j = 2 pi delta_ij (reciplat)."""
    return reciplat(avec)[0]


def sort_index_1d(a: np.ndarray) -> np.ndarray:
    """0-based index map sorting a ascending with the reference's heapsort
    (src/sorting.f90:74-117; exs_sort_index_1d in the library)."""
    import ctypes
    from . import abi
    a = np.ascontiguousarray(a, dtype=np.float64)
    idx = np.zeros(a.size, dtype=np.int32)
    rc = abi.load().exs_sort_index_1d(a.size, a.ctypes.data_as(ctypes.c_void_p), 1,
                                      idx.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise abi.ExsError(rc, "exs_sort_index_1d")
    return idx.astype(np.int64) - 1


def gridsize(avec: np.ndarray, gmaxvr: float):
    """FFT box sizes and integer G ranges (src/gridsize.f90:27-50).

    ``avec[:, j]`` is lattice vector j.  Returns (ngrid[3], intgv[3,2]).
    """
    lens = np.sqrt(avec[0, :] ** 2 + avec[1, :] ** 2 + avec[2, :] ** 2)
    ngrid = [nfftifc(int(gmaxvr * lens[j] / math.pi) + 1) for j in range(3)]
    intgv = np.zeros((3, 2), dtype=np.int32)
    for j in range(3):
        intgv[j, 0] = ngrid[j] // 2 - ngrid[j] + 1
        intgv[j, 1] = ngrid[j] // 2
    return np.array(ngrid, dtype=np.int32), intgv


@dataclass
class GVectors:
    """Output of ``gengvec`` (src/gengvec.f90)."""

    ngrid: np.ndarray          # (3,) int32
    intgv: np.ndarray          # (3, 2) int32, inclusive bounds
    ivg: np.ndarray            # (3, ngrtot) int32, sorted by |G|
    ivgig: np.ndarray          # box (n1, n2, n3) int32, 1-based G index, Fortran order
    vgc: np.ndarray            # (3, ngrtot) float64, Cartesian G
    gc: np.ndarray             # (ngrtot,) float64, |G|
    ngvec: int                 # number of G with |G| < gmaxvr

    @property
    def ngrtot(self) -> int:
        return int(self.ivg.shape[1])

    def ivgig_lookup(self, iv: np.ndarray) -> np.ndarray:
        """ivgig(iv1, iv2, iv3) for integer triples iv (3, ...) inside the box."""
        lo = self.intgv[:, 0]
        return self.ivgig[iv[0] - lo[0], iv[1] - lo[1], iv[2] - lo[2]]


def gengvec(avec: np.ndarray, gmaxvr: float) -> GVectors:
    """G-vector tables (src/gengvec.f90:33-122)."""
    bvec = reciprocal(avec)
    ngrid, intgv = gridsize(avec, gmaxvr)
    r1 = np.arange(intgv[0, 0], intgv[0, 1] + 1)
    r2 = np.arange(intgv[1, 0], intgv[1, 1] + 1)
    r3 = np.arange(intgv[2, 0], intgv[2, 1] + 1)
    # loop order i1 (outer), i2, i3 (inner), as the reference's triple loop
    i1, i2, i3 = np.meshgrid(r1, r2, r3, indexing="ij")
    i1 = i1.ravel(); i2 = i2.ravel(); i3 = i3.ravel()
    v = (i1[None, :] * bvec[:, 0:1] + i2[None, :] * bvec[:, 1:2]
         + i3[None, :] * bvec[:, 2:3])
    gc = np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    idx = sort_index_1d(gc)                     # gengvec.f90:74, the reference's heapsort
    gc = gc[idx]
    ivg = np.stack([i1[idx], i2[idx], i3[idx]]).astype(np.int32)
    ngrtot = ivg.shape[1]
    ivgig = np.zeros((ngrid[0], ngrid[1], ngrid[2]), dtype=np.int32, order="F")
    ivgig[ivg[0] - intgv[0, 0], ivg[1] - intgv[1, 0], ivg[2] - intgv[2, 0]] = \
        np.arange(1, ngrtot + 1, dtype=np.int32)
    vgc = (ivg[0][None, :] * bvec[:, 0:1] + ivg[1][None, :] * bvec[:, 1:2]
           + ivg[2][None, :] * bvec[:, 2:3])
    below = np.nonzero(gc < gmaxvr)[0]
    ngvec = int(below[-1] + 1) if below.size else 1
    return GVectors(ngrid=ngrid, intgv=intgv, ivg=ivg, ivgig=ivgig,
                    vgc=np.ascontiguousarray(vgc), gc=gc, ngvec=ngvec)


def sphcrd(v: np.ndarray):
    """Spherical coordinates of vectors v (3, n) (src/src_lib/sphcrd.f90:30-56)."""
    eps = 1e-14
    r = np.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
    tp = np.zeros((2, v.shape[1]))
    ok = r > eps
    t1 = np.where(ok, v[2] / np.where(ok, r, 1.0), 0.0)
    t1 = np.clip(t1, -1.0, 1.0)
    tp[0] = np.where(ok, np.arccos(t1), 0.0)
    has_phi = ok & ((np.abs(v[0]) > eps) | (np.abs(v[1]) > eps))
    phi = np.arctan2(v[1], v[0])
    phi = np.where(phi < 0.0, phi + TWOPI, phi)
    tp[1] = np.where(has_phi, phi, 0.0)
    return r, tp


@dataclass
class GkSet:
    """Output of ``gengpvec`` for one k-point (src/gengpvec.f90:29-50)."""

    vpl: np.ndarray            # (3,) k in lattice coordinates
    ngp: int
    igpig: np.ndarray          # (ngp,) int32, 1-based G index
    vgpc: np.ndarray           # (3, ngp) Cartesian G+k
    gpc: np.ndarray            # (ngp,) |G+k|
    tpgpc: np.ndarray          # (2, ngp) (theta, phi)


def gengpvec(vpl, bvec: np.ndarray, gv: GVectors, gkmax: float) -> GkSet:
    """G+k vectors with |G+k| < gkmax, in ``ivg`` order (src/gengpvec.f90:29-50)."""
    vpl = np.asarray(vpl, dtype=np.float64)
    vpc = bvec @ vpl
    v = gv.vgc[:, : gv.ngvec] + vpc[:, None]
    t2 = v[0] ** 2 + v[1] ** 2 + v[2] ** 2
    sel = np.nonzero(t2 < gkmax ** 2)[0]
    vgpc = np.ascontiguousarray(v[:, sel])
    gpc, tpgpc = sphcrd(vgpc)
    return GkSet(vpl=vpl, ngp=int(sel.size), igpig=(sel + 1).astype(np.int32),
                 vgpc=vgpc, gpc=gpc, tpgpc=tpgpc)


def gensfacgp(vgpc: np.ndarray, atposc: np.ndarray) -> np.ndarray:
    """Structure factors exp(i (G+k).tau_a), shape (ngp, natmtot) (src/gensfacgp.f90:33-45)."""
    t1 = vgpc.T @ atposc  # (ngp, natmtot)
    return np.cos(t1) + 1j * np.sin(t1)


def ffacg_species(gc: np.ndarray, rmt: float, omega: float, cfdamp: float = 0.0,
                  gmaxvr: float = 12.0, epslat: float = 1e-6) -> np.ndarray:
    """Step-function form factor of one sphere (src/genffacg.f90:20-33)."""
    t1 = FOURPI / omega
    out = np.empty_like(gc)
    big = gc > epslat
    g = gc[big]
    t3 = np.exp(-((cfdamp / gmaxvr) * g) ** 2) if cfdamp != 0.0 else 1.0
    t4 = g * rmt
    out[big] = t1 * t3 * (np.sin(t4) - t4 * np.cos(t4)) / g ** 3
    out[~big] = (t1 / 3.0) * rmt ** 3
    return out


def gencfun(gv: GVectors, species_rmt, atom_species, atposc, omega: float,
            epslat: float = 1e-6) -> np.ndarray:
    """Characteristic function of the interstitial in G-space, ``cfunig(ngrtot)``.

    src/gencfun.f90:33-58 (``cfdamp`` = 0, the default).
    """
    cfunig = np.zeros(gv.ngrtot, dtype=np.complex128)
    cfunig[0] = 1.0
    for isp, rmt in enumerate(species_rmt):
        ff = ffacg_species(gv.gc, rmt, omega, epslat=epslat)
        for ias in np.nonzero(np.asarray(atom_species) == isp)[0]:
            t2 = -(gv.vgc.T @ atposc[:, ias])
            cfunig -= (np.cos(t2) + 1j * np.sin(t2)) * ff
    return cfunig


def radial_mesh_cubic(rmt: float, nrmt: int, rmin: float) -> np.ndarray:
    """Default ("cubic") muffin-tin radial mesh up to rmt (src/genrmesh.f90:37-46)."""
    ir = np.arange(1, nrmt + 1, dtype=np.float64)
    return ((ir - 1) / (nrmt - 1)) ** 3 * (rmt - rmin * nrmt) + rmin * ir


def gkmax_of(rgkmax: float, species_rmt) -> float:
    """gkmax = rgkmax / rmt of the species with the smallest sphere (src/init1.f90:333-339)."""
    return rgkmax / float(min(species_rmt))


@dataclass
class Crystal:
    """Lattice and atoms.  ``avec[:, j]`` is lattice vector j (Bohr)."""

    avec: np.ndarray
    species_rmt: list
    atom_species: list          # species index per atom (0-based)
    atposl: np.ndarray          # (3, natmtot) lattice coordinates
    bvec: np.ndarray = field(init=False)
    omega: float = field(init=False)
    atposc: np.ndarray = field(init=False)

    def __post_init__(self):
        self.avec = np.asarray(self.avec, dtype=np.float64)
        self.atposl = np.asarray(self.atposl, dtype=np.float64)
        self.bvec, self.omega = reciplat(self.avec)
        self.atposc = self.avec @ self.atposl

    @property
    def natmtot(self) -> int:
        return int(self.atposl.shape[1])

    @property
    def nspecies(self) -> int:
        return len(self.species_rmt)
