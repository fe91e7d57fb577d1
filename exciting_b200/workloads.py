"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No converged potential of the reference is available, so every workload is
synthetic, built from fixed seeds (numpy PCG64):

* ``si_fcc``        -- diamond Si, fcc a = 10.26 Bohr, 2 atoms, rmt 2.1,
                       rgkmax 7, gmaxvr 12, lmaxapw = lmaxmat = 8, the 8
                       irreducible k-points of the 4x4x4 mesh.  Two basis
                       variants: "shipped" (Si.xml: apw+lo for l <= 1, lapw
                       above, 4 lo per atom, maxaa 158) and "text" (apword 2
                       for all l, one lo per l <= 2, maxaa 162).
* ``si_cube8``      -- 8-atom simple-cubic Si cell, a = 10.26, sites displaced
                       by U(+-0.02) Bohr, rgkmax 8, lmaxapw = lmaxmat = 10,
                       apword 2, 3 lo per l <= 2, shifted 3x3x3 mesh (27 k).
* ``si_fcc_random`` -- one instance of the uneven-size batch: 2-atom fcc with
                       a in U[9.8, 10.8] and rgkmax in {6, 7, 8, 9}.
* ``si_cube216``    -- 3x3x3 supercell of the 8-atom cube (a = 30.78), 216
                       atoms, U(+-0.02) displacements, rgkmax 8, lmaxapw 8.

Synthetic SCF inputs: MT integrals h_a complex Hermitian with entries
N(0,1)*exp(-(l+l')/2); APW-lo and lo-lo integrals likewise; oalo ~ N(0, 0.1);
ololo a Gram matrix (positive definite); V(G) complex with V(-G) = conj V(G)
and amplitude 0.5*exp(-|G|^2/8)*N(0,1); Theta(G) the analytic step function
of the spheres (gencfun); radial function tails smooth analytic r^l e^{-r/2}
and r^{l+1} e^{-r/3} on the default cubic mesh (300 points, rmin 1e-5).
"""
from __future__ import annotations

import math

import numpy as np

from .basis import Basis
from .crystal import Crystal, gencfun, gengvec, gkmax_of, radial_mesh_cubic
from .system import LapwSystem, farr

ALPHA = 1.0 / 137.03599911
A2 = 0.5 * ALPHA ** 2

FCC_IRREDUCIBLE_4x4x4 = np.array([
    [0.00, 0.00, 0.00], [0.25, 0.00, 0.00], [0.50, 0.00, 0.00], [0.25, 0.25, 0.00],
    [0.50, 0.25, 0.00], [0.75, 0.25, 0.00], [0.50, 0.50, 0.00], [0.75, 0.50, 0.25]])
FCC_IRREDUCIBLE_4x4x4_WEIGHTS = np.array([
    0.015625, 0.125, 0.0625, 0.09375, 0.375, 0.1875, 0.046875, 0.09375])

DIAMOND_CUBE_SITES = np.array([
    [0.00, 0.00, 0.00], [0.00, 0.50, 0.50], [0.50, 0.00, 0.50], [0.50, 0.50, 0.00],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25]])


def _apw_l_of_rows(basis: Basis, is_: int, size: int) -> np.ndarray:
    ls = np.zeros(size, dtype=np.int64)
    rows = basis.apw_rows(is_)
    for f, (l, _m, _io) in enumerate(rows):
        ls[f] = l
    return ls, len(rows)


def _lo_l_of_rows(basis: Basis, is_: int, size: int) -> np.ndarray:
    ls = np.zeros(size, dtype=np.int64)
    r = 0
    for l in basis.lorbl[is_]:
        for _m in range(-l, l + 1):
            ls[r] = l
            r += 1
    return ls, r


def _hermitian(rng, n, weight):
    z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2.0)
    return 0.5 * (z + z.conj().T) * weight


def build_system(crystal: Crystal, basis: Basis, *, rgkmax: float, gmaxvr: float = 12.0,
                 relativity: str = "none", kpoints=None, seed: int = 1,
                 nrmt: int = 300, rmin: float = 1e-5, name: str = "") -> LapwSystem:
    """Assemble a LapwSystem with seeded synthetic per-SCF inputs."""
    rng = np.random.default_rng(seed)
    gv = gengvec(crystal.avec, gmaxvr)
    gkmax = gkmax_of(rgkmax, crystal.species_rmt)
    if 2.0 * gkmax > gmaxvr + 1e-6:
        raise ValueError("2*gkmax > gmaxvr (src/init1.f90:340)")
    nsp = crystal.nspecies
    nat = crystal.natmtot
    lmaxapw = basis.lmaxapw
    apwordmax = basis.apwordmax
    np_tail = max(apwordmax + 1, 4)
    rmt = np.array(crystal.species_rmt, dtype=np.float64)

    # radial mesh tails and smooth radial functions u_{l,io}(r)
    spr_tail = np.zeros((np_tail, nsp), order="F")
    for is_ in range(nsp):
        spr_tail[:, is_] = radial_mesh_cubic(rmt[is_], nrmt, rmin)[-np_tail:]
    apwfr_tail = np.zeros((np_tail, apwordmax, lmaxapw + 1, nat), order="F")
    for ias in range(nat):
        is_ = crystal.atom_species[ias]
        r = spr_tail[:, is_]
        for l in range(lmaxapw + 1):
            scale = 1.0 + 0.05 * rng.standard_normal()
            apwfr_tail[:, 0, l, ias] = scale * r ** l * np.exp(-r / 2.0) / rmt[is_] ** l
            if apwordmax > 1:
                apwfr_tail[:, 1, l, ias] = scale * r ** (l + 1) * np.exp(-r / 3.0) / rmt[is_] ** (l + 1)
            for io in range(2, apwordmax):
                apwfr_tail[:, io, l, ias] = r ** (l + io) * np.exp(-r / (2.0 + io)) / rmt[is_] ** (l + io)

    maxaa, maxnlo, nlomax = basis.maxaa, max(basis.maxnlo, 1), basis.nlomax
    mt_aa = np.zeros((maxaa, maxaa, nat), dtype=np.complex128, order="F")
    mt_loa = np.zeros((maxnlo, maxaa, nat), dtype=np.complex128, order="F")
    mt_lolo = np.zeros((maxnlo, maxnlo, nat), dtype=np.complex128, order="F")
    oalo = np.zeros((apwordmax, nlomax, nat), order="F")
    ololo = np.zeros((nlomax, nlomax, nat), order="F")
    for ias in range(nat):
        is_ = crystal.atom_species[ias]
        la, na = _apw_l_of_rows(basis, is_, maxaa)
        w = np.exp(-(la[:na, None] + la[None, :na]) / 2.0)
        mt_aa[:na, :na, ias] = _hermitian(rng, na, w)
        ll, nl = _lo_l_of_rows(basis, is_, maxnlo)
        if nl:
            wl = np.exp(-(ll[:nl, None] + la[None, :na]) / 2.0)
            mt_loa[:nl, :na, ias] = (rng.standard_normal((nl, na))
                                     + 1j * rng.standard_normal((nl, na))) / math.sqrt(2.0) * wl
            mt_lolo[:nl, :nl, ias] = _hermitian(rng, nl, np.exp(-(ll[:nl, None] + ll[None, :nl]) / 2.0))
            nlo = len(basis.lorbl[is_])
            oalo[:, :nlo, ias] = 0.1 * rng.standard_normal((apwordmax, nlo))
            g = rng.standard_normal((nlo + 2, nlo))
            ololo[:nlo, :nlo, ias] = g.T @ g / (nlo + 2) + np.eye(nlo)

    # V(G): Hermitian in G, amplitude 0.5 exp(-|G|^2/8) N(0,1)
    ngvec = gv.ngvec
    ivg = gv.ivg[:, :ngvec]
    mig = gv.ivgig_lookup(-ivg) - 1         # index of -G (always inside the box)
    raw = (rng.standard_normal(ngvec) + 1j * rng.standard_normal(ngvec))
    amp = 0.5 * np.exp(-gv.gc[:ngvec] ** 2 / 8.0)
    veffig = 0.5 * (raw + np.conj(raw[mig])) * amp
    veffig[0] = veffig[0].real
    cfunig = gencfun(gv, crystal.species_rmt, crystal.atom_species, crystal.atposc, crystal.omega)

    meffig = m2effig = h1aa = h1loa = h1lolo = None
    if relativity != "none":
        # Theta/(1 - a2 V) to first order in a2: Theta + a2 (Theta * V); a
        # Hermitian-symmetric perturbation of cfunig of the same size.
        pert = 0.5 * (raw + np.conj(raw[mig])) * np.exp(-gv.gc[:ngvec] ** 2 / 4.0)
        meffig = cfunig[:ngvec] + 50.0 * A2 * pert
    if relativity == "iora*":
        m2effig = cfunig[:ngvec] + 100.0 * A2 * pert
        h1aa = np.zeros((apwordmax, apwordmax, lmaxapw + 1, nat), order="F")
        h1loa = np.zeros((apwordmax, nlomax, nat), order="F")
        h1lolo = np.zeros((nlomax, nlomax, nat), order="F")
        for ias in range(nat):
            for l in range(lmaxapw + 1):
                g = 1e-3 * rng.standard_normal((apwordmax, apwordmax))
                h1aa[:, :, l, ias] = g + g.T
            h1loa[:, :, ias] = 1e-3 * rng.standard_normal((apwordmax, nlomax))
            g = 1e-3 * rng.standard_normal((nlomax, nlomax))
            h1lolo[:, :, ias] = g + g.T

    return LapwSystem(
        crystal=crystal, basis=basis, gv=gv, gmaxvr=gmaxvr, rgkmax=rgkmax, gkmax=gkmax,
        relativity=relativity, np_tail=np_tail, spr_tail=spr_tail, apwfr_tail=apwfr_tail,
        rmt=rmt, mt_aa=mt_aa, mt_loa=mt_loa, mt_lolo=mt_lolo, oalo=oalo, ololo=ololo,
        veffig=farr(veffig, np.complex128), cfunig=farr(cfunig, np.complex128),
        meffig=None if meffig is None else farr(meffig, np.complex128),
        m2effig=None if m2effig is None else farr(m2effig, np.complex128),
        h1aa=h1aa, h1loa=h1loa, h1lolo=h1lolo,
        kpoints=None if kpoints is None else np.asarray(kpoints, dtype=np.float64), name=name)


def si_fcc(variant: str = "shipped", *, relativity: str = "none", seed: int = 1,
           a: float = 10.26, rgkmax: float = 7.0, lmaxapw: int = 8) -> LapwSystem:
    """Diamond Si, fcc, 2 atoms at (0,0,0) and (1/4,1/4,1/4), rmt 2.1."""
    h = a / 2.0
    avec = np.array([[h, h, 0.0], [h, 0.0, h], [0.0, h, h]]).T
    crystal = Crystal(avec, [2.1], [0, 0], np.array([[0, 0, 0], [0.25, 0.25, 0.25]]).T)
    if variant == "shipped":
        apword = [[1, 1] + [2] * (lmaxapw - 1)]
        lorbl = [[0, 1]]
    elif variant == "text":
        apword = [[2] * (lmaxapw + 1)]
        lorbl = [[0, 1, 2]]
    else:
        raise ValueError(variant)
    basis = Basis(lmaxapw=lmaxapw, lmaxmat=lmaxapw, apword=apword, lorbl=lorbl, atom_species=[0, 0])
    return build_system(crystal, basis, rgkmax=rgkmax, relativity=relativity,
                        kpoints=FCC_IRREDUCIBLE_4x4x4, seed=seed, name=f"si_fcc_{variant}")


def si_fcc_random(instance: int, *, relativity: str = "none") -> LapwSystem:
    """Instance i of the uneven-size batch: a ~ U[9.8, 10.8], rgkmax in {6,7,8,9}, seed 4+i."""
    rng = np.random.default_rng(4 + instance)
    a = float(rng.uniform(9.8, 10.8))
    rgkmax = float(rng.choice([6.0, 7.0, 8.0, 9.0]))
    s = si_fcc("text", relativity=relativity, seed=4 + instance, a=a, rgkmax=rgkmax)
    s.name = f"si_fcc_random_{instance}"
    s.kpoints = FCC_IRREDUCIBLE_4x4x4[:1] + 0.0
    return s


def shifted_mesh(n: int) -> np.ndarray:
    g = (np.arange(n) + 0.5) / n
    return np.array([[x, y, z] for x in g for y in g for z in g])


def si_cube8(*, relativity: str = "none", seed: int = 2, nk: int = 3,
             lmaxapw: int = 10, rgkmax: float = 8.0) -> LapwSystem:
    """8-atom simple-cubic Si cell a = 10.26, U(+-0.02) Bohr displacements."""
    a = 10.26
    rng = np.random.default_rng(seed)
    disp = rng.uniform(-0.02, 0.02, size=(8, 3)) / a       # Bohr -> lattice units
    atposl = (DIAMOND_CUBE_SITES + disp).T
    crystal = Crystal(np.eye(3) * a, [2.1], [0] * 8, atposl)
    basis = Basis(lmaxapw=lmaxapw, lmaxmat=lmaxapw, apword=[[2] * (lmaxapw + 1)],
                  lorbl=[[0, 0, 0, 1, 1, 1, 2, 2, 2]], atom_species=[0] * 8)
    return build_system(crystal, basis, rgkmax=rgkmax, relativity=relativity,
                        kpoints=shifted_mesh(nk), seed=seed, name="si_cube8")


def si_cube216(*, relativity: str = "none", seed: int = 5) -> LapwSystem:
    """3x3x3 supercell of the 8-atom cube, a = 30.78, 216 atoms."""
    a = 30.78
    rng = np.random.default_rng(seed)
    sites = []
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for s in DIAMOND_CUBE_SITES:
                    sites.append((s + np.array([i, j, k])) / 3.0)
    sites = np.array(sites)
    disp = rng.uniform(-0.02, 0.02, size=sites.shape) / a
    crystal = Crystal(np.eye(3) * a, [2.1], [0] * len(sites), (sites + disp).T)
    basis = Basis(lmaxapw=8, lmaxmat=8, apword=[[2] * 9], lorbl=[[0, 1, 2]],
                  atom_species=[0] * len(sites))
    kpts = np.array([[0, 0, 0], [0.5, 0, 0], [0.5, 0.5, 0], [0.5, 0.5, 0.5]])
    return build_system(crystal, basis, rgkmax=8.0, relativity=relativity,
                        kpoints=kpts, seed=seed, name="si_cube216")


Y00 = 0.28209479177387814347


def _pow_exp(r, p, a):
    """r^p exp(-r/a) and its derivative."""
    f = r ** p * np.exp(-r / a)
    d = (p * r ** (p - 1) if p > 0 else 0.0) * np.exp(-r / a) - f / a
    return f, d


def mt_radial(sys: LapwSystem, *, lmaxvr: int = 8, seed: int = 11, nrmt=300,
              rmin: float = 1e-5, nrmtmax: int | None = None):
    """Seeded full radial functions and potential for ``hmlint``.

    The APW functions continue the tails of ``sys`` (same analytic forms
    r^l e^{-r/2} and r^{l+1} e^{-r/3}, same per-(l, atom) scale), so that the
    matching coefficients and the muffin-tin integrals describe one basis.
    Local orbitals (r/R)^{l+1} (1 - r/R) e^{-r/(2+i)} vanish at the sphere
    boundary.  Potential: V_00 = (-14 e^{-2r}/r - 1)/Y00, and for l >= 1
    V_lm = 0.3 N(0,1) (r/R)^l e^{-r/R}.  lmaxvr = 8 is the reference's
    default (xml/schema/groundstate.xsd, attribute lmaxvr).  ``nrmt`` is one
    count for every species or a list per species; the arrays are padded
    with zeros to ``nrmtmax`` radial points (default: the largest nrmt)."""
    from .system import MtRadial
    rng = np.random.default_rng(seed)
    b, cr = sys.basis, sys.crystal
    nsp, nat = cr.nspecies, cr.natmtot
    nr_s = [int(nrmt)] * nsp if np.isscalar(nrmt) else [int(x) for x in nrmt]
    nrmax = int(nrmtmax or max(nr_s))
    spr = np.zeros((nrmax, nsp), order="F")
    for is_ in range(nsp):
        spr[:nr_s[is_], is_] = radial_mesh_cubic(sys.rmt[is_], nr_s[is_], rmin)
        if abs(spr[nr_s[is_] - 1, is_] - sys.spr_tail[-1, is_]) > 1e-12:
            raise ValueError("radial mesh does not end on the tail mesh")
    apwfr = np.zeros((nrmax, 2, b.apwordmax, b.lmaxapw + 1, nat), order="F")
    lofr = np.zeros((nrmax, 2, b.nlomax, nat), order="F")
    lmmaxvr = (lmaxvr + 1) ** 2
    veffmt = np.zeros((lmmaxvr, nrmax, nat), order="F")
    for ias in range(nat):
        is_ = cr.atom_species[ias]
        R = sys.rmt[is_]
        n = nr_s[is_]
        r = spr[:n, is_]
        for l in range(b.lmaxapw + 1):
            for io in range(b.apword[is_][l]):
                p, a = l + io, 2.0 + io
                f, d = _pow_exp(r, p, a)
                # scale so that the tail points are reproduced
                scale = sys.apwfr_tail[-1, io, l, ias] / f[-1]
                apwfr[:n, 0, io, l, ias] = scale * f
                apwfr[:n, 1, io, l, ias] = scale * d
        for ilo, l in enumerate(b.lorbl[is_]):
            x = r / R
            e = np.exp(-r / (2.0 + ilo))
            v = x ** (l + 1) * (1.0 - x) * e
            dv = ((l + 1) * x ** l * (1.0 - x) / R - x ** (l + 1) / R) * e - v / (2.0 + ilo)
            lofr[:n, 0, ilo, ias] = v
            lofr[:n, 1, ilo, ias] = dv
        veffmt[0, :n, ias] = (-14.0 * np.exp(-2.0 * r) / r - 1.0) / Y00
        for l in range(1, lmaxvr + 1):
            for m in range(-l, l + 1):
                veffmt[l * (l + 1) + m, :n, ias] = 0.3 * rng.standard_normal() * (r / R) ** l * np.exp(-r / R)
    return MtRadial(lmaxvr=lmaxvr, nrmt=np.array(nr_s, dtype=np.int32), spr=spr,
                    apwfr=apwfr, lofr=lofr, veffmt=veffmt)



def sic_two_species(*, relativity: str = "none", seed: int = 3) -> LapwSystem:
    """Zincblende two-species cell (a = 8.24 Bohr) with different bases per
    species: rmt 1.9 / 1.6, lmaxapw 8 with lmaxmat 7, apword 1 for l <= 1
    and 2 above with lo l = 0, 1, 2 on species 0; apword 2 with one lo
    (l = 0) on species 1.  Two k-points."""
    h = 8.24 / 2.0
    avec = np.array([[h, h, 0.0], [h, 0.0, h], [0.0, h, h]]).T
    crystal = Crystal(avec, [1.9, 1.6], [0, 1], np.array([[0, 0, 0], [0.25, 0.25, 0.25]]).T)
    basis = Basis(lmaxapw=8, lmaxmat=7, apword=[[1, 1] + [2] * 7, [2] * 9], lorbl=[[0, 1, 2], [0]],
                  atom_species=[0, 1])
    return build_system(crystal, basis, rgkmax=6.0, relativity=relativity,
                        kpoints=np.array([[0.0, 0.0, 0.0], [0.25, 0.125, 0.0]]), seed=seed, name="sic_two_species")
