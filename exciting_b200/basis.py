"""APW/lo basis bookkeeping: orders, local-orbital index map and block sizes.

Mirrors of the reference's index set-up, used by the host side of the library
and by the test harness:

* ``idxlm``     -- packed lm = l(l+1)+m (0-based here; the reference is 1-based)
* ``MaxAPWs``   -- src/mod_eigensystem.F90:151-184 (``maxaa``)
* ``MTInitAll`` -- src/mod_eigensystem.F90:194-235 (``losize``, ``maxnlo``)
* ``genidxlo``  -- src/genidxlo.f90:13-40 (``idxlo``, ``nlotot``)

The APW row order inside one atom's block is (l, m, io) with io fastest, l up
to ``lmaxmat`` (src/src_eigensystem/hamiltonsetup.f90:59-71).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def idxlm(l: int, m: int) -> int:
    """0-based packed (l, m) index; the reference's idxlm(l, m) minus one."""
    return l * (l + 1) + m


@dataclass
class Basis:
    """Per-species APW orders and local orbitals.

    ``apword[is_][l]`` for l = 0..lmaxapw; ``lorbl[is_]`` lists the l of each
    local orbital of species is_ (its length is ``nlorb``).
    """

    lmaxapw: int
    lmaxmat: int
    apword: list                 # [nspecies][lmaxapw+1]
    lorbl: list                  # [nspecies][nlorb]
    atom_species: list           # species index per atom
    # derived
    apwordmax: int = field(init=False)
    maxaa: int = field(init=False)
    losize: list = field(init=False)
    maxnlo: int = field(init=False)
    nlomax: int = field(init=False)
    lolmax: int = field(init=False)
    idxlo: np.ndarray = field(init=False)   # (lolmmax, nlomax, natmtot), 1-based values, 0 = unused
    nlotot: int = field(init=False)

    def __post_init__(self):
        if self.lmaxmat > self.lmaxapw:
            raise ValueError("lmaxmat must not exceed lmaxapw")
        nsp = len(self.apword)
        self.apwordmax = max(max(a) for a in self.apword)
        # MaxAPWs
        self.maxaa = max(self.napw_species(is_) for is_ in range(nsp))
        self.nlomax = max([len(x) for x in self.lorbl] + [1])
        self.lolmax = max([max(x) for x in self.lorbl if len(x)] + [0])
        lolmmax = (self.lolmax + 1) ** 2
        nat = len(self.atom_species)
        # genidxlo: running index over species -> atoms -> lo -> m
        self.idxlo = np.zeros((lolmmax, self.nlomax, nat), dtype=np.int32, order="F")
        i = 0
        for is_ in range(nsp):
            for ias in self.atoms_of(is_):
                for ilo, l in enumerate(self.lorbl[is_]):
                    for m in range(-l, l + 1):
                        i += 1
                        self.idxlo[idxlm(l, m), ilo, ias] = i
        self.nlotot = i
        # MTInitAll: losize per species
        self.losize = [sum(2 * l + 1 for l in self.lorbl[is_]) for is_ in range(nsp)]
        self.maxnlo = max(self.losize + [0])

    @property
    def nspecies(self) -> int:
        return len(self.apword)

    @property
    def natmtot(self) -> int:
        return len(self.atom_species)

    @property
    def lmmaxapw(self) -> int:
        return (self.lmaxapw + 1) ** 2

    def atoms_of(self, is_: int):
        return [ias for ias, s in enumerate(self.atom_species) if s == is_]

    def napw_species(self, is_: int) -> int:
        """Number of APW functions of one atom of species is_ (l <= lmaxmat)."""
        return sum((2 * l + 1) * self.apword[is_][l] for l in range(self.lmaxmat + 1))

    def napw_atom(self, ias: int) -> int:
        return self.napw_species(self.atom_species[ias])

    def lo_offset(self, ias: int) -> int:
        """0-based first lo row of atom ias within the lo block (idxlo of its first function - 1)."""
        is_ = self.atom_species[ias]
        if not self.lorbl[is_]:
            return -1
        l = self.lorbl[is_][0]
        return int(self.idxlo[idxlm(l, -l), 0, ias]) - 1

    def apw_rows(self, is_: int):
        """List of (l, m, io) in the APW row order of one atom of species is_."""
        rows = []
        for l in range(self.lmaxmat + 1):
            for m in range(-l, l + 1):
                for io in range(self.apword[is_][l]):
                    rows.append((l, m, io))
        return rows
