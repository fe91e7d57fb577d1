"""The oracle's restatement of src/wavefmt.f90 (no GPU): a state that is
one local-orbital row gives that local orbital's radial function in its
(l, m) row and nothing else (idxlo, lorbl and the lrstp sub-mesh of
wavefmt_add); a state on the G rows gives sum_io (sum_G b_G A) u_io; the
result is linear in the state."""
import numpy as np

import lapw_oracle as O
from exciting_b200 import workloads as W


def test_wavefmt_lo_row_and_apw_rows():
    s = W.si_fcc("shipped")
    b = s.basis
    rad = W.mt_radial(s)
    gk = s.gkset(s.kpoints[2])
    apwalm, _ = O.match(s, gk)
    ngp, nmat, lmax, ld, lrstp = gk.ngp, s.nmat(gk), b.lmaxapw, (b.lmaxapw + 1) ** 2, 2
    ias = 1
    is_ = b.atom_species[ias]
    ilo = len(b.lorbl[is_]) - 1
    l = b.lorbl[is_][ilo]
    lm = l * (l + 1) + 0
    e = np.zeros(nmat, dtype=np.complex128)
    e[ngp + int(b.idxlo[lm, ilo, ias]) - 1] = 2.0 - 1.0j
    wf = O.wavefmt(s, rad, lrstp, lmax, ias, ngp, apwalm, e, ld)
    rs = np.arange(0, int(rad.nrmt[is_]), lrstp)
    assert wf.shape == (ld, len(rs))
    assert np.array_equal(wf[lm], (2.0 - 1.0j) * rad.lofr[rs, 0, ilo, ias])
    assert not np.any(np.delete(wf, lm, axis=0))
    # G rows only: the APW part with zdotu (no conjugation)
    rng = np.random.default_rng(3)
    g = np.zeros(nmat, dtype=np.complex128)
    g[:ngp] = rng.standard_normal(ngp) + 1j * rng.standard_normal(ngp)
    wf2 = O.wavefmt(s, rad, 1, 3, 0, ngp, apwalm, g, 16)
    l, m, io = 2, -1, 0
    lm = l * (l + 1) + m
    z = np.sum(g[:ngp] * apwalm[:ngp, io, lm, 0])
    want = sum(np.sum(g[:ngp] * apwalm[:ngp, j, lm, 0]) * rad.apwfr[: int(rad.nrmt[0]), 0, j, l, 0]
               for j in range(b.apword[0][l]))
    assert abs(z) > 0
    assert np.allclose(wf2[lm], want, rtol=1e-13, atol=1e-13 * np.abs(want).max())
    # linear in the state
    wf3 = O.wavefmt(s, rad, 1, 3, 0, ngp, apwalm, g + 3 * e, 16)
    wf4 = O.wavefmt(s, rad, 1, 3, 0, ngp, apwalm, e, 16)
    assert np.allclose(wf3, wf2 + 3 * wf4, rtol=0, atol=1e-12 * np.abs(wf3).max())
