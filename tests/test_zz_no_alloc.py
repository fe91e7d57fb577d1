"""exs_mt_contract_noalloc, the entry point for callers that cannot allocate.

Some host programs must not call cudaMalloc once they are running (a
framework whose memory pool owns the device, a plug-in inside a host that
reserved its memory up front).  For them the library offers one entry point
that keeps its work space in a static device array instead of allocating.

Checked against the existing context entry point: on a system without local
orbitals and with the interstitial tables set to zero, the APW-APW block of
exs_hamiltonandoverlapsetup is exactly the muffin-tin sum this entry point
computes.  Two checked calls must both agree (the shared array keeps the
previous call's contents); between them a call with another layout (one
atom, fewer G+k, so other offsets, padding and tile tables) runs and its
outputs are discarded, and the second checked call runs on a non-default
stream.  Same tolerance as the other parity tests.
"""
import ctypes

import numpy as np
import pytest

from exciting_b200 import workloads as W
from exciting_b200.basis import Basis
from exciting_b200.crystal import Crystal

pytestmark = pytest.mark.gpu

TOL_FRO = 1e-12


def _system_without_lo_or_interstitial():
    h = 10.26 / 2.0
    avec = np.array([[h, h, 0.0], [h, 0.0, h], [0.0, h, h]]).T
    crystal = Crystal(avec, [2.1], [0, 0], np.array([[0, 0, 0], [0.25, 0.25, 0.25]]).T)
    basis = Basis(lmaxapw=8, lmaxmat=8, apword=[[1, 1] + [2] * 7], lorbl=[[]], atom_species=[0, 0])
    s = W.build_system(crystal, basis, rgkmax=7.0, kpoints=W.FCC_IRREDUCIBLE_4x4x4, seed=11)
    s.veffig[:] = 0.0
    s.cfunig[:] = 0.0
    return s


def test_noalloc_matches_context_entry_point_twice():
    import torch

    from exciting_b200.fvsystem import Setup

    s = _system_without_lo_or_interstitial()
    st = Setup(s)
    b = s.basis
    gk = s.gkset(s.kpoints[5])
    ngp = gk.ngp
    h_ref, o_ref = st.hamiltonandoverlapsetup(gk)
    apwalm, _ = st.match(gk)
    # the reference's apwi rows (l, m, io) of every atom (hamiltonsetup.f90:59-71)
    maxaa = b.maxaa
    apwi = np.zeros((maxaa, ngp, s.natmtot), dtype=np.complex128, order="F")
    napw = np.zeros(s.natmtot, dtype=np.int32)
    for ias in range(s.natmtot):
        f = 0
        for l in range(b.lmaxmat + 1):
            for m in range(-l, l + 1):
                for io in range(b.apword[b.atom_species[ias]][l]):
                    apwi[f, :, ias] = apwalm[:ngp, io, l * (l + 1) + m, ias]
                    f += 1
        napw[ias] = f
    dev = torch.device("cuda", 0)
    d_apwi = torch.from_numpy(np.ascontiguousarray(apwi.transpose(2, 1, 0)).view(np.float64)).to(dev)
    d_aa = torch.from_numpy(np.ascontiguousarray(s.mt_aa.transpose(2, 1, 0)).view(np.float64)).to(dev)
    lib = st.lib
    side = torch.cuda.Stream(device=dev)
    for call in range(2):
        if call == 1:
            # another layout in between: atom 0 only, 100 G+k (the first 100 columns of its apwi)
            n2 = 100
            d_a2 = torch.from_numpy(np.ascontiguousarray(apwi[:, :n2, 0].T).view(np.float64)).to(dev)
            d_h2 = torch.empty((n2, n2, 2), dtype=torch.float64, device=dev)
            d_o2 = torch.empty_like(d_h2)
            rc = lib.exs_mt_contract_noalloc(1, maxaa, napw.ctypes.data_as(ctypes.c_void_p), n2,
                                             ctypes.c_void_p(d_a2.data_ptr()), ctypes.c_void_p(d_aa.data_ptr()),
                                             ctypes.c_void_p(d_h2.data_ptr()), ctypes.c_void_p(d_o2.data_ptr()),
                                             n2, None)
            assert rc == 0
            torch.cuda.synchronize()
        d_h = torch.full((ngp, ngp, 2), float("nan"), dtype=torch.float64, device=dev)
        d_o = torch.full((ngp, ngp, 2), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        stream = None if call == 0 else ctypes.c_void_p(side.cuda_stream)
        rc = lib.exs_mt_contract_noalloc(s.natmtot, maxaa, napw.ctypes.data_as(ctypes.c_void_p), ngp,
                                         ctypes.c_void_p(d_apwi.data_ptr()), ctypes.c_void_p(d_aa.data_ptr()),
                                         ctypes.c_void_p(d_h.data_ptr()), ctypes.c_void_p(d_o.data_ptr()),
                                         ngp, stream)
        assert rc == 0
        side.synchronize()
        torch.cuda.synchronize()
        # device arrays are za(ld, ngp) column-major: [col][row][re/im]
        h = d_h.cpu().numpy().view(np.complex128)[..., 0].T
        o = d_o.cpu().numpy().view(np.complex128)[..., 0].T
        hr = h_ref[:ngp, :ngp]
        orf = o_ref[:ngp, :ngp]
        assert np.linalg.norm(h - hr) / np.linalg.norm(hr) <= TOL_FRO, call
        assert np.linalg.norm(o - orf) / np.linalg.norm(orf) <= TOL_FRO, call
    st.close()


def test_noalloc_rejects_oversized_work_space():
    from exciting_b200 import abi
    lib = abi.load()
    napw = np.full(8, 242, dtype=np.int32)
    # 8 atoms x 242 rows x 4096 G+k does not fit in the 32 MiB work space: rejected
    # before any device pointer is touched
    rc = lib.exs_mt_contract_noalloc(8, 242, napw.ctypes.data_as(ctypes.c_void_p), 4096,
                                     ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                     ctypes.c_void_p(16), 4096, None)
    assert rc == -3
