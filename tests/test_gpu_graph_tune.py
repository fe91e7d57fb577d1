"""Autotuner, kernel configurations and CUDA-graph replay of the batched setup.

* every split-precision pipeline configuration gives bit-identical H and O
  (the int32 slice sums are exact, so the order of the K chunks cannot
  change them) within 1e-12 of the FP64 oracle;
* exs_autotune returns a valid configuration and leaves correct results;
* a captured graph replays the same bits as the direct call, follows new
  SCF inputs written in place (exs_set_scf_inputs), and refuses to launch
  after exs_set_precision.
"""
import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FRO = 1e-12
NK = 3


def rel_fro(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


class DeviceBatch:
    """Device buffers of a batched call (torch allocations)."""

    def __init__(self, st, gks):
        import torch
        self.torch = torch
        nk = len(gks)
        ig = np.zeros((nk, st.ngkmax), dtype=np.int32)
        vg = np.zeros((nk, st.ngkmax, 3))
        for k, g in enumerate(gks):
            ig[k, : g.ngp] = g.igpig
            vg[k, : g.ngp] = g.vgpc.T
        self.d_ig = torch.from_numpy(ig).cuda()
        self.d_vg = torch.from_numpy(vg).cuda()
        self.ngp = [g.ngp for g in gks]
        self.nmat = [n + st.nlotot for n in self.ngp]
        self.d_h = [torch.zeros(2 * m * m, dtype=torch.float64, device="cuda") for m in self.nmat]
        self.d_o = [torch.zeros(2 * m * m, dtype=torch.float64, device="cuda") for m in self.nmat]

    def args(self):
        return (self.ngp, self.d_ig.data_ptr(), self.d_vg.data_ptr(), [t.data_ptr() for t in self.d_h],
                [t.data_ptr() for t in self.d_o])

    def result(self, k):
        m = self.nmat[k]
        h = self.d_h[k].cpu().numpy().view(np.complex128).reshape(m, m).T.copy()
        o = self.d_o[k].cpu().numpy().view(np.complex128).reshape(m, m).T.copy()
        return h, o

    def clear(self):
        for t in self.d_h + self.d_o:
            t.zero_()


def _system():
    s = W.si_cube8()
    return s, s.gksets()[:NK]


@pytest.mark.parametrize("mode,n", [("ozaki", 7), ("ozaki_mod", 0)])
def test_ozaki_configurations_bit_identical(mode, n):
    from exciting_b200.fvsystem import Setup
    s, gks = _system()
    st = Setup(s, max_batch=NK)
    st.set_precision(mode, n)
    b = DeviceBatch(st, gks)
    outs = []
    for cfg in range(32):
        st.set_kernel_config(cfg)
        b.clear()
        st.setup_batched_device(*b.args())
        st.synchronize()
        outs.append([b.result(k) for k in range(NK)])
    # the same arithmetic for h_a A (bit 4) gives the same bits
    for cfg in range(1, 32):
        ref = outs[cfg & 16]
        for k in range(NK):
            assert np.array_equal(ref[k][0], outs[cfg][k][0]), cfg
            assert np.array_equal(ref[k][1], outs[cfg][k][1]), cfg
    hr, orf = O.hamiltonandoverlapsetup(s, gks[1])
    for cfg in (1, 17):
        assert rel_fro(outs[cfg][1][0], hr) <= TOL_FRO
        assert rel_fro(outs[cfg][1][1], orf) <= TOL_FRO
    with pytest.raises(Exception):
        st.set_kernel_config(32)


@pytest.mark.parametrize("prec", ["fp64", "ozaki", "ozaki_mod"])
def test_autotune_keeps_results_correct(prec):
    from exciting_b200.fvsystem import Setup
    s, gks = _system()
    st = Setup(s, max_batch=NK)
    n = 0 if prec == "ozaki_mod" else 7
    st.set_precision(prec, n)
    b = DeviceBatch(st, gks)
    choice = st.autotune(*b.args())
    assert choice in ((0,) if prec == "fp64" else tuple(range(32)))
    h, o = b.result(2)
    hr, orf = O.hamiltonandoverlapsetup(s, gks[2])
    assert rel_fro(h, hr) <= TOL_FRO and rel_fro(o, orf) <= TOL_FRO
    # the choice sticks for this shape after switching precision back and forth
    st.set_precision("fp64")
    st.set_precision(prec, n)
    b.clear()
    st.setup_batched_device(*b.args())
    st.synchronize()
    h2, o2 = b.result(2)
    assert np.array_equal(h, h2) and np.array_equal(o, o2)


@pytest.mark.parametrize("prec", ["fp64", "ozaki", "ozaki_mod"])
def test_graph_replay(prec):
    from exciting_b200.abi import ExsError
    from exciting_b200.fvsystem import Setup
    s, gks = _system()
    st = Setup(s, max_batch=NK)
    st.set_precision(prec, 0 if prec == "ozaki_mod" else 7)
    b = DeviceBatch(st, gks)
    st.setup_batched_device(*b.args())
    st.synchronize()
    ref = [b.result(k) for k in range(NK)]
    g = st.graph(*b.args())
    for _ in range(2):
        b.clear()
        g.launch()
        st.synchronize()
    for k in range(NK):
        h, o = b.result(k)
        assert np.array_equal(h, ref[k][0]) and np.array_equal(o, ref[k][1])
    # new SCF inputs are written in place: the same graph follows them
    s.veffig = s.veffig * 0.5
    st.set_scf_inputs(s)
    b.clear()
    g.launch()
    st.synchronize()
    hg, og = b.result(0)
    hr, orf = O.hamiltonandoverlapsetup(s, gks[0])
    assert rel_fro(hg, hr) <= TOL_FRO and rel_fro(og, orf) <= TOL_FRO
    # a precision change replaces buffers the graph uses
    st.set_precision("fp64")
    with pytest.raises(ExsError):
        g.launch()
    g.close()
