"""Failure detection on the device, without a GPU fault.

* Bounded pipeline waits: with the split-precision kernels' wait limit set
  to one cycle (exs_set_wait_limit), the first wait on a tensor-core stage,
  a finished product or a free stage runs out; the kernel gives up cleanly
  (its copies and products drain under the default limit, tensor memory is
  freed) and the call returns EXS_ERR_TIMEOUT from the device flag.  With
  the default limit restored the same context sets up the same k-point
  correctly.
* Index checks: a context whose G-vector table holds a corrupted vector
  (one coordinate moved far outside the FFT box) makes the G - G' lookups of
  the interstitial term leave the ivgig box; the kernels skip those reads
  and raise the device flag, and the call returns EXS_ERR_INDEX, in the FP64
  and in the split-precision contraction.
"""
import copy

import numpy as np
import pytest

import lapw_oracle as O
from exciting_b200 import workloads as W
from exciting_b200.abi import ExsError

pytestmark = pytest.mark.gpu

EXS_ERR_INDEX = -4
EXS_ERR_TIMEOUT = -7


def rel_fro(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_pipeline_wait_runs_out_and_context_stays_usable():
    from exciting_b200.fvsystem import Setup
    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[2])
    st = Setup(s)
    st.set_precision("ozaki_mod", 0)
    st.set_wait_limit(1)
    with pytest.raises(ExsError) as e:
        st.hamiltonandoverlapsetup(gk)
    assert e.value.code == EXS_ERR_TIMEOUT
    st.set_wait_limit(0)
    h, o = st.hamiltonandoverlapsetup(gk)
    hr, orf = O.hamiltonandoverlapsetup(s, gk)
    assert rel_fro(h, hr) <= 1e-12 and rel_fro(o, orf) <= 1e-12
    st.close()


@pytest.mark.parametrize("precision", ["fp64", "ozaki_mod"])
def test_corrupted_gvector_raises_index_error(precision):
    from exciting_b200.fvsystem import Setup
    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[1])
    bad = copy.copy(s)
    bad.gv = copy.copy(s.gv)
    bad.gv.ivg = np.array(s.gv.ivg, copy=True)
    g = int(gk.igpig[7]) - 1                       # a G-vector of this k-point's basis
    bad.gv.ivg[0, g] += 10 * int(np.max(np.abs(s.gv.intgv)) + 1)
    st = Setup(bad)
    if precision != "fp64":
        st.set_precision(precision, 0)
    with pytest.raises(ExsError) as e:
        st.hamiltonandoverlapsetup(gk)
    assert e.value.code == EXS_ERR_INDEX
    st.close()
