"""The host-side G-vector / G+k construction against numbers the reference printed.

tests/golden/reference_counts.json was extracted from the reference's own
test-farm outputs (INFO.OUT, KPOINTS.OUT) by tests/golden/make_golden.py.
"""
import json
import os

import numpy as np
import pytest

from exciting_b200.crystal import Crystal, gengpvec, gengvec, gkmax_of

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_counts.json")))


def _crystal(info):
    avec = np.array(info["avec_rows"]).T
    rmts = [s["rmt"] for s in info["species"]]
    sp, pos = [], []
    for i, s in enumerate(info["species"]):
        for a in s["atoms"]:
            sp.append(i)
            pos.append(a)
    return Crystal(avec, rmts, sp, np.array(pos).T), rmts


@pytest.mark.parametrize("case", sorted(GOLD))
def test_gvectors_and_nmat(case):
    info = GOLD[case]
    cr, rmts = _crystal(info)
    assert abs(cr.omega - info["omega"]) < 1e-6
    gv = gengvec(cr.avec, info["gmaxvr"])
    assert list(gv.ngrid) == info["ngrid"]                      # gridsize.f90
    assert gv.ngvec == info["ngvec"]                            # gengvec.f90
    gk = gkmax_of(info["rgkmax"], rmts)
    assert abs(gk - info["gkmax"]) < 1e-7                       # init1.f90:333-339
    ngk = []
    for k in info["kpoints"]:
        s = gengpvec(k["vkl"], cr.bvec, gv, gk)
        assert s.ngp + info["nlotot"] == k["nmat"], k          # init1.f90:474
        ngk.append(s.ngp)
    assert max(ngk) == info["ngkmax"]
    assert max(ngk) + info["nlotot"] == info["nmatmax"]


def test_ivgig_inverts_ivg():
    info = GOLD["groundstate-GGA_PBE-properties-Si"]
    cr, _ = _crystal(info)
    gv = gengvec(cr.avec, info["gmaxvr"])
    idx = gv.ivgig_lookup(gv.ivg)
    assert np.array_equal(idx, np.arange(1, gv.ngrtot + 1))
    assert np.all(np.diff(gv.gc) >= 0)                          # sorted by |G|
