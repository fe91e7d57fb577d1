"""G-vector numbering as the reference's gengvec leaves it (no GPU).

src/gengvec.f90:73-74 sorts the FFT box by |G| with sort_index_1d, the
heapsort of src/sorting.f90:74-117, which is not stable: G-vectors of equal
length come out in an order set by the heapsort's steps.  The library's
exs_sort_index_1d must reproduce that order exactly; it is checked against a
line-by-line Python transcription of the Fortran routine below (1-based
positions kept), on inputs full of ties.  The host's gengvec must then sort
by length with it, with bvec and omega from reciplat's arithmetic.
"""
import numpy as np
import pytest

from exciting_b200 import crystal as C


def sort_index_1d_real(a):
    """src/sorting.f90:74-117 transcribed (1-based idx, strict '<')."""
    n = len(a)
    idx = [0] + list(range(1, n + 1))           # idx[1..n]
    if n == 1:
        return idx[1:]
    l, k = n // 2 + 1, n
    while True:
        if l > 1:
            l = l - 1
            m = idx[l]
        else:
            m = idx[k]
            idx[k] = idx[1]
            k = k - 1
            if k == 1:
                idx[1] = m
                break
        i, j = l, l + l
        while j <= k:
            if j < k and a[idx[j] - 1] < a[idx[j + 1] - 1]:
                j = j + 1
            if a[m - 1] < a[idx[j] - 1]:
                idx[i] = idx[j]
                i = j
                j = j + j
            else:
                j = k + 1
        idx[i] = m
    return idx[1:]


@pytest.mark.parametrize("n,levels", [(1, 1), (2, 1), (5, 2), (64, 3), (999, 7), (4096, 40)])
def test_heapsort_matches_the_fortran_routine(n, levels):
    rng = np.random.default_rng(n)
    a = rng.integers(0, levels, n).astype(np.float64)
    got = C.sort_index_1d(a) + 1
    assert list(got) == sort_index_1d_real(list(a))
    assert np.all(np.diff(a[got - 1]) >= 0)


def test_heapsort_is_not_the_stable_order():
    a = np.array([1.0, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, 0.0])
    heap = C.sort_index_1d(a)
    assert list(heap) != list(np.argsort(a, kind="stable"))
    assert np.all(np.diff(a[heap]) >= 0)


def test_gengvec_numbers_by_the_heapsort():
    avec = np.array([[5.13, 5.13, 0.0], [5.13, 0.0, 5.13], [0.0, 5.13, 5.13]]).T
    gv = C.gengvec(avec, 12.0)
    bvec, omega = C.reciplat(avec)
    assert np.array_equal(C.reciprocal(avec), bvec)
    assert abs(omega - abs(np.linalg.det(avec))) <= 1e-12 * omega
    # lengths recomputed in the box's loop order, then the heapsort's order
    r = [np.arange(gv.intgv[j, 0], gv.intgv[j, 1] + 1) for j in range(3)]
    i1, i2, i3 = [x.ravel() for x in np.meshgrid(*r, indexing="ij")]
    v = i1[None, :] * bvec[:, 0:1] + i2[None, :] * bvec[:, 1:2] + i3[None, :] * bvec[:, 2:3]
    gc = np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    order = np.array(sort_index_1d_real(list(gc))) - 1
    assert np.array_equal(gv.ivg, np.stack([i1[order], i2[order], i3[order]]))
    assert np.array_equal(gv.gc, gc[order])
    # ivgig inverts ivg
    lo = gv.intgv[:, 0]
    assert np.array_equal(gv.ivgig[gv.ivg[0] - lo[0], gv.ivg[1] - lo[1], gv.ivg[2] - lo[2]],
                          np.arange(1, gv.ngrtot + 1))
