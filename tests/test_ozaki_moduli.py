"""The modular split-precision scheme (EXS_PREC_OZAKI_MOD), checked on the CPU.

The library's plan (exs_ozaki_moduli: moduli, bits per operand, the per-atom
fold's constants and headroom bits) is checked against exact integer
arithmetic, and the device arithmetic is emulated in numpy with that plan:
columns scaled by a power of two above their 2-norms, residues in
[-127, 127], one exact integer product per modulus; for the H/O products the
residues x = v mod p in [0, p) recombined with 96-bit constants C_m =
round(2^96 y_m / p_m) (the top 64 bits of sum x_m C_m mod 2^96 read as a
signed integer times M 2^-64, oz_crt_kernel); for the per-atom products the
kernel's multiply-high fold into the 64-bit wrapping sum t += r c_m with
c_m = round(2^(64+h) y_m / p_m).  The emulated products must reconstruct the
exact integer products within the stated bounds, and an emulated setup must
meet the 1e-12 Frobenius bar and keep the lowest generalized eigenvalues
within 1e-8 Ha.  No GPU is touched.
"""
import ctypes
import math

import numpy as np
import pytest

from exciting_b200 import abi


def plan(n, K, kx):
    lib = abi.load()
    n_out = ctypes.c_int()
    p = np.zeros(16, dtype=np.int32)
    c = np.zeros(16, dtype=np.uint64)
    b, bx, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = lib.exs_ozaki_moduli(n, K, kx, ctypes.byref(n_out), p.ctypes.data_as(ctypes.c_void_p),
                              c.ctypes.data_as(ctypes.c_void_p), ctypes.byref(b), ctypes.byref(bx), ctypes.byref(h))
    if rc != 0:
        return None
    m = n_out.value
    return [int(x) for x in p[:m]], [int(x) for x in c[:m]], b.value, bx.value, h.value


@pytest.mark.parametrize("n,K,kx", [(14, 1936, 242), (12, 1936, 242), (0, 1936, 242), (0, 34992, 162),
                                    (16, 65536, 512), (8, 200, 50), (0, 324, 162)])
def test_plan_constants_and_bounds(n, K, kx):
    ps, cs, b, bx, h = plan(n, K, kx)
    if n:
        assert len(ps) == n
    for i in range(len(ps)):
        assert ps[i] % 2 == 1 and ps[i] < 256
        for j in range(i):
            assert math.gcd(ps[i], ps[j]) == 1
    M = math.prod(ps)
    for p, c in zip(ps, cs):
        y = pow(M // p, -1, p)
        assert c == (((y << (64 + h)) + p // 2) // p) % 2 ** 64      # round(2^(64+h) y / p) mod 2^64
    # H/O: |X| <= 2^(2b) (1 + eps)^2, one bit of margin beyond 2|X| < M; per-atom fold: h headroom bits
    assert 2 ** (2 * b + 2) <= M and 2 ** (b + bx + h + 2) <= M
    assert h >= 5 and b <= 52 and bx <= 52
    # b, bx and h are the largest that fit (unless capped at 52)
    assert b == 52 or 2 ** (2 * (b + 1) + 2) > M
    assert bx == 52 or 2 ** (b + (bx + 1) + 5 + 2) > M
    assert 2 ** (b + bx + (h + 1) + 2) > M
    if n == 0:
        want = math.ceil(41 + 0.5 * math.log2(K) - 1e-9)
        assert b >= want and bx >= 44
        if len(ps) > 6:    # one modulus fewer would not keep the bits
            q = plan(len(ps) - 1, K, kx)
            assert q[2] < want or q[3] < 44


def test_plan_counts_of_the_benchmark_cells():
    """13 moduli at 49 bits (45 for the h_a rows, 5 headroom bits in the
    per-atom fold) for both the 8-atom cell (K = 1936) and the 216-atom cell
    (K = 34,992)."""
    for K, kx in ((1936, 242), (34992, 162)):
        ps, _, b, bx, h = plan(0, K, kx)
        assert (len(ps), b, bx, h) == (13, 49, 45, 5)


def test_plan_rejects_bad_arguments():
    assert plan(5, 1936, 242) is None          # too few moduli
    assert plan(17, 1936, 242) is None         # more than the table holds
    assert plan(14, 70000, 242) is None        # 2 K 127^2 would overflow int32
    assert plan(14, 1936, 0) is None           # no per-atom window
    assert plan(14, 0, 242) is None


def _residues(x, p):
    r = np.mod(x, p)
    return np.where(r > p // 2, r - p, r)


def _fold_reduce(v, p):
    """The kernel's reduction of an int32 sum: q = floor(v round(2^32 / p) / 2^32)."""
    mg = ((1 << 32) + p // 2) // p
    return v - ((v * mg) >> 32) * p


def emulate(X, Y, ps, cs):
    """Integer product X^T Y by the per-atom kernel's 64-bit fold."""
    t = np.zeros((X.shape[1], Y.shape[1]), dtype=np.uint64)
    rsum = np.zeros(t.shape)
    for p, c in zip(ps, cs):
        v = np.rint(_residues(X, p).T @ _residues(Y, p)).astype(np.int64)     # exact: |v| < 2^31
        assert np.abs(v).max() < 2 ** 31
        r = _fold_reduce(v, p)
        assert r.min() >= -p / 4 and r.max() <= 5 * p / 4
        rsum += np.abs(r)
        with np.errstate(over="ignore"):
            t += r.astype(np.int64).view(np.uint64) * np.uint64(c)
    return t.view(np.int64), rsum


def c96(ps):
    """The H/O recombination constants C_m = round(2^96 y_m / p_m) as three 32-bit words."""
    M = math.prod(ps)
    out = []
    for p in ps:
        y = pow(M // p, -1, p)
        c = ((y << 96) + p // 2) // p
        out.append([(c >> (32 * w)) & 0xffffffff for w in range(3)])
    return out


def crt_shift(ps, b):
    """Bits the recombination skips below the top of the 96-bit sum: the sign
    copies that |X| <= 2^2b leaves when M is far above 2^2b (at most 20)."""
    return max(0, min(20, math.floor(sum(math.log2(p) for p in ps) - 1e-9 - 2 * b - 3)))


def emulate_crt(X, Y, ps, sh=0):
    """Integer product X^T Y as the residue tiles give it: per modulus the
    residue x = (X^T Y) mod p in [0, p) (the kernel's multiply-high reduction
    of the exact int32 sum, then moved into [0, p)), recombined by the 96-bit
    sum of oz_crt_kernel (three 64-bit accumulators, carries at the end); the
    result is the signed 64-bit window sh bits below the top (2^(64+sh) X / M)."""
    C = c96(ps)
    a = [np.zeros((X.shape[1], Y.shape[1]), dtype=np.uint64) for _ in range(3)]
    for p, cw in zip(ps, C):
        v = np.rint(_residues(X, p).T @ _residues(Y, p)).astype(np.int64)
        x = _fold_reduce(v, p)
        x = np.where(x < 0, x + p, x)
        x = np.where(x >= p, x - p, x).astype(np.uint64)
        with np.errstate(over="ignore"):
            for w in range(3):
                a[w] += x * np.uint64(cw[w])
    with np.errstate(over="ignore"):
        a1 = a[1] + (a[0] >> np.uint64(32))
        a2 = a[2] + (a1 >> np.uint64(32))
        top = (a2 << np.uint64(32)) | (a1 & np.uint64(0xffffffff))
        top = (top << np.uint64(sh)) | ((a[0] & np.uint64(0xffffffff)) >> np.uint64(32 - sh))
    return top.view(np.int64)


def _norm_columns(rng, K, ncol, b):
    """Integer columns of 2-norm <= 2^b (random directions, rounded)."""
    Z = rng.standard_normal((K, ncol))
    Z *= (2.0 ** b) * (1 - 1e-9) / np.linalg.norm(Z, axis=0)
    return np.trunc(Z)


@pytest.mark.parametrize("n", [8, 12, 14])
def test_emulated_fold_reconstructs_per_atom_products(n):
    """The 64-bit fold of the per-atom products: |X| <= 2^(b + bx), t =
    2^(64+h) X / M + e with |e| <= sum |r| / 2 + 1."""
    rng = np.random.default_rng(n)
    K = 300
    ps, cs, b, bx, h = plan(n, K // 2, 8)
    X = _norm_columns(rng, K, 5, b)
    Y = _norm_columns(rng, K, 4, bx)
    Y[:, 0] = -np.trunc(X[:, 0] * 2.0 ** (bx - b))    # the bound's extreme: a nearly parallel pair
    t, rsum = emulate(X, Y, ps, cs)
    M = math.prod(ps)
    for i in range(X.shape[1]):
        for j in range(Y.shape[1]):
            exact = sum(int(a) * int(bb) for a, bb in zip(X[:, i], Y[:, j]))
            assert 2 ** (h + 1) * abs(exact) < M
            err = int(t[i, j]) * M - exact * 2 ** (64 + h)
            assert abs(err) <= (rsum[i, j] / 2 + 1) * M, (i, j)


@pytest.mark.parametrize("n", [8, 12, 13, 14, 15, 16])
def test_emulated_crt_reconstructs_ho_products(n):
    """The residue tiles' recombination: |X| <= 2^(2b), the 64-bit window sh
    bits below the top of the 96-bit sum equals floor(2^(64+sh) X / M) up to
    one unit (the constants' rounding is below 2^-85 of M), and that unit,
    M 2^-(64+sh), is at most 2^(2b-58): the window keeps ~58 bits of the
    bound 2^2b for every plan (with sh = 0, 16 moduli and b = 52 would keep
    only 42)."""
    rng = np.random.default_rng(100 + n)
    K = 300
    ps, _, b, _, _ = plan(n, K // 2, 8)
    sh = crt_shift(ps, b)
    assert sh == 0 or n >= 14
    X = _norm_columns(rng, K, 5, b)
    Y = _norm_columns(rng, K, 4, b)
    Y[:, 0] = -X[:, 0]
    top = emulate_crt(X, Y, ps, sh)
    M = math.prod(ps)
    assert M <= 2 ** (2 * b - 58 + 64 + sh)
    for i in range(X.shape[1]):
        for j in range(Y.shape[1]):
            exact = sum(int(a) * int(bb) for a, bb in zip(X[:, i], Y[:, j]))
            assert 2 ** (sh + 1) * abs(exact) < M
            assert abs(int(top[i, j]) * M - exact * 2 ** (64 + sh)) <= 2 * M, (i, j)


def _split_scaled(Z, b):
    """Columns scaled by a power of two above their 2-norm, then to integers (norm <= 2^b)."""
    m = np.sqrt((np.abs(Z) ** 2).sum(0)) * (1 + 2.0 ** -30)
    sig = np.ldexp(1.0, np.frexp(np.where(m > 0, m, 1.0))[1])
    return np.rint(Z.real / sig * 2.0 ** b), np.rint(Z.imag / sig * 2.0 ** b), sig


def _rows_scaled(X, b):
    m = np.sqrt((np.abs(X) ** 2).sum(1)) * (1 + 2.0 ** -30)
    sx = np.ldexp(1.0, np.frexp(np.where(m > 0, m, 1.0))[1])
    return np.rint(X.real / sx[:, None] * 2.0 ** b), np.rint(X.imag / sx[:, None] * 2.0 ** b), sx


def _emulated_setup(s, gk, apwalm):
    """H and O of one k-point with the APW-APW block (and B = h_a A) taken
    through the emulated integer path of the default plan."""
    import lapw_oracle as O
    N = gk.ngp
    apwi = [O._apwi(s, apwalm, N, a) for a in range(s.natmtot)]
    A = np.concatenate(apwi)
    K, kx = A.shape[0], s.basis.maxaa
    ps, cs, b, bx, h = plan(0, K, kx)
    M = float(math.prod(ps))
    ar, ai, sa = _split_scaled(A, b)
    Bs = []
    for a in range(s.natmtot):      # the per-atom products B_a = h_a A_a (A residues over the atom's rows)
        f0 = sum(x.shape[0] for x in apwi[:a])
        war, wai = ar[f0:f0 + apwi[a].shape[0]], ai[f0:f0 + apwi[a].shape[0]]
        hr, hi, sx = _rows_scaled(s.mt_aa[:, :, a], bx)
        X = np.concatenate([hr.T, hi.T])
        re = emulate(X, np.concatenate([war, -wai]), ps, cs)[0].astype(np.float64)
        im = emulate(X, np.concatenate([wai, war]), ps, cs)[0].astype(np.float64)
        Bs.append((re + 1j * im) * (M * 2.0 ** (-64 - h - b - bx)) * np.outer(sx, sa))
    B = np.concatenate(Bs)
    br, bi, sb = _split_scaled(B, b)
    XA = np.concatenate([ar, ai])                   # [Ar; Ai]
    YH = [np.concatenate([br, bi]), np.concatenate([bi, -br])]    # Re H, Im H
    YO = [np.concatenate([ar, ai]), np.concatenate([ai, -ar])]    # Re O, Im O
    sh = crt_shift(ps, b)
    scale = M * 2.0 ** (-64 - sh - 2 * b)
    out = []
    for Ys, sy in ((YH, sb), (YO, sa)):
        parts = [emulate_crt(XA, Y, ps, sh).astype(np.float64) * scale for Y in Ys]
        out.append((parts[0] + 1j * parts[1]) * np.outer(sa, sy))
    Bx = np.concatenate([s.mt_aa[:, :, a] @ apwi[a] for a in range(s.natmtot)])
    return out[0], out[1], A.conj().T @ Bx, A.conj().T @ A, B, Bx


def test_emulated_setup_meets_the_bars():
    """One Si k-point (2 atoms, K = 2 x 81 x 2): the emulated integer path
    (B = h_a A included) within 1e-12 of the FP64 products in Frobenius norm,
    and the lowest 20 generalized eigenvalues of the whole H, O within
    1e-8 Ha of the FP64 ones (the metric's absolute bar)."""
    import scipy.linalg as sl
    import lapw_oracle as O
    from exciting_b200 import workloads as W
    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[3])
    apwalm, _ = O.match(s, gk)
    Hm, Om, Href, Oref, B, Bx = _emulated_setup(s, gk, apwalm)
    assert np.linalg.norm(B - Bx) / np.linalg.norm(Bx) <= 1e-12
    assert np.linalg.norm(Hm - Href) / np.linalg.norm(Href) <= 1e-12
    assert np.linalg.norm(Om - Oref) / np.linalg.norm(Oref) <= 1e-12
    H, Ov = O.hamiltonandoverlapsetup(s, gk, apwalm)
    N = gk.ngp
    H2, O2 = H.copy(), Ov.copy()
    H2[:N, :N] += Hm - Href
    O2[:N, :N] += Om - Oref
    w0 = sl.eigh(H, Ov, eigvals_only=True, subset_by_index=[0, 19])
    w = sl.eigh(H2, O2, eigvals_only=True, subset_by_index=[0, 19])
    assert np.abs(w - w0).max() <= 1e-8


def test_split_residue_formula():
    """The split kernels' FP32 residue: 13-bit limbs, v = x3 (2^39 mod p) + x2 (2^26 mod p)
    + x1 (2^13 mod p) + x0 with integer partial sums below 2^24 (exact in FP32), q =
    round(v / p) as one FMA v * fl(1/p) + 1.5 2^23 rounded once to FP32, r = v - q p:
    r = x (mod p) and |r| <= 127 for |x| <= 2^52 and every modulus of the table."""
    ps = plan(16, 1000, 100)[0]
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.integers(-2 ** 52, 2 ** 52, size=20000, dtype=np.int64),
                         np.array([0, 1, -1, 2 ** 52, -2 ** 52, 2 ** 39 - 1, -2 ** 39, 2 ** 48 + 12345],
                                  dtype=np.int64)])
    limbs = [(xs & 0x1fff), (xs >> 13) & 0x1fff, (xs >> 26) & 0x1fff, xs >> 39]
    magic = np.float64(1.5 * 2 ** 23)
    for p in ps:
        assert p <= 253
        c = [(1 << 13) % p, (1 << 26) % p, (1 << 39) % p]
        v = limbs[0] + limbs[1] * c[0] + limbs[2] * c[1] + limbs[3] * c[2]
        assert np.abs(v).max() < 2 ** 23
        inv = np.float64(np.float32(1.0 / p))
        q = (v * inv + magic).astype(np.float32).astype(np.float64) - magic   # exact product, one rounding
        r = (v - q * p).astype(np.int64)
        assert np.abs(r).max() <= 127
        assert np.all(np.mod(r - xs, p) == 0)


def test_emulated_eight_atom_eigenvalues():
    """The 8-atom cell (K = 1936, O conditioned ~2.5e4, eigenvalues down to
    about -1600 Ha), k-point 0: H/O products through the emulated residue
    tiles of the default plan (13 moduli, 49 bits, 96-bit recombination), the
    lowest 40 generalized eigenvalues within the absolute 1e-8 Ha of FP64.
    A 64-bit recombination with column-maximum scaling and no headroom is
    4.3e-8 Ha off on the same k-point: the recombination, not the operand
    bits, limited the eigenvalues."""
    import scipy.linalg as sl
    import lapw_oracle as O
    from exciting_b200 import workloads as W
    s = W.si_cube8()
    gk = s.gkset(s.kpoints[0])
    apwalm, _ = O.match(s, gk)
    H, Ov = O.hamiltonandoverlapsetup(s, gk, apwalm)
    N = gk.ngp
    apwi = [O._apwi(s, apwalm, N, a) for a in range(s.natmtot)]
    A = np.concatenate(apwi)
    B = np.concatenate([s.mt_aa[:, :, a] @ apwi[a] for a in range(s.natmtot)])
    ps, cs, b, _, h = plan(0, A.shape[0], s.basis.maxaa)
    assert (len(ps), b) == (13, 49)
    M = float(math.prod(ps))
    ar, ai, sa = _split_scaled(A, b)
    br, bi, sb = _split_scaled(B, b)
    XA = np.concatenate([ar, ai])
    assert crt_shift(ps, b) == 0
    scale = M * 2.0 ** (-64 - 2 * b)
    got = []
    for Ys, sy in (([np.concatenate([br, bi]), np.concatenate([bi, -br])], sb),
                   ([np.concatenate([ar, ai]), np.concatenate([ai, -ar])], sa)):
        parts = [emulate_crt(XA, Y, ps).astype(np.float64) * scale for Y in Ys]
        got.append((parts[0] + 1j * parts[1]) * np.outer(sa, sy))
    Href, Oref = A.conj().T @ B, A.conj().T @ A
    assert np.linalg.norm(got[0] - Href) / np.linalg.norm(Href) <= 1e-12
    assert np.linalg.norm(got[1] - Oref) / np.linalg.norm(Oref) <= 1e-12
    H2, O2 = H.copy(), Ov.copy()
    H2[:N, :N] += got[0] - Href
    O2[:N, :N] += got[1] - Oref
    w0 = sl.eigh(H, Ov, eigvals_only=True, subset_by_index=[0, 39])
    w = sl.eigh(H2, O2, eigvals_only=True, subset_by_index=[0, 39])
    assert np.abs(w - w0).max() <= 1e-8
