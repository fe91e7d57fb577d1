"""The modular split-precision scheme (EXS_PREC_OZAKI_MOD), checked on the CPU.

The library's plan (exs_ozaki_moduli: moduli, Chinese-remainder constants,
bits per operand) is checked against exact integer arithmetic, and the
device arithmetic is emulated in numpy with that plan: residues in
[-127, 127], one exact integer product per modulus, the multiply-high
quotient of the fold, the 64-bit wrapping sum t += r c_m and the final
t / 2^64 * M.  The emulated products must reconstruct the exact integer
product within the stated bound (sum |r| / 2 + 1 units of 2^-64 M), and an
emulated H = A^H B on a Si k-point must meet the 1e-12 bar.  No GPU is
touched.
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
    b, bx = ctypes.c_int(), ctypes.c_int()
    rc = lib.exs_ozaki_moduli(n, K, kx, ctypes.byref(n_out), p.ctypes.data_as(ctypes.c_void_p),
                              c.ctypes.data_as(ctypes.c_void_p), ctypes.byref(b), ctypes.byref(bx))
    if rc != 0:
        return None
    m = n_out.value
    return [int(x) for x in p[:m]], [int(x) for x in c[:m]], b.value, bx.value


@pytest.mark.parametrize("n,K,kx", [(14, 1936, 242), (12, 1936, 242), (0, 1936, 242), (0, 34992, 162),
                                    (16, 65536, 512), (6, 200, 50)])
def test_plan_constants_and_bounds(n, K, kx):
    ps, cs, b, bx = plan(n, K, kx)
    if n:
        assert len(ps) == n
    for i in range(len(ps)):
        assert ps[i] % 2 == 1 and ps[i] < 256
        for j in range(i):
            assert math.gcd(ps[i], ps[j]) == 1
    M = math.prod(ps)
    for p, c in zip(ps, cs):
        y = pow(M // p, -1, p)
        assert c == ((y << 64) + p // 2) // p          # round(2^64 y / p)
    # |X| <= 2K 2^(2b) < M / 2 for the H/O products, 2 kx 2^(b + bx) for the per-atom ones
    assert 2 * K * 2 ** (2 * b) < M // 2 and 2 * kx * 2 ** (b + bx) < M // 2
    assert b <= 52 and bx <= 52
    # b is the largest that fits (unless capped at 52)
    assert b == 52 or 2 * K * 2 ** (2 * (b + 1)) >= M // 2
    if n == 0:
        assert b >= 44
        if len(ps) > 6:    # one modulus fewer would not keep 44 bits
            Mf = math.prod(ps[:-1])
            assert 2 * K * 2 ** 88 >= Mf // 2


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
    """Integer product X^T Y (entries of X, Y integers as float64) by the modular fold."""
    t = np.zeros((X.shape[1], Y.shape[1]), dtype=np.uint64)
    rsum = np.zeros(t.shape)
    for p, c in zip(ps, cs):
        v = (_residues(X, p).T @ _residues(Y, p)).astype(np.int64)     # exact: |v| < 2^31
        assert np.abs(v).max() < 2 ** 31
        r = _fold_reduce(v, p)
        assert r.min() >= -p / 4 and r.max() <= 5 * p / 4
        rsum += np.abs(r)
        with np.errstate(over="ignore"):
            t += r.astype(np.int64).view(np.uint64) * np.uint64(c)
    return t.view(np.int64), rsum


@pytest.mark.parametrize("n", [8, 12, 14])
def test_emulated_fold_reconstructs_integer_products(n):
    rng = np.random.default_rng(n)
    K = 300
    ps, cs, b, _ = plan(n, K // 2, 8)
    lim = 2 ** b
    X = rng.integers(-lim, lim + 1, size=(K, 5), dtype=np.int64)
    Y = rng.integers(-lim, lim + 1, size=(K, 4), dtype=np.int64)
    X[:, 0] = lim                      # the bound's extreme: one column pair at +-2^b everywhere
    Y[:, 0] = -lim
    t, rsum = emulate(X.astype(np.float64), Y.astype(np.float64), ps, cs)
    M = math.prod(ps)
    for i in range(X.shape[1]):
        for j in range(Y.shape[1]):
            exact = sum(int(a) * int(bb) for a, bb in zip(X[:, i], Y[:, j]))
            assert abs(exact) < M // 2
            # t = 2^64 X / M + e, |e| <= sum |r| / 2 (rounded constants) + 1 (the exact quotient's fraction)
            err = int(t[i, j]) * M - exact * 2 ** 64
            assert abs(err) <= (rsum[i, j] / 2 + 1) * M, (i, j)


def _split_scaled(Z, b):
    """Columns scaled by a power of two above their maximum, then to b-bit integers."""
    m = np.maximum(np.abs(Z.real).max(0), np.abs(Z.imag).max(0))
    sig = np.ldexp(1.0, np.frexp(np.where(m > 0, m, 1.0))[1])
    return np.rint(Z.real / sig * 2.0 ** b), np.rint(Z.imag / sig * 2.0 ** b), sig


def test_emulated_contraction_meets_the_bar():
    """H = A^H B and O = A^H A for one Si k-point (2 atoms, K = 2 x 81 x 2)."""
    import lapw_oracle as O
    from exciting_b200 import workloads as W
    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[3])
    apwalm, _ = O.match(s, gk)
    N = gk.ngp
    A = np.concatenate([O._apwi(s, apwalm, N, a) for a in range(s.natmtot)])
    B = np.concatenate([s.mt_aa[:, :, a] @ O._apwi(s, apwalm, N, a) for a in range(s.natmtot)])
    K = A.shape[0]
    ps, cs, b, _ = plan(0, K, 8)
    M = float(math.prod(ps))
    ar, ai, sa = _split_scaled(A, b)
    br, bi, sb = _split_scaled(B, b)
    XA = np.concatenate([ar, ai])                   # [Ar; Ai]
    YH = [np.concatenate([br, bi]), np.concatenate([bi, -br])]    # Re H, Im H
    YO = [np.concatenate([ar, ai]), np.concatenate([ai, -ar])]    # Re O, Im O
    scale = M * 2.0 ** (-64 - 2 * b)
    for Ys, ref, sy in ((YH, A.conj().T @ B, sb), (YO, A.conj().T @ A, sa)):
        parts = [emulate(XA, Y, ps, cs)[0].astype(np.float64) * scale for Y in Ys]
        got = (parts[0] + 1j * parts[1]) * np.outer(sa, sy)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12


def test_split_residue_formula():
    """The split kernels' FP32 residue: 13-bit limbs, v = x3 (2^39 mod p) + x2 (2^26 mod p)
    + x1 (2^13 mod p) + x0 with integer partial sums below 2^24 (exact in FP32), q =
    round(v / p) as one FMA v * fl(1/p) + 1.5 2^23 rounded once to FP32, r = v - q p:
    r = x (mod p) and |r| <= 127 for |x| <= 2^52 and every modulus of the table."""
    ps, _, _, _ = plan(16, 1000, 100)
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


def test_emulated_per_atom_product_meets_the_bar():
    """B_a = h_a A_a as the per-atom kernel forms it: rows of h_a scaled to bx
    bits (a power of two above each row's maximum), A to b bits by its column
    maxima over all atoms, the same moduli; |X| <= 2 maxaa 2^(b + bx) < M / 2."""
    import lapw_oracle as O
    from exciting_b200 import workloads as W
    s = W.si_fcc("text")
    gk = s.gkset(s.kpoints[3])
    apwalm, _ = O.match(s, gk)
    N = gk.ngp
    apwi = [O._apwi(s, apwalm, N, a) for a in range(s.natmtot)]
    A = np.concatenate(apwi)
    K, kx = A.shape[0], s.basis.maxaa
    ps, cs, b, bx = plan(0, K, kx)
    M = float(math.prod(ps))
    _, _, sa = _split_scaled(A, b)
    for a in range(s.natmtot):
        h = s.mt_aa[:, :, a]
        Aa = apwi[a]
        ar, ai = np.rint(Aa.real / sa * 2.0 ** b), np.rint(Aa.imag / sa * 2.0 ** b)
        hm = np.maximum(np.abs(h.real).max(1), np.abs(h.imag).max(1))
        sx = np.ldexp(1.0, np.frexp(np.where(hm > 0, hm, 1.0))[1])
        hr = np.rint(h.real / sx[:, None] * 2.0 ** bx).T           # (f', f)
        hi = np.rint(h.imag / sx[:, None] * 2.0 ** bx).T
        X = np.concatenate([hr, hi])
        re = emulate(X, np.concatenate([ar, -ai]), ps, cs)[0].astype(np.float64)
        im = emulate(X, np.concatenate([ai, ar]), ps, cs)[0].astype(np.float64)
        got = (re + 1j * im) * (M * 2.0 ** (-64 - b - bx)) * np.outer(sx, sa)
        ref = h @ Aa
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-13
