// Split-precision MT contraction on the 5th-gen tensor cores (tcgen05.mma
// kind::i8, int32 accumulators in tensor memory): int8 slices (Ozaki scheme)
// or int8 residues modulo coprime moduli (the modular scheme, the default
// of the benchmark).
//
// H = A^H B and O = A^H A in real arithmetic: with the real and imaginary
// planes of A and B,
//   Re H = Ar^T Br + Ai^T Bi    Im H = Ar^T Bi - Ai^T Br
//   Re O = Ar^T Ar + Ai^T Ai    Im O = Ar^T Ai - Ai^T Ar
// so one B operand tile [Br | Bi | Ar | Ai] (32 columns G_j each, N = 128)
// against the two A operands Ar and Ai (two int32 accumulators r and i)
// yields all four: Re H = r0 + i1, Im H = r1 - i0, Re O = r2 + i3,
// Im O = r3 - i2 (rq = block q of accumulator r).
//
// Every column G of A (and of B) is scaled by a power of two sigma(G) >
// max|column| and cut into S int8 slices of 7 bits each by truncation,
//   x = sigma * sum_s q_s 2^{-7s} + rest,  |q_s| <= 127,  |rest| < sigma 2^{-7S}
// (exact in FP64).  The product keeps the slice pairs s + t <= S + 1.  Pairs
// are accumulated in int32 in segments short enough to be exact (the pairs of
// one diagonal d = s + t in groups of P with P * K * 127^2 < 2^31), and each
// finished segment is added in FP64 as 2^{-7d} times its int32 sums to an
// FP64 accumulator that also lives in tensor memory.  The final epilogue
// multiplies by sigma_A(i) sigma_B(j), adds the interstitial term and writes
// the upper triangle and its conjugate mirror, as the FP64 path does.
//
// Modular arithmetic (OzScheme.mod = 1) replaces the slices by residues:
// every column is scaled by sigma = a power of two above its 2-norm and
// rounded to integers of b bits, x' = rint(x 2^b / sigma) (exact in FP64;
// the scaled column has norm <= 2^b (1 + eps)), and stored as n int8 planes
// x' mod p_m in [-127, 127] for pairwise coprime odd moduli p_m.  One int8
// product per modulus gives r +- i = X (mod p_m) for the integer product X,
// and |X| <= 2^(2b) (1 + eps)^2 by the Cauchy-Schwarz inequality.  With M =
// prod p_m >= 2^(2b + h + 2), 2^h X / M is the signed fraction of
// sum_m (X mod p_m) 2^h y_m / p_m, y_m = (M / p_m)^-1 mod p_m (the Chinese
// remainder theorem).  The kernel keeps that fraction as a 64-bit fixed-point
// sum t += r c_m (mod 2^64), c_m = round(2^(64+h) y_m / p_m) mod 2^64, in the
// tensor-memory columns of the FP64 sums; the rounded constants err by at
// most sum |r| / 2 units of 2^-(64+h) M, so the h headroom bits (at least 5)
// divide the recombination error by 2^h.  That error adds to H and O like
// noise, which the generalized eigenvalues feel far more than the rounding
// of the operands (a perturbation of A itself), hence the headroom.  n
// products replace the n(n+1)/2 slice pairs (13 moduli keep 47 bits per
// operand at K = 1936, 14 keep 51 at K = 34,992; 7 slices cost 28
// products).  The fold runs in two phases: phase 1 reads r and i, reduces
// v = r +- i below 16 bits and releases the accumulators to the next
// modulus's MMAs; phase 2 updates the 64-bit sums meanwhile.
//
// Slice storage (int8, K contiguous, K padded to kp8 = multiple of 256):
//   [slot][slice][array: Br, Bi, Ar, Ai][G (npad rows)][kp8]
// viewed by TMA as 5D (K byte in a 128-byte chunk, G, array, K chunk,
// slot x slice), so that both A operands of a stage (Ar and Ai, 128 G rows
// each) are ONE box and the B operand (32 G rows of all four arrays) is
// another: two boxes per stage.  Rows past npad fall outside the view and
// arrive as zeros.  Boxes are written with 128-byte swizzling; the MMA
// descriptors use the matching SWIZZLE_128B K-major layout (8-row x 128-byte
// atoms, 1024 B between 8-row groups, K advanced 32 bytes per MMA).
//
// Configurations (chosen per problem by the autotuner): KCH K chunks per
// stage x NST stages, 192 KB in all: (2, 2) or (1, 4) for the H/O tiles;
// one CTA per tile or a persistent grid of one CTA per SM, for the H/O tiles
// and the per-atom tiles separately.
//
// Roles (one CTA per 128 x 32 output tile, 384 threads):
//   warps 0-1  one TMA producer thread each (the A box and the B box of a stage)
//   warp 3     MMA issuer (one thread); allocates tensor memory
//   warps 4-11 epilogue: segment folds and the final store, two warps per
//              tensor-memory lane quadrant, each with two of the four value
//              blocks (H/O tiles: half 0 Re H, Im H, half 1 Re O, Im O;
//              per-atom tiles: half h the re and im blocks of rows 32h..32h+31)
// The same kernel (MODE OZ_ATOM) forms the per-atom products B_a = h_a A_a
// and the APW-lo rows loa_a A_a from int8 slices (or residues) of h_a and loa.
// Tensor memory (512 columns): r at [0,128), i at [128,256), the running sums
// (FP64 for slices, 64-bit fixed point for moduli; two 32-bit columns per
// value) at [256,512).  With one tile per CTA the H/O tile's conjugate
// mirror is staged in the stage buffers (idle by then) and written as whole
// columns.  Every wait on an mbarrier is
// bounded (about one second) and gives up early once another role has given
// up; the kernel then records an error, lets its own copies and MMAs drain
// (bounded), frees tensor memory and returns.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "exs_internal.cuh"
#include "interstitial.cuh"

namespace exs {

constexpr int OZ_BM = 128;                       // tile rows (G_i)
constexpr int OZ_BJ = 32;                        // tile columns (G_j); MMA N = 4 * OZ_BJ
constexpr int OZ_N = 4 * OZ_BJ;
constexpr int OZ_NARR = 4;                       // Br, Bi, Ar, Ai (the B box: four arrays)
constexpr int OZ_CHUNK = 128;                    // bytes of K in one swizzle row
constexpr int OZ_TILE = 128 * OZ_CHUNK;          // 16 KB: one K chunk of a 128-row operand
constexpr int OZ_THREADS = 384;                  // 12 warps: see the roles below
constexpr int OZ_MAX_KCH = 2;                    // K chunks per stage of the widest configuration
constexpr int OZ_TMEM_COLS = 512;
constexpr int OZ_FP64_COL = 256;
constexpr long long OZ_WAIT_CYCLES = 2000000000LL;   // ~1 s at 2 GHz

// ------------------------------------------------------------ device helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait (limit cycles; 0: OZ_WAIT_CYCLES) that also gives up as soon
// as another role raised `abort`.
__device__ __forceinline__ bool mbar_wait_ab(uint64_t *bar, uint32_t parity, volatile int *abort, long long limit)
{
    const long long t0 = clock64();
    const long long lim = limit > 0 ? limit : OZ_WAIT_CYCLES;
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (*abort) return false;
        if (clock64() - t0 > lim) {
            *abort = 1;
            return false;
        }
    }
}

// Bounded wait used while draining after an abort.
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity) && clock64() - t0 < OZ_WAIT_CYCLES) {
    }
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];\n" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// K-major SWIZZLE_128B descriptor (8-row x 128-byte atoms, 1024 B between 8-row groups).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                   // leading byte offset (unused by swizzled K-major): 16 B
    d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset
    d |= (uint64_t)1 << 46;                   // descriptor version of sm_100
    d |= (uint64_t)2 << 61;                   // SWIZZLE_128B
    return d;
}

// kind::i8 instruction descriptor: s8 x s8 -> s32, K-major A and B, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tm_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tm_st16(uint32_t taddr, const uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(
            taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]));
}

__device__ __forceinline__ void tm_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// ------------------------------------------------------------ preparation
// Column scale sigma(G) = 2^e with m < 2^e (frexp) for the column bound m in
// oz_scale: with slices the column maximum that the producers of the A and B
// planes raise (the matching kernels for A, the h_a A epilogue for B), with
// moduli the column 2-norm (oz_colnorm_kernel).  An all-zero column gets
// sigma = 1.
__host__ __device__ __forceinline__ double oz_sigma(double m)
{
    int e = 0;
    if (m > 0.0) frexp(m, &e);
    return ldexp(1.0, e);
}

// Arrays of one slice of a slot: Br, Bi, Ar, Ai, or with iora* (O = A^H C,
// C = (I + h1aa) A) Br, Bi, Cr, Ci, Ar, Ai, so that the B box is always the
// first four arrays and the A operand the last two.
__host__ __device__ __forceinline__ int oz_narr(int relativity) { return relativity == EXS_REL_IORA ? 6 : 4; }

// Byte offset of (slice s, array a, row G, K index f) inside one slot.
__device__ __forceinline__ size_t oz_off(int s, int a, int g, int f, int npad, int kp8, int narr)
{
    return (((size_t)s * narr + a) * npad + g) * (size_t)kp8 + f;
}

// Residues of an integer x (|x| <= 2^52) in exact FP32 arithmetic: with
// 13-bit limbs x = x3 2^39 + x2 2^26 + x1 2^13 + x0 (x3 signed, |x3| <=
// 2^13; the others in [0, 2^13)), v = x3 (2^39 mod p) + x2 (2^26 mod p) +
// x1 (2^13 mod p) + x0 = x (mod p) has every partial sum an integer below
// 2^23, so each FMA is exact.  q = round(v / p) by one FMA with 1.5 * 2^23
// (|v / p| < 2^15; the error of 1/p in FP32 moves v/p by under 2^-9), and
// r = v - q p is exact with |r| <= (p + 1) / 2 <= 127 for odd p <= 253.
// The byte of r is the low byte of the FP32 bits of 1.5 * 2^23 + r.
struct OzLimbs {
    float l[4];
};

__device__ __forceinline__ OzLimbs oz_limbs(long long x)
{
    OzLimbs t;
    t.l[0] = (float)(int)(x & 0x1fff);
    t.l[1] = (float)(int)((x >> 13) & 0x1fff);
    t.l[2] = (float)(int)((x >> 26) & 0x1fff);
    t.l[3] = (float)(int)(x >> 39);
    return t;
}

__device__ __forceinline__ uint32_t oz_residue_byte(const OzLimbs &x, const OzScheme &sch, int m)
{
    constexpr float MAGIC = 12582912.0f;           // 1.5 * 2^23
    const float v = fmaf(x.l[3], sch.fc[2][m], fmaf(x.l[2], sch.fc[1][m], fmaf(x.l[1], sch.fc[0][m], x.l[0])));
    const float q = fmaf(v, sch.finv[m], MAGIC) - MAGIC;
    const float r = fmaf(-q, sch.fp[m], v);
    return __float_as_uint(r + MAGIC) & 0xffu;
}

__device__ __forceinline__ void oz_put(uint32_t (&o0)[16], uint32_t (&o1)[16], int e, uint32_t w0, uint32_t w1)
{
    if (e < 8) {
        o0[2 * e] = w0;
        o0[2 * e + 1] = w1;
    } else {
        o1[2 * (e - 8)] = w0;
        o1[2 * (e - 8) + 1] = w1;
    }
}

// Fold 16 finished int32 sums of diagonal g (slices) into the FP64 running
// sums (two 32-bit tensor-memory words each, low word first; lo / hi hold
// the previous values unless init): a += 2^{-7(g+2)} (r + sg i), r + sg i
// exact in FP64, one rounding per fold.
__device__ __forceinline__ void oz_fold16(int g, bool init, int sg, const uint32_t (&rv)[16], const uint32_t (&iv)[16],
                                          const uint32_t (&lo)[16], const uint32_t (&hi)[16], uint32_t (&o0)[16],
                                          uint32_t (&o1)[16])
{
    const double scale = ldexp(1.0, -7 * (g + 2));
    const double sgd = (double)sg;
#pragma unroll
    for (int e = 0; e < 16; e++) {
        double a = 0.0;
        if (!init) {
            const uint32_t w0 = e < 8 ? lo[2 * e] : hi[2 * (e - 8)];
            const uint32_t w1 = e < 8 ? lo[2 * e + 1] : hi[2 * (e - 8) + 1];
            a = __hiloint2double((int)w1, (int)w0);
        }
        a += scale * ((double)(int)rv[e] + sgd * (double)(int)iv[e]);
        oz_put(o0, o1, e, (uint32_t)__double2loint(a), (uint32_t)__double2hiint(a));
    }
}

// Modular fold of modulus g in two phases, so that the MMAs of the next
// modulus need wait only for the first.
// Phase 1 reads the int32 sums (r at columns [0, 128), i at [128, 256)) of
// the 128 values of this lane, v = r +- i (exact: |v| <= 2 K 127^2 < 2^31),
// and keeps v - q p_g, q = floor(v mg / 2^32), mg = round(2^32 / p_g):
// |v (mg - 2^32 / p_g)| / 2^32 <= 1/4, so the residue lies in
// [-p_g / 4, 5 p_g / 4], 16 bits, packed two per word (value q at half
// q & 1 of word q >> 1).  Value block o (32 values) = r block o +- i block
// (o ^ 1) for the H/O tiles (Re H, Im H, Re O, Im O), (o ^ 2) for the
// per-atom tiles (Re rows 0-63, Im rows 0-63).
// Value blocks of an epilogue half: H/O tiles {2h, 2h + 1} (Re H, Im H or
// Re O, Im O); per-atom tiles {h, h + 2} (re and im of rows 32h..32h+31).
template <int MODE>
__device__ __forceinline__ int oz_block(int half, int k)
{
    return MODE == OZ_HO ? 2 * half + k : half + 2 * k;
}

template <int MODE>
__device__ __forceinline__ void oz_mod_read(uint32_t t_lane, const OzScheme &sch, int g, int half, uint32_t (&rp)[32])
{
    const int pm = sch.p[g], mg = sch.mg[g];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int o = oz_block<MODE>(half, k);
        const int oi = (MODE == OZ_HO) ? (o ^ 1) : (o ^ 2);
        const bool minus = (MODE == OZ_HO) ? (o & 1) != 0 : o < 2;
        uint32_t r0[16], r1[16], i0[16], i1[16];
        tm_ld16(t_lane + o * 32, r0);
        tm_ld16(t_lane + o * 32 + 16, r1);
        tm_ld16(t_lane + 128 + oi * 32, i0);
        tm_ld16(t_lane + 128 + oi * 32 + 16, i1);
        tm_wait_ld();
#pragma unroll
        for (int e = 0; e < 32; e += 2) {
            int res[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int q = e + h;
                const int rv = (int)(q < 16 ? r0[q] : r1[q - 16]), iv = (int)(q < 16 ? i0[q] : i1[q - 16]);
                const int v = minus ? rv - iv : rv + iv;
                res[h] = v - __mulhi(v, mg) * pm;
            }
            rp[k * 16 + e / 2] = ((uint32_t)res[0] & 0xffffu) | ((uint32_t)res[1] << 16);
        }
    }
}

// Phase 2: the 64-bit running sums t += r c_g (mod 2^64) in the FP64
// columns of this half's blocks, two 32-bit words per value (low first);
// t = r c_g for g = 0.
template <int MODE>
__device__ __forceinline__ void oz_mod_accumulate(uint32_t t_lane, const OzScheme &sch, int g, int half,
                                                  const uint32_t (&rp)[32])
{
    const unsigned long long cm = sch.c[g];
    const bool init = g == 0;
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int jc = 0; jc < 32; jc += 16) {
            const uint32_t fcol = OZ_FP64_COL + 2 * (oz_block<MODE>(half, k) * 32 + jc);
            uint32_t lo[16], hi[16];            // updated in place
            if (!init) {
                tm_ld16(t_lane + fcol, lo);
                tm_ld16(t_lane + fcol + 16, hi);
                tm_wait_ld();
            }
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const int q = k * 32 + jc + e;
                const int r = (int)(int16_t)(uint16_t)(rp[q >> 1] >> (16 * (q & 1)));
                uint32_t &w0 = e < 8 ? lo[2 * e] : hi[2 * (e - 8)];
                uint32_t &w1 = e < 8 ? lo[2 * e + 1] : hi[2 * (e - 8) + 1];
                unsigned long long t = init ? 0ull : (((unsigned long long)w1 << 32) | w0);
                t += (unsigned long long)(long long)r * cm;
                w0 = (uint32_t)t;
                w1 = (uint32_t)(t >> 32);
            }
            tm_st16(t_lane + fcol, lo);
            tm_st16(t_lane + fcol + 16, hi);
        }
    tm_wait_st();
}

// A finished running sum as a value: the FP64 sum of the slices, or the
// signed 64-bit fraction t / 2^64 = X / M times fin = M 2^-64 2^-(bits).
__device__ __forceinline__ double oz_final(const OzScheme &sch, double fin, uint32_t w0, uint32_t w1)
{
    if (!sch.mod) return __hiloint2double((int)w1, (int)w0);
    return (double)(long long)(((unsigned long long)w1 << 32) | w0) * fin;
}


// Final store of one row of a 128 x 32 H/O tile by epilogue half `half`:
// half 0 writes H (Re H, Im H scaled by sigma_A(i) sigma_B(j), plus the
// hmlistln term), half 1 writes O (sigma_A(i) sigma_A(j), plus olpistln);
// the upper triangle and its conjugate mirror, like the FP64 path.  With
// T (shared memory, OZ_MIRROR_LD x 64 values) the mirror values go to
// T[(half * 32 + j - j0) * OZ_MIRROR_LD + row] instead, for oz_store_mirror.
constexpr int OZ_MIRROR_LD = 129;                 // 16-byte values; odd stride: no bank conflicts

__device__ __forceinline__ void oz_store_ho(const DevParams &p, const KDesc &kd, const OzScheme &sch, int i0, int j0,
                                            uint32_t t_lane, int row, int half, exs_complex *T)
{
    const int i = i0 + row;
    int ivi[3] = {0, 0, 0};
    double vi[3] = {0.0, 0.0, 0.0};
    const bool row_ok = i < kd.ngp;
    if (row_ok) {
        int g = kd.igpig[i] - 1;
        if (g < 0 || g >= p.ngrtot) {
            atomicOr(p.err, DEV_ERR_INDEX);
            g = 0;
        }
        for (int x = 0; x < 3; x++) {
            ivi[x] = p.ivg[3 * g + x];
            vi[x] = kd.vgpc[3 * i + x];
        }
    }
    const double sai = row_ok ? oz_sigma(kd.oz_scale[i]) : 0.0;
    const int kind = half == 0 ? EPI_HAM : EPI_OVL;
    exs_complex *out = half == 0 ? kd.h : kd.o;
    // H: sigma_B(j); O: sigma_A(j), or sigma_C(j) with iora* (O = A^H C)
    const double *scol = kd.oz_scale + (half == 0 ? p.npad : (p.relativity == EXS_REL_IORA ? 2 * p.npad : 0));
#pragma unroll 1
    for (int jc = 0; jc < OZ_BJ; jc += 8) {
        double val[2][8];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            uint32_t w[16];
            tm_ld16(t_lane + OZ_FP64_COL + 2 * ((2 * half + k) * 32 + jc), w);
            tm_wait_ld();
#pragma unroll
            for (int e = 0; e < 8; e++) val[k][e] = oz_final(sch, sch.fin, w[2 * e], w[2 * e + 1]);
        }
        if (!row_ok) continue;
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int j = j0 + jc + e;
            if (j >= kd.ngp || i > j) continue;
            // column data (the same for the whole warp: broadcast loads)
            int gj = kd.igpig[j] - 1;
            if (gj < 0 || gj >= p.ngrtot) {
                atomicOr(p.err, DEV_ERR_INDEX);
                gj = 0;
            }
            const int ivj[3] = {p.ivg[3 * gj], p.ivg[3 * gj + 1], p.ivg[3 * gj + 2]};
            const double vj[3] = {kd.vgpc[3 * j], kd.vgpc[3 * j + 1], kd.vgpc[3 * j + 2]};
            const double sj = oz_sigma(scol[j]);
            double re = val[0][e] * sai * sj, im = val[1][e] * sai * sj;
            double ar, ai;
            if (interstitial(p, kind, ivi, ivj, vi, vj, ar, ai)) {
                re += ar;
                im += ai;
            }
            exs_complex v;
            v.re = re;
            v.im = im;
            out[(size_t)i + (size_t)kd.nmat * j] = v;
            if (i < j) {
                v.im = -im;
                if (T)
                    T[(half * 32 + jc + e) * OZ_MIRROR_LD + row] = v;
                else
                    out[(size_t)j + (size_t)kd.nmat * i] = v;
            }
        }
    }
}

// The staged mirror of a 128 x 32 H/O tile, written as whole columns: the
// 256 (matrix, row i) pairs are split over the eight epilogue warps (ew =
// 0..7); lane l writes element (j0 + l, i), so each warp store covers 32
// consecutive rows of one column (512 contiguous bytes).
__device__ __forceinline__ void oz_store_mirror(const KDesc &kd, int i0, int j0, const exs_complex *T, int ew, int lane)
{
    const int j = j0 + lane;
#pragma unroll 4
    for (int q = 0; q < 32; q++) {
        const int pr = ew * 32 + q, h = pr >> 7, il = pr & 127;
        const int i = i0 + il;
        if (i < kd.ngp && j < kd.ngp && i < j)
            (h ? kd.o : kd.h)[(size_t)j + (size_t)kd.nmat * i] = T[(h * 32 + lane) * OZ_MIRROR_LD + il];
    }
}

// Planes and scale block of operand `which` (0: A, 1: B, 2: C = (I + h1aa) A).
__device__ __forceinline__ void oz_operand(const KDesc &k, int which, const double *&pr, const double *&pi)
{
    pr = which == 0 ? k.ar : (which == 1 ? k.br : k.cr);
    pi = which == 0 ? k.ai : (which == 1 ? k.bi : k.ci);
}

// Column bounds of the A, B or C planes (which = 0, 1, 2) written into
// oz_scale block `which`: 2-norms (norm != 0; the modular scheme, over the
// maxima the producers raised) or maxima of |re|, |im| (the slices, for C
// whose producer raises none).  One column per thread column of a 32 x 8
// block, the eight rows of threads covering interleaved rows f (stride 8),
// the eight partial results combined in a fixed order, so that the scales,
// and every result, are the same from run to run.  The factor 1 + 2^-30
// covers the rounding of a sum of squares.
__global__ void __launch_bounds__(256) oz_colnorm_kernel(DevParams p, const KDesc *ks, int which, int norm)
{
    __shared__ double part[8][33];
    const KDesc k = ks[blockIdx.y];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int g = blockIdx.x * 32 + tx;
    const double *pr, *pi;
    oz_operand(k, which, pr, pi);
    double s = 0.0;
    if (g < k.ngp) {
#pragma unroll 4
        for (int f = ty; f < p.K; f += 8) {
            const size_t i = (size_t)f * p.npad + g;
            const double xr = pr[i], xi = pi[i];
            s = norm ? fma(xr, xr, fma(xi, xi, s)) : fmax(s, fmax(fabs(xr), fabs(xi)));
        }
    }
    part[ty][tx] = s;
    __syncthreads();
    if (ty == 0 && g < p.npad) {
        double t = 0.0;
        for (int q = 0; q < 8; q++) t = norm ? t + part[q][tx] : fmax(t, part[q][tx]);
        k.oz_scale[(size_t)which * p.npad + g] = norm ? sqrt(t) * (1.0 + 0x1p-30) : t;
    }
}

// The S slices of one operand (which = 0: A into the last two arrays of the
// slot; 1: B into arrays 0, 1; 2: C into arrays 2, 3 (iora*)).
// A 64(f) x 32(G) tile per block, transposed through shared memory: reads
// G-contiguous planes (a warp reads 32 consecutive G; 16 loads per thread in
// flight), writes K-contiguous int8 rows eight bytes per thread (8 threads
// cover the tile's 64 K bytes of one G row).
constexpr int SPLIT_F = 64;

__global__ void __launch_bounds__(256) oz_split_kernel(DevParams p, const KDesc *ks,
                                                       const __grid_constant__ OzScheme sch, int kp8, int which)
{
    const int S = sch.n;
    __shared__ double t[2][SPLIT_F][33];
    const KDesc k = ks[blockIdx.z];
    const int f0 = blockIdx.x * SPLIT_F, g0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;      // 32 x 8
    const int narr = oz_narr(p.relativity);
    const int a0 = which == 0 ? narr - 2 : (which == 1 ? 0 : 2);
    const double *pr, *pi;
    oz_operand(k, which, pr, pi);
    {
        double vr[SPLIT_F / 8], vi[SPLIT_F / 8];
#pragma unroll
        for (int q = 0; q < SPLIT_F / 8; q++) {
            const int f = f0 + ty + 8 * q, g = g0 + tx;
            const bool v = f < p.K && g < k.ngp;
            const size_t i = (size_t)f * p.npad + g;
            vr[q] = v ? pr[i] : 0.0;
            vi[q] = v ? pi[i] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < SPLIT_F / 8; q++) {
            t[0][ty + 8 * q][tx] = vr[q];
            t[1][ty + 8 * q][tx] = vi[q];
        }
    }
    __syncthreads();
    const int tid = ty * 32 + tx;
    const int gl = tid >> 3, fl = (tid & 7) * 8;
    const int g = g0 + gl, f = f0 + fl;
    if (g >= p.npad || f >= kp8) return;
    // 1/sigma is a power of two: the scaling is exact
    const double rs = 1.0 / oz_sigma(k.oz_scale[(size_t)which * p.npad + g]);
    if (sch.mod) {
        // x' = rint(x 2^b / sigma) (power-of-two scaling: exact), then its residues
        const double sc = rs * ldexp(1.0, sch.b);
        OzLimbs xq[2][8];
#pragma unroll
        for (int e = 0; e < 8; e++)
#pragma unroll
            for (int a = 0; a < 2; a++) xq[a][e] = oz_limbs(__double2ll_rn(t[a][fl + e][gl] * sc));
        for (int m = 0; m < S; m++) {
#pragma unroll
            for (int a = 0; a < 2; a++) {
                uint32_t w[2] = {0, 0};
#pragma unroll
                for (int e = 0; e < 8; e++) w[e >> 2] |= oz_residue_byte(xq[a][e], sch, m) << (8 * (e & 3));
                *reinterpret_cast<uint2 *>(k.oz_slices + oz_off(m, a0 + a, g, f, p.npad, kp8, narr)) = make_uint2(w[0], w[1]);
            }
        }
        return;
    }
    // The slices are the base-128 digits of |x| 2^(7S) truncated, with the
    // sign of x: the same digits as S steps of (x *= 128, q = trunc(x),
    // x -= q) in exact FP64, taken from one integer (7S <= 63 bits).
    const double two7s = ldexp(1.0, 7 * S);
    unsigned long long mag[2][8];
    uint32_t neg[2] = {0, 0};
#pragma unroll
    for (int e = 0; e < 8; e++)
#pragma unroll
        for (int a = 0; a < 2; a++) {
            const long long X = (long long)(t[a][fl + e][gl] * rs * two7s);   // |.| < 2^63, truncated
            neg[a] |= (X < 0 ? 1u : 0u) << e;
            mag[a][e] = (unsigned long long)(X < 0 ? -X : X);
        }
    for (int s = 0; s < S; s++) {
        const int sh = 7 * (S - 1 - s);
#pragma unroll
        for (int a = 0; a < 2; a++) {
            uint32_t w[2] = {0, 0};
#pragma unroll
            for (int e = 0; e < 8; e++) {
                int q = (int)((mag[a][e] >> sh) & 127u);
                if ((neg[a] >> e) & 1u) q = -q;
                w[e >> 2] |= ((uint32_t)(uint8_t)(int8_t)q) << (8 * (e & 3));
            }
            *reinterpret_cast<uint2 *>(k.oz_slices + oz_off(s, a0 + a, g, f, p.npad, kp8, narr)) = make_uint2(w[0], w[1]);
        }
    }
}

// ------------------------------------------------------------ per-atom operands
// Slices of the per-atom MT integrals that multiply A from the left in the
// per-atom products B_a = h_a A_a (hamiltonsetup.f90:75-88) and
// H_lo,a = loa_a A_a (hamiltonsetup.f90:131-145):
//   X(n, k) for n = output row (f of h_a in blocks of 64, then the lo rows r
//   of loa in blocks of 64 from block nfb on), k = K byte of the atom's window: the window starts
//   at oz_x0 (apw_off rounded down to 16) so that X(n, k) = 0 unless
//   0 <= k - (apw_off - oz_x0) < napw.
// Layout [atom][slice][block xb][array re, im][64 rows][lw bytes], one scale
// sigma per row (power of two above the row maximum with slices, above the
// row 2-norm with moduli).
__device__ __forceinline__ void x_value(const DevParams &p, const OzAtomArgs &xa, int ias, int xb, int n, int fp,
                                        double &re, double &im)
{
    re = im = 0.0;
    const AtomDesc at = p.atoms[ias];
    if (fp < 0 || fp >= at.napw) return;
    if (xb < xa.nfb) {
        const int f = xb * 64 + n;
        if (f >= at.napw) return;
        const size_t i = (size_t)ias * xa.ldh * xa.ldh + (size_t)fp * xa.ldh + f;   // h(f, f') at [ias][f'][f]
        re = xa.hr[i];
        im = xa.hi[i];
    } else {
        const int r = (xb - xa.nfb) * 64 + n;
        if (r >= at.losize) return;
        const size_t i = (size_t)ias * xa.ldlo * xa.maxaa + (size_t)fp * xa.ldlo + r;   // loa(r, f) at [ias][f][r]
        re = xa.lr[i];
        im = xa.li[i];
    }
}

// sigma of every X row: one thread per (atom, block, row); the row maximum
// (slices) or the row 2-norm (moduli, norm != 0).
__global__ void oz_xsig_kernel(DevParams p, OzAtomArgs xa, int norm)
{
    const int n = threadIdx.x, xb = blockIdx.x, ias = blockIdx.y;
    double m = 0.0, s = 0.0;
    for (int fp = 0; fp < p.atoms[ias].napw; fp++) {
        double re, im;
        x_value(p, xa, ias, xb, n, fp, re, im);
        m = fmax(m, fmax(fabs(re), fabs(im)));
        s = fma(re, re, fma(im, im, s));
    }
    xa.xsig[((size_t)ias * xa.nxb + xb) * 64 + n] = oz_sigma(norm ? sqrt(s) * (1.0 + 0x1p-30) : m);
}

// The slices of X: one thread per (atom, block, row, 4 window bytes).
__global__ void oz_xsplit_kernel(DevParams p, OzAtomArgs xa, const __grid_constant__ OzScheme sch)
{
    const int S = sch.n;
    const int ias = blockIdx.z, xb = blockIdx.y;
    const int n = threadIdx.y + blockIdx.x * blockDim.y;        // row 0..63
    const int k4 = threadIdx.x * 4;                             // window byte
    if (n >= 64 || k4 >= xa.lw) return;
    const AtomDesc at = p.atoms[ias];
    const int delta = at.apw_off - at.oz_x0;
    const double r = 1.0 / xa.xsig[((size_t)ias * xa.nxb + xb) * 64 + n];
    double x[2][4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        double re, im;
        x_value(p, xa, ias, xb, n, k4 + e - delta, re, im);
        x[0][e] = re * r;
        x[1][e] = im * r;
    }
    if (sch.mod) {
        const double sc = ldexp(1.0, sch.bx);
        OzLimbs xq[2][4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            xq[0][e] = oz_limbs(__double2ll_rn(x[0][e] * sc));
            xq[1][e] = oz_limbs(__double2ll_rn(x[1][e] * sc));
        }
        for (int m = 0; m < S; m++)
#pragma unroll
            for (int a = 0; a < 2; a++) {
                uint32_t w = 0;
#pragma unroll
                for (int e = 0; e < 4; e++) w |= oz_residue_byte(xq[a][e], sch, m) << (8 * e);
                const size_t row = ((((size_t)ias * S + m) * xa.nxb + xb) * 2 + a) * 64 + n;
                *reinterpret_cast<uint32_t *>(xa.xs + row * xa.lw + k4) = w;
            }
        return;
    }
    for (int s = 0; s < S; s++)
#pragma unroll
        for (int a = 0; a < 2; a++) {
            uint32_t w = 0;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                x[a][e] *= 128.0;
                const double tq = trunc(x[a][e]);
                x[a][e] -= tq;
                w |= ((uint32_t)(uint8_t)(int8_t)tq) << (8 * e);
            }
            const size_t row = ((((size_t)ias * S + s) * xa.nxb + xb) * 2 + a) * 64 + n;
            *reinterpret_cast<uint32_t *>(xa.xs + row * xa.lw + k4) = w;
        }
}

// ------------------------------------------------------------ main kernel

// MODE OZ_HO: tiles {k, ib, jb}: H and O, 128 G_i x 32 G_j, B operand
//   [Br | Bi | Ar | Ai] of one G block, contraction over all K.
// MODE OZ_ATOM: tiles {k, atom, ib, xb}: 128 G x 64 output rows n of one
//   atom, B operand [X re | X im] (64 rows each), contraction over the
//   atom's K window; writes B planes (xb < nfb) or the APW-lo rows of H.
struct OzTileInfo {
    int k, i0, j0, ias, xb, nst;
};

template <int MODE, int KCH>
__device__ __forceinline__ OzTileInfo oz_tile(const DevParams &p, const int *tiles, int t, int kp8)
{
    OzTileInfo ti{};
    if (MODE == OZ_HO) {
        ti.k = tiles[3 * t];
        ti.i0 = tiles[3 * t + 1] * OZ_BM;
        ti.j0 = tiles[3 * t + 2] * OZ_BJ;
        ti.nst = kp8 / (KCH * OZ_CHUNK);
    } else {
        ti.k = tiles[4 * t];
        ti.ias = tiles[4 * t + 1];
        ti.i0 = tiles[4 * t + 2] * OZ_BM;
        ti.xb = tiles[4 * t + 3];
        ti.nst = p.atoms[ti.ias].oz_nch / KCH;
    }
    return ti;
}

// Persistent: each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// and every role walks the same sequence (tile, diagonal d = 2..S+1, left
// slice s = 1..d-1 with t = d - s on the right, K stages), so the mbarrier
// phases simply continue from tile to tile.  The MMAs of a tile's first
// segment overlap the final epilogue of the previous tile (the int32
// accumulators are free once the last fold has read them).
template <int MODE, int KCH, int NST>
__global__ void __launch_bounds__(OZ_THREADS, 1)
oz_mma_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, DevParams p,
              const KDesc *ks, const int *tiles, int ntiles, const __grid_constant__ OzScheme sch, int kp8,
              OzAtomArgs xa)
{
    const int S = sch.n;
    const bool mod = sch.mod != 0;
    const int seg_pairs = mod ? 1 : (MODE == OZ_HO ? sch.seg : sch.segx);
    constexpr int BOX = KCH * OZ_TILE;          // one operand of a stage
    constexpr int STAGE = 3 * BOX;              // A box [chunk][Ar, Ai][128 rows], B box [chunk][128 rows]
    extern __shared__ __align__(1024) uint8_t oz_smem[];
    __shared__ uint64_t full[NST], empty[NST], accf, acce, stg;
    __shared__ uint32_t tmem_sh;
    __shared__ int abort_sh;
    volatile int *abort = &abort_sh;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = (smem_u32(oz_smem) + 1023u) & ~1023u;
    // one tile per CTA: at the final store the stage buffers are idle and
    // hold the H/O mirror (2 x 32 x OZ_MIRROR_LD values, below the stages' size)
    static_assert(2 * 32 * OZ_MIRROR_LD * 16 <= NST * 3 * KCH * OZ_TILE, "mirror staging fits the stages");
    const bool staged = MODE == OZ_HO && (int)gridDim.x >= ntiles;
    exs_complex *mirror = reinterpret_cast<exs_complex *>(oz_smem + (sbase - smem_u32(oz_smem)));

    if (warp == 3) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_sh)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 2);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accf, 1);
        mbar_init(&acce, 8);                  // the eight epilogue warps
        mbar_init(&stg, 8);                   // the mirror is staged (one tile per CTA only)
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tmem_sh;

    if (warp < 3) {
        // ------------------------------------------------ TMA producers: warp 0 the A box, warp 1 the B box
        if (lane == 0 && warp < 2) {
            const int role = warp;
            uint32_t fills[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) fills[q] = 0;
            int st = 0;
            bool bad = false;
            for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
                const OzTileInfo ti = oz_tile<MODE, KCH>(p, tiles, tile, kp8);
                const int slot = ks[ti.k].oz_slot;
                const int x0 = (MODE == OZ_ATOM) ? p.atoms[ti.ias].oz_x0 : 0;
                // group g: slices, the pairs (s, t) of diagonal s + t = g + 2; moduli, plane g with itself
                for (int g = 0; g < S && !bad; g++)
                    for (int j = 0; j < (mod ? 1 : g + 1) && !bad; j++) {
                        const int s = mod ? g + 1 : j + 1, t = mod ? g + 1 : g + 1 - j;
                        for (int kb = 0; kb < ti.nst; kb++) {
                            if (fills[st] > 0 && !mbar_wait_ab(&empty[st], (fills[st] - 1) & 1, abort, sch.wait)) {
                                bad = true;
                                break;
                            }
                            mbar_expect_tx(&full[st], role == 0 ? 2 * BOX : BOX);
                            const uint32_t dst = sbase + st * STAGE + role * 2 * BOX;
                            if (role == 0) {   // Ar and Ai (the slot's last two arrays) of G rows i0 .. i0+127, slice s
                                if (MODE == OZ_HO)
                                    tma_load_5d(dst, &mapA, 0, ti.i0, oz_narr(p.relativity) - 2, kb * KCH, slot * S + s - 1, &full[st]);
                                else
                                    tma_load_4d(dst, &mapA, x0 + kb * OZ_CHUNK, ti.i0, oz_narr(p.relativity) - 2, slot * S + s - 1,
                                                &full[st]);
                            } else if (MODE == OZ_HO) {   // the four arrays of G rows j0 .. j0+31, slice t
                                tma_load_5d(dst, &mapB, 0, ti.j0, 0, kb * KCH, slot * S + t - 1, &full[st]);
                            } else {                      // X rows of block xb, slice t
                                const int grp = (ti.ias * S + (t - 1)) * xa.nxb + ti.xb;
                                tma_load_4d(dst, &mapB, 0, 0, grp, kb * KCH, &full[st]);
                            }
                            fills[st]++;
                            st = (st + 1 == NST) ? 0 : st + 1;
                        }
                    }
            }
            if (bad)   // copies already issued must land before the CTA goes away
                for (int q = 0; q < NST; q++)
                    if (fills[q] > 0) mbar_drain(&full[q], (fills[q] - 1) & 1);
        }
    } else if (warp == 3) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_i8(128, OZ_N);
            uint32_t uses[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) uses[q] = 0;
            int nseg = 0, st = 0;
            bool bad = false;
            for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
                const int nst = oz_tile<MODE, KCH>(p, tiles, tile, kp8).nst;
                for (int g = 0; g < S && !bad; g++)
                    for (int s0 = 1; s0 <= (mod ? 1 : g + 1) && !bad; s0 += seg_pairs) {
                        const int s1 = min(mod ? 1 : g + 1, s0 + seg_pairs - 1);
                        // the epilogue must have folded the previous segment
                        if (nseg > 0 && !mbar_wait_ab(&acce, (nseg - 1) & 1, abort, sch.wait)) {
                            bad = true;
                            break;
                        }
                        tc_fence_after();
                        bool first = true;
                        for (int s = s0; s <= s1 && !bad; s++)
                            for (int kb = 0; kb < nst; kb++) {
                                if (!mbar_wait_ab(&full[st], uses[st] & 1, abort, sch.wait)) {
                                    bad = true;
                                    break;
                                }
                                tc_fence_after();
                                const uint32_t sa = sbase + st * STAGE;
#pragma unroll
                                for (int c = 0; c < KCH; c++)
#pragma unroll
                                    for (int q = 0; q < OZ_CHUNK / 32; q++) {
                                        const uint32_t ao = c * 2 * OZ_TILE + q * 32;   // Ar; Ai one tile on
                                        const uint64_t bd = umma_desc_sw128(sa + 2 * BOX + c * OZ_TILE + q * 32);
                                        const uint32_t acc = (first && c == 0 && q == 0) ? 0u : 1u;
                                        umma_i8(tbase, umma_desc_sw128(sa + ao), bd, idesc, acc);
                                        umma_i8(tbase + 128, umma_desc_sw128(sa + ao + OZ_TILE), bd, idesc, acc);
                                    }
                                first = false;
                                umma_commit(&empty[st]);
                                uses[st]++;
                                st = (st + 1 == NST) ? 0 : st + 1;
                            }
                        if (!bad) {
                            umma_commit(&accf);
                            nseg++;
                        }
                    }
            }
            if (bad)   // MMAs already issued must finish before tensor memory is freed
                for (int q = 0; q < NST; q++)
                    if (uses[q] > 0) mbar_drain(&empty[q], (uses[q] - 1) & 1);
        }
    } else {
        // ------------------------------------------------ epilogue (warps 4..11)
        const int qd = warp & 3;                                    // tensor-memory lane quadrant
        const int half = (warp - 4) >> 2;                           // which two value blocks
        const uint32_t t_lane = tbase + ((uint32_t)(qd * 32) << 16);
        int nseg = 0;
        bool bad = false;
        for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
            const OzTileInfo ti = oz_tile<MODE, KCH>(p, tiles, tile, kp8);
            for (int g = 0; g < S && !bad; g++) {
                for (int s0 = 1; s0 <= (mod ? 1 : g + 1); s0 += seg_pairs) {
                    const bool ok = __all_sync(0xffffffffu, mbar_wait_ab(&accf, nseg & 1, abort, sch.wait));
                    if (!ok) {
                        bad = true;
                        break;
                    }
                    tc_fence_after();
                    if (mod) {
                        uint32_t rp[32];
                        oz_mod_read<MODE>(t_lane, sch, g, half, rp);
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&acce);          // the accumulators are free
                        nseg++;
                        oz_mod_accumulate<MODE>(t_lane, sch, g, half, rp);
                        continue;
                    }
                    const bool init = (g == 0 && s0 == 1);      // first segment of the tile
                    // running-sum block o (32 values) = r block o +- i block (o ^ 1) (HO:
                    // Re H, Im H, Re O, Im O) or (o ^ 2) (ATOM: Re rows 0-63, Im rows 0-63)
#pragma unroll 1
                    for (int k = 0; k < 2; k++) {
                        const int o = oz_block<MODE>(half, k);
                        const int sg = (MODE == OZ_HO) ? ((o & 1) ? -1 : 1) : ((o < 2) ? -1 : 1);
                        const int oi = (MODE == OZ_HO) ? (o ^ 1) : (o ^ 2);
#pragma unroll 1
                        for (int jc = 0; jc < 32; jc += 16) {
                            uint32_t rv[16], iv[16], lo[16], hi[16];
                            const uint32_t fcol = OZ_FP64_COL + 2 * (o * 32 + jc);
                            tm_ld16(t_lane + o * 32 + jc, rv);
                            tm_ld16(t_lane + 128 + oi * 32 + jc, iv);
                            if (!init) {
                                tm_ld16(t_lane + fcol, lo);
                                tm_ld16(t_lane + fcol + 16, hi);
                            }
                            tm_wait_ld();
                            uint32_t o0[16], o1[16];
                            oz_fold16(g, init, sg, rv, iv, lo, hi, o0, o1);
                            tm_st16(t_lane + fcol, o0);
                            tm_st16(t_lane + fcol + 16, o1);
                        }
                    }
                    tm_wait_st();
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acce);
                    nseg++;
                }
            }
            if (!__all_sync(0xffffffffu, !bad && !*abort)) {
                bad = true;
                break;
            }
            const KDesc kd = ks[ti.k];
            if (MODE == OZ_HO) {
                oz_store_ho(p, kd, sch, ti.i0, ti.j0, t_lane, qd * 32 + lane, half, staged ? mirror : nullptr);
                if (staged) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&stg);
                    if (__all_sync(0xffffffffu, mbar_wait_ab(&stg, 0, abort, sch.wait)))
                        oz_store_mirror(kd, ti.i0, ti.j0, mirror, warp - 4, lane);
                }
            } else {
                // row G of the tile; values v = 0..63 real, 64..127 imaginary parts of the 64 output
                // rows, of which this half holds rows 32 half .. 32 half + 31
                const int g = ti.i0 + qd * 32 + lane;
                const bool g_ok = g < p.npad;
                const AtomDesc at = p.atoms[ti.ias];
                const bool lorows = ti.xb >= xa.nfb;
                const double sa = g_ok ? oz_sigma(kd.oz_scale[g]) : 0.0;
                const double *sig = xa.xsig + ((size_t)ti.ias * xa.nxb + ti.xb) * 64;
                const size_t row0 = (size_t)kd.ngp + at.lo_off;
                double bmax = 0.0;
#pragma unroll 1
                for (int jc = 32 * half; jc < 32 * half + 32; jc += 8) {
                    uint32_t wr[16], wi[16];
                    tm_ld16(t_lane + OZ_FP64_COL + 2 * jc, wr);
                    tm_ld16(t_lane + OZ_FP64_COL + 2 * (64 + jc), wi);
                    tm_wait_ld();
                    if (!g_ok) continue;
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        const int n = jc + e;
                        const double sc = sa * sig[n];
                        const double re = oz_final(sch, sch.finx, wr[2 * e], wr[2 * e + 1]) * sc;
                        const double im = oz_final(sch, sch.finx, wi[2 * e], wi[2 * e + 1]) * sc;
                        if (!lorows) {
                            const int f = ti.xb * 64 + n;
                            if (f >= at.napw) continue;
                            const size_t off = (size_t)(at.apw_off + f) * p.npad + g;
                            kd.br[off] = re;
                            kd.bi[off] = im;
                            bmax = fmax(bmax, fmax(fabs(re), fabs(im)));
                        } else {
                            const int r = (ti.xb - xa.nfb) * 64 + n;
                            if (r >= at.losize || g >= kd.ngp) continue;
                            exs_complex v;
                            v.re = re;
                            v.im = im;
                            kd.h[(row0 + r) + (size_t)kd.nmat * g] = v;
                            v.im = -im;
                            kd.h[(size_t)g + (size_t)kd.nmat * (row0 + r)] = v;
                        }
                    }
                }
                if (!lorows && g_ok) atomic_max_nonneg(kd.oz_scale + p.npad + g, bmax);
            }
            // the FP64 region is read; the next tile's first fold may overwrite it
            tc_fence_before();
        }
    }
    if (tid == 0 && *abort) atomicOr(p.err, DEV_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 3) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(OZ_TMEM_COLS));
    }
}

// ------------------------------------------------------------ two-SM H/O tiles
// A cluster of two CTAs computes a 256 (G_i) x 32 (G_j) tile with
// tcgen05.mma.cta_group::2 (M = 256): each CTA holds its own 128 rows of the
// A operands (Ar, Ai) and half of the B operand (CTA 0: Br, Bi; CTA 1: Ar,
// Ai of the 32 G_j), so each SM fetches 320 instead of 384 operand rows per
// K byte.  CTA 0 issues the MMAs; its full barriers count the bytes of both
// CTAs' copies (the copies of CTA 1 signal CTA 0's barrier); MMA completion
// is signalled to both CTAs (multicast commit); both CTAs' epilogues fold
// their own 128 rows and report to CTA 0's barrier.  Each CTA loads its own operands.
constexpr uint32_t OZ_PEER_BIT_MASK = 0xFEFFFFFFu;   // shared::cluster address of CTA 0's copy

__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ void tma_load_5d_2sm(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                                int c4, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3, %4, %5, %6}], [%7];\n" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar & OZ_PEER_BIT_MASK)
        : "memory");
}

__device__ __forceinline__ void umma_i8_2sm(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

// Arrive on the barrier at this offset in both CTAs of the pair.
__device__ __forceinline__ void umma_commit_2sm(uint64_t *bar)
{
    const uint16_t mask = 3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n" ::"r"(
            smem_u32(bar)),
        "h"(mask)
        : "memory");
}

template <int KCH, int NST>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(OZ_THREADS, 1)
oz_mma2_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB2, DevParams p,
               const KDesc *ks, const int *tiles, const __grid_constant__ OzScheme sch, int kp8)
{
    const int S = sch.n;
    const bool mod = sch.mod != 0;
    const int seg_pairs = mod ? 1 : sch.seg;
    constexpr int ABOX = 2 * KCH * OZ_TILE;          // Ar, Ai of this CTA's 128 rows
    constexpr int BBOX = KCH * OZ_TILE / 2;          // this CTA's 64 rows of B
    constexpr int STAGE = ABOX + BBOX;
    extern __shared__ __align__(1024) uint8_t oz_smem[];
    __shared__ uint64_t full[NST], empty[NST], accf, acce, stg;
    __shared__ uint32_t tmem_sh;
    __shared__ int abort_sh;
    volatile int *abort = &abort_sh;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_ctarank();
    static_assert(2 * 32 * OZ_MIRROR_LD * 16 <= NST * STAGE, "mirror staging fits the stages");
    const uint32_t sbase = (smem_u32(oz_smem) + 1023u) & ~1023u;
    const int t3 = 3 * (blockIdx.x >> 1);
    const KDesc kd = ks[tiles[t3]];
    const int i0 = (2 * tiles[t3 + 1] + (int)rank) * OZ_BM, j0 = tiles[t3 + 2] * OZ_BJ;
    const int nst = kp8 / (KCH * OZ_CHUNK);

    if (warp == 3) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_sh)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);      // CTA 0: one arrive (with the bytes of both CTAs)
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accf, 1);
        mbar_init(&acce, 16);            // CTA 0: eight epilogue warps in each CTA
        mbar_init(&stg, 8);              // this CTA's epilogue warps: the mirror is staged
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();                  // the peer's barriers are initialised before anyone signals them
    tc_fence_after();
    const uint32_t tbase = tmem_sh;

    if (warp < 2) {
        // ------------------------------------------------ TMA producers (both CTAs)
        if (lane == 0) {
            const int role = warp;       // 0: this CTA's A rows, 1: this CTA's half of B
            uint32_t fills[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) fills[q] = 0;
            int st = 0;
            bool bad = false;
            const int slot = kd.oz_slot;
            for (int g = 0; g < S && !bad; g++)
                for (int j = 0; j < (mod ? 1 : g + 1) && !bad; j++) {
                    const int s = mod ? g + 1 : j + 1, t = mod ? g + 1 : g + 1 - j;
                    for (int kb = 0; kb < nst; kb++) {
                        if (fills[st] > 0 && !mbar_wait_ab(&empty[st], (fills[st] - 1) & 1, abort, sch.wait)) {
                            bad = true;
                            break;
                        }
                        if (rank == 0 && role == 0) mbar_expect_tx(&full[st], 2 * STAGE);
                        const uint32_t bar = smem_u32(&full[st]);
                        if (role == 0)
                            tma_load_5d_2sm(sbase + st * STAGE, &mapA, 0, i0, oz_narr(p.relativity) - 2, kb * KCH,
                                            slot * S + s - 1, bar);
                        else
                            tma_load_5d_2sm(sbase + st * STAGE + ABOX, &mapB2, 0, j0, 2 * (int)rank, kb * KCH,
                                            slot * S + t - 1, bar);
                        fills[st]++;
                        st = (st + 1 == NST) ? 0 : st + 1;
                    }
                }
            // CTA 0: copies already issued (both CTAs') must land before the pair goes away;
            // CTA 1 stopped issuing at least one bounded wait ago
            if (bad && rank == 0)
                for (int q = 0; q < NST; q++)
                    if (fills[q] > 0) mbar_drain(&full[q], (fills[q] - 1) & 1);
        }
    } else if (warp == 3) {
        // ------------------------------------------------ MMA issuer (CTA 0)
        if (lane == 0 && rank == 0) {
            const uint32_t idesc = umma_idesc_i8(256, OZ_N);
            uint32_t uses[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) uses[q] = 0;
            int nseg = 0, st = 0;
            bool bad = false;
            for (int g = 0; g < S && !bad; g++)
                for (int s0 = 1; s0 <= (mod ? 1 : g + 1) && !bad; s0 += seg_pairs) {
                    const int s1 = min(mod ? 1 : g + 1, s0 + seg_pairs - 1);
                    if (nseg > 0 && !mbar_wait_ab(&acce, (nseg - 1) & 1, abort, sch.wait)) {
                        bad = true;
                        break;
                    }
                    tc_fence_after();
                    bool first = true;
                    for (int s = s0; s <= s1 && !bad; s++)
                        for (int kb = 0; kb < nst; kb++) {
                            if (!mbar_wait_ab(&full[st], uses[st] & 1, abort, sch.wait)) {
                                bad = true;
                                break;
                            }
                            tc_fence_after();
                            const uint32_t sa = sbase + st * STAGE;
#pragma unroll
                            for (int c = 0; c < KCH; c++)
#pragma unroll
                                for (int q = 0; q < OZ_CHUNK / 32; q++) {
                                    const uint32_t ao = c * 2 * OZ_TILE + q * 32;
                                    const uint64_t bd = umma_desc_sw128(sa + ABOX + c * (OZ_TILE / 2) + q * 32);
                                    const uint32_t acc = (first && c == 0 && q == 0) ? 0u : 1u;
                                    umma_i8_2sm(tbase, umma_desc_sw128(sa + ao), bd, idesc, acc);
                                    umma_i8_2sm(tbase + 128, umma_desc_sw128(sa + ao + OZ_TILE), bd, idesc, acc);
                                }
                            first = false;
                            umma_commit_2sm(&empty[st]);
                            uses[st]++;
                            st = (st + 1 == NST) ? 0 : st + 1;
                        }
                    if (!bad) {
                        umma_commit_2sm(&accf);
                        nseg++;
                    }
                }
            if (bad)
                for (int q = 0; q < NST; q++)
                    if (uses[q] > 0) mbar_drain(&empty[q], (uses[q] - 1) & 1);
        }
    } else if (warp >= 4) {
        // ------------------------------------------------ epilogue (both CTAs, warps 4..11)
        const int qd = warp & 3;
        const int half = (warp - 4) >> 2;
        const uint32_t t_lane = tbase + ((uint32_t)(qd * 32) << 16);
        const uint32_t acce0 = mapa_shared(smem_u32(&acce), 0);
        int nseg = 0;
        bool bad = false;
        for (int g = 0; g < S && !bad; g++) {
            for (int s0 = 1; s0 <= (mod ? 1 : g + 1); s0 += seg_pairs) {
                const bool ok = __all_sync(0xffffffffu, mbar_wait_ab(&accf, nseg & 1, abort, sch.wait));
                if (!ok) {
                    bad = true;
                    break;
                }
                tc_fence_after();
                if (mod) {
                    uint32_t rp[32];
                    oz_mod_read<OZ_HO>(t_lane, sch, g, half, rp);
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_remote(acce0);      // the accumulators are free
                    nseg++;
                    oz_mod_accumulate<OZ_HO>(t_lane, sch, g, half, rp);
                    continue;
                }
                const bool init = (nseg == 0);
#pragma unroll 1
                for (int k = 0; k < 2; k++) {
                    const int o = oz_block<OZ_HO>(half, k);
                    const int sg = (o & 1) ? -1 : 1;
#pragma unroll 1
                    for (int jc = 0; jc < 32; jc += 16) {
                        uint32_t rv[16], iv[16], lo[16], hi[16];
                        const uint32_t fcol = OZ_FP64_COL + 2 * (o * 32 + jc);
                        tm_ld16(t_lane + o * 32 + jc, rv);
                        tm_ld16(t_lane + 128 + (o ^ 1) * 32 + jc, iv);
                        if (!init) {
                            tm_ld16(t_lane + fcol, lo);
                            tm_ld16(t_lane + fcol + 16, hi);
                        }
                        tm_wait_ld();
                        uint32_t o0[16], o1[16];
                        oz_fold16(g, init, sg, rv, iv, lo, hi, o0, o1);
                        tm_st16(t_lane + fcol, o0);
                        tm_st16(t_lane + fcol + 16, o1);
                    }
                }
                tm_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_remote(acce0);      // CTA 0's barrier (also from CTA 0)
                nseg++;
            }
        }
        exs_complex *mirror = reinterpret_cast<exs_complex *>(oz_smem + (sbase - smem_u32(oz_smem)));
        if (__all_sync(0xffffffffu, !bad && !*abort))
            oz_store_ho(p, kd, sch, i0, j0, t_lane, qd * 32 + lane, half, mirror);
        __syncwarp();
        if (lane == 0) mbar_arrive(&stg);
        if (__all_sync(0xffffffffu, mbar_wait_ab(&stg, 0, abort, sch.wait) && !*abort))
            oz_store_mirror(kd, i0, j0, mirror, warp - 4, lane);
    }
    if (tid == 0 && *abort) atomicOr(p.err, DEV_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();                  // neither CTA leaves while the pair still uses its memory
    if (warp == 3) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(OZ_TMEM_COLS));
    }
}

// ------------------------------------------------------------ residue tiles (modular H/O)
// The modular H/O contraction in two kernels.  oz_res_kernel forms, per
// 128 (G_i) x BJ (G_j) tile and per modulus, the int32 products
// r = Ar^T [Br|Bi|Ar|Ai] and i = Ai^T [Br|Bi|Ar|Ai] (MMA N = 4 BJ) and writes
// the residues x = v mod p in [0, p) of the four values
// v = Re H (r0 + i1), Im H (r1 - i0), Re O (r2 + i3), Im O (r3 - i2) as bytes.
// oz_crt_kernel recombines the n residues of each value by the Chinese
// remainder theorem with 96-bit constants (exact but for 2^-(64+s) M, the
// 64-bit window s bits below the top of the sum, s = 0 up to 13 moduli; no
// headroom bits needed), scales by sigma_A(i) sigma_B(j) (sigma_A(j) for O),
// adds the interstitial term and writes the upper triangle and its mirror.
// With no running sums in tensor memory the tile is 128 x 64 (N = 256: r and
// i fill the 512 columns) or 128 x 32 with two accumulator pairs, so that
// the MMAs of one modulus run while the epilogue reduces the previous one.
//
// Residues of a tile (n * 4 * 128 * BJ bytes): [modulus g][value o]
// [16-column chunk][row 0..127][16 bytes]: an epilogue warp (32 rows) stores
// 512 contiguous bytes, a thread of oz_crt_kernel reads 8 of the 16 bytes of
// one vector per (g, o).
template <int BJ>
struct ResCfg {
    static constexpr int N = 4 * BJ;                     // MMA N
    static constexpr int NACC = BJ == 32 ? 2 : 1;        // accumulator pairs (r, i) in tensor memory
    static constexpr int ABOX = 2 * OZ_TILE;             // Ar, Ai of 128 G rows, one K chunk
    static constexpr int BBOX = 4 * BJ * OZ_CHUNK;       // four arrays of BJ G rows, one K chunk
    static constexpr int STAGE = ABOX + BBOX;
    static constexpr int NST = (192 * 1024) / STAGE;     // 4 stages (BJ 32) or 3 (BJ 64)
    static constexpr int NCH = BJ / 16;                  // 16-column chunks of a value block
    static constexpr int MOD_BYTES = 4 * 128 * BJ;       // residues of one modulus of a tile
    static constexpr int SMEM = NST * STAGE + 1024;
};

__device__ __forceinline__ uint32_t oz_res4(const uint32_t (&rv)[16], const uint32_t (&iv)[16], int e0, bool minus,
                                            int pm, int mg)
{
    uint32_t w = 0;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int v = minus ? (int)rv[e0 + e] - (int)iv[e0 + e] : (int)rv[e0 + e] + (int)iv[e0 + e];
        int x = v - __mulhi(v, mg) * pm;          // in [-p/4, 5p/4]
        x += x < 0 ? pm : 0;
        x -= x >= pm ? pm : 0;                    // in [0, p)
        w |= (uint32_t)x << (8 * e);
    }
    return w;
}

template <int BJ>
__global__ void __launch_bounds__(OZ_THREADS, 1)
oz_res_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, DevParams p,
              const KDesc *ks, const int *tiles, int ntiles, const __grid_constant__ OzScheme sch, int kp8,
              uint8_t *res)
{
    using C = ResCfg<BJ>;
    constexpr int NST = C::NST, NACC = C::NACC, N = C::N;
    const int S = sch.n;
    const int nch = kp8 / OZ_CHUNK;
    extern __shared__ __align__(1024) uint8_t oz_smem[];
    __shared__ uint64_t full[NST], empty[NST], accf[NACC], acce[NACC];
    __shared__ uint32_t tmem_sh;
    __shared__ int abort_sh;
    volatile int *abort = &abort_sh;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = (smem_u32(oz_smem) + 1023u) & ~1023u;

    if (warp == 3) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_sh)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int q = 0; q < NST; q++) {
            mbar_init(&full[q], 2);
            mbar_init(&empty[q], 1);
        }
        for (int a = 0; a < NACC; a++) {
            mbar_init(&accf[a], 1);
            mbar_init(&acce[a], 8);              // the eight epilogue warps
        }
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tmem_sh;

    if (warp < 3) {
        // ------------------------------------------------ TMA producers: warp 0 the A box, warp 1 the B box
        if (lane == 0 && warp < 2) {
            const int role = warp;
            uint32_t fills[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) fills[q] = 0;
            int st = 0;
            bool bad = false;
            for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
                const int slot = ks[tiles[3 * tile]].oz_slot;
                const int i0 = tiles[3 * tile + 1] * OZ_BM, j0 = tiles[3 * tile + 2] * BJ;
                for (int g = 0; g < S && !bad; g++)
                    for (int kb = 0; kb < nch; kb++) {
                        if (fills[st] > 0 && !mbar_wait_ab(&empty[st], (fills[st] - 1) & 1, abort, sch.wait)) {
                            bad = true;
                            break;
                        }
                        mbar_expect_tx(&full[st], role == 0 ? C::ABOX : C::BBOX);
                        const uint32_t dst = sbase + st * C::STAGE + (role == 0 ? 0 : C::ABOX);
                        if (role == 0)          // Ar and Ai (the slot's last two arrays) of G rows i0 .. i0+127, modulus g
                            tma_load_5d(dst, &mapA, 0, i0, oz_narr(p.relativity) - 2, kb, slot * S + g, &full[st]);
                        else                    // the four arrays of G rows j0 .. j0+BJ-1
                            tma_load_5d(dst, &mapB, 0, j0, 0, kb, slot * S + g, &full[st]);
                        fills[st]++;
                        st = (st + 1 == NST) ? 0 : st + 1;
                    }
            }
            if (bad)   // copies already issued must land before the CTA goes away
                for (int q = 0; q < NST; q++)
                    if (fills[q] > 0) mbar_drain(&full[q], (fills[q] - 1) & 1);
        }
    } else if (warp == 3) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_i8(128, N);
            uint32_t uses[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) uses[q] = 0;
            int st = 0, u = 0;
            bool bad = false;
            for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x)
                for (int g = 0; g < S && !bad; g++, u++) {
                    const int buf = u % NACC, use = u / NACC;
                    // the epilogue must have read this accumulator pair's previous modulus
                    if (use > 0 && !mbar_wait_ab(&acce[buf], (use - 1) & 1, abort, sch.wait)) {
                        bad = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t tacc = tbase + (uint32_t)(buf * 2 * N);
                    for (int kb = 0; kb < nch; kb++) {
                        if (!mbar_wait_ab(&full[st], uses[st] & 1, abort, sch.wait)) {
                            bad = true;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sa = sbase + st * C::STAGE;
#pragma unroll
                        for (int q = 0; q < OZ_CHUNK / 32; q++) {
                            const uint64_t bd = umma_desc_sw128(sa + C::ABOX + q * 32);
                            const uint32_t acc = (kb == 0 && q == 0) ? 0u : 1u;
                            umma_i8(tacc, umma_desc_sw128(sa + q * 32), bd, idesc, acc);
                            umma_i8(tacc + N, umma_desc_sw128(sa + OZ_TILE + q * 32), bd, idesc, acc);
                        }
                        umma_commit(&empty[st]);
                        uses[st]++;
                        st = (st + 1 == NST) ? 0 : st + 1;
                    }
                    if (!bad) umma_commit(&accf[buf]);
                }
            if (bad)   // MMAs already issued must finish before tensor memory is freed
                for (int q = 0; q < NST; q++)
                    if (uses[q] > 0) mbar_drain(&empty[q], (uses[q] - 1) & 1);
        }
    } else {
        // ------------------------------------------------ epilogue (warps 4..11): residues of two value blocks
        const int qd = warp & 3;                                    // tensor-memory lane quadrant
        const int half = (warp - 4) >> 2;                           // 0: Re H, Im H; 1: Re O, Im O
        const int row = qd * 32 + lane;
        const uint32_t t_lane = tbase + ((uint32_t)(qd * 32) << 16);
        int u = 0;
        bool bad = false;
        for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
            uint8_t *tres = res + (size_t)tile * S * C::MOD_BYTES;
            for (int g = 0; g < S; g++, u++) {
                const int buf = u % NACC, use = u / NACC;
                if (!__all_sync(0xffffffffu, mbar_wait_ab(&accf[buf], use & 1, abort, sch.wait))) {
                    bad = true;
                    break;
                }
                tc_fence_after();
                const int pm = sch.p[g], mg = sch.mg[g];
                const uint32_t tacc = t_lane + (uint32_t)(buf * 2 * N);
                uint4 out[2][C::NCH];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int o = 2 * half + k, oi = o ^ 1;
                    const bool minus = (o & 1) != 0;
#pragma unroll
                    for (int c = 0; c < C::NCH; c++) {
                        uint32_t rv[16], iv[16];
                        tm_ld16(tacc + o * BJ + c * 16, rv);
                        tm_ld16(tacc + N + oi * BJ + c * 16, iv);
                        tm_wait_ld();
                        out[k][c] = make_uint4(oz_res4(rv, iv, 0, minus, pm, mg), oz_res4(rv, iv, 4, minus, pm, mg),
                                               oz_res4(rv, iv, 8, minus, pm, mg), oz_res4(rv, iv, 12, minus, pm, mg));
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acce[buf]);             // the accumulator pair is free
                uint8_t *gres = tres + (size_t)g * C::MOD_BYTES;
#pragma unroll
                for (int k = 0; k < 2; k++)
#pragma unroll
                    for (int c = 0; c < C::NCH; c++)
                        *reinterpret_cast<uint4 *>(gres + ((size_t)((2 * half + k) * C::NCH + c) * 128 + row) * 16) =
                            out[k][c];
            }
        }
    }
    if (tid == 0 && *abort) atomicOr(p.err, DEV_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 3) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(OZ_TMEM_COLS));
    }
}

// ------------------------------------------------------------ two-SM residue tiles
// A cluster of two CTAs computes a 256 (G_i) x BJ (G_j) tile with
// tcgen05.mma.cta_group::2 (M = 256, N = 4 BJ): each CTA holds its own 128
// rows of Ar, Ai and two of the four B arrays (CTA 0: Br, Bi; CTA 1: Ar, Ai
// of the G_j, or Cr, Ci with iora*), 48 KB per K chunk instead of 64 KB, and
// each CTA writes the residues of its own 128 rows as the 128-row residue
// tile 2 pair + rank.  CTA 0 issues the MMAs; its full barriers count the
// bytes of both CTAs' copies; MMA completion is signalled to both CTAs
// (multicast commit); both CTAs' epilogues report to CTA 0's barrier.
// Pacing of the persistent pair kernel: every cluster publishes, every
// OZ_PACE_CHUNKS K chunks it issues, its step count in pace[cluster] and,
// before a new step, waits until the slowest cluster is at most OZ_PACE_LAG
// steps behind, so that the pairs running at one time read the same row and
// column blocks within a few MB of each other's position and the L2 serves
// the repeats.  216-atom cell, setups/s by (lag, chunks): (1, 32) 0.955,
// (2, 32) 0.944, (2, 16) 0.943, (2, 64) 0.935, (4, 16) 0.915; a 200,000
// cycle cap 0.943.  The wait is a hint, not a dependency: it gives up after
// OZ_PACE_CYCLES (a cluster that is not resident, or a slow one, delays the
// others by that much per step at most) and never raises an error.  A
// finished cluster publishes INT_MAX.
constexpr int OZ_PACE_CHUNKS = 32;
constexpr int OZ_PACE_LAG = 1;
constexpr long long OZ_PACE_CYCLES = 40000;
constexpr int OZ_PACE_MAX = 1024;                 // clusters (ints of the pace array)

__device__ __forceinline__ int ld_relaxed_gpu(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_gpu(int *p, int v)
{
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void oz_pace(int *pace, int me, int ncl, int step)
{
    const long long t0 = clock64();
    while (true) {
        int mn = 0x7fffffff;
        for (int c = 0; c < ncl; c++) mn = min(mn, ld_relaxed_gpu(pace + c));
        if (mn >= step - OZ_PACE_LAG || clock64() - t0 > OZ_PACE_CYCLES) break;
    }
    st_relaxed_gpu(pace + me, step);
}

template <int BJ>
struct Res2Cfg {
    static constexpr int N = 4 * BJ;                     // MMA N: both CTAs' halves of B
    static constexpr int ABOX = 2 * OZ_TILE;             // this CTA's Ar, Ai (128 rows), one K chunk
    static constexpr int BBOX = 2 * BJ * OZ_CHUNK;       // this CTA's two arrays of B (BJ rows each)
    static constexpr int STAGE = ABOX + BBOX;
    static constexpr int NST = (192 * 1024) / STAGE;     // BJ 64: 4 stages of 48 KB
    static constexpr int SMEM = NST * STAGE + 1024;
};

template <int BJ>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(OZ_THREADS, 1)
oz_res2_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapBh, DevParams p,
               const KDesc *ks, const int *tiles, int npairs, const __grid_constant__ OzScheme sch, int kp8,
               uint8_t *res, int *pace)
{
    using C = Res2Cfg<BJ>;
    using R = ResCfg<BJ>;
    constexpr int NST = C::NST, N = C::N;
    static_assert(2 * N <= OZ_TMEM_COLS, "r and i fit tensor memory");
    const int S = sch.n;
    const int nch = kp8 / OZ_CHUNK;
    extern __shared__ __align__(1024) uint8_t oz_smem[];
    __shared__ uint64_t full[NST], empty[NST], accf, acce;
    __shared__ uint32_t tmem_sh;
    __shared__ int abort_sh;
    volatile int *abort = &abort_sh;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_ctarank();
    const uint32_t sbase = (smem_u32(oz_smem) + 1023u) & ~1023u;
    // pairs pair0, pair0 + npc, ...: one pair per cluster, or (persistent launch) the clusters walk the
    // list together, so that the pairs running at one time share row and column blocks in the L2; the
    // 128-row tile list holds the pair's tiles at 2 pair and 2 pair + 1 (this CTA's: 2 pair + rank), with
    // the same k-point and column block
    const int pair0 = (int)(blockIdx.x >> 1), npc = (int)(gridDim.x >> 1);

    if (warp == 3) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_sh)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int q = 0; q < NST; q++) {
            mbar_init(&full[q], 1);      // CTA 0: one arrive (with the bytes of both CTAs)
            mbar_init(&empty[q], 1);
        }
        mbar_init(&accf, 1);
        mbar_init(&acce, 16);            // CTA 0: eight epilogue warps in each CTA
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();                  // the peer's barriers are initialised before anyone signals them
    tc_fence_after();
    const uint32_t tbase = tmem_sh;

    if (warp < 2) {
        // ------------------------------------------------ TMA producers (both CTAs)
        if (lane == 0) {
            const int role = warp;       // 0: this CTA's A rows, 1: this CTA's half of B
            uint32_t fills[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) fills[q] = 0;
            int st = 0, chunk = 0;
            bool bad = false;
            const bool pacer = pace != nullptr && rank == 0 && role == 0;
            for (int pr = pair0; pr < npairs && !bad; pr += npc) {
                const int tile = 2 * pr + (int)rank;
                const int slot = ks[tiles[3 * tile]].oz_slot;
                const int i0 = tiles[3 * tile + 1] * OZ_BM, j0 = tiles[3 * tile + 2] * BJ;
                for (int g = 0; g < S && !bad; g++)
                    for (int kb = 0; kb < nch; kb++, chunk++) {
                        if (pacer && chunk % OZ_PACE_CHUNKS == 0) oz_pace(pace, pair0, npc, chunk / OZ_PACE_CHUNKS);
                        if (fills[st] > 0 && !mbar_wait_ab(&empty[st], (fills[st] - 1) & 1, abort, sch.wait)) {
                            bad = true;
                            break;
                        }
                        if (rank == 0 && role == 0) mbar_expect_tx(&full[st], 2 * C::STAGE);
                        const uint32_t bar = smem_u32(&full[st]);
                        if (role == 0)
                            tma_load_5d_2sm(sbase + st * C::STAGE, &mapA, 0, i0, oz_narr(p.relativity) - 2, kb,
                                            slot * S + g, bar);
                        else
                            tma_load_5d_2sm(sbase + st * C::STAGE + C::ABOX, &mapBh, 0, j0, 2 * (int)rank, kb,
                                            slot * S + g, bar);
                        fills[st]++;
                        st = (st + 1 == NST) ? 0 : st + 1;
                    }
            }
            if (pacer) st_relaxed_gpu(pace + pair0, 0x7fffffff);     // done: nobody waits for this cluster
            // CTA 0: copies already issued (both CTAs') must land before the pair goes away;
            // CTA 1 stopped issuing at least one bounded wait ago
            if (bad && rank == 0)
                for (int q = 0; q < NST; q++)
                    if (fills[q] > 0) mbar_drain(&full[q], (fills[q] - 1) & 1);
        }
    } else if (warp == 3) {
        // ------------------------------------------------ MMA issuer (CTA 0)
        if (lane == 0 && rank == 0) {
            const uint32_t idesc = umma_idesc_i8(256, N);
            uint32_t uses[NST];
#pragma unroll
            for (int q = 0; q < NST; q++) uses[q] = 0;
            int st = 0, u = 0;
            bool bad = false;
            for (int pr = pair0; pr < npairs && !bad; pr += npc)
                for (int g = 0; g < S && !bad; g++, u++) {
                    // the epilogues of both CTAs must have read the previous modulus
                    if (u > 0 && !mbar_wait_ab(&acce, (u - 1) & 1, abort, sch.wait)) {
                        bad = true;
                        break;
                    }
                    tc_fence_after();
                    for (int kb = 0; kb < nch; kb++) {
                        if (!mbar_wait_ab(&full[st], uses[st] & 1, abort, sch.wait)) {
                            bad = true;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sa = sbase + st * C::STAGE;
#pragma unroll
                        for (int q = 0; q < OZ_CHUNK / 32; q++) {
                            const uint64_t bd = umma_desc_sw128(sa + C::ABOX + q * 32);
                            const uint32_t acc = (kb == 0 && q == 0) ? 0u : 1u;
                            umma_i8_2sm(tbase, umma_desc_sw128(sa + q * 32), bd, idesc, acc);
                            umma_i8_2sm(tbase + N, umma_desc_sw128(sa + OZ_TILE + q * 32), bd, idesc, acc);
                        }
                        umma_commit_2sm(&empty[st]);
                        uses[st]++;
                        st = (st + 1 == NST) ? 0 : st + 1;
                    }
                    if (!bad) umma_commit_2sm(&accf);
                }
            if (bad)
                for (int q = 0; q < NST; q++)
                    if (uses[q] > 0) mbar_drain(&empty[q], (uses[q] - 1) & 1);
        }
    } else if (warp >= 4) {
        // ------------------------------------------------ epilogue (both CTAs, warps 4..11)
        const int qd = warp & 3;
        const int half = (warp - 4) >> 2;                           // 0: Re H, Im H; 1: Re O, Im O
        const int row = qd * 32 + lane;
        const uint32_t t_lane = tbase + ((uint32_t)(qd * 32) << 16);
        const uint32_t acce0 = mapa_shared(smem_u32(&acce), 0);
        int u = 0;
        bool bad = false;
        for (int pr = pair0; pr < npairs && !bad; pr += npc) {
            uint8_t *tres = res + (size_t)(2 * pr + (int)rank) * S * R::MOD_BYTES;
            for (int g = 0; g < S; g++, u++) {
                if (!__all_sync(0xffffffffu, mbar_wait_ab(&accf, u & 1, abort, sch.wait))) {
                    bad = true;
                    break;
                }
                tc_fence_after();
                const int pm = sch.p[g], mg = sch.mg[g];
                uint4 out[2][R::NCH];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int o = 2 * half + k, oi = o ^ 1;
                    const bool minus = (o & 1) != 0;
#pragma unroll
                    for (int c = 0; c < R::NCH; c++) {
                        uint32_t rv[16], iv[16];
                        tm_ld16(t_lane + o * BJ + c * 16, rv);
                        tm_ld16(t_lane + N + oi * BJ + c * 16, iv);
                        tm_wait_ld();
                        out[k][c] = make_uint4(oz_res4(rv, iv, 0, minus, pm, mg), oz_res4(rv, iv, 4, minus, pm, mg),
                                               oz_res4(rv, iv, 8, minus, pm, mg), oz_res4(rv, iv, 12, minus, pm, mg));
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_remote(acce0);           // CTA 0's barrier (also from CTA 0)
                uint8_t *gres = tres + (size_t)g * R::MOD_BYTES;
#pragma unroll
                for (int k = 0; k < 2; k++)
#pragma unroll
                    for (int c = 0; c < R::NCH; c++)
                        *reinterpret_cast<uint4 *>(gres + ((size_t)((2 * half + k) * R::NCH + c) * 128 + row) * 16) =
                            out[k][c];
            }
        }
    }
    if (tid == 0 && *abort) atomicOr(p.err, DEV_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();                  // neither CTA leaves while the pair still uses its memory
    if (warp == 3) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(OZ_TMEM_COLS));
    }
}

// Eight values from their n residues (w[m]: the 8 bytes of modulus m): per
// value the 96-bit fixed-point sum t = sum_m x_m C_m (mod 2^96), C_m =
// round(2^96 y_m / p_m) in three 32-bit words (three 32 x 32 -> 64-bit
// multiply-adds per term, the carries propagated once at the end), whose top
// 64 bits read as a signed integer are 2^64 X / M (the constants' rounding
// moves t by at most sum x_m / 2 units of 2^-96); X 2^-2b = that times
// fin96 = M 2^-64 2^-2b.
__device__ __forceinline__ void oz_crt8(const OzScheme &sch, const uint2 (&w)[OZ_MAX_MODULI], double (&v)[8])
{
    unsigned long long a[8][3];
#pragma unroll
    for (int e = 0; e < 8; e++) a[e][0] = a[e][1] = a[e][2] = 0ull;
#pragma unroll
    for (int m = 0; m < OZ_MAX_MODULI; m++) {
        if (m >= sch.n) break;
        const unsigned long long c0 = sch.c96[0][m], c1 = sch.c96[1][m], c2 = sch.c96[2][m];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const unsigned long long x = ((e < 4 ? w[m].x : w[m].y) >> (8 * (e & 3))) & 0xffu;
            a[e][0] += x * c0;
            a[e][1] += x * c1;
            a[e][2] += x * c2;
        }
    }
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const unsigned long long a1 = a[e][1] + (a[e][0] >> 32);
        const unsigned long long a2 = a[e][2] + (a1 >> 32);
        const unsigned long long top = (((a2 << 32) | (a1 & 0xffffffffull)) << sch.crt_shift) |
                                       ((a[e][0] & 0xffffffffull) >> (32 - sch.crt_shift));
        v[e] = (double)(long long)top * sch.fin96;
    }
}

// Recombination, scaling, interstitial term and store of the residue tiles:
// one thread per (row of the tile, 8-column group, matrix: 0 = H, 1 = O):
// blocks of 128 threads (the rows), blockIdx.y = (matrix, column group).
// Every thread first issues the 2n loads of its residue bytes (8 per modulus
// and part), then recombines: the loads of a warp cover 32 rows, 256
// contiguous bytes per modulus and part.  158 registers: three blocks per SM.
template <int BJ>
__global__ void __launch_bounds__(128) oz_crt_kernel(DevParams p, const KDesc *ks, const int *tiles,
                                                     const __grid_constant__ OzScheme sch, const uint8_t *res)
{
    using C = ResCfg<BJ>;
    constexpr int NG = BJ / 8;                                   // 8-column groups
    const int tile = blockIdx.x;
    const int row = threadIdx.x;
    const int cg = blockIdx.y % NG, half = blockIdx.y / NG;
    const KDesc kd = ks[tiles[3 * tile]];
    const int i = tiles[3 * tile + 1] * OZ_BM + row;
    const int jb = tiles[3 * tile + 2] * BJ + cg * 8;
    if (i >= kd.ngp || jb >= kd.ngp || jb + 7 < i) return;     // no element i <= j < ngp here
    const uint8_t *tres = res + (size_t)tile * sch.n * C::MOD_BYTES;
    const size_t stride = C::MOD_BYTES;                          // between moduli
    const size_t o_re = ((size_t)((2 * half) * C::NCH + (cg >> 1)) * 128 + row) * 16 + (cg & 1) * 8;
    const size_t o_im = ((size_t)((2 * half + 1) * C::NCH + (cg >> 1)) * 128 + row) * 16 + (cg & 1) * 8;
    uint2 wr[OZ_MAX_MODULI], wi[OZ_MAX_MODULI];
#pragma unroll
    for (int m = 0; m < OZ_MAX_MODULI; m++)
        if (m < sch.n) {
            wr[m] = *reinterpret_cast<const uint2 *>(tres + (size_t)m * stride + o_re);
            wi[m] = *reinterpret_cast<const uint2 *>(tres + (size_t)m * stride + o_im);
        }
    // row data
    int gi = kd.igpig[i] - 1;
    if (gi < 0 || gi >= p.ngrtot) {
        atomicOr(p.err, DEV_ERR_INDEX);
        gi = 0;
    }
    const int ivi[3] = {p.ivg[3 * gi], p.ivg[3 * gi + 1], p.ivg[3 * gi + 2]};
    const double vi[3] = {kd.vgpc[3 * i], kd.vgpc[3 * i + 1], kd.vgpc[3 * i + 2]};
    const double sai = oz_sigma(kd.oz_scale[i]);
    // H: sigma_B(j); O: sigma_A(j), or sigma_C(j) with iora* (O = A^H C)
    const double *scol = kd.oz_scale + (half == 0 ? p.npad : (p.relativity == EXS_REL_IORA ? 2 * p.npad : 0));
    const int kind = half == 0 ? EPI_HAM : EPI_OVL;
    exs_complex *out = half == 0 ? kd.h : kd.o;
    double vre[8], vim[8];
    oz_crt8(sch, wr, vre);
    oz_crt8(sch, wi, vim);
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const int j = jb + e;
        if (j >= kd.ngp || j < i) continue;
        int gj = kd.igpig[j] - 1;
        if (gj < 0 || gj >= p.ngrtot) {
            atomicOr(p.err, DEV_ERR_INDEX);
            gj = 0;
        }
        const int ivj[3] = {p.ivg[3 * gj], p.ivg[3 * gj + 1], p.ivg[3 * gj + 2]};
        const double vj[3] = {kd.vgpc[3 * j], kd.vgpc[3 * j + 1], kd.vgpc[3 * j + 2]};
        const double sc = sai * oz_sigma(scol[j]);
        double re = vre[e] * sc, im = vim[e] * sc;
        double ar, ai;
        if (interstitial(p, kind, ivi, ivj, vi, vj, ar, ai)) {
            re += ar;
            im += ai;
        }
        exs_complex v;
        v.re = re;
        v.im = im;
        out[(size_t)i + (size_t)kd.nmat * j] = v;
        if (i < j) {
            v.im = -im;
            out[(size_t)j + (size_t)kd.nmat * i] = v;
        }
    }
}

// ------------------------------------------------------------ host side
int oz_kpad(int K) { return (K + OZ_MAX_KCH * OZ_CHUNK - 1) / (OZ_MAX_KCH * OZ_CHUNK) * (OZ_MAX_KCH * OZ_CHUNK); }

size_t oz_slot_bytes(int S, int npad, int kp8, int narr) { return (size_t)S * npad * narr * (size_t)kp8; }

int oz_seg_pairs(int S, int kp8)
{
    // pairs whose int32 sums over K stay exact: pairs * kp8 * 127^2 < 2^31
    const long long per = (long long)kp8 * 127 * 127;
    long long n = (((long long)1 << 31) - 1) / per;
    return (int)(n < 1 ? 0 : (n > S ? S : n));
}

// Pairwise coprime odd moduli up to 253, largest first (253 = 11 * 23,
// 247 = 13 * 19, 217 = 7 * 31, 185 = 5 * 37; the others are primes).  At
// most 253 so that a rounded residue |r| <= (p + 1) / 2 fits int8.
static const int OZ_MODULI[OZ_MAX_MODULI] = {253, 251, 247, 241, 239, 233, 229, 227,
                                             223, 217, 211, 199, 197, 193, 191, 185};

// log2 M for the first n moduli (a sum of logarithms: the plan keeps a
// margin of one bit beyond it).
static double oz_log2_modulus(int n)
{
    double lm = 0.0;
    for (int m = 0; m < n; m++) lm += std::log2((double)OZ_MODULI[m]);
    return lm;
}

static int oz_inverse_mod(long long a, long long p)
{
    // extended Euclid on (a mod p, p); gcd is 1 for coprime moduli
    long long r0 = p, r1 = ((a % p) + p) % p, t0 = 0, t1 = 1;
    while (r1 != 0) {
        const long long q = r0 / r1, r2 = r0 - q * r1, t2 = t0 - q * t1;
        r0 = r1; r1 = r2; t0 = t1; t1 = t2;
    }
    return r0 == 1 ? (int)(((t0 % p) + p) % p) : -1;
}

// The modular scheme for n moduli, contraction length K (H/O tiles) and
// per-atom window kx.  Columns are scaled by their 2-norms, so the integer
// products obey |X| <= 2^(2b) (1 + eps)^2 (H/O) and 2^(b + bx) (1 + eps)^2
// (per-atom) whatever K.  The H/O products are recombined exactly (96-bit
// constants), so b = min(52, floor((log2 M - 2) / 2)) keeps one bit of
// margin beyond 2|X| < M; the per-atom products are folded in 64 bits with
// h >= 5 headroom bits: bx = min(52, floor(log2 M - 7 - b)),
// h = floor(log2 M - 2 - b - bx).  The quantisation error of the operands
// grows like 2^-b sqrt(K), so n = 0 takes the fewest moduli in 6..16 with
// b >= 41 + log2(K) / 2 and bx >= 44 (13 moduli, b = 49 and bx = 45, at both
// K = 1936 and K = 34,992).  Returns 0, or -1 if no valid plan exists (n out
// of range, b or bx below 8, or K past the exact int32 range of one product:
// 2 K 127^2 < 2^31).
static void oz_mod_bits(int n, int *b, int *h, int *bx)
{
    const double lm = oz_log2_modulus(n) - 1e-9;
    *b = std::min(52, (int)std::floor((lm - 2.0) / 2.0));
    *bx = std::min(52, (int)std::floor(lm - 7.0 - *b));
    *h = (int)std::floor(lm - 2.0 - *b - *bx);
}

int oz_mod_plan(int n, int K, int kx, OzScheme *sch)
{
    if (K < 1 || kx < 1 || K > 65536 || kx > 65536) return -1;
    int b = 0, h = 0, bx = 0;
    if (n == 0) {
        const int want = (int)std::ceil(41.0 + 0.5 * std::log2((double)K) - 1e-9);
        n = OZ_MAX_MODULI;
        for (int q = 6; q <= OZ_MAX_MODULI; q++) {
            oz_mod_bits(q, &b, &h, &bx);
            if (b >= want && bx >= 44) {
                n = q;
                break;
            }
        }
    }
    if (n < 6 || n > OZ_MAX_MODULI) return -1;
    oz_mod_bits(n, &b, &h, &bx);
    if (b < 8 || bx < 8 || h < 5) return -1;
    OzScheme s{};
    s.mod = 1;
    s.n = n;
    s.seg = s.segx = 1;
    s.b = b;
    s.bx = bx;
    s.h = h;
    double M = 1.0;
    for (int m = 0; m < n; m++) M *= (double)OZ_MODULI[m];
    s.fin = std::ldexp(M, -64 - h - 2 * b);
    s.finx = std::ldexp(M, -64 - h - b - bx);
    // |X| / M <= 2^(2b - log2 M) (1 + eps)^2 < 2^-(crt_shift + 1): the window's top bit is still the sign;
    // its lowest bit, 2^(32 - crt_shift) units of 2^-96, stays above the constants' rounding (< 2^11 units)
    s.crt_shift = std::max(0, std::min(20, (int)std::floor(oz_log2_modulus(n) - 1e-9 - 2.0 * b - 3.0)));
    s.fin96 = std::ldexp(M, -64 - s.crt_shift - 2 * b);
    for (int m = 0; m < n; m++) {
        const int p = OZ_MODULI[m];
        long long mm = 1;   // (M / p) mod p
        for (int q = 0; q < n; q++)
            if (q != m) mm = mm * OZ_MODULI[q] % p;
        const int y = oz_inverse_mod(mm, p);
        if (y < 0) return -1;
        s.p[m] = p;
        s.mg[m] = (int)((((long long)1 << 32) + p / 2) / p);
        s.fp[m] = (float)p;
        s.finv[m] = 1.0f / (float)p;
        for (int j = 0; j < 3; j++) s.fc[j][m] = (float)((1LL << (13 * (j + 1))) % p);
        // round(2^(64+h) y / p) mod 2^64 (y < p < 2^8 and h <= 18: the numerator fits 128 bits)
        const unsigned __int128 num = ((unsigned __int128)y << (64 + h)) + (unsigned)(p / 2);
        s.c[m] = (unsigned long long)(num / (unsigned)p);
        // round(2^96 y / p) < 2^96 in three 32-bit words
        const unsigned __int128 c96 = (((unsigned __int128)y << 96) + (unsigned)(p / 2)) / (unsigned)p;
        for (int w = 0; w < 3; w++) s.c96[w][m] = (unsigned)(c96 >> (32 * w));
    }
    *sch = s;
    return 0;
}

// configuration index: bit 0 = pipeline shape (KCH, NST) of the H/O tiles,
// bit 1 = persistent launch (one CTA per SM) of the H/O tiles, bit 2 =
// persistent launch of the per-atom tiles, bit 3 = two-SM H/O tiles (256 x 32
// per CTA pair; bit 1 unused then)
// bit 0 of a configuration: two 96 KB stages of 2 K chunks, or four 48 KB stages of 1
const int OZ_CFG_KCH[OZ_NCFG] = {2, 1, 2, 1, 2, 1, 2, 1, 2, 1, 2, 1, 2, 1, 2, 1,
                                 2, 1, 2, 1, 2, 1, 2, 1, 2, 1, 2, 1, 2, 1, 2, 1};
const int OZ_CFG_NST[OZ_NCFG] = {2, 4, 2, 4, 2, 4, 2, 4, 2, 4, 2, 4, 2, 4, 2, 4,
                                 2, 4, 2, 4, 2, 4, 2, 4, 2, 4, 2, 4, 2, 4, 2, 4};

cudaError_t launch_oz_split(const DevParams &p, const KDesc *d_k, int nk, const OzScheme &sch, int kp8, int which,
                            cudaStream_t s)
{
    oz_split_kernel<<<dim3(kp8 / SPLIT_F, p.npad / 32, nk), dim3(32, 8), 0, s>>>(p, d_k, sch, kp8, which);
    return cudaGetLastError();
}

cudaError_t launch_oz_colnorm(const DevParams &p, const KDesc *d_k, int nk, int which, int norm, cudaStream_t s)
{
    oz_colnorm_kernel<<<dim3(p.npad / 32, nk), dim3(32, 8), 0, s>>>(p, d_k, which, norm);
    return cudaGetLastError();
}

cudaError_t launch_oz_x(const DevParams &p, const OzAtomArgs &xa, const OzScheme &sch, cudaStream_t s)
{
    oz_xsig_kernel<<<dim3(xa.nxb, p.natmtot), 64, 0, s>>>(p, xa, sch.mod);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    oz_xsplit_kernel<<<dim3(8, xa.nxb, p.natmtot), dim3(xa.lw / 4, 8), 0, s>>>(p, xa, sch);
    return cudaGetLastError();
}

template <int MODE, int KCH, int NST>
static cudaError_t launch_cfg(const CUtensorMap *mapA, const CUtensorMap *mapB, const DevParams &p, const KDesc *d_k,
                              const void *d_tiles, int ntiles, const OzScheme &sch, int kp8, const OzAtomArgs &xa,
                              bool persistent, cudaStream_t s)
{
    constexpr int smem = NST * 3 * KCH * OZ_TILE + 1024;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        return cudaFuncSetAttribute(oz_mma_kernel<MODE, KCH, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // persistent: one CTA per SM walking the tiles; else one CTA per tile
    const int grid = (persistent && nsm < ntiles) ? nsm : ntiles;
    oz_mma_kernel<MODE, KCH, NST><<<grid, OZ_THREADS, smem, s>>>(*mapA, *mapB, p, d_k, (const int *)d_tiles, ntiles,
                                                                 sch, kp8, xa);
    return cudaGetLastError();
}

template <int KCH, int NST>
static cudaError_t launch_2sm(const CUtensorMap *mapA, const CUtensorMap *mapB2, const DevParams &p, const KDesc *d_k,
                              const void *d_tiles, int ntiles, const OzScheme &sch, int kp8, cudaStream_t s)
{
    constexpr int smem = NST * (2 * KCH * OZ_TILE + KCH * OZ_TILE / 2) + 1024;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        return cudaFuncSetAttribute(oz_mma2_kernel<KCH, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (e != cudaSuccess) return e;
    oz_mma2_kernel<KCH, NST><<<2 * ntiles, OZ_THREADS, smem, s>>>(*mapA, *mapB2, p, d_k, (const int *)d_tiles, sch,
                                                                  kp8);
    return cudaGetLastError();
}

cudaError_t launch_oz_mma(int cfg, const CUtensorMap *mapA, const CUtensorMap *mapB, const DevParams &p,
                          const KDesc *d_k, const void *d_tiles, int ntiles, const OzScheme &sch, int kp8,
                          cudaStream_t s)
{
    if (ntiles <= 0) return cudaSuccess;
    if (cfg & 8) {   // two-SM tiles: mapB is the half-B view
        if (cfg & 1) return launch_2sm<1, 4>(mapA, mapB, p, d_k, d_tiles, ntiles, sch, kp8, s);
        return launch_2sm<2, 2>(mapA, mapB, p, d_k, d_tiles, ntiles, sch, kp8, s);
    }
    const OzAtomArgs none{};
    const bool persistent = (cfg & 2) != 0;
    switch (cfg & 1) {
    case 0: return launch_cfg<OZ_HO, 2, 2>(mapA, mapB, p, d_k, d_tiles, ntiles, sch, kp8, none, persistent, s);
    default: return launch_cfg<OZ_HO, 1, 4>(mapA, mapB, p, d_k, d_tiles, ntiles, sch, kp8, none, persistent, s);
    }
}

template <int BJ>
static cudaError_t launch_res_bj(const CUtensorMap *mapA, const CUtensorMap *mapB, const DevParams &p,
                                 const KDesc *d_k, const void *d_tiles, int ntiles, const OzScheme &sch, int kp8,
                                 uint8_t *res, bool persistent, cudaStream_t s)
{
    constexpr int smem = ResCfg<BJ>::SMEM;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        return cudaFuncSetAttribute(oz_res_kernel<BJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (persistent && nsm < ntiles) ? nsm : ntiles;
    oz_res_kernel<BJ><<<grid, OZ_THREADS, smem, s>>>(*mapA, *mapB, p, d_k, (const int *)d_tiles, ntiles, sch, kp8,
                                                     res);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    oz_crt_kernel<BJ><<<dim3(ntiles, 2 * (BJ / 8)), 128, 0, s>>>(p, d_k, (const int *)d_tiles, sch, res);
    return cudaGetLastError();
}

static cudaError_t launch_res2(const CUtensorMap *mapA, const CUtensorMap *mapBh, const DevParams &p,
                               const KDesc *d_k, const void *d_tiles, int ntiles, const OzScheme &sch, int kp8,
                               uint8_t *res, int *pace, bool persistent, cudaStream_t s)
{
    constexpr int BJ = 64;
    constexpr int smem = Res2Cfg<BJ>::SMEM;
    if (ntiles % 2 != 0) return cudaErrorInvalidValue;      // whole pairs
    const int npairs = ntiles / 2;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        return cudaFuncSetAttribute(oz_res2_kernel<BJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (e != cudaSuccess) return e;
    int ncl = npairs;
    if (persistent) {   // as many pairs as can be resident at once (one cluster of two per SM pair)
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(ntiles);
        lc.blockDim = dim3(OZ_THREADS);
        lc.dynamicSmemBytes = smem;
        lc.stream = s;
        int act = 0;
        if (cudaOccupancyMaxActiveClusters(&act, (void *)oz_res2_kernel<BJ>, &lc) != cudaSuccess || act < 1) {
            (void)cudaGetLastError();
            int dev = 0, nsm = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            act = nsm / 2;
        }
        ncl = std::min(std::min(npairs, act), OZ_PACE_MAX);
        if (pace) {
            e = cudaMemsetAsync(pace, 0, sizeof(int) * ncl, s);
            if (e != cudaSuccess) return e;
        }
    }
    oz_res2_kernel<BJ><<<2 * ncl, OZ_THREADS, smem, s>>>(*mapA, *mapBh, p, d_k, (const int *)d_tiles, npairs, sch,
                                                          kp8, res, persistent ? pace : nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    oz_crt_kernel<BJ><<<dim3(ntiles, 2 * (BJ / 8)), 128, 0, s>>>(p, d_k, (const int *)d_tiles, sch, res);
    return cudaGetLastError();
}

// The modular H/O products: residue tiles then their recombination.
// Configuration bit 0: 128 x 32 tiles (two accumulator pairs) instead of
// 128 x 64; bit 1: persistent residue kernel (one CTA per SM, or one
// cluster per SM pair); bit 3: 256 x 64 tiles on two SMs (the tile list then
// holds each pair's two 128-row tiles next to each other; bit 0 does not
// apply).
cudaError_t launch_oz_res(int cfg, const CUtensorMap *mapA, const CUtensorMap *mapB32, const CUtensorMap *mapB64,
                          const CUtensorMap *mapB64h, const DevParams &p, const KDesc *d_k, const void *d_tiles,
                          int ntiles, const OzScheme &sch, int kp8, uint8_t *res, int *pace, cudaStream_t s)
{
    if (ntiles <= 0) return cudaSuccess;
    if (cfg & 8) return launch_res2(mapA, mapB64h, p, d_k, d_tiles, ntiles, sch, kp8, res, pace, (cfg & 2) != 0, s);
    const bool persistent = (cfg & 2) != 0;
    if (cfg & 1) return launch_res_bj<32>(mapA, mapB32, p, d_k, d_tiles, ntiles, sch, kp8, res, persistent, s);
    return launch_res_bj<64>(mapA, mapB64, p, d_k, d_tiles, ntiles, sch, kp8, res, persistent, s);
}

int oz_res_cols(int cfg) { return (cfg & 1) && !(cfg & 8) ? 32 : 64; }

int oz_res_rows(int cfg) { return (cfg & 8) ? 256 : 128; }

size_t oz_pace_bytes() { return sizeof(int) * OZ_PACE_MAX; }

size_t oz_res_tile_bytes(int n, int cfg) { return (size_t)n * 4 * 128 * oz_res_cols(cfg); }

cudaError_t launch_oz_atom(int cfg, const CUtensorMap *mapArow, const CUtensorMap *mapX, const DevParams &p,
                           const KDesc *d_k, const void *d_tiles, int ntiles, const OzScheme &sch, int kp8,
                           const OzAtomArgs &xa, cudaStream_t s)
{
    if (ntiles <= 0) return cudaSuccess;
    return launch_cfg<OZ_ATOM, 1, 4>(mapArow, mapX, p, d_k, d_tiles, ntiles, sch, kp8, xa, (cfg & 4) != 0, s);
}

// TMA views of the slices of all slots (int8, 5D):
//   d0: K byte within a 128-byte chunk                       stride 1
//   d1: G row (npad)                                         stride kp8
//   d2: array (Br, Bi, Ar, Ai; iora*: Br, Bi, Cr, Ci, Ar, Ai) stride npad kp8
//   d3: K chunk                                              stride 128
//   d4: slot x slice                                         stride narr npad kp8
// A box {128, 128, 2, kch, 1}: Ar and Ai of 128 G rows; B box
// {128, 32, 4, kch, 1}: the four arrays of 32 G rows.  d3 is outside d1, d2
// in the box, so each K chunk lands in shared memory as contiguous
// 128-byte rows (A: 2 x 128 rows, B: 4 x 32 rows).
bool make_oz_tensor_maps(void *base, size_t nss, int npad, int kp8, int kch, int narr, CUtensorMap *mapA,
                         CUtensorMap *mapB, CUtensorMap *mapB2)
{
    typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
        return false;
    EncodeFn encode = (EncodeFn)fn;
    if (kch < 1 || kch > OZ_MAX_KCH || kp8 % (OZ_MAX_KCH * OZ_CHUNK) != 0) return false;
    const cuuint64_t dims[5] = {(cuuint64_t)OZ_CHUNK, (cuuint64_t)npad, (cuuint64_t)narr, (cuuint64_t)(kp8 / OZ_CHUNK),
                                (cuuint64_t)nss};
    const cuuint64_t strides[4] = {(cuuint64_t)kp8, (cuuint64_t)npad * kp8, (cuuint64_t)OZ_CHUNK,
                                   (cuuint64_t)narr * npad * kp8};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const cuuint32_t boxA[5] = {OZ_CHUNK, OZ_BM, 2, (cuuint32_t)kch, 1};
    const cuuint32_t boxB[5] = {OZ_CHUNK, OZ_BJ, OZ_NARR, (cuuint32_t)kch, 1};
    if (encode(mapA, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, base, dims, strides, boxA, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (encode(mapB, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, base, dims, strides, boxB, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    // half of B (two of the four arrays) for the two-SM tiles
    const cuuint32_t boxB2[5] = {OZ_CHUNK, OZ_BJ, 2, (cuuint32_t)kch, 1};
    if (encode(mapB2, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, base, dims, strides, boxB2, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    return true;
}

// The B operand of the 128 x 64 residue tiles: the four arrays of 64 G rows,
// one 128-byte K chunk (the 5D view of make_oz_tensor_maps, box {128, 64, 4, 1, 1});
// and the half of it that one CTA of a 256 x 64 pair holds (box {128, 64, 2, 1, 1}).
bool make_oz_b64_map(void *base, size_t nss, int npad, int kp8, int narr, CUtensorMap *mapB64, CUtensorMap *mapB64h)
{
    typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
        return false;
    EncodeFn encode = (EncodeFn)fn;
    if (kp8 % OZ_CHUNK != 0 || npad % 64 != 0) return false;
    const cuuint64_t dims[5] = {(cuuint64_t)OZ_CHUNK, (cuuint64_t)npad, (cuuint64_t)narr, (cuuint64_t)(kp8 / OZ_CHUNK),
                                (cuuint64_t)nss};
    const cuuint64_t strides[4] = {(cuuint64_t)kp8, (cuuint64_t)npad * kp8, (cuuint64_t)OZ_CHUNK,
                                   (cuuint64_t)narr * npad * kp8};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const cuuint32_t box[5] = {OZ_CHUNK, 64, OZ_NARR, 1, 1};
    const cuuint32_t boxh[5] = {OZ_CHUNK, 64, 2, 1, 1};
    return encode(mapB64, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
           encode(mapB64h, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, base, dims, strides, boxh, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// TMA views for the per-atom products:
//   mapArow: the slices as [slot x slice][array][G][kp8 bytes] (4D), box
//     {128, 128, 2, 1}: Ar and Ai of 128 G rows, one 128-byte K chunk
//     starting at any multiple of 16 bytes (the atom windows are not chunk
//     aligned);
//   mapX: the X slices as [group][128 rows][lw bytes] viewed like the B tiles
//     (4D, K chunked), box {128, 128, 1, 1}.
bool make_oz_atom_maps(void *base, size_t nss, int npad, int kp8, int narr, void *xbase, size_t xgroups, int lw,
                       CUtensorMap *mapArow, CUtensorMap *mapX)
{
    typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
        return false;
    EncodeFn encode = (EncodeFn)fn;
    if (kp8 % OZ_CHUNK != 0 || lw % OZ_CHUNK != 0) return false;
    const cuuint32_t es[4] = {1, 1, 1, 1};
    {
        const cuuint64_t dims[4] = {(cuuint64_t)kp8, (cuuint64_t)npad, (cuuint64_t)narr, (cuuint64_t)nss};
        const cuuint64_t strides[3] = {(cuuint64_t)kp8, (cuuint64_t)npad * kp8, (cuuint64_t)narr * npad * kp8};
        const cuuint32_t box[4] = {OZ_CHUNK, OZ_BM, 2, 1};
        if (encode(mapArow, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, base, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    {
        const cuuint64_t dims[4] = {(cuuint64_t)OZ_CHUNK, 128, (cuuint64_t)xgroups, (cuuint64_t)(lw / OZ_CHUNK)};
        const cuuint64_t strides[3] = {(cuuint64_t)lw, (cuuint64_t)128 * lw, (cuuint64_t)OZ_CHUNK};
        const cuuint32_t box[4] = {OZ_CHUNK, 128, 1, 1};
        if (encode(mapX, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, xbase, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

}  // namespace exs

extern "C" int exs_ozaki_moduli(int n, int K, int kx, int *n_out, int *p, unsigned long long *c, int *b, int *bx,
                                int *h)
{
    exs::OzScheme s{};
    if (exs::oz_mod_plan(n, K, kx, &s) != 0) return EXS_ERR_ARG;
    if (n_out) *n_out = s.n;
    for (int m = 0; m < s.n; m++) {
        if (p) p[m] = s.p[m];
        if (c) c[m] = s.c[m];
    }
    if (b) *b = s.b;
    if (bx) *bx = s.bx;
    if (h) *h = s.h;
    return EXS_OK;
}
