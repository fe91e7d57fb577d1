// Split-precision (Ozaki scheme, int8 slices) MT contraction on the 5th-gen
// tensor cores (tcgen05.mma kind::i8, int32 accumulators in tensor memory).
//
// The APW-APW blocks H = A^H B and O = A^H A are written as one real product
// with the contraction index K' = 2K (real and imaginary rows stacked):
//   L  = [Ar; Ai]                      (left operand, shared)
//   R1 = [Br; Bi],  R2 = [Bi; -Br]      Re H = L^T R1,  Im H = L^T R2
//   R3 = [Ar; Ai],  R4 = [Ai; -Ar]      Re O = L^T R3,  Im O = L^T R4
// Every column G of A (and of B) is scaled by a power of two sigma(G) >
// max|column| and cut into S int8 slices of 7 bits each by truncation,
//   x = sigma * sum_s q_s 2^{-7s} + r,  |q_s| <= 127,  |r| < sigma 2^{-7S}
// (exact in FP64).  The product keeps the slice pairs s + t <= S + 1; pairs
// of one diagonal d = s + t share one int32 accumulator (exact: at most S
// products of K' <= 2^17 terms of |q q'| <= 127^2 stay below 2^31), and each
// finished diagonal is added in FP64 as 2^{-7d} times the int32 sum into an
// FP64 accumulator that also lives in tensor memory.  The final epilogue
// multiplies by sigma_A(i) sigma_B(j), adds the interstitial term and writes
// the upper triangle and its conjugate mirror, as the FP64 path does.
//
// Tile: 128 rows (G_i) x 32 columns (G_j) x 4 outputs (Re H, Im H, Re O,
// Im O) = one M=128, N=128 MMA shape; K staged 128 bytes at a time through a
// 4-deep cp.async pipeline in the canonical no-swizzle K-major layout
// (8-row x 16-byte core matrices).  Tensor memory: int32 accumulator in
// columns [0,128), FP64 accumulator (two 32-bit columns per value) in
// [128,384) of a 512-column allocation.  Every wait on an mbarrier is bounded
// (about one second); on expiry the kernel records an error, drains its own
// copies, frees tensor memory and returns.
#include <cuda.h>

#include <cstdint>

#include "exs_internal.cuh"
#include "interstitial.cuh"

namespace exs {

constexpr int OZ_BM = 128;                       // tile rows (G_i)
constexpr int OZ_BJ = 32;                        // tile columns (G_j); MMA N = 4 * OZ_BJ
constexpr int OZ_N = 4 * OZ_BJ;
constexpr int OZ_BK = 128;                       // bytes of K per pipeline stage (4 MMAs of K = 32)
constexpr int OZ_STAGES = 4;
constexpr int OZ_PREFETCH = 2;                  // loads run two iterations ahead of the MMAs
constexpr int OZ_TILE = 128 * OZ_BK;             // 16 KB per operand tile
constexpr int OZ_STAGE = 2 * OZ_TILE;            // A + B
constexpr int OZ_SMEM = OZ_STAGES * OZ_STAGE + 1024;
constexpr int OZ_TMEM_COLS = 512;
constexpr int OZ_NARR = 6;                       // Ar, Ai, Br, Bi, -Br, -Ar
constexpr long long OZ_WAIT_CYCLES = 2000000000LL;   // ~1 s at 2 GHz

// ------------------------------------------------------------ device helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void oz_cp16(uint32_t dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait for the phase with the given parity; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > OZ_WAIT_CYCLES) return false;
    }
}

// K-major, no-swizzle shared-memory matrix descriptor: core matrices of
// 8 rows x 16 bytes; lbo = byte step between the two 16-byte K chunks of one
// MMA, sbo = byte step between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                  // descriptor version of sm_100
    return d;                                // base offset 0, layout type 0 (no swizzle)
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
// Column scales sigma(G) = 2^e with max|column| < 2^e (frexp), for A (Ar, Ai)
// and for B (Br, Bi).  One thread per (G, k-point).
__global__ void oz_colscale_kernel(DevParams p, const KDesc *ks)
{
    const KDesc k = ks[blockIdx.y];
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= p.npad) return;
    double ma = 0.0, mb = 0.0;
    if (g < k.ngp)
        for (int f = 0; f < p.K; f++) {
            const size_t i = (size_t)f * p.npad + g;
            ma = fmax(ma, fmax(fabs(k.ar[i]), fabs(k.ai[i])));
            mb = fmax(mb, fmax(fabs(k.br[i]), fabs(k.bi[i])));
        }
    int ea = 0, eb = 0;
    if (ma > 0.0) frexp(ma, &ea);
    if (mb > 0.0) frexp(mb, &eb);
    k.oz_scale[g] = ldexp(1.0, ea);
    k.oz_scale[p.npad + g] = ldexp(1.0, eb);
}

// Slices of the six operand arrays, K-major int8 [arr][s][G][f], f padded to
// kp8 with zeros.  A 32(f) x 32(G) tile per block, transposed through shared
// memory.
__global__ void oz_split_kernel(DevParams p, const KDesc *ks, int S, int kp8)
{
    __shared__ double t[4][32][33];
    const KDesc k = ks[blockIdx.z];
    const int f0 = blockIdx.x * 32, g0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;      // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int f = f0 + r, g = g0 + tx;
        const bool v = f < p.K && g < k.ngp;
        const size_t i = (size_t)f * p.npad + g;
        t[0][r][tx] = v ? k.ar[i] : 0.0;
        t[1][r][tx] = v ? k.ai[i] : 0.0;
        t[2][r][tx] = v ? k.br[i] : 0.0;
        t[3][r][tx] = v ? k.bi[i] : 0.0;
    }
    __syncthreads();
    // thread (tx = f within tile, ty..): one G per pass
    for (int r = ty; r < 32; r += 8) {
        const int g = g0 + r, f = f0 + tx;
        if (g >= p.npad || f >= kp8) continue;
        const double sa = k.oz_scale[g], sb = k.oz_scale[p.npad + g];
        double x[4] = {t[0][tx][r] / sa, t[1][tx][r] / sa, t[2][tx][r] / sb, t[3][tx][r] / sb};
        for (int s = 0; s < S; s++) {
            int8_t q[4];
            for (int a = 0; a < 4; a++) {
                x[a] *= 128.0;
                const double tq = trunc(x[a]);
                x[a] -= tq;
                q[a] = (int8_t)tq;
            }
            // arrays: 0 Ar, 1 Ai, 2 Br, 3 Bi, 4 -Br, 5 -Ar
            const int8_t vals[OZ_NARR] = {q[0], q[1], q[2], q[3], (int8_t)(-q[2]), (int8_t)(-q[0])};
            for (int a = 0; a < OZ_NARR; a++)
                k.oz_slices[(((size_t)a * S + s) * p.npad + g) * kp8 + f] = vals[a];
        }
    }
}

// ------------------------------------------------------------ main kernel
struct OzTile {
    int k, ib, jb;
};

// Source array of sub-block q of the B tile, K half h (see the header).
__device__ __forceinline__ int oz_barr(int q, int h)
{
    const int t0[4] = {2, 3, 0, 1}, t1[4] = {3, 4, 1, 5};
    return h == 0 ? t0[q] : t1[q];
}

__global__ void __launch_bounds__(128, 1)
oz_mma_kernel(DevParams p, const KDesc *ks, const OzTile *tiles, int S, int kp8)
{
    extern __shared__ __align__(1024) uint8_t oz_smem[];
    __shared__ uint64_t bars[OZ_STAGES];
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;
    __shared__ int jiv[OZ_BJ][3];
    __shared__ double jv[OZ_BJ][3];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const OzTile tl = tiles[blockIdx.x];
    const KDesc kd = ks[tl.k];
    const int i0 = tl.ib * OZ_BM, j0 = tl.jb * OZ_BJ;
    // stage buffers at a 1024-byte aligned offset
    const uint32_t sbase = (smem_u32(oz_smem) + 1023u) & ~1023u;
    uint8_t *sgen = oz_smem + (sbase - smem_u32(oz_smem));

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < OZ_STAGES; s++) mbar_init(&bars[s], 1);
        fail_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tmem_base_sh;
    const uint32_t t_lane = tbase + ((uint32_t)(warp * 32) << 16);   // this warp's 32 lanes
    const uint32_t idesc = umma_idesc_i8(128, OZ_N);
    const int nkb_half = kp8 / OZ_BK;
    const int nkb = 2 * nkb_half;                    // k-blocks per slice pair (both K halves)
    const size_t arr_stride = (size_t)S * p.npad * kp8;
    const size_t slice_stride = (size_t)p.npad * kp8;
    uint32_t uses[OZ_STAGES] = {0, 0, 0, 0};          // completed-commit count per stage
    long git = 0;                                     // global pipeline iteration
    bool failed = false;

    // Load the A and B tiles of flat iteration `it` of diagonal d into stage st.
    auto load_stage = [&](int d, int s_lo, int it, int st) {
        const int pair = it / nkb, kb = it % nkb;
        const int s = s_lo + pair, t = d - s;        // 1-based slice indices
        const int h = kb / nkb_half, kk = (kb % nkb_half) * OZ_BK;
        const uint32_t sa = sbase + st * OZ_STAGE, sb = sa + OZ_TILE;
        const int8_t *abase = kd.oz_slices + (size_t)h * arr_stride + (size_t)(s - 1) * slice_stride;
#pragma unroll
        for (int it2 = 0; it2 < 8; it2++) {
            const int qd = tid + 128 * it2;          // chunk 0..1023
            const int r8 = qd & 7, c = (qd >> 3) & 7, grp = qd >> 6;
            const int row = grp * 8 + r8;            // 0..127
            const uint32_t soff = grp * 1024 + c * 128 + r8 * 16;
            // A: row -> G_i = i0 + row (rows past npad read row npad-1: in bounds, results discarded)
            const int gi = min(i0 + row, p.npad - 1);
            oz_cp16(sa + soff, abase + (size_t)gi * kp8 + kk + c * 16);
            // B: row -> sub-block q = row / 32, G_j = j0 + row % 32
            const int q = row >> 5;
            const int gj = min(j0 + (row & 31), p.npad - 1);
            const int8_t *bb = kd.oz_slices + (size_t)oz_barr(q, h) * arr_stride + (size_t)(t - 1) * slice_stride;
            oz_cp16(sb + soff, bb + (size_t)gj * kp8 + kk + c * 16);
        }
    };

    for (int d = 2; d <= S + 1 && !failed; d++) {
        const int s_lo = max(1, d - S), s_hi = min(S, d - 1);
        const int total = (s_hi - s_lo + 1) * nkb;
        // prologue: the first OZ_PREFETCH iterations
        for (int it = 0; it < OZ_PREFETCH; it++) {
            if (it < total) {
                const int st = (int)((git + it) % OZ_STAGES);
                if (uses[st] > 0 && !mbar_wait(&bars[st], (uses[st] - 1) & 1)) failed = true;
                load_stage(d, s_lo, it, st);
            }
            asm volatile("cp.async.commit_group;\n" ::);
        }
        for (int it = 0; it < total; it++) {
            const int st = (int)((git + it) % OZ_STAGES);
            asm volatile("cp.async.wait_group %0;\n" ::"n"(OZ_PREFETCH - 1));   // iteration it has landed
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            if (__syncthreads_or(failed)) { failed = true; break; }
            if (tid == 0) {
                tc_fence_after();
                const uint32_t sa = sbase + st * OZ_STAGE, sb = sa + OZ_TILE;
#pragma unroll
                for (int q = 0; q < OZ_BK / 32; q++) {
                    const uint64_t ad = umma_desc(sa + q * 256, 128, 1024);
                    const uint64_t bd = umma_desc(sb + q * 256, 128, 1024);
                    umma_i8(tbase, ad, bd, idesc, (it == 0 && q == 0) ? 0u : 1u);
                }
                umma_commit(&bars[st]);
            }
            uses[st]++;
            // prefetch iteration it + OZ_PREFETCH into the stage the MMAs of
            // iteration it + OZ_PREFETCH - OZ_STAGES read (two batches ago)
            const int nt = it + OZ_PREFETCH;
            if (nt < total) {
                const int sn = (int)((git + nt) % OZ_STAGES);
                if (uses[sn] > 0 && !mbar_wait(&bars[sn], (uses[sn] - 1) & 1)) failed = true;
                load_stage(d, s_lo, nt, sn);
            }
            asm volatile("cp.async.commit_group;\n" ::);
        }
        git += total;
        // all MMAs of this diagonal done: the last commit completes after every earlier one
        if (!failed) {
            const int stl = (int)((git - 1) % OZ_STAGES);
            if (!mbar_wait(&bars[stl], (uses[stl] - 1) & 1)) failed = true;
        }
        if (__syncthreads_or(failed)) { failed = true; break; }
        tc_fence_after();
        // fold the int32 diagonal sum into the FP64 accumulator: acc += 2^{-7d} C_d
        const double scale = ldexp(1.0, -7 * d);
#pragma unroll 1
        for (int c = 0; c < OZ_N / 16; c++) {
            uint32_t iv[16], lo[16], hi[16];
            tm_ld16(t_lane + c * 16, iv);
            if (d > 2) {
                tm_ld16(t_lane + 128 + c * 32, lo);
                tm_ld16(t_lane + 128 + c * 32 + 16, hi);
            }
            tm_wait_ld();
            uint32_t o0[16], o1[16];
#pragma unroll
            for (int e = 0; e < 16; e++) {
                double a = 0.0;
                if (d > 2) {
                    const uint32_t w0 = e < 8 ? lo[2 * e] : hi[2 * (e - 8)];
                    const uint32_t w1 = e < 8 ? lo[2 * e + 1] : hi[2 * (e - 8) + 1];
                    a = __hiloint2double((int)w1, (int)w0);
                }
                a += scale * (double)(int)iv[e];
                const uint32_t w0 = (uint32_t)__double2loint(a), w1 = (uint32_t)__double2hiint(a);
                if (e < 8) { o0[2 * e] = w0; o0[2 * e + 1] = w1; }
                else { o1[2 * (e - 8)] = w0; o1[2 * (e - 8) + 1] = w1; }
            }
            tm_st16(t_lane + 128 + c * 32, o0);
            tm_st16(t_lane + 128 + c * 32 + 16, o1);
        }
        tm_wait_st();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }

    if (!failed) {
        // ---------------- final epilogue: scale, interstitial, store H and O
        if (tid < OZ_BJ) {
            const int j = j0 + tid;
            if (j < kd.ngp) {
                int g = kd.igpig[j] - 1;
                if (g < 0 || g >= p.ngrtot) { atomicOr(p.err, DEV_ERR_INDEX); g = 0; }
                for (int x = 0; x < 3; x++) {
                    jiv[tid][x] = p.ivg[3 * g + x];
                    jv[tid][x] = kd.vgpc[3 * j + x];
                }
            }
        }
        __syncthreads();
        const int i = i0 + warp * 32 + lane;            // this thread's row
        int ivi[3] = {0, 0, 0};
        double vi[3] = {0.0, 0.0, 0.0};
        const bool row_ok = i < kd.ngp;
        if (row_ok) {
            int g = kd.igpig[i] - 1;
            if (g < 0 || g >= p.ngrtot) { atomicOr(p.err, DEV_ERR_INDEX); g = 0; }
            for (int x = 0; x < 3; x++) {
                ivi[x] = p.ivg[3 * g + x];
                vi[x] = kd.vgpc[3 * i + x];
            }
        }
        const double sai = row_ok ? kd.oz_scale[i] : 0.0;
        // FP64 accumulator columns: value v at TMEM columns 128 + 2v, 129 + 2v;
        // v = q * 32 + jj for output q (Re H, Im H, Re O, Im O) and column jj.
#pragma unroll 1
        for (int jc = 0; jc < OZ_BJ; jc += 8) {
            double val[4][8];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint32_t w[16];
                tm_ld16(t_lane + 128 + 2 * (q * 32 + jc), w);
                tm_wait_ld();
#pragma unroll
                for (int e = 0; e < 8; e++) val[q][e] = __hiloint2double((int)w[2 * e + 1], (int)w[2 * e]);
            }
            if (!row_ok) continue;
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int jj = jc + e, j = j0 + jj;
                if (j >= kd.ngp || i > j) continue;
                const double sbj = kd.oz_scale[p.npad + j], saj = kd.oz_scale[j];
                double hr = val[0][e] * sai * sbj, hi = val[1][e] * sai * sbj;
                double orr = val[2][e] * sai * saj, oi = val[3][e] * sai * saj;
                double ar, ai;
                if (interstitial(p, EPI_HAM, ivi, jiv[jj], vi, jv[jj], ar, ai)) { hr += ar; hi += ai; }
                if (interstitial(p, EPI_OVL, ivi, jiv[jj], vi, jv[jj], ar, ai)) { orr += ar; oi += ai; }
                exs_complex h, o;
                h.re = hr; h.im = hi;
                o.re = orr; o.im = oi;
                kd.h[(size_t)i + (size_t)kd.nmat * j] = h;
                kd.o[(size_t)i + (size_t)kd.nmat * j] = o;
                if (i < j) {
                    h.im = -hi;
                    o.im = -oi;
                    kd.h[(size_t)j + (size_t)kd.nmat * i] = h;
                    kd.o[(size_t)j + (size_t)kd.nmat * i] = o;
                }
            }
        }
    } else if (tid == 0) {
        atomicOr(p.err, DEV_ERR_TIMEOUT);
    }
    // teardown: drain own copies, make sure no MMA is still reading, free TMEM
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (failed && tid == 0) {
        for (int st = 0; st < OZ_STAGES; st++)
            if (uses[st] > 0) (void)mbar_wait(&bars[st], (uses[st] - 1) & 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(OZ_TMEM_COLS));
    }
}

// ------------------------------------------------------------ launchers
cudaError_t launch_oz_prepare(const DevParams &p, const KDesc *d_k, int nk, int S, int kp8, cudaStream_t s)
{
    oz_colscale_kernel<<<dim3((p.npad + 127) / 128, nk), 128, 0, s>>>(p, d_k);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    oz_split_kernel<<<dim3(kp8 / 32, p.npad / 32, nk), dim3(32, 8), 0, s>>>(p, d_k, S, kp8);
    return cudaGetLastError();
}

cudaError_t launch_oz_mma(const DevParams &p, const KDesc *d_k, const void *d_tiles, int ntiles, int S, int kp8,
                          cudaStream_t s)
{
    if (ntiles <= 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(oz_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    oz_mma_kernel<<<ntiles, 128, OZ_SMEM, s>>>(p, d_k, (const OzTile *)d_tiles, S, kp8);
    return cudaGetLastError();
}

}  // namespace exs

namespace exs {

// ============================================================================
// Warp-specialised variant: TMA-fed 6-stage pipeline, one producer warp, one
// MMA warp, four epilogue warps, and two int32 accumulators in tensor memory
// so that the FP64 fold of diagonal d overlaps the MMAs of diagonal d+1.
//
// Operand tiles are loaded by TMA with 128-byte swizzling from the same int8
// slice array (viewed as a 2D tensor [rows][kp8 bytes]); the MMA descriptors
// use the matching SWIZZLE_128B K-major layout (8-row x 128-byte atoms,
// 1024-byte stride between 8-row groups, K advanced 32 bytes per MMA).
// Tensor memory (512 columns): int32 accumulators at [0,128) and [128,256),
// FP64 accumulator (two 32-bit words per value) at [256,512).
// ============================================================================
constexpr int WS_STAGES = 6;
constexpr int WS_THREADS = 192;
constexpr int WS_SMEM = WS_STAGES * OZ_STAGE + 1024;
constexpr int WS_FP64_COL = 256;

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            dst),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait that also gives up as soon as another role raised `abort`.
__device__ __forceinline__ bool mbar_wait_ab(uint64_t *bar, uint32_t parity, volatile int *abort)
{
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*abort) return false;
        if (clock64() - t0 > OZ_WAIT_CYCLES) {
            *abort = 1;
            return false;
        }
    }
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

__global__ void __launch_bounds__(WS_THREADS, 1)
oz_mma_ws_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, DevParams p,
                 const KDesc *ks, const OzTile *tiles, int S, int kp8)
{
    extern __shared__ __align__(1024) uint8_t ws_smem[];
    __shared__ uint64_t full[WS_STAGES], empty[WS_STAGES], accf[2], acce[2];
    __shared__ uint32_t tmem_sh;
    __shared__ int abort_sh;
    __shared__ int jiv[OZ_BJ][3];
    __shared__ double jv[OZ_BJ][3];
    volatile int *abort = &abort_sh;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const OzTile tl = tiles[blockIdx.x];
    const KDesc kd = ks[tl.k];
    const int i0 = tl.ib * OZ_BM, j0 = tl.jb * OZ_BJ;
    const uint32_t sbase = (smem_u32(ws_smem) + 1023u) & ~1023u;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_sh)),
                     "r"(OZ_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < WS_STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int b = 0; b < 2; b++) { mbar_init(&accf[b], 1); mbar_init(&acce[b], 4); }
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (tid >= 64 && tid < 64 + OZ_BJ) {        // column data of the final epilogue
        const int c = tid - 64, j = j0 + c;
        if (j < kd.ngp) {
            int g = kd.igpig[j] - 1;
            if (g < 0 || g >= p.ngrtot) { atomicOr(p.err, DEV_ERR_INDEX); g = 0; }
            for (int x = 0; x < 3; x++) { jiv[c][x] = p.ivg[3 * g + x]; jv[c][x] = kd.vgpc[3 * j + x]; }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tmem_sh;
    const int nkb_half = kp8 / OZ_BK, nkb = 2 * nkb_half;
    const int npad = p.npad;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t fills[WS_STAGES] = {0, 0, 0, 0, 0, 0};
            long it = 0;
            bool bad = false;
            for (int d = 2; d <= S + 1 && !bad; d++) {
                const int s_lo = max(1, d - S), s_hi = min(S, d - 1);
                for (int s = s_lo; s <= s_hi && !bad; s++) {
                    const int t = d - s;
                    for (int kb = 0; kb < nkb; kb++, it++) {
                        const int st = (int)(it % WS_STAGES);
                        if (fills[st] > 0 && !mbar_wait_ab(&empty[st], (fills[st] - 1) & 1, abort)) { bad = true; break; }
                        mbar_expect_tx(&full[st], OZ_STAGE);
                        const int h = kb / nkb_half, kk = (kb % nkb_half) * OZ_BK;
                        const uint32_t sa = sbase + st * OZ_STAGE;
                        tma_load_2d(sa, &mapA, kk, kd.oz_row0 + (h * S + (s - 1)) * npad + i0, &full[st]);
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            tma_load_2d(sa + OZ_TILE + q * 4096, &mapB, kk,
                                        kd.oz_row0 + (oz_barr(q, h) * S + (t - 1)) * npad + j0, &full[st]);
                        fills[st]++;
                    }
                }
            }
            if (bad)   // let the copies already issued land before the CTA goes away
                for (int st = 0; st < WS_STAGES; st++)
                    if (fills[st] > 0) (void)mbar_wait(&full[st], (fills[st] - 1) & 1);
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_i8(128, OZ_N);
            uint32_t uses[WS_STAGES] = {0, 0, 0, 0, 0, 0};
            int accuse[2] = {0, 0};
            long it = 0;
            bool bad = false;
            for (int d = 2; d <= S + 1 && !bad; d++) {
                const int b = (d - 2) & 1;
                if (accuse[b] > 0 && !mbar_wait_ab(&acce[b], (accuse[b] - 1) & 1, abort)) { bad = true; break; }
                tc_fence_after();
                const uint32_t dtm = tbase + b * 128;
                const int s_lo = max(1, d - S), s_hi = min(S, d - 1);
                bool first = true;
                for (int s = s_lo; s <= s_hi && !bad; s++)
                    for (int kb = 0; kb < nkb; kb++, it++) {
                        const int st = (int)(it % WS_STAGES);
                        if (!mbar_wait_ab(&full[st], uses[st] & 1, abort)) { bad = true; break; }
                        tc_fence_after();
                        const uint32_t sa = sbase + st * OZ_STAGE, sb = sa + OZ_TILE;
#pragma unroll
                        for (int q = 0; q < OZ_BK / 32; q++) {
                            umma_i8(dtm, umma_desc_sw128(sa + q * 32), umma_desc_sw128(sb + q * 32), idesc,
                                    (first && q == 0) ? 0u : 1u);
                        }
                        first = false;
                        umma_commit(&empty[st]);
                        uses[st]++;
                    }
                if (!bad) {
                    umma_commit(&accf[b]);
                    accuse[b]++;
                }
            }
            if (bad)   // MMAs already issued must finish before tensor memory is freed
                for (int st = 0; st < WS_STAGES; st++)
                    if (uses[st] > 0) (void)mbar_wait(&empty[st], (uses[st] - 1) & 1);
        }
    } else {
        // ------------------------------------------------ epilogue (warps 2..5)
        const int qd = warp & 3;                                   // tensor-memory lane quadrant
        const uint32_t t_lane = tbase + ((uint32_t)(qd * 32) << 16);
        int accn[2] = {0, 0};
        bool bad = false;
        for (int d = 2; d <= S + 1; d++) {
            const int b = (d - 2) & 1;
            // warp-uniform outcome: the tcgen05.ld/st below need the whole warp
            const bool ok = __all_sync(0xffffffffu, mbar_wait_ab(&accf[b], accn[b] & 1, abort));
            if (!ok) { bad = true; break; }
            accn[b]++;
            tc_fence_after();
            const double scale = ldexp(1.0, -7 * d);
#pragma unroll 1
            for (int c = 0; c < OZ_N / 16; c++) {
                uint32_t iv[16], lo[16], hi[16];
                tm_ld16(t_lane + b * 128 + c * 16, iv);
                if (d > 2) {
                    tm_ld16(t_lane + WS_FP64_COL + c * 32, lo);
                    tm_ld16(t_lane + WS_FP64_COL + c * 32 + 16, hi);
                }
                tm_wait_ld();
                uint32_t o0[16], o1[16];
#pragma unroll
                for (int e = 0; e < 16; e++) {
                    double a = 0.0;
                    if (d > 2) {
                        const uint32_t w0 = e < 8 ? lo[2 * e] : hi[2 * (e - 8)];
                        const uint32_t w1 = e < 8 ? lo[2 * e + 1] : hi[2 * (e - 8) + 1];
                        a = __hiloint2double((int)w1, (int)w0);
                    }
                    a += scale * (double)(int)iv[e];
                    const uint32_t w0 = (uint32_t)__double2loint(a), w1 = (uint32_t)__double2hiint(a);
                    if (e < 8) { o0[2 * e] = w0; o0[2 * e + 1] = w1; }
                    else { o1[2 * (e - 8)] = w0; o1[2 * (e - 8) + 1] = w1; }
                }
                tm_st16(t_lane + WS_FP64_COL + c * 32, o0);
                tm_st16(t_lane + WS_FP64_COL + c * 32 + 16, o1);
            }
            tm_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[b]);
        }
        if (__all_sync(0xffffffffu, !bad && !*abort)) {
            const int i = i0 + qd * 32 + lane;
            int ivi[3] = {0, 0, 0};
            double vi[3] = {0.0, 0.0, 0.0};
            const bool row_ok = i < kd.ngp;
            if (row_ok) {
                int g = kd.igpig[i] - 1;
                if (g < 0 || g >= p.ngrtot) { atomicOr(p.err, DEV_ERR_INDEX); g = 0; }
                for (int x = 0; x < 3; x++) { ivi[x] = p.ivg[3 * g + x]; vi[x] = kd.vgpc[3 * i + x]; }
            }
            const double sai = row_ok ? kd.oz_scale[i] : 0.0;
#pragma unroll 1
            for (int jc = 0; jc < OZ_BJ; jc += 8) {
                double val[4][8];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    uint32_t w[16];
                    tm_ld16(t_lane + WS_FP64_COL + 2 * (q * 32 + jc), w);
                    tm_wait_ld();
#pragma unroll
                    for (int e = 0; e < 8; e++) val[q][e] = __hiloint2double((int)w[2 * e + 1], (int)w[2 * e]);
                }
                if (!row_ok) continue;
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int jj = jc + e, j = j0 + jj;
                    if (j >= kd.ngp || i > j) continue;
                    const double sbj = kd.oz_scale[npad + j], saj = kd.oz_scale[j];
                    double hr = val[0][e] * sai * sbj, hi = val[1][e] * sai * sbj;
                    double orr = val[2][e] * sai * saj, oi = val[3][e] * sai * saj;
                    double ar, ai;
                    if (interstitial(p, EPI_HAM, ivi, jiv[jj], vi, jv[jj], ar, ai)) { hr += ar; hi += ai; }
                    if (interstitial(p, EPI_OVL, ivi, jiv[jj], vi, jv[jj], ar, ai)) { orr += ar; oi += ai; }
                    exs_complex hv, ov;
                    hv.re = hr; hv.im = hi;
                    ov.re = orr; ov.im = oi;
                    kd.h[(size_t)i + (size_t)kd.nmat * j] = hv;
                    kd.o[(size_t)i + (size_t)kd.nmat * j] = ov;
                    if (i < j) {
                        hv.im = -hi;
                        ov.im = -oi;
                        kd.h[(size_t)j + (size_t)kd.nmat * i] = hv;
                        kd.o[(size_t)j + (size_t)kd.nmat * i] = ov;
                    }
                }
            }
        }
    }
    if (tid == 0 && *abort) atomicOr(p.err, DEV_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(OZ_TMEM_COLS));
    }
}

cudaError_t launch_oz_mma_ws(const CUtensorMap *mapA, const CUtensorMap *mapB, const DevParams &p, const KDesc *d_k,
                             const void *d_tiles, int ntiles, int S, int kp8, cudaStream_t s)
{
    if (ntiles <= 0) return cudaSuccess;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(oz_mma_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, WS_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    oz_mma_ws_kernel<<<ntiles, WS_THREADS, WS_SMEM, s>>>(*mapA, *mapB, p, d_k, (const OzTile *)d_tiles, S, kp8);
    return cudaGetLastError();
}

// Tensor maps over the int8 slices of all slots: [rows][kp8] bytes, boxes of
// 128 x 128 (A tile) and 32 x 128 (one B sub-block), 128-byte swizzle.
bool make_oz_tensor_maps(void *base, size_t rows, int kp8, CUtensorMap *mapA, CUtensorMap *mapB)
{
    typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeFn encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return false;
        encode = (EncodeFn)fn;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)kp8, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kp8};
    const cuuint32_t es[2] = {1, 1};
    const cuuint32_t boxA[2] = {128, 128}, boxB[2] = {128, 32};
    if (encode(mapA, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, boxA, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
        return false;
    if (encode(mapB, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, boxB, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
        return false;
    return true;
}

}  // namespace exs
