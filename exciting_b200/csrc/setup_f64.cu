// Native-FP64 path of the H/O setup: grouped complex contractions on the
// FP64 tensor instruction (DMMA m8n8k4), with the epilogues that place the
// results into the reference's za(nmat, nmat) layout.
//
// Stages of one k-point (the reference's per-atom loop of
// src/src_eigensystem/hamiltonsetup.f90:53-168 and overlapsetup.f90:47-154,
// regrouped so that all atoms and k-points of a call share one launch):
//   1. B_a = h_a A_a per atom              (hamiltonsetup.f90:75-88)
//   2. H = A^H B, O = A^H A (or A^H C, iora*), K = all atoms' APW rows at
//      once; upper tiles only; the epilogue adds the interstitial term
//      (hmlistln.f90 / olpistln.f90) and writes the conjugate mirror
//      (hamiltonoverlapocopy_UL.f90)
//   3. APW-lo rows of H (hamiltonsetup.f90:131-149) as a grouped GEMM,
//      APW-lo of O (overlapsetup.f90:111-127) and the lo-lo blocks
//      (hamiltonsetup.f90:154-161, overlapsetup.f90:131-146) elementwise.
//
// Operand layout: real and imaginary parts in separate planes; an operand
// X of an M x K product is stored [k][m] (m contiguous), i.e. X^T, which is
// how both the matching coefficients (G contiguous) and the Fortran MT
// integrals (first index contiguous) already lie in memory.
#include <algorithm>

#include "exs_internal.cuh"
#include "interstitial.cuh"

namespace exs {

constexpr int GB_M = 64, GB_N = 64, GB_K = 16, GB_LDS = GB_M + 8, GB_STAGES = 3, GB_THREADS = 128;
constexpr int GB_PLANE = GB_K * GB_LDS;                 // doubles per plane per stage
constexpr int GB_STAGE = 4 * GB_PLANE;                  // xr, xi, yr, yi
constexpr size_t GB_SMEM = (size_t)GB_STAGES * GB_STAGE * sizeof(double);

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Load one K-slab (GB_K rows) of the four operand planes into stage buffer s.
__device__ __forceinline__ void load_stage(double *st, const GemmProb &P, int m0, int n0, int k0)
{
    const int tid = threadIdx.x;
#pragma unroll
    for (int it = 0; it < (GB_K * GB_M / 2) / GB_THREADS; it++) {
        const int c = tid + it * GB_THREADS;
        const int row = c / (GB_M / 2);
        const int col = (c % (GB_M / 2)) * 2;
        const int gk = k0 + row;
        {
            const int gm = m0 + col;
            const bool v = gk < P.K && gm < P.M;
            const size_t off = v ? (size_t)gk * P.ldx + gm : 0;
            cp_async16(st + 0 * GB_PLANE + row * GB_LDS + col, P.xr + off, v);
            cp_async16(st + 1 * GB_PLANE + row * GB_LDS + col, P.xi + off, v);
        }
        {
            const int gn = n0 + col;
            const bool v = gk < P.K && gn < P.N;
            const size_t off = v ? (size_t)gk * P.ldy + gn : 0;
            cp_async16(st + 2 * GB_PLANE + row * GB_LDS + col, P.yr + off, v);
            cp_async16(st + 3 * GB_PLANE + row * GB_LDS + col, P.yi + off, v);
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(GB_THREADS, 2)
zgemm_dmma_kernel(DevParams p, const GemmProb *probs, const TileWork *work, const KDesc *ks)
{
    extern __shared__ __align__(16) double smem[];
    const TileWork tw = work[blockIdx.x];
    const GemmProb P = probs[tw.prob];
    const int m0 = tw.tm * GB_M, n0 = tw.tn * GB_N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp >> 1, wn = warp & 1;

    double cre[4][4][2], cim[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) { cre[i][j][0] = cre[i][j][1] = cim[i][j][0] = cim[i][j][1] = 0.0; }

    const int nkt = (P.K + GB_K - 1) / GB_K;
#pragma unroll
    for (int s = 0; s < GB_STAGES - 1; s++) {
        if (s < nkt) load_stage(smem + s * GB_STAGE, P, m0, n0, s * GB_K);
        cp_async_commit();
    }
    const double sgn = P.conjx ? 1.0 : -1.0;
    for (int kt = 0; kt < nkt; kt++) {
        cp_async_wait<GB_STAGES - 2>();
        __syncthreads();
        {
            const int nt = kt + GB_STAGES - 1;
            if (nt < nkt) load_stage(smem + (nt % GB_STAGES) * GB_STAGE, P, m0, n0, nt * GB_K);
            cp_async_commit();
        }
        const double *st = smem + (kt % GB_STAGES) * GB_STAGE;
#pragma unroll
        for (int kk = 0; kk < GB_K / 4; kk++) {
            const int kr = kk * 4 + (lane & 3);
            double ar[4], aim[4], naim[4], br[4], bi[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int mm = wm * 32 + i * 8 + (lane >> 2);
                ar[i] = st[0 * GB_PLANE + kr * GB_LDS + mm];
                aim[i] = sgn * st[1 * GB_PLANE + kr * GB_LDS + mm];   // conj: +ai, plain: -ai
                naim[i] = -aim[i];
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int nn = wn * 32 + j * 8 + (lane >> 2);
                br[j] = st[2 * GB_PLANE + kr * GB_LDS + nn];
                bi[j] = st[3 * GB_PLANE + kr * GB_LDS + nn];
            }
            // four passes over the 4x4 sub-tiles so that the two products
            // accumulated into one register pair are 16 DMMAs apart
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(cre[i][j][0], cre[i][j][1], ar[i], br[j]);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(cim[i][j][0], cim[i][j][1], ar[i], bi[j]);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(cre[i][j][0], cre[i][j][1], aim[i], bi[j]);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(cim[i][j][0], cim[i][j][1], naim[i], br[j]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();

    if (KIND == EPI_PLANAR) {
        // split-precision path: column maxima of |B| (rows m of this tile),
        // reduced over the 8 row groups of a warp, then one atomic per column
        double *bmax = P.colmax;
        if (bmax) {
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    double mx = 0.0;
#pragma unroll
                    for (int i = 0; i < 4; i++) mx = fmax(mx, fmax(fabs(cre[i][j][h]), fabs(cim[i][j][h])));
                    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
                    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
                    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
                    const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + h;
                    if (lane < 4 && n < P.N) atomic_max_nonneg(bmax + n, mx);
                }
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int m = m0 + wm * 32 + i * 8 + (lane >> 2);
                const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3);
                if (m >= P.M) continue;
                if (n + 1 < P.N) {
                    *reinterpret_cast<double2 *>(P.outr + (size_t)m * P.ldo + n) = make_double2(cre[i][j][0], cre[i][j][1]);
                    *reinterpret_cast<double2 *>(P.outi + (size_t)m * P.ldo + n) = make_double2(cim[i][j][0], cim[i][j][1]);
                } else if (n < P.N) {
                    P.outr[(size_t)m * P.ldo + n] = cre[i][j][0];
                    P.outi[(size_t)m * P.ldo + n] = cim[i][j][0];
                }
            }
        return;
    }
    if (KIND == EPI_LOROWS) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int r = m0 + wm * 32 + i * 8 + (lane >> 2);
                    const int g = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + h;
                    if (r >= P.M || g >= P.N) continue;
                    exs_complex v; v.re = cre[i][j][h]; v.im = cim[i][j][h];
                    exs_complex vc; vc.re = v.re; vc.im = -v.im;
                    P.z[(size_t)(P.row0 + r) + (size_t)P.ldz * g] = v;
                    P.z[(size_t)g + (size_t)P.ldz * (P.row0 + r)] = vc;
                }
        return;
    }
    // EPI_HAM / EPI_OVL: APW-APW block, upper tiles, interstitial + mirror.
    int *s_iv = reinterpret_cast<int *>(smem);                 // [128][3]
    double *s_v = smem + 2 * 128;                              // [128][3] (after 1536 bytes)
    const KDesc kd = ks[P.kidx];
    {
        const int t = threadIdx.x;                             // 0..63 rows, 64..127 cols
        const int idx = (t < 64) ? (m0 + t) : (n0 + t - 64);
        if (idx < kd.ngp) {
            int g = kd.igpig[idx] - 1;
            if (g < 0 || g >= p.ngrtot) {      // caller's index table out of range
                atomicOr(p.err, DEV_ERR_INDEX);
                g = 0;
            }
            s_iv[3 * t + 0] = p.ivg[3 * g + 0];
            s_iv[3 * t + 1] = p.ivg[3 * g + 1];
            s_iv[3 * t + 2] = p.ivg[3 * g + 2];
            s_v[3 * t + 0] = kd.vgpc[3 * idx + 0];
            s_v[3 * t + 1] = kd.vgpc[3 * idx + 1];
            s_v[3 * t + 2] = kd.vgpc[3 * idx + 2];
        }
    }
    __syncthreads();
    const int ngp = kd.ngp;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int li = wm * 32 + i * 8 + (lane >> 2);
                const int lj = wn * 32 + j * 8 + 2 * (lane & 3) + h;
                const int gi = m0 + li, gj = n0 + lj;
                if (gi >= ngp || gj >= ngp || gi > gj) continue;
                double zr = cre[i][j][h], zi = cim[i][j][h];
                double ar, ai;
                if (interstitial(p, KIND, s_iv + 3 * li, s_iv + 3 * (64 + lj), s_v + 3 * li, s_v + 3 * (64 + lj), ar, ai)) {
                    zr += ar;
                    zi += ai;
                }
                exs_complex v; v.re = zr; v.im = zi;
                P.z[(size_t)gi + (size_t)P.ldz * gj] = v;
                if (gi < gj) {
                    exs_complex vc; vc.re = zr; vc.im = -zi;
                    P.z[(size_t)gj + (size_t)P.ldz * gi] = vc;
                }
            }
}

// ---------------------------------------------------------------- host side
template <int KIND>
static cudaError_t launch_kind(const DevParams &p, const GemmProb *d_probs, const TileWork *d_work, int nwork,
                               const KDesc *d_k, cudaStream_t s)
{
    if (nwork <= 0) return cudaSuccess;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        return cudaFuncSetAttribute(zgemm_dmma_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GB_SMEM);
    });
    if (e != cudaSuccess) return e;
    zgemm_dmma_kernel<KIND><<<(unsigned)nwork, GB_THREADS, GB_SMEM, s>>>(p, d_probs, d_work, d_k);
    return cudaGetLastError();
}

// Problem and tile tables of the three GEMM stages of one batched call.
void build_gemm_tables(const exs_ctx *c, const std::vector<KDesc> &ks, GemmTables &t)
{
    for (int q = 0; q < 4; q++) { t.probs[q].clear(); t.work[q].clear(); }
    for (size_t k = 0; k < ks.size(); k++) {
        const int ncols = std::min(c->npad, (ks[k].ngp + GB_N - 1) / GB_N * GB_N);
        for (int ias = 0; ias < c->natmtot; ias++) {
            const AtomDesc &a = c->atoms[ias];
            // stage 1: B_a = h_a A_a  (planar output, all padded columns)
            {
                GemmProb P{};
                P.xr = c->d_haa_r + (size_t)ias * c->ldh * c->ldh;
                P.xi = c->d_haa_i + (size_t)ias * c->ldh * c->ldh;
                P.ldx = c->ldh;
                P.yr = ks[k].ar + (size_t)a.apw_off * c->npad;
                P.yi = ks[k].ai + (size_t)a.apw_off * c->npad;
                P.ldy = c->npad;
                P.M = a.napw; P.N = ncols; P.K = a.napw;
                P.conjx = 0;
                P.outr = ks[k].br + (size_t)a.apw_off * c->npad;
                P.outi = ks[k].bi + (size_t)a.apw_off * c->npad;
                P.ldo = c->npad;
                P.kidx = (int)k;
                P.colmax = ks[k].oz_scale ? ks[k].oz_scale + c->npad : nullptr;
                const int pi = (int)t.probs[EPI_PLANAR].size();
                t.probs[EPI_PLANAR].push_back(P);
                for (int tm = 0; tm < (P.M + GB_M - 1) / GB_M; tm++)
                    for (int tn = 0; tn < (P.N + GB_N - 1) / GB_N; tn++) t.work[EPI_PLANAR].push_back({pi, tm, tn});
            }
            // stage 3: APW-lo rows of H
            if (a.losize > 0) {
                GemmProb P{};
                P.xr = c->d_loa_r + (size_t)ias * c->ldlo * c->maxaa;
                P.xi = c->d_loa_i + (size_t)ias * c->ldlo * c->maxaa;
                P.ldx = c->ldlo;
                P.yr = ks[k].ar + (size_t)a.apw_off * c->npad;
                P.yi = ks[k].ai + (size_t)a.apw_off * c->npad;
                P.ldy = c->npad;
                P.M = a.losize; P.N = ks[k].ngp; P.K = a.napw;
                P.conjx = 0;
                P.z = ks[k].h;
                P.ldz = ks[k].nmat;
                P.row0 = ks[k].ngp + a.lo_off;
                P.kidx = (int)k;
                const int pi = (int)t.probs[EPI_LOROWS].size();
                t.probs[EPI_LOROWS].push_back(P);
                for (int tm = 0; tm < (P.M + GB_M - 1) / GB_M; tm++)
                    for (int tn = 0; tn < (P.N + GB_N - 1) / GB_N; tn++) t.work[EPI_LOROWS].push_back({pi, tm, tn});
            }
        }
        // stage 2: H = A^H B and O = A^H A (A^H C for iora*), upper tiles
        for (int which = 0; which < 2; which++) {
            const int kind = which == 0 ? EPI_HAM : EPI_OVL;
            GemmProb P{};
            P.xr = ks[k].ar; P.xi = ks[k].ai; P.ldx = c->npad;
            if (which == 0) { P.yr = ks[k].br; P.yi = ks[k].bi; }
            else { P.yr = ks[k].cr; P.yi = ks[k].ci; }
            P.ldy = c->npad;
            P.M = P.N = ks[k].ngp;
            P.K = c->K;
            P.conjx = 1;
            P.z = which == 0 ? ks[k].h : ks[k].o;
            P.ldz = ks[k].nmat;
            P.kidx = (int)k;
            const int pi = (int)t.probs[kind].size();
            t.probs[kind].push_back(P);
            const int nt = (P.M + GB_M - 1) / GB_M;
            for (int tm = 0; tm < nt; tm++)
                for (int tn = tm; tn < nt; tn++) t.work[kind].push_back({pi, tm, tn});
        }
    }
}

cudaError_t launch_gemm_kind(int kind, const DevParams &p, const void *d_probs, const void *d_work, int nwork,
                             const KDesc *d_k, cudaStream_t s)
{
    const GemmProb *P = (const GemmProb *)d_probs;
    const TileWork *W = (const TileWork *)d_work;
    switch (kind) {
    case EPI_PLANAR: return launch_kind<EPI_PLANAR>(p, P, W, nwork, d_k, s);
    case EPI_HAM: return launch_kind<EPI_HAM>(p, P, W, nwork, d_k, s);
    case EPI_OVL: return launch_kind<EPI_OVL>(p, P, W, nwork, d_k, s);
    default: return launch_kind<EPI_LOROWS>(p, P, W, nwork, d_k, s);
    }
}

// ------------------------------------------- lo blocks that need no product
// O APW-lo (overlapsetup.f90:111-127): for lo function j = (ilo, m) of atom
// ias, O(G, ngp+idxlo) = sum_io conj(A(G, io, lm) (oalo(io,ilo) + h1loa)),
// lower = conjugate.  One thread per (G, lo row of the whole lo block).
__global__ void olp_apwlo_kernel(DevParams p, const KDesc *ks)
{
    const KDesc k = ks[blockIdx.z];
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;                     // global lo row 0..nlotot-1
    if (g >= k.ngp) return;
    // find the atom owning lo row r
    int ias = 0;
    while (ias + 1 < p.natmtot && (p.atoms[ias].losize == 0 || r >= p.atoms[ias].lo_off + p.atoms[ias].losize)) ias++;
    const AtomDesc at = p.atoms[ias];
    const int is = at.species;
    const int rl = r - at.lo_off;
    // decode (ilo, m) of the local lo row
    int ilo = 0, base = 0, l = 0;
    for (; ilo < p.nlorb[is]; ilo++) {
        l = p.lorbl[ilo + p.nlomax * is];
        if (rl < base + 2 * l + 1) break;
        base += 2 * l + 1;
    }
    const int m = rl - base - l;
    // APW row f of (l, m, io=0) inside the atom
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * is;
    int f = at.apw_off;
    for (int ll = 0; ll < l; ll++) f += (2 * ll + 1) * apw[ll];
    f += (m + l) * apw[l];
    double sr = 0.0, si = 0.0;
    for (int io = 0; io < apw[l]; io++) {
        double w = p.oalo[io + (size_t)p.apwordmax * (ilo + (size_t)p.nlomax * ias)];
        if (p.h1loa) w += p.h1loa[io + (size_t)p.apwordmax * (ilo + (size_t)p.nlomax * ias)];
        const double are = k.ar[(size_t)(f + io) * p.npad + g], aim = k.ai[(size_t)(f + io) * p.npad + g];
        sr += are * w;
        si -= aim * w;
    }
    const int j = k.ngp + r;
    exs_complex v; v.re = sr; v.im = si;
    exs_complex vc; vc.re = sr; vc.im = -si;
    k.o[(size_t)g + (size_t)k.nmat * j] = v;
    k.o[(size_t)j + (size_t)k.nmat * g] = vc;
}

// lo-lo blocks of H and O, every element of the nlotot x nlotot block.
__global__ void lolo_kernel(DevParams p, const KDesc *ks)
{
    const KDesc k = ks[blockIdx.z];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= p.nlotot) return;
    double hr = 0.0, hi = 0.0, orr = 0.0;
    int ia = 0, ib = 0;
    while (ia + 1 < p.natmtot && (p.atoms[ia].losize == 0 || r >= p.atoms[ia].lo_off + p.atoms[ia].losize)) ia++;
    while (ib + 1 < p.natmtot && (p.atoms[ib].losize == 0 || c >= p.atoms[ib].lo_off + p.atoms[ib].losize)) ib++;
    if (ia == ib) {
        const AtomDesc at = p.atoms[ia];
        const int rl = r - at.lo_off, cl = c - at.lo_off;
        // H: upper from lolo(r, c); lower = conj(lolo(c, r))   (copy_UL)
        if (rl <= cl) {
            const exs_complex v = p.lolo[rl + (size_t)p.maxnlo * (cl + (size_t)p.maxnlo * ia)];
            hr = v.re; hi = v.im;
        } else {
            const exs_complex v = p.lolo[cl + (size_t)p.maxnlo * (rl + (size_t)p.maxnlo * ia)];
            hr = v.re; hi = -v.im;
        }
        // O: ololo(ilo1, ilo2) + h1lolo on equal l and m (taken from the upper element)
        const int is = at.species;
        const int ru = rl <= cl ? rl : cl, cu = rl <= cl ? cl : rl;
        int i1 = 0, b1 = 0, l1 = 0, i2 = 0, b2 = 0, l2 = 0;
        for (; i1 < p.nlorb[is]; i1++) { l1 = p.lorbl[i1 + p.nlomax * is]; if (ru < b1 + 2 * l1 + 1) break; b1 += 2 * l1 + 1; }
        for (; i2 < p.nlorb[is]; i2++) { l2 = p.lorbl[i2 + p.nlomax * is]; if (cu < b2 + 2 * l2 + 1) break; b2 += 2 * l2 + 1; }
        if (l1 == l2 && (ru - b1) == (cu - b2)) {
            orr = p.ololo[i1 + (size_t)p.nlomax * (i2 + (size_t)p.nlomax * ia)];
            if (p.h1lolo) orr += p.h1lolo[i1 + (size_t)p.nlomax * (i2 + (size_t)p.nlomax * ia)];
        }
    }
    const size_t idx = (size_t)(k.ngp + r) + (size_t)k.nmat * (k.ngp + c);
    exs_complex hv; hv.re = hr; hv.im = hi;
    exs_complex ov; ov.re = orr; ov.im = 0.0;
    k.h[idx] = hv;
    k.o[idx] = ov;
}

cudaError_t launch_olp_apwlo(const DevParams &p, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s)
{
    if (p.nlotot == 0 || ngp_max == 0) return cudaSuccess;
    dim3 grid((ngp_max + 127) / 128, p.nlotot, nk);
    olp_apwlo_kernel<<<grid, 128, 0, s>>>(p, d_k);
    return cudaGetLastError();
}

cudaError_t launch_lolo_blocks(const DevParams &p, const KDesc *d_k, int nk, cudaStream_t s)
{
    if (p.nlotot == 0) return cudaSuccess;
    dim3 grid((p.nlotot + 127) / 128, p.nlotot, nk);
    lolo_kernel<<<grid, 128, 0, s>>>(p, d_k);
    return cudaGetLastError();
}

}  // namespace exs
