// IBS force (src/forcek.f90) and the adjoint of the H/O setup on the device.
//
// The reference builds, per atom a and direction x, the full nmat x nmat
// derivative matrices dlh and dlo (forcek.f90:262-287) and projects them on
// the eigenvectors with three zgemm calls each (:295-337), i.e.
// O(natoms * 3 * nmat^2 * nstfv).  Here the same quantity
//     F(x, a) = sum_n w_n Re[ c_n^H (dlh + eps_n dlo) c_n ],  w_n = wkpt occ_n
// is evaluated in factored form, never forming dlh/dlo:
//   * MT APW-APW (dlh = i(G_i-G_j)_x H_a, dlo = -i(G_i-G_j)_x O_a):
//       with U = A_a C_G and U_x = A_a V_x C_G (V_x = diag((k+G)_x)),
//       term = sum_n w_n Re{ i (u_x^H h u - u^H h u_x) - i eps_n (u_x^H M u - u^H M u_x) }
//       (M = 1, or 1 + h1aa for iora*; C_G the APW rows of the eigenvectors);
//   * APW-lo (dlh = i(k+G_i)_x H_a(i, lo), dlo = -i(k+G_i)_x O_a(i, lo), mirrored):
//       term = 2 Re sum_n w_n sum_j C_lo(j,n) conj( i (loa U_x)(j,n) - i eps_n (S U_x)(j,n) )^*
//       with S the oalo(+h1loa) map of overlapsetup.f90:111-127;
//   * interstitial step function (the zt1 = -ffacg conj(sfacg) terms):
//       R_H(g) = sum_{G_i-G_j=g} dp_ij P(j,i), R_O(g) = sum_{G_i-G_j=g} Q(j,i),
//       P = C_G W C_G^H, Q = C_G W eps C_G^H, then
//       term = sum_g Re[ i g_x zt1_a(g) (R_H(g) - R_O(g)) ].
// The scatter sums also give the gradient of L = sum_n w_n c_n^H (H - eps_n O) c_n
// with respect to V(G), and U gives the gradient with respect to h_a.
#include <algorithm>
#include <cstring>
#include <vector>

#include "exs_internal.cuh"

namespace exs {

struct ForceWork {
    int ngp, nst, nstp, ldt;         // ldt = Kpad (leading dim of At)
    int ldu;                         // 4 nstp: row stride of Ct, U, hU, MU, whose four blocks q sit side by side
    const KDesc *k;                  // A planes of the k-point (slot 0)
    double *atr, *ati;               // At [G][f]
    double *ct[4][2];                // Ct, Ct_x [G][ldu], block q at column q nstp (q = 0: plain, 1..3: x (k+G)_x)
    double *cn[2], *wc[2], *wec[2];  // [n][G]
    double *u[4][2];                 // U_q [f][ldu], block q at column q nstp
    double *hu[4][2];                // h_a U_q, same layout
    double *mu[4][2];                // M U_q (iora*) or == u, same layout
    double *pt[2], *qt[2];           // one band of rows of P^T, Q^T [i - i0][j], ld npad
    exs_complex *evec;               // (nmat, nst) dense
    const double *w, *eps;           // (nst)
    exs_complex *rh, *ro, *rv;       // (ngvec)
    const double *ffacg;             // (ngvec, nspecies)
    const double *vgc;               // (3, ngvec)
    double *force;                   // (3, natmtot)
};

__global__ void fk_transpose_a(int K, int ngp, int npad, int ldt, const double *ar, const double *ai, double *atr,
                               double *ati)
{
    __shared__ double tr[32][33], ti[32][33];
    const int f0 = blockIdx.y * 32, g0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int f = f0 + r, g = g0 + threadIdx.x;
        tr[r][threadIdx.x] = (f < K && g < ngp) ? ar[(size_t)f * npad + g] : 0.0;
        ti[r][threadIdx.x] = (f < K && g < ngp) ? ai[(size_t)f * npad + g] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int g = g0 + r, f = f0 + threadIdx.x;
        if (g < ngp && f < K) {
            atr[(size_t)g * ldt + f] = tr[threadIdx.x][r];
            ati[(size_t)g * ldt + f] = ti[threadIdx.x][r];
        }
    }
}

// Eigenvector packings: Ct_q[G][n] (q=0 plain, q=1..3 times (k+G)_x),
// C[n][G], w C[n][G], w eps C[n][G]; zero for n >= nst.
__global__ void fk_pack_evec(ForceWork fw, int npad, const double *vgpc, int nmat)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = blockIdx.y;
    if (g >= fw.ngp || n >= fw.nstp) return;
    double re = 0.0, im = 0.0, w = 0.0, we = 0.0;
    if (n < fw.nst) {
        const exs_complex z = fw.evec[g + (size_t)nmat * n];
        re = z.re;
        im = z.im;
        w = fw.w[n];
        we = fw.w[n] * fw.eps[n];
    }
    const size_t it = (size_t)g * fw.ldu + n;
    fw.ct[0][0][it] = re;
    fw.ct[0][1][it] = im;
    for (int x = 0; x < 3; x++) {
        const double v = vgpc[3 * g + x];
        fw.ct[1 + x][0][it] = v * re;
        fw.ct[1 + x][1][it] = v * im;
    }
    const size_t in = (size_t)n * npad + g;
    fw.cn[0][in] = re;
    fw.cn[1][in] = im;
    fw.wc[0][in] = w * re;
    fw.wc[1][in] = w * im;
    fw.wec[0][in] = we * re;
    fw.wec[1][in] = we * im;
}

// M U_q = U_q + h1aa U_q per (l, m) block (overlapsetup.f90:72-87), iora* only.
__global__ void fk_iora_u(DevParams p, ForceWork fw)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int ias = blockIdx.y;
    const int q = blockIdx.z;
    if (n >= fw.nstp) return;
    const AtomDesc at = p.atoms[ias];
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * at.species;
    int f = at.apw_off;
    for (int l = 0; l <= p.lmaxmat; l++) {
        const int no = apw[l];
        const double *h1 = p.h1aa + (size_t)p.apwordmax * p.apwordmax * (l + (size_t)(p.lmaxapw + 1) * ias);
        for (int m = -l; m <= l; m++, f += no)
            for (int io2 = 0; io2 < no; io2++) {
                double re = fw.u[q][0][(size_t)(f + io2) * fw.ldu + n];
                double im = fw.u[q][1][(size_t)(f + io2) * fw.ldu + n];
                for (int io1 = 0; io1 < no; io1++) {
                    const double w = h1[io1 + (size_t)p.apwordmax * io2];
                    re += w * fw.u[q][0][(size_t)(f + io1) * fw.ldu + n];
                    im += w * fw.u[q][1][(size_t)(f + io1) * fw.ldu + n];
                }
                fw.mu[q][0][(size_t)(f + io2) * fw.ldu + n] = re;
                fw.mu[q][1][(size_t)(f + io2) * fw.ldu + n] = im;
            }
    }
}

__device__ inline double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
    return s;
}

// conj(a) . b over the f rows [f0, f0+nf) of column n of two planar [f][n] arrays
__device__ inline void cdot(const double *ar, const double *ai, const double *br, const double *bi, int f0, int nf,
                            int ld, int n, double &re, double &im)
{
    re = 0.0;
    im = 0.0;
    for (int f = f0; f < f0 + nf; f++) {
        const size_t i = (size_t)f * ld + n;
        re += ar[i] * br[i] + ai[i] * bi[i];
        im += ar[i] * bi[i] - ai[i] * br[i];
    }
}

// The force terms are sums over the atom's APW rows f, so each block takes
// FK_FROWS of them and adds its share to the force atomically: many blocks
// per (atom, direction) instead of one long serial loop over the rows.
constexpr int FK_FROWS = 16;

// MT APW-APW terms, one block per (atom, direction, chunk of FK_FROWS rows).
__global__ void fk_terms_mt(DevParams p, ForceWork fw)
{
    __shared__ double sh[32];
    const int ias = blockIdx.x, x = blockIdx.y;
    const AtomDesc at = p.atoms[ias];
    const int fc = blockIdx.z * FK_FROWS;
    if (fc >= at.napw) return;                  // the whole block: no barrier is skipped by part of it
    const int f0 = at.apw_off + fc, nf = min(FK_FROWS, at.napw - fc);
    double acc = 0.0;
    for (int n = threadIdx.x; n < fw.nst; n += blockDim.x) {
        double zr, zi, z2r, z2i, yr, yi, y2r, y2i;
        // z = u_x^H h u, z' = u^H h u_x, y = u_x^H M u, y' = u^H M u_x (this block's rows)
        cdot(fw.u[1 + x][0], fw.u[1 + x][1], fw.hu[0][0], fw.hu[0][1], f0, nf, fw.ldu, n, zr, zi);
        cdot(fw.u[0][0], fw.u[0][1], fw.hu[1 + x][0], fw.hu[1 + x][1], f0, nf, fw.ldu, n, z2r, z2i);
        cdot(fw.u[1 + x][0], fw.u[1 + x][1], fw.mu[0][0], fw.mu[0][1], f0, nf, fw.ldu, n, yr, yi);
        cdot(fw.u[0][0], fw.u[0][1], fw.mu[1 + x][0], fw.mu[1 + x][1], f0, nf, fw.ldu, n, y2r, y2i);
        // Re[i w (z - z')] + Re[-i w eps (y - y')]
        acc += -fw.w[n] * (zi - z2i) + fw.w[n] * fw.eps[n] * (yi - y2i);
    }
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(&fw.force[x + 3 * ias], s);
}

// APW-lo terms, one block per (atom, direction, chunk of FK_FROWS APW rows
// of the loa U_x product); threads over (lo row, state).  The S U_x part,
// a few rows per lo row, is added by the blocks of the first chunk.
__global__ void fk_terms_lo(DevParams p, ForceWork fw, const double *loa_r, const double *loa_i, int ldlo, int maxaa)
{
    __shared__ double sh[32];
    const int ias = blockIdx.x, x = blockIdx.y;
    const AtomDesc at = p.atoms[ias];
    const int fc = blockIdx.z * FK_FROWS;
    if (fc >= at.napw) return;                  // the whole block
    const int fe = min(at.napw, fc + FK_FROWS);
    const int is = at.species;
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * is;
    const int nmat = fw.ngp + p.nlotot;
    double acc = 0.0;
    const double *uxr = fw.u[1 + x][0], *uxi = fw.u[1 + x][1];
    for (int t = threadIdx.x; t < at.losize * fw.nst; t += blockDim.x) {
        const int r = t % at.losize, n = t / at.losize;
        // (loa U_x)(r, n)
        double lr = 0.0, li = 0.0;
        const double *lar = loa_r + (size_t)ldlo * maxaa * ias, *lai = loa_i + (size_t)ldlo * maxaa * ias;
        for (int f = fc; f < fe; f++) {
            const double ar = lar[r + (size_t)ldlo * f], ai = lai[r + (size_t)ldlo * f];
            const size_t iu = (size_t)(at.apw_off + f) * fw.ldu + n;
            lr += ar * uxr[iu] - ai * uxi[iu];
            li += ar * uxi[iu] + ai * uxr[iu];
        }
        // (S U_x)(r, n): lo row r = (ilo, m), S picks the APW rows (l, m, io) with oalo(io, ilo)
        int ilo = 0, base = 0, l = 0;
        for (; ilo < p.nlorb[is]; ilo++) {
            l = p.lorbl[ilo + p.nlomax * is];
            if (r < base + 2 * l + 1) break;
            base += 2 * l + 1;
        }
        const int m = r - base - l;
        int f = at.apw_off;
        for (int ll = 0; ll < l; ll++) f += (2 * ll + 1) * apw[ll];
        f += (m + l) * apw[l];
        double sr = 0.0, si = 0.0;
        for (int io = 0; io < (blockIdx.z == 0 ? apw[l] : 0); io++) {
            double w = p.oalo[io + (size_t)p.apwordmax * (ilo + (size_t)p.nlomax * ias)];
            if (p.h1loa) w += p.h1loa[io + (size_t)p.apwordmax * (ilo + (size_t)p.nlomax * ias)];
            const size_t iu = (size_t)(f + io) * fw.ldu + n;
            sr += w * uxr[iu];
            si += w * uxi[iu];
        }
        const exs_complex cl = fw.evec[(size_t)(fw.ngp + at.lo_off + r) + (size_t)nmat * n];
        // 2 Re[ i w cl conj(L) ] + 2 Re[ -i w eps cl conj(S) ];  Re(i z) = -Im z
        const double im_l = cl.im * lr - cl.re * li;      // Im(cl * conj(L))
        const double im_s = cl.im * sr - cl.re * si;      // Im(cl * conj(S))
        acc += -2.0 * fw.w[n] * im_l + 2.0 * fw.w[n] * fw.eps[n] * im_s;
    }
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(&fw.force[x + 3 * ias], s);
}

// Scatter of P(j,i), dp_ij P(j,i) and Q(j,i) onto G_i - G_j for the rows
// i0 <= i < i1 of one band of P^T and Q^T (held from row i0 on) and all j < ngp.
__global__ void fk_scatter(DevParams p, ForceWork fw, const KDesc *kd, int i0, int i1)
{
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = i0 + blockIdx.y;                  // the band holds the columns j >= i0
    if (i >= i1 || i >= fw.ngp || j < i) return;    // upper triangle; fk_fold_conj adds the lower one
    const int gi = kd->igpig[i] - 1, gj = kd->igpig[j] - 1;
    if (gi < 0 || gi >= p.ngrtot || gj < 0 || gj >= p.ngrtot) { atomicOr(p.err, DEV_ERR_INDEX); return; }
    const int d0 = p.ivg[3 * gi] - p.ivg[3 * gj] - p.intgv_lo[0];
    const int d1 = p.ivg[3 * gi + 1] - p.ivg[3 * gj + 1] - p.intgv_lo[1];
    const int d2 = p.ivg[3 * gi + 2] - p.ivg[3 * gj + 2] - p.intgv_lo[2];
    if ((unsigned)d0 >= (unsigned)p.intgv_n[0] || (unsigned)d1 >= (unsigned)p.intgv_n[1] ||
        (unsigned)d2 >= (unsigned)p.intgv_n[2]) {
        atomicOr(p.err, DEV_ERR_INDEX);
        return;
    }
    const int ig = p.ivgig[d0 + p.intgv_n[0] * (d1 + p.intgv_n[1] * d2)];
    if (ig <= 0 || ig > p.ngvec) return;
    const double *vi = kd->vgpc + 3 * i, *vj = kd->vgpc + 3 * j;
    const double dp = 0.5 * (vi[0] * vj[0] + vi[1] * vj[1] + vi[2] * vj[2]);
    const size_t e = (size_t)(i - i0) * p.npad + (j - i0);
    // the diagonal (g = 0) is folded onto itself: half of it here, the fold doubles the real part
    const double hf = (j == i) ? 0.5 : 1.0;
    const double pr = hf * fw.pt[0][e], pi = hf * fw.pt[1][e], qr = hf * fw.qt[0][e], qi = hf * fw.qt[1][e];
    double *rh = reinterpret_cast<double *>(fw.rh + (ig - 1));
    double *ro = reinterpret_cast<double *>(fw.ro + (ig - 1));
    double *rv = reinterpret_cast<double *>(fw.rv + (ig - 1));
    atomicAdd(rh, dp * pr);
    atomicAdd(rh + 1, dp * pi);
    atomicAdd(ro, qr);
    atomicAdd(ro + 1, qi);
    atomicAdd(rv, pr);
    atomicAdd(rv + 1, pi);
}

// P^T and Q^T are Hermitian and dp is symmetric in (i, j), so the lower
// triangle's share of a G-vector g = G_i - G_j is the conjugate of the upper
// triangle's share of -g: R(g) = R_up(g) + conj(R_up(-g)) for rh, ro, rv.
// One thread per pair {g, -g} (the one with g <= -g in the list order).
__global__ void fk_fold_conj(DevParams p, ForceWork fw)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= p.ngvec) return;
    const int d0 = -p.ivg[3 * g] - p.intgv_lo[0], d1 = -p.ivg[3 * g + 1] - p.intgv_lo[1],
              d2 = -p.ivg[3 * g + 2] - p.intgv_lo[2];
    if ((unsigned)d0 >= (unsigned)p.intgv_n[0] || (unsigned)d1 >= (unsigned)p.intgv_n[1] ||
        (unsigned)d2 >= (unsigned)p.intgv_n[2]) {
        atomicOr(p.err, DEV_ERR_INDEX);
        return;
    }
    const int ng = p.ivgig[d0 + p.intgv_n[0] * (d1 + p.intgv_n[1] * d2)] - 1;
    if (ng < 0 || ng >= p.ngvec) {
        atomicOr(p.err, DEV_ERR_INDEX);
        return;
    }
    if (ng < g) return;                             // the partner thread does the pair
    exs_complex *arr[3] = {fw.rh, fw.ro, fw.rv};
    for (int k = 0; k < 3; k++) {
        const exs_complex a = arr[k][g], b = arr[k][ng];
        exs_complex x, y;
        x.re = a.re + b.re;
        x.im = a.im - b.im;
        y.re = b.re + a.re;
        y.im = b.im - a.im;
        arr[k][g] = x;
        if (ng != g) arr[k][ng] = y;
    }
}

// Interstitial step-function terms, one block per atom, the three directions.
__global__ void fk_terms_theta(DevParams p, ForceWork fw, int ngvec)
{
    __shared__ double sh[32];
    const int ias = blockIdx.x;
    const AtomDesc at = p.atoms[ias];
    double acc[3] = {0.0, 0.0, 0.0};
    // blockIdx.y: one of gridDim.y interleaved shares of the G-vectors
    for (int g = blockIdx.y * blockDim.x + threadIdx.x; g < ngvec; g += gridDim.y * blockDim.x) {
        const double *v = fw.vgc + 3 * (size_t)g;
        const double ff = fw.ffacg[g + (size_t)ngvec * at.species];
        double s, c;
        sincos(v[0] * at.pos[0] + v[1] * at.pos[1] + v[2] * at.pos[2], &s, &c);
        // zt1 = -ffacg conj(sfacg) = -ff (c - i s)
        const double zr = -ff * c, zi = ff * s;
        const double dr = fw.rh[g].re - fw.ro[g].re, di = fw.rh[g].im - fw.ro[g].im;
        const double im = zr * di + zi * dr;          // Im(zt1 * D)
        for (int x = 0; x < 3; x++) acc[x] += -v[x] * im;   // Re(i g_x zt1 D) = -g_x Im(zt1 D)
    }
    for (int x = 0; x < 3; x++) {
        const double s = block_sum(acc[x], sh);
        if (threadIdx.x == 0) atomicAdd(&fw.force[x + 3 * ias], s);
    }
}

// dL/dh_a(f, f') = sum_n w_n conj(U(f, n)) U(f', n) per atom, into (maxaa, maxaa, natmtot).
// One block per 32 x 32 tile (f, f') of one atom, 32 x 8 threads: chunks of
// 32 states of the rows f and f' are staged in shared memory (coalesced over
// n), and each thread sums four outputs f = tile + tx, f' = tile + ty + 8 j.
__global__ void fk_dh(DevParams p, ForceWork fw, exs_complex *dh, int maxaa)
{
    __shared__ double ar[32][33], ai[32][33], br[32][33], bi[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int fb = blockIdx.x * 32, f2b = blockIdx.y * 32, ias = blockIdx.z;
    const AtomDesc at = p.atoms[ias];
    const double *ur = fw.u[0][0], *ui = fw.u[0][1];
    double re[4] = {0.0, 0.0, 0.0, 0.0}, im[4] = {0.0, 0.0, 0.0, 0.0};
    for (int n0 = 0; n0 < fw.nst; n0 += 32) {
        const int n = n0 + tx;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int r = ty + 8 * k;
            const int f = fb + r, f2 = f2b + r;
            const bool vn = n < fw.nst;
            const double w = vn ? fw.w[n] : 0.0;
            const bool va = vn && f < at.napw, vb = vn && f2 < at.napw;
            const size_t ia = (size_t)(at.apw_off + f) * fw.ldu + n, ib = (size_t)(at.apw_off + f2) * fw.ldu + n;
            ar[r][tx] = va ? ur[ia] : 0.0;
            ai[r][tx] = va ? ui[ia] : 0.0;
            br[r][tx] = vb ? w * ur[ib] : 0.0;
            bi[r][tx] = vb ? w * ui[ib] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < 32; c++) {
            const double xr = ar[tx][c], xi = ai[tx][c];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const double yr = br[ty + 8 * j][c], yi = bi[ty + 8 * j][c];
                re[j] += xr * yr + xi * yi;                 // conj(x) y
                im[j] += xr * yi - xi * yr;
            }
        }
        __syncthreads();
    }
    const int f = fb + tx;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int f2 = f2b + ty + 8 * j;
        if (f >= maxaa || f2 >= maxaa) continue;
        exs_complex z;
        z.re = re[j];
        z.im = im[j];
        dh[f + (size_t)maxaa * (f2 + (size_t)maxaa * ias)] = z;
    }
}

}  // namespace exs

// ---------------------------------------------------------------- host side
namespace {

using exs::ForceWork;
using exs::GemmProb;
using exs::KDesc;
using exs::TileWork;

int ffail(exs_ctx *c, int code, const char *msg)
{
    c->last_error = msg;
    return code;
}

#define FK_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            c->last_error = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return EXS_ERR_CUDA;                                                           \
        }                                                                                  \
    } while (0)

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

cudaError_t grow(void **p, size_t *cap, size_t need, bool pinned)
{
    if (need <= *cap) return cudaSuccess;
    if (*p) { if (pinned) cudaFreeHost(*p); else cudaFree(*p); }
    *p = nullptr;
    *cap = 0;
    cudaError_t e = pinned ? cudaMallocHost(p, need) : cudaMalloc(p, need);
    if (e == cudaSuccess) *cap = need;
    return e;
}

void add_tiles(std::vector<TileWork> &w, int pi, int M, int N, bool upper)
{
    const int tm = (M + 63) / 64, tn = (N + 63) / 64;
    for (int a = 0; a < tm; a++)
        for (int b = upper ? a : 0; b < tn; b++) w.push_back({pi, a, b});
}

// The whole adjoint of one k-point.  Fills c->fk_force (device, 3*natmtot),
// the scatter sums and U; returns an EXS_ code.
int run_adjoint(exs_ctx *c, int ngp, const int *igpig, const double *vgpc, int nst, const exs_complex *evec, int ldv,
                const double *w_host, const double *eps_host, const double *ffacg, const double *vgc,
                ForceWork &fw, exs_complex **d_rv_out)
{
    cudaStream_t s = c->stream;
    const int nmat = ngp + c->nlotot;
    const int nstp = (nst + 1) / 2 * 2;
    const int npad = c->npad, Kp = c->Kpad;
    // ---- device work space
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = al256(off + bytes); return o; };
    const size_t o_at = take(2 * sizeof(double) * (size_t)npad * Kp);
    const size_t o_ct = take(8 * sizeof(double) * (size_t)npad * nstp);
    const size_t o_cn = take(6 * sizeof(double) * (size_t)nstp * npad);
    const size_t o_u = take(8 * sizeof(double) * (size_t)Kp * nstp);
    const size_t o_hu = take(8 * sizeof(double) * (size_t)Kp * nstp);
    const bool iora = c->relativity == EXS_REL_IORA;
    const size_t o_mu = take(iora ? 8 * sizeof(double) * (size_t)Kp * nstp : 0);
    // P^T and Q^T in bands of rows of at most ~1 GiB (one band below ~5,800 G+k)
    const int band = std::max(64, std::min(npad, (int)((((size_t)1 << 30) / (4 * sizeof(double) * (size_t)npad)) / 64 * 64)));
    const size_t o_pq = take(4 * sizeof(double) * (size_t)band * npad);
    const size_t o_ev = take(sizeof(exs_complex) * (size_t)nmat * nst);
    const size_t o_we = take(2 * sizeof(double) * (size_t)nst);
    const size_t o_r = take(3 * sizeof(exs_complex) * (size_t)c->ngvec);
    const size_t o_ff = take(sizeof(double) * (size_t)c->ngvec * c->nspecies);
    const size_t o_vg = take(3 * sizeof(double) * (size_t)c->ngvec);
    const size_t o_f = take(3 * sizeof(double) * (size_t)c->natmtot);
    FK_CUDA(cudaStreamSynchronize(s));
    FK_CUDA(grow(&c->fk_dev, &c->fk_bytes, off, false));
    char *b = (char *)c->fk_dev;
    fw.ngp = ngp; fw.nst = nst; fw.nstp = nstp; fw.ldt = Kp;
    const int ldu = 4 * nstp;
    fw.ldu = ldu;
    fw.atr = (double *)(b + o_at); fw.ati = fw.atr + (size_t)npad * Kp;
    for (int q = 0; q < 4; q++)
        for (int r = 0; r < 2; r++) fw.ct[q][r] = (double *)(b + o_ct) + (size_t)r * npad * ldu + (size_t)q * nstp;
    double *cn = (double *)(b + o_cn);
    fw.cn[0] = cn; fw.cn[1] = cn + (size_t)nstp * npad;
    fw.wc[0] = cn + 2 * (size_t)nstp * npad; fw.wc[1] = cn + 3 * (size_t)nstp * npad;
    fw.wec[0] = cn + 4 * (size_t)nstp * npad; fw.wec[1] = cn + 5 * (size_t)nstp * npad;
    for (int q = 0; q < 4; q++)
        for (int r = 0; r < 2; r++) {
            fw.u[q][r] = (double *)(b + o_u) + (size_t)r * Kp * ldu + (size_t)q * nstp;
            fw.hu[q][r] = (double *)(b + o_hu) + (size_t)r * Kp * ldu + (size_t)q * nstp;
            fw.mu[q][r] = iora ? (double *)(b + o_mu) + (size_t)r * Kp * ldu + (size_t)q * nstp : fw.u[q][r];
        }
    double *pq = (double *)(b + o_pq);
    fw.pt[0] = pq; fw.pt[1] = pq + (size_t)band * npad;
    fw.qt[0] = pq + 2 * (size_t)band * npad; fw.qt[1] = pq + 3 * (size_t)band * npad;
    fw.evec = (exs_complex *)(b + o_ev);
    double *we = (double *)(b + o_we);
    fw.w = we;
    fw.eps = we + nst;
    fw.rh = (exs_complex *)(b + o_r);
    fw.ro = fw.rh + c->ngvec;
    fw.rv = fw.ro + c->ngvec;
    fw.ffacg = (const double *)(b + o_ff);
    fw.vgc = (const double *)(b + o_vg);
    fw.force = (double *)(b + o_f);
    *d_rv_out = fw.rv;

    // ---- uploads
    FK_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
    FK_CUDA(cudaMemcpyAsync(c->d_igpig, igpig, sizeof(int) * ngp, cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemcpyAsync(c->d_vgpc, vgpc, sizeof(double) * 3 * ngp, cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemcpy2DAsync(fw.evec, sizeof(exs_complex) * nmat, evec, sizeof(exs_complex) * ldv,
                              sizeof(exs_complex) * nmat, nst, cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemcpyAsync(we, w_host, sizeof(double) * nst, cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemcpyAsync(we + nst, eps_host, sizeof(double) * nst, cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemcpyAsync((void *)fw.ffacg, ffacg, sizeof(double) * (size_t)c->ngvec * c->nspecies,
                            cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemcpyAsync((void *)fw.vgc, vgc, 3 * sizeof(double) * (size_t)c->ngvec, cudaMemcpyHostToDevice, s));
    FK_CUDA(cudaMemsetAsync(fw.rh, 0, 3 * sizeof(exs_complex) * (size_t)c->ngvec, s));
    FK_CUDA(cudaMemsetAsync(fw.force, 0, 3 * sizeof(double) * (size_t)c->natmtot, s));

    // ---- k descriptor (slot 0 work planes) and GEMM tables, one upload
    KDesc kd{};
    kd.ngp = ngp;
    kd.nmat = nmat;
    kd.igpig = c->d_igpig;
    kd.vgpc = c->d_vgpc;
    double *wk = c->d_work;
    kd.ar = wk; kd.ai = wk + c->plane; kd.br = wk + 2 * c->plane; kd.bi = wk + 3 * c->plane;
    kd.cr = kd.ar; kd.ci = kd.ai;
    std::vector<GemmProb> probs;
    std::vector<TileWork> w1, w2, wb;
    std::vector<size_t> wb_off;
    {                                          // [U_0 .. U_3] = A [C_0 .. C_3]: one product over G, N = 4 nstp
        GemmProb P{};
        P.xr = fw.atr; P.xi = fw.ati; P.ldx = Kp;
        P.yr = fw.ct[0][0]; P.yi = fw.ct[0][1]; P.ldy = ldu;
        P.M = c->K; P.N = ldu; P.K = ngp; P.conjx = 0;
        P.outr = fw.u[0][0]; P.outi = fw.u[0][1]; P.ldo = ldu;
        add_tiles(w1, (int)probs.size(), P.M, P.N, false);
        probs.push_back(P);
    }
    for (int i0 = 0; i0 < ngp; i0 += band) {   // P^T = conj(C)^T (w C), Q^T = conj(C)^T (w eps C): rows i0..,
        wb_off.push_back(wb.size());             // columns j >= i0 (the scatter takes the upper triangle)
        for (int which = 0; which < 2; which++) {
            GemmProb P{};
            P.xr = fw.cn[0] + i0; P.xi = fw.cn[1] + i0; P.ldx = npad;
            P.yr = (which == 0 ? fw.wc[0] : fw.wec[0]) + i0; P.yi = (which == 0 ? fw.wc[1] : fw.wec[1]) + i0;
            P.ldy = npad;
            P.M = std::min(band, ngp - i0); P.N = ngp - i0; P.K = nst; P.conjx = 1;
            P.outr = which == 0 ? fw.pt[0] : fw.qt[0]; P.outi = which == 0 ? fw.pt[1] : fw.qt[1]; P.ldo = npad;
            add_tiles(wb, (int)probs.size(), P.M, P.N, false);
            probs.push_back(P);
        }
    }
    wb_off.push_back(wb.size());
    for (int ias = 0; ias < c->natmtot; ias++) {   // h_a [U_0 .. U_3] per atom, N = 4 nstp
        const exs::AtomDesc &a = c->atoms[ias];
        GemmProb P{};
        P.xr = c->d_haa_r + (size_t)ias * c->ldh * c->ldh; P.xi = c->d_haa_i + (size_t)ias * c->ldh * c->ldh;
        P.ldx = c->ldh;
        P.yr = fw.u[0][0] + (size_t)a.apw_off * ldu; P.yi = fw.u[0][1] + (size_t)a.apw_off * ldu; P.ldy = ldu;
        P.M = a.napw; P.N = ldu; P.K = a.napw; P.conjx = 0;
        P.outr = fw.hu[0][0] + (size_t)a.apw_off * ldu; P.outi = fw.hu[0][1] + (size_t)a.apw_off * ldu;
        P.ldo = ldu;
        add_tiles(w2, (int)probs.size(), P.M, P.N, false);
        probs.push_back(P);
    }
    const size_t kb = al256(sizeof(KDesc)), pb = al256(sizeof(GemmProb) * probs.size());
    const size_t wbytes = sizeof(TileWork) * (w1.size() + w2.size() + wb.size());
    const size_t tb = kb + pb + wbytes;
    FK_CUDA(grow(&c->fk_tab_h, &c->fk_tab_hbytes, tb, true));
    FK_CUDA(grow(&c->fk_tab_d, &c->fk_tab_dbytes, tb, false));
    char *th = (char *)c->fk_tab_h;
    std::memcpy(th, &kd, sizeof(KDesc));
    std::memcpy(th + kb, probs.data(), sizeof(GemmProb) * probs.size());
    std::memcpy(th + kb + pb, w1.data(), sizeof(TileWork) * w1.size());
    std::memcpy(th + kb + pb + sizeof(TileWork) * w1.size(), w2.data(), sizeof(TileWork) * w2.size());
    std::memcpy(th + kb + pb + sizeof(TileWork) * (w1.size() + w2.size()), wb.data(), sizeof(TileWork) * wb.size());
    FK_CUDA(cudaMemcpyAsync(c->fk_tab_d, th, tb, cudaMemcpyHostToDevice, s));
    char *td = (char *)c->fk_tab_d;
    const KDesc *d_k = (const KDesc *)td;
    const GemmProb *d_p = (const GemmProb *)(td + kb);
    const TileWork *d_w1 = (const TileWork *)(td + kb + pb);
    const TileWork *d_w2 = d_w1 + w1.size();
    const TileWork *d_wb = d_w2 + w2.size();

    // ---- launches
    (void)cudaGetLastError();   // launch checks below read the last error: start clean
    const exs::DevParams p = c->params();
    FK_CUDA(exs::launch_match_planes(p, d_k, 1, ngp, s));
    {
        dim3 blk(32, 8), grd((ngp + 31) / 32, (c->K + 31) / 32);
        exs::fk_transpose_a<<<grd, blk, 0, s>>>(c->K, ngp, npad, Kp, kd.ar, kd.ai, fw.atr, fw.ati);
        exs::fk_pack_evec<<<dim3((ngp + 127) / 128, nstp), 128, 0, s>>>(fw, npad, c->d_vgpc, nmat);
        FK_CUDA(cudaGetLastError());
    }
    FK_CUDA(exs::launch_gemm_kind(exs::EPI_PLANAR, p, d_p, d_w1, (int)w1.size(), d_k, s));
    FK_CUDA(exs::launch_gemm_kind(exs::EPI_PLANAR, p, d_p, d_w2, (int)w2.size(), d_k, s));
    if (iora) exs::fk_iora_u<<<dim3((nstp + 63) / 64, c->natmtot, 4), 64, 0, s>>>(p, fw);
    const unsigned fch = (unsigned)((c->maxaa + exs::FK_FROWS - 1) / exs::FK_FROWS);
    exs::fk_terms_mt<<<dim3(c->natmtot, 3, fch), 64, 0, s>>>(p, fw);
    if (c->nlotot > 0)
        exs::fk_terms_lo<<<dim3(c->natmtot, 3, fch), 256, 0, s>>>(p, fw, c->d_loa_r, c->d_loa_i, c->ldlo, c->maxaa);
    for (size_t b = 0; b + 1 < wb_off.size(); b++) {   // one band of P^T, Q^T, then its scatter
        const int i0 = (int)b * band, i1 = std::min(ngp, i0 + band);
        FK_CUDA(exs::launch_gemm_kind(exs::EPI_PLANAR, p, d_p, d_wb + wb_off[b], (int)(wb_off[b + 1] - wb_off[b]),
                                      d_k, s));
        exs::fk_scatter<<<dim3((i1 - i0 + 127) / 128, ngp - i0), 128, 0, s>>>(p, fw, d_k, i0, i1);
        FK_CUDA(cudaGetLastError());
    }
    exs::fk_fold_conj<<<(c->ngvec + 255) / 256, 256, 0, s>>>(p, fw);
    // about two waves of blocks whatever the number of atoms, at least 2,048 G-vectors per block
    const int gsh = std::max(1, std::min((c->ngvec + 2047) / 2048, (2 * 148 * 8 + c->natmtot - 1) / c->natmtot));
    exs::fk_terms_theta<<<dim3(c->natmtot, gsh), 256, 0, s>>>(p, fw, c->ngvec);
    FK_CUDA(cudaGetLastError());
    return EXS_OK;
}

int check_adjoint_args(exs_ctx *c, int ngp, const int *igpig, const double *vgpc, int nst, const exs_complex *evec,
                       int ldv, const double *ffacg, const double *vgc)
{
    if (!igpig || !vgpc || !evec || !ffacg || !vgc) return ffail(c, EXS_ERR_ARG, "null argument");
    if (ngp <= 0 || ngp > c->ngkmax) return ffail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax");
    if (nst <= 0 || ldv < ngp + c->nlotot) return ffail(c, EXS_ERR_ARG, "nstfv <= 0 or ldv < nmat");
    if (!c->have_inputs) return ffail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    for (int i = 0; i < ngp; i++)
        if (igpig[i] < 1 || igpig[i] > c->ngrtot) return ffail(c, EXS_ERR_INDEX, "igpig entry outside 1..ngrtot");
    return EXS_OK;
}

}  // namespace

extern "C" int exs_forcek(exs_ctx *c, int ngp, const int *igpig, const double *vgpc, int nstfv,
                          const exs_complex *evecfv, int ldv, const double *evalfv, const double *occsv,
                          double wkpt, const double *ffacg, const double *vgc, double *forceibs)
{
    if (!c) return EXS_ERR_ARG;
    if (!evalfv || !occsv || !forceibs) return ffail(c, EXS_ERR_ARG, "null argument");
    int rc = check_adjoint_args(c, ngp, igpig, vgpc, nstfv, evecfv, ldv, ffacg, vgc);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    std::vector<double> w(nstfv);
    for (int n = 0; n < nstfv; n++) w[n] = wkpt * occsv[n];
    ForceWork fw{};
    exs_complex *rv = nullptr;
    rc = run_adjoint(c, ngp, igpig, vgpc, nstfv, evecfv, ldv, w.data(), evalfv, ffacg, vgc, fw, &rv);
    if (rc != EXS_OK) return rc;
    std::vector<double> f(3 * (size_t)c->natmtot);
    FK_CUDA(cudaMemcpyAsync(f.data(), fw.force, sizeof(double) * f.size(), cudaMemcpyDeviceToHost, c->stream));
    rc = exs_synchronize(c);
    if (rc < 0) return rc;
    for (size_t i = 0; i < f.size(); i++) forceibs[i] += f[i];    // forcek accumulates (forcek.f90:373-383)
    return rc;
}

extern "C" int exs_adjoint(exs_ctx *c, int ngp, const int *igpig, const double *vgpc, int nst, const exs_complex *cvec,
                           int ldv, const double *w, const double *eps, const double *ffacg, const double *vgc,
                           double *dtau, exs_complex *dveffig, exs_complex *dh)
{
    if (!c) return EXS_ERR_ARG;
    if (!w || !eps || !dtau) return ffail(c, EXS_ERR_ARG, "null argument");
    int rc = check_adjoint_args(c, ngp, igpig, vgpc, nst, cvec, ldv, ffacg, vgc);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    ForceWork fw{};
    exs_complex *rv = nullptr;
    rc = run_adjoint(c, ngp, igpig, vgpc, nst, cvec, ldv, w, eps, ffacg, vgc, fw, &rv);
    if (rc != EXS_OK) return rc;
    cudaStream_t s = c->stream;
    std::vector<double> f(3 * (size_t)c->natmtot);
    FK_CUDA(cudaMemcpyAsync(f.data(), fw.force, sizeof(double) * f.size(), cudaMemcpyDeviceToHost, s));
    if (dveffig)
        FK_CUDA(cudaMemcpyAsync(dveffig, rv, sizeof(exs_complex) * (size_t)c->ngvec, cudaMemcpyDeviceToHost, s));
    if (dh) {   // the work buffer stays with the context between calls
        const size_t n = (size_t)c->maxaa * c->maxaa * c->natmtot;
        FK_CUDA(grow(&c->fk_dh, &c->fk_dh_bytes, sizeof(exs_complex) * n, false));
        exs_complex *d_dh = (exs_complex *)c->fk_dh;
        exs::fk_dh<<<dim3((c->maxaa + 31) / 32, (c->maxaa + 31) / 32, c->natmtot), dim3(32, 8), 0, s>>>(c->params(), fw, d_dh,
                                                                                                   c->maxaa);
        FK_CUDA(cudaGetLastError());
        FK_CUDA(cudaMemcpyAsync(dh, d_dh, sizeof(exs_complex) * n, cudaMemcpyDeviceToHost, s));
    }
    rc = exs_synchronize(c);
    if (rc < 0) return rc;
    for (size_t i = 0; i < f.size(); i++) dtau[i] = -f[i];          // dL/dtau = -F_IBS
    return rc;
}
