// Muffin-tin integral generation on the device: the per-SCF-iteration
// mt_hscf%main = {aa, loa, lolo} that the setup contracts with the matching
// coefficients.  Replaces  call hmlint  (src/src_eigensystem/hmlint.f90:53-55,
// the spin-unpolarised main part: mt_kin then mt_pot on zeroed arrays).
//
// The reference integrates every product u_p u_q r^2 V_lm2 with its own
// cubic-spline call (fderiv, m = -1) and contracts with the nonzero Gaunt
// coefficients gntyry(lm2, lm3, lm1) (init1.f90:559-595).  Here:
//   * the spline integral is a linear functional of the integrand, so it is
//     applied as a weight vector w_r per species (built once on the host from
//     the radial mesh): I = sum_r w_r f_r;
//   * the radial integrals of one atom are then small dense contractions
//     I[lm2][p][q] = sum_r phi_p(r) (phi_q(r) w_r r^2 V_lm2(r)) over all radial
//     functions p, q (APW u_{l,io} of l <= lmaxmat, then the local orbitals),
//     plus one kinetic channel; mt_radial_kernel computes them tile by tile;
//   * mt_angular_kernel contracts them with a compressed Gaunt list for each
//     (lm1, lm3) pair and writes h_a, loa and lolo straight into the context's
//     device copies, where the next setup reads them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "exs_internal.cuh"
#include "host_spline.h"

namespace {

using exs::spline_integral;
using exs::spline_weights;

constexpr double Y00 = 0.28209479177387814347;   // 1/sqrt(4 pi)
constexpr double PI = 3.14159265358979323846;
constexpr double ALPHA = 1.0 / 137.03599911;     // fine-structure constant (mt_kin.f90:38)

int mfail(exs_ctx *c, int code, const std::string &msg)
{
    if (c) c->last_error = msg;
    return code;
}

#define MT_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return mfail(c, EXS_ERR_CUDA, std::string(#call ": ") + \
                                                                 cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ Gaunt coefficients
// theta(l, m, x), m >= 0: Y_lm(theta, phi) = theta_lm(cos theta) e^{i m phi}
// with the Condon-Shortley phase, by the standard normalised recurrences
//   theta_00 = 1/sqrt(4 pi),  theta_mm = -sqrt((2m+1)/(2m)) sin(theta) theta_{m-1,m-1},
//   theta_lm = a_lm (x theta_{l-1,m} - theta_{l-2,m} / a_{l-1,m}),
//   a_lm = sqrt((4 l^2 - 1) / (l^2 - m^2)).
// Then for any m, Y_lm = s_m theta_{l|m|} e^{i m phi} with s_m = (-1)^m for m < 0.
struct LegendreTable {
    int lmax = -1, n = 0;
    std::vector<double> x, w;      // Gauss-Legendre nodes and weights on [-1, 1]
    std::vector<double> th;        // [(l(l+1)/2 + m) * n + k]
    const double *at(int l, int m) const { return th.data() + (size_t)(l * (l + 1) / 2 + m) * n; }

    void build(int lmax_, int npts)
    {
        lmax = lmax_;
        n = npts;
        x.assign(n, 0.0);
        w.assign(n, 0.0);
        // nodes: Newton on P_n from the Tricomi estimate cos(pi (k + 3/4) / (n + 1/2))
        for (int k = 0; k < n; k++) {
            double z = std::cos(PI * (k + 0.75) / (n + 0.5)), dp = 1.0;
            for (int it = 0; it < 100; it++) {
                double p0 = 1.0, p1 = z;
                for (int j = 2; j <= n; j++) {
                    const double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                    p0 = p1;
                    p1 = p2;
                }
                dp = n * (z * p1 - p0) / (z * z - 1.0);
                const double dz = p1 / dp;
                z -= dz;
                if (std::fabs(dz) < 1e-16) break;
            }
            // weight from the derivative at the converged node
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= n; j++) {
                const double p2 = ((2 * j - 1) * z * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            x[k] = z;
            w[k] = 2.0 / ((1.0 - z * z) * dp * dp);
        }
        th.assign((size_t)(lmax + 1) * (lmax + 2) / 2 * n, 0.0);
        for (int k = 0; k < n; k++) {
            const double z = x[k], sn = std::sqrt(std::max(0.0, 1.0 - z * z));
            double diag = 1.0 / std::sqrt(4.0 * PI);
            for (int m = 0; m <= lmax; m++) {
                if (m > 0) diag *= -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * sn;
                double pm2 = 0.0, pm1 = diag, a_prev = 0.0;
                th[(size_t)(m * (m + 1) / 2 + m) * n + k] = diag;
                for (int l = m + 1; l <= lmax; l++) {
                    const double a = std::sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
                    const double v = a * (z * pm1 - (l == m + 1 ? 0.0 : pm2 / a_prev));
                    th[(size_t)(l * (l + 1) / 2 + m) * n + k] = v;
                    pm2 = pm1;
                    pm1 = v;
                    a_prev = a;
                }
            }
        }
    }

    // int_{-1}^{1} theta_{l1|m1|} theta_{l2|m2|} theta_{l3|m3|} dx, exact while
    // l1 + l2 + l3 <= 2n - 1 (the product is a polynomial when
    // |m1| + |m2| + |m3| is even)
    double triple(int l1, int m1, int l2, int m2, int l3, int m3) const
    {
        const double *a = at(l1, std::abs(m1)), *b = at(l2, std::abs(m2)), *c = at(l3, std::abs(m3));
        double t = 0.0;
        for (int k = 0; k < n; k++) t += w[k] * a[k] * b[k] * c[k];
        return t;
    }
};

// The integral of conj(Y_l1m1) R_l2m2 Y_l3m3 over the sphere (the quantity of
// src/src_lib/gauntyry.f90), R the real harmonics of src/src_lib/genrlm.f90:
// R_l0 = Y_l0, R_lm = sqrt(2) Re Y_lm (m > 0), sqrt(2) Im Y_lm (m < 0).  The
// azimuthal integral is done analytically: with d = m3 - m1,
//   m2 = 0:   2 pi delta_{d,0}
//   m2 = k:   sqrt(2) pi (delta_{d,k} + delta_{d,-k})           (cos k phi)
//   m2 = -k: -sqrt(2) (-1)^k i pi (delta_{d,k} - delta_{d,-k})   (sin k phi)
// and the polar integral by the exact Gauss-Legendre rule of LegendreTable.
void gaunt_yry(const LegendreTable &t, int l1, int l2, int l3, int m1, int m2, int m3, double *re, double *im)
{
    *re = 0.0;
    *im = 0.0;
    if (std::abs(m1) > l1 || std::abs(m2) > l2 || std::abs(m3) > l3) return;
    if (l2 < std::abs(l1 - l3) || l2 > l1 + l3 || ((l1 + l2 + l3) & 1)) return;
    const int d = m3 - m1, k = std::abs(m2);
    if (std::abs(d) != k) return;
    const double s1 = (m1 < 0 && (m1 & 1)) ? -1.0 : 1.0;
    const double s3 = (m3 < 0 && (m3 & 1)) ? -1.0 : 1.0;
    const double T = s1 * s3 * t.triple(l1, m1, l2, m2, l3, m3);
    if (m2 == 0) {
        *re = 2.0 * PI * T;
    } else if (m2 > 0) {
        *re = std::sqrt(2.0) * PI * T;
    } else {
        const double sk = (k & 1) ? -1.0 : 1.0;
        *im = -std::sqrt(2.0) * sk * PI * T * (d > 0 ? 1.0 : -1.0);
    }
}

int legendre_points(int lsum) { return lsum / 2 + 2; }

// ------------------------------------------------------------------ device tables
struct RadFun {      // one radial function of a species
    int kind;        // 0: APW u_{l,io}, 1: local orbital
    int l;
    int idx;         // io or ilo
};

struct MtArgs {
    int natmtot, lmmaxvr, nslot, nradmax, nrmtmax, apwordmax, lmaxapw, nlomax, lmmaxmat;
    int g0;                        // first channel group of the launch (mt_radial_kernel)
    double a;                      // 0.5 alpha^2 for a relativistic valence, else 0
    const int *species;            // [natmtot]
    const int *nrmt;               // [nspecies]
    const int *nrad;               // [nspecies]
    const int4 *rfun;              // [nspecies][nradmax] {kind, l, idx, 0}
    const int *nrow_apw, *nrow_lo; // [nspecies]
    const int2 *rows;              // [nspecies][maxrows] {lm, p}
    int maxrows;
    const double *wr;              // [nspecies][2][nrmtmax]: spline weights, radii
    const double *apwfr, *lofr, *veffmt;
    double *rint;                  // [natmtot][nradmax (p)][nradmax (q)][nslot]
    int nsplit;                    // radial ranges per integral (mt_radial_kernel)
    double *rpart;                 // nsplit > 1: partial sums [split][natmtot][p][q][nslot]
    const int *gnt_off;            // [lmmaxmat^2 + 1]
    const int *gnt_lm2;            // [nnz]
    const double2 *gnt_val;        // [nnz]
    double *haa_r, *haa_i;         // [ias][f'][f], leading dim ldh
    int ldh;
    double *loa_r, *loa_i;         // [ias][f][r], leading dim ldlo
    int ldlo, maxaa, maxnlo;
    exs_complex *lolo;             // (maxnlo, maxnlo, natmtot)
    exs_complex *out_aa, *out_loa; // optional copies in the reference layouts
    double *oalo, *ololo;          // olprad outputs, reference layouts
    double *h1aa, *h1loa, *h1lolo; // iora* only (else null)
};

// Channels after the lmmaxvr potential channels of the radial integrals.
constexpr int CH_KIN = 0, CH_OVL = 1, CH_H1 = 2, NSPECIAL = 3;

constexpr int RC = 32;   // radial points per chunk

__device__ __forceinline__ const double *radfun(const MtArgs &a, int4 f, int ias)
{
    if (f.x == 0)
        return a.apwfr + (size_t)a.nrmtmax * 2 * (f.z + (size_t)a.apwordmax * (f.y + (size_t)(a.lmaxapw + 1) * ias));
    return a.lofr + (size_t)a.nrmtmax * 2 * (f.z + (size_t)a.nlomax * ias);
}

constexpr int SG = 8;    // potential channels per block of mt_radial_kernel

// grid (tile pairs tp <= tq, channel groups of the launch, natmtot), 8 T
// threads; group g = g0 + blockIdx.y.  Group g < ngroup: channels lm2 =
// SG g .. SG g + SG - 1 (< lmmaxvr),
//   I[lm2][p][q] = sum_r phi_p (phi_q w_r r^2) V_lm2(r);
// the staged radial functions serve all SG channels of the block.  Groups
// ngroup + CH_*: one channel each, stored at slot lmmaxvr + CH_*, with
// rm = 1 / (1 - a V_00 Y00):
//   CH_KIN (mt_kin.f90:98-150)  sum_r w_r rm (phi'_p phi'_q r^2 + l(l+1) phi_p phi_q) / 2
//   CH_OVL (olprad.f90:52-56)   sum_r w_r r^2 phi_p phi_q
//   CH_H1  (olprad.f90:30-44)   sum_r w_r a rm^2 (phi'_p phi'_q r^2 + l(l+1) phi_p phi_q) / 2
// the l(l+1) terms meaningful for equal l.  Tiles are T x T function
// pairs, T = 16, 24 or 32 chosen to fit the basis (the 21 radial functions
// of an lmaxmat 8 atom fill a 24 tile to 77 %, a 32 tile to 43 %); thread
// (tx, ty) = (i % T, i / T) owns q = tx and p = ty + 8 k, k < T / 8.  With
// nsplit > 1 (few atoms), blockIdx.y also selects one of nsplit contiguous
// ranges of 32-point chunks, and the block writes its partial sums to rpart
// (mt_reduce_kernel adds them in a fixed order).
template <int T>
__global__ void __launch_bounds__(8 * T, T == 16 ? 4 : (T == 24 ? 3 : 2)) mt_radial_kernel(MtArgs a)
{
    constexpr int KP = T / 8, NT = 8 * T;
    const int ias = blockIdx.z, grp = blockIdx.y / a.nsplit + a.g0, split = blockIdx.y % a.nsplit;
    const int is = a.species[ias];
    const int nrad = a.nrad[is], nr = a.nrmt[is];
    const int ntile = (a.nradmax + T - 1) / T;
    int t = blockIdx.x, tp = 0;
    while (tp < ntile && t >= ntile - tp) { t -= ntile - tp; tp++; }
    if (tp >= ntile) return;
    const int tq = tp + t;
    if (tp * T >= nrad || tq * T >= nrad) return;
    const int ngroup = (a.lmmaxvr + SG - 1) / SG;
    const bool kin = grp >= ngroup;             // one of the single-channel groups
    const int special = grp - ngroup;
    const int lm0 = grp * SG;
    __shared__ double sA[RC][T + 1], sB[RC][T + 1], sAd[RC][T + 1], sBd[RC][T + 1];
    __shared__ double sV[SG][RC];
    const int tx = threadIdx.x % T, ty = threadIdx.x / T;
    const double *w = a.wr + (size_t)is * 2 * a.nrmtmax, *rr = w + a.nrmtmax;
    const double *vat = a.veffmt + (size_t)a.lmmaxvr * a.nrmtmax * ias;
    double acc[KP][SG];
#pragma unroll
    for (int k = 0; k < KP; k++)
#pragma unroll
        for (int c = 0; c < SG; c++) acc[k][c] = 0.0;
    const int nchunk = (nr + RC - 1) / RC;
    const int c_end = (split + 1) * nchunk / a.nsplit;
    for (int r0 = split * nchunk / a.nsplit * RC; r0 < c_end * RC; r0 += RC) {
#pragma unroll
        for (int k = 0; k < (RC * T) / NT; k++) {
            const int i = threadIdx.x + NT * k;
            const int rl = i % RC, col = i / RC, r = r0 + rl;
            const int p = tp * T + col, q = tq * T + col;
            double fa = 0.0, fad = 0.0, fb = 0.0, fbd = 0.0;
            if (r < nr) {
                const double wt = w[r], x = rr[r];
                if (p < nrad) {
                    const double *f = radfun(a, a.rfun[is * a.nradmax + p], ias);
                    fa = f[r];
                    if (kin) fad = f[r + a.nrmtmax];
                }
                if (q < nrad) {
                    const int4 fq = a.rfun[is * a.nradmax + q];
                    const double *f = radfun(a, fq, ias);
                    if (!kin || special == CH_OVL) {
                        fb = f[r] * (wt * x * x);
                    } else {
                        const double rm = 1.0 / (1.0 - a.a * vat[(size_t)a.lmmaxvr * r] * Y00);
                        const double g = special == CH_KIN ? wt * rm * 0.5 : wt * a.a * rm * rm * 0.5;
                        fb = f[r] * (g * (double)(fq.y * (fq.y + 1)));
                        fbd = f[r + a.nrmtmax] * (g * x * x);
                    }
                }
            }
            sA[rl][col] = fa;
            sB[rl][col] = fb;
            sAd[rl][col] = fad;
            sBd[rl][col] = fbd;
        }
        if (!kin)   // V_lm2(r) of the block's channels: 8 consecutive lm2 per r
            for (int i = threadIdx.x; i < SG * RC; i += NT) {
                const int c = i % SG, rl = i / SG, r = r0 + rl;
                sV[c][rl] = (r < nr && lm0 + c < a.lmmaxvr) ? vat[lm0 + c + (size_t)a.lmmaxvr * r] : 0.0;
            }
        __syncthreads();
        if (kin) {
#pragma unroll 4
            for (int rl = 0; rl < RC; rl++) {
                const double b = sB[rl][tx], bd = sBd[rl][tx];
#pragma unroll
                for (int k = 0; k < KP; k++) acc[k][0] += sA[rl][ty + 8 * k] * b + sAd[rl][ty + 8 * k] * bd;
            }
        } else {
#pragma unroll 2
            for (int rl = 0; rl < RC; rl++) {
                const double b = sB[rl][tx];
                double bv[SG];
#pragma unroll
                for (int c = 0; c < SG; c++) bv[c] = b * sV[c][rl];
#pragma unroll
                for (int k = 0; k < KP; k++) {
                    const double av = sA[rl][ty + 8 * k];
#pragma unroll
                    for (int c = 0; c < SG; c++) acc[k][c] += av * bv[c];
                }
            }
        }
        __syncthreads();
    }
    const size_t nr2 = (size_t)a.nradmax * a.nradmax;
    double *out = (a.nsplit > 1 ? a.rpart + (size_t)split * a.natmtot * nr2 * a.nslot : a.rint) +
                  (size_t)ias * nr2 * a.nslot;
    const int q = tq * T + tx;
    const int nch = kin ? 1 : (a.lmmaxvr - lm0 < SG ? a.lmmaxvr - lm0 : SG);
#pragma unroll
    for (int k = 0; k < KP; k++) {
        const int p = tp * T + ty + 8 * k;
        if (p < nrad && q < nrad) {
#pragma unroll
            for (int c = 0; c < SG; c++) {
                if (c >= nch) break;
                const int slot = kin ? a.lmmaxvr + special : lm0 + c;
                out[((size_t)p * a.nradmax + q) * a.nslot + slot] = acc[k][c];
                if (tp != tq) out[((size_t)q * a.nradmax + p) * a.nslot + slot] = acc[k][c];
            }
        }
    }
}

// rint[x][s] = sum over the splits of rpart[split][x][s] for the channels
// s0 <= s < s1 of a launch, splits added in order.
__global__ void __launch_bounds__(256) mt_reduce_kernel(MtArgs a, int s0, int s1)
{
    const int ns = s1 - s0;
    const size_t nx = (size_t)a.natmtot * a.nradmax * a.nradmax, stride = nx * a.nslot;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nx * ns; i += (size_t)gridDim.x * blockDim.x) {
        const size_t o = (i / ns) * a.nslot + s0 + i % ns;
        double v = a.rpart[o];
        for (int sp = 1; sp < a.nsplit; sp++) v += a.rpart[sp * stride + o];
        a.rint[o] = v;
    }
}

// grid (row blocks of 32, column blocks of 8, natmtot), 256 threads: element
// (i, j) of the combined [APW rows | lo rows] matrix of one atom,
//   sum over the Gaunt list of (lm_i, lm_j) of g * I[lm2][p_i][p_j]
//   + I[kinetic][p_i][p_j] when lm_i = lm_j        (mt_kin.f90:150-225,
// mt_pot.f90:232-306); the APW x lo block (alo) is not stored.
__global__ void __launch_bounds__(256) mt_angular_kernel(MtArgs a)
{
    const int ias = blockIdx.z, is = a.species[ias];
    const int napw = a.nrow_apw[is], nrow = napw + a.nrow_lo[is];
    const int i = blockIdx.x * 32 + (threadIdx.x & 31), j = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (i >= nrow || j >= nrow || (i < napw && j >= napw)) return;
    const int2 ri = a.rows[is * a.maxrows + i], rj = a.rows[is * a.maxrows + j];
    const size_t nr2 = (size_t)a.nradmax * a.nradmax;
    const double *I = a.rint + ((size_t)ias * nr2 + (size_t)ri.y * a.nradmax + rj.y) * a.nslot;
    const int e0 = a.gnt_off[ri.x * a.lmmaxmat + rj.x], e1 = a.gnt_off[ri.x * a.lmmaxmat + rj.x + 1];
    double re = 0.0, im = 0.0;
    for (int e = e0; e < e1; e++) {
        const double v = I[a.gnt_lm2[e]];
        const double2 g = a.gnt_val[e];
        re += g.x * v;
        im += g.y * v;
    }
    if (ri.x == rj.x) re += I[a.lmmaxvr];
    if (i < napw) {                  // aa(i, j)
        const size_t o = (size_t)i + (size_t)a.ldh * (j + (size_t)a.ldh * ias);
        a.haa_r[o] = re;
        a.haa_i[o] = im;
        if (a.out_aa) a.out_aa[i + (size_t)a.maxaa * (j + (size_t)a.maxaa * ias)] = exs_complex{re, im};
    } else if (j < napw) {           // loa(i - napw, j)
        const int r = i - napw;
        const size_t o = (size_t)r + (size_t)a.ldlo * (j + (size_t)a.maxaa * ias);
        a.loa_r[o] = re;
        a.loa_i[o] = im;
        if (a.out_loa) a.out_loa[r + (size_t)a.maxnlo * (j + (size_t)a.maxaa * ias)] = exs_complex{re, im};
    } else {                         // lolo(i - napw, j - napw)
        a.lolo[(i - napw) + (size_t)a.maxnlo * ((j - napw) + (size_t)a.maxnlo * ias)] = exs_complex{re, im};
    }
}

__device__ __forceinline__ int find_radfun(const MtArgs &a, int is, int kind, int l, int idx)
{
    const int n = a.nrad[is];
    for (int p = 0; p < n; p++) {
        const int4 f = a.rfun[is * a.nradmax + p];
        if (f.x == kind && f.z == idx && (kind == 1 || f.y == l)) return p;
    }
    return -1;
}

// grid (natmtot), 256 threads: the olprad arrays of one atom from the
// overlap (and, for iora*, h1) channels; entries the reference does not
// visit (l > lmaxmat, io >= apword, lo pairs of different l) are zero.
__global__ void __launch_bounds__(256) mt_olprad_kernel(MtArgs a)
{
    const int ias = blockIdx.x, is = a.species[ias];
    const size_t nr2 = (size_t)a.nradmax * a.nradmax;
    const double *I = a.rint + (size_t)ias * nr2 * a.nslot;
    const double *Io = I + a.lmmaxvr + CH_OVL, *Ih = I + a.lmmaxvr + CH_H1;   // stride nslot per (p, q)
    const int ao = a.apwordmax, nlo = a.nlomax;
    for (int t = threadIdx.x; t < ao * nlo; t += blockDim.x) {        // oalo, h1loa (io, ilo)
        const int io = t % ao, ilo = t / ao;
        const int q = find_radfun(a, is, 1, 0, ilo);
        const int p = q < 0 ? -1 : find_radfun(a, is, 0, a.rfun[is * a.nradmax + q].y, io);
        const size_t o = (size_t)t + (size_t)ao * nlo * ias;
        a.oalo[o] = p < 0 ? 0.0 : Io[((size_t)p * a.nradmax + q) * a.nslot];
        if (a.h1loa) a.h1loa[o] = p < 0 ? 0.0 : Ih[((size_t)p * a.nradmax + q) * a.nslot];
    }
    for (int t = threadIdx.x; t < nlo * nlo; t += blockDim.x) {       // ololo, h1lolo (ilo1, ilo2)
        const int i1 = t % nlo, i2 = t / nlo;
        const int p = find_radfun(a, is, 1, 0, i1), q = find_radfun(a, is, 1, 0, i2);
        const bool ok = p >= 0 && q >= 0 && a.rfun[is * a.nradmax + p].y == a.rfun[is * a.nradmax + q].y;
        const size_t o = (size_t)t + (size_t)nlo * nlo * ias;
        a.ololo[o] = ok ? Io[((size_t)p * a.nradmax + q) * a.nslot] : 0.0;
        if (a.h1lolo) a.h1lolo[o] = ok ? Ih[((size_t)p * a.nradmax + q) * a.nslot] : 0.0;
    }
    if (a.h1aa)                                                        // h1aa (io1, io2, l)
        for (int t = threadIdx.x; t < ao * ao * (a.lmaxapw + 1); t += blockDim.x) {
            const int io1 = t % ao, io2 = (t / ao) % ao, l = t / (ao * ao);
            const int p = find_radfun(a, is, 0, l, io1), q = find_radfun(a, is, 0, l, io2);
            a.h1aa[(size_t)t + (size_t)ao * ao * (a.lmaxapw + 1) * ias] =
                (p < 0 || q < 0) ? 0.0 : Ih[((size_t)p * a.nradmax + q) * a.nslot];
        }
}

// ------------------------------------------------------------------ context state
struct MtState {
    // basis tables (fixed per context)
    bool basis_ready = false;
    int nradmax = 0, maxrows = 0;
    std::vector<int> nrad, nrow_apw, nrow_lo;
    std::vector<int4> rfun;
    std::vector<int2> rows;
    // Gaunt list for the current lmaxvr
    int lmaxvr = -1;
    std::vector<int> gnt_off, gnt_lm2;
    std::vector<double2> gnt_val;
    // spline weights for the current meshes
    std::vector<double> mesh_key;
    std::vector<int> nrmt_key;
    std::vector<double> wr;        // [nspecies][2][nrmtmax]
    int nrmtmax = 0;
    bool tables_dirty = true;
    // device buffers
    void *d_tab = nullptr;
    size_t tab_cap = 0;
    size_t off_species = 0, off_nrmt = 0, off_nrad = 0, off_rfun = 0, off_napw = 0, off_nlo = 0, off_rows = 0,
           off_wr = 0, off_goff = 0, off_glm2 = 0, off_gval = 0;
    double *d_rint = nullptr;
    size_t rint_cap = 0;
    double *d_rpart = nullptr;     // partial sums of split radial ranges
    size_t rpart_cap = 0;
    double *d_in = nullptr;        // uploaded apwfr | lofr | veffmt of the host-pointer call
    size_t in_cap = 0;
    exs_complex *d_out = nullptr;  // aa | loa in the reference layouts
    size_t out_cap = 0;
};

template <class T>
cudaError_t grow(T **p, size_t *cap, size_t n)
{
    if (n <= *cap && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) *cap = n;
    return e;
}

void build_basis_tables(const exs_ctx *c, MtState &m)
{
    const int nsp = c->nspecies;
    m.nrad.assign(nsp, 0);
    m.nrow_apw.assign(nsp, 0);
    m.nrow_lo.assign(nsp, 0);
    std::vector<std::vector<int4>> fun(nsp);
    std::vector<std::vector<int2>> rw(nsp);
    for (int is = 0; is < nsp; is++) {
        const int *apw = c->apword.data() + (size_t)(c->lmaxapw + 1) * is;
        std::vector<int> first(c->lmaxmat + 1, 0);
        for (int l = 0; l <= c->lmaxmat; l++) {
            first[l] = (int)fun[is].size();
            for (int io = 0; io < apw[l]; io++) fun[is].push_back(int4{0, l, io, 0});
        }
        const int nlo = c->nlorb[is];
        const int lo0 = (int)fun[is].size();
        for (int ilo = 0; ilo < nlo; ilo++) fun[is].push_back(int4{1, c->lorbl[ilo + (size_t)c->nlomax * is], ilo, 0});
        // APW rows in the order l, m, io (mt_pot.f90:236-241); lo rows ilo, m
        for (int l = 0; l <= c->lmaxmat; l++)
            for (int mm = -l; mm <= l; mm++)
                for (int io = 0; io < apw[l]; io++) rw[is].push_back(int2{l * (l + 1) + mm, first[l] + io});
        m.nrow_apw[is] = (int)rw[is].size();
        for (int ilo = 0; ilo < nlo; ilo++) {
            const int l = c->lorbl[ilo + (size_t)c->nlomax * is];
            for (int mm = -l; mm <= l; mm++) rw[is].push_back(int2{l * (l + 1) + mm, lo0 + ilo});
        }
        m.nrow_lo[is] = (int)rw[is].size() - m.nrow_apw[is];
        m.nrad[is] = (int)fun[is].size();
        m.nradmax = std::max(m.nradmax, m.nrad[is]);
        m.maxrows = std::max(m.maxrows, (int)rw[is].size());
    }
    m.rfun.assign((size_t)nsp * m.nradmax, int4{0, 0, 0, 0});
    m.rows.assign((size_t)nsp * m.maxrows, int2{0, 0});
    for (int is = 0; is < nsp; is++) {
        std::copy(fun[is].begin(), fun[is].end(), m.rfun.begin() + (size_t)is * m.nradmax);
        std::copy(rw[is].begin(), rw[is].end(), m.rows.begin() + (size_t)is * m.maxrows);
    }
    m.basis_ready = true;
    m.tables_dirty = true;
}

// Nonzero Gaunt coefficients gntyry(lm2, lm3, lm1) for lm1, lm3 of l <= lmaxmat
// and lm2 of l <= lmaxvr, grouped by (lm1, lm3) with lm2 ascending (the order
// of the reference's gntnonz list, init1.f90:575-595).
void build_gaunt_list(const exs_ctx *c, MtState &m, int lmaxvr)
{
    const int lmaxmat = c->lmaxmat, lmmaxmat = (lmaxmat + 1) * (lmaxmat + 1);
    LegendreTable t;
    t.build(std::max(lmaxmat, lmaxvr), legendre_points(2 * lmaxmat + lmaxvr));
    m.gnt_off.assign((size_t)lmmaxmat * lmmaxmat + 1, 0);
    m.gnt_lm2.clear();
    m.gnt_val.clear();
    for (int l1 = 0; l1 <= lmaxmat; l1++)
        for (int m1 = -l1; m1 <= l1; m1++)
            for (int l3 = 0; l3 <= lmaxmat; l3++)
                for (int m3 = -l3; m3 <= l3; m3++) {
                    const int lm1 = l1 * (l1 + 1) + m1, lm3 = l3 * (l3 + 1) + m3;
                    m.gnt_off[(size_t)lm1 * lmmaxmat + lm3] = (int)m.gnt_lm2.size();
                    const int k = std::abs(m3 - m1);
                    for (int l2 = std::max(k, std::abs(l1 - l3)); l2 <= std::min(lmaxvr, l1 + l3); l2++) {
                        const int cand[2] = {-k, k};
                        for (int ci = (k == 0 ? 1 : 0); ci < 2; ci++) {
                            double re, im;
                            gaunt_yry(t, l1, l2, l3, m1, cand[ci], m3, &re, &im);
                            if (std::hypot(re, im) > 1e-20) {
                                m.gnt_lm2.push_back(l2 * (l2 + 1) + cand[ci]);
                                m.gnt_val.push_back(double2{re, im});
                            }
                        }
                    }
                }
    // offsets were recorded at the start of each (lm1, lm3) group in loop
    // order, which is lm1-major and lm3-minor: the same as the index order
    m.gnt_off[(size_t)lmmaxmat * lmmaxmat] = (int)m.gnt_lm2.size();
    m.lmaxvr = lmaxvr;
    m.tables_dirty = true;
}

// Spline weights of each species' mesh (recomputed when a mesh changes).
bool update_weights(const exs_ctx *c, MtState &m, int nrmtmax, const int *nrmt, const double *spr)
{
    const int nsp = c->nspecies;
    std::vector<double> key(spr, spr + (size_t)nrmtmax * nsp);
    std::vector<int> nkey(nrmt, nrmt + nsp);
    if (m.nrmtmax == nrmtmax && key == m.mesh_key && nkey == m.nrmt_key) return false;
    m.wr.assign((size_t)nsp * 2 * nrmtmax, 0.0);
    for (int is = 0; is < nsp; is++) {
        const double *x = spr + (size_t)nrmtmax * is;
        double *w = m.wr.data() + (size_t)is * 2 * nrmtmax;
        spline_weights(nrmt[is], x, w);
        std::memcpy(w + nrmtmax, x, sizeof(double) * nrmt[is]);
    }
    m.mesh_key.swap(key);
    m.nrmt_key.swap(nkey);
    m.nrmtmax = nrmtmax;
    m.tables_dirty = true;
    return true;
}

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

int upload_tables(exs_ctx *c, MtState &m, cudaStream_t s)
{
    if (!m.tables_dirty) return EXS_OK;
    const int nsp = c->nspecies, nat = c->natmtot;
    std::vector<int> species(nat);
    for (int ias = 0; ias < nat; ias++) species[ias] = c->atom_species[ias];
    size_t o = 0;
    m.off_species = o; o = align_up(o + sizeof(int) * nat);
    m.off_nrmt = o;    o = align_up(o + sizeof(int) * nsp);
    m.off_nrad = o;    o = align_up(o + sizeof(int) * nsp);
    m.off_napw = o;    o = align_up(o + sizeof(int) * nsp);
    m.off_nlo = o;     o = align_up(o + sizeof(int) * nsp);
    m.off_rfun = o;    o = align_up(o + sizeof(int4) * m.rfun.size());
    m.off_rows = o;    o = align_up(o + sizeof(int2) * m.rows.size());
    m.off_wr = o;      o = align_up(o + sizeof(double) * m.wr.size());
    m.off_goff = o;    o = align_up(o + sizeof(int) * m.gnt_off.size());
    m.off_glm2 = o;    o = align_up(o + sizeof(int) * std::max<size_t>(m.gnt_lm2.size(), 1));
    m.off_gval = o;    o = align_up(o + sizeof(double2) * std::max<size_t>(m.gnt_val.size(), 1));
    std::vector<char> h(o, 0);
    auto put = [&](size_t off, const void *src, size_t bytes) { if (bytes) std::memcpy(h.data() + off, src, bytes); };
    put(m.off_species, species.data(), sizeof(int) * nat);
    put(m.off_nrmt, m.nrmt_key.data(), sizeof(int) * nsp);
    put(m.off_nrad, m.nrad.data(), sizeof(int) * nsp);
    put(m.off_napw, m.nrow_apw.data(), sizeof(int) * nsp);
    put(m.off_nlo, m.nrow_lo.data(), sizeof(int) * nsp);
    put(m.off_rfun, m.rfun.data(), sizeof(int4) * m.rfun.size());
    put(m.off_rows, m.rows.data(), sizeof(int2) * m.rows.size());
    put(m.off_wr, m.wr.data(), sizeof(double) * m.wr.size());
    put(m.off_goff, m.gnt_off.data(), sizeof(int) * m.gnt_off.size());
    put(m.off_glm2, m.gnt_lm2.data(), sizeof(int) * m.gnt_lm2.size());
    put(m.off_gval, m.gnt_val.data(), sizeof(double2) * m.gnt_val.size());
    MT_CUDA(cudaStreamSynchronize(s));   // the previous tables may still be read
    MT_CUDA(grow((char **)&m.d_tab, &m.tab_cap, o));
    MT_CUDA(cudaMemcpyAsync(m.d_tab, h.data(), o, cudaMemcpyHostToDevice, s));
    MT_CUDA(cudaStreamSynchronize(s));   // h is a pageable temporary
    m.tables_dirty = false;
    return EXS_OK;
}

template <class T>
cudaError_t ensure_dev(T **p, size_t n)
{
    if (*p || n == 0) return cudaSuccess;
    return cudaMalloc((void **)p, n * sizeof(T));
}

// Host-side preparation shared by both entry points; validates the sizes.
int prepare(exs_ctx *c, const exs_mt_radial *in, MtState **out)
{
    if (!c || !in || !in->nrmt || !in->spr || !in->apwfr || !in->veffmt)
        return mfail(c, EXS_ERR_ARG, "exs_hmlint: missing input array");
    if (c->nlotot > 0 && !in->lofr) return mfail(c, EXS_ERR_ARG, "exs_hmlint: lofr is required with local orbitals");
    if (in->lmaxvr < 0 || in->lmaxvr > 50) return mfail(c, EXS_ERR_SIZE, "exs_hmlint: lmaxvr outside 0..50");
    if (in->nrmtmax < 4) return mfail(c, EXS_ERR_SIZE, "exs_hmlint: nrmtmax < 4");
    for (int is = 0; is < c->nspecies; is++)
        if (in->nrmt[is] < 4 || in->nrmt[is] > in->nrmtmax)
            return mfail(c, EXS_ERR_SIZE, "exs_hmlint: nrmt outside 4..nrmtmax");
    MtState *m = (MtState *)c->mt;
    if (!m) {
        m = new MtState;
        c->mt = m;
    }
    if (!m->basis_ready) build_basis_tables(c, *m);
    if (m->lmaxvr != in->lmaxvr) build_gaunt_list(c, *m, in->lmaxvr);
    update_weights(c, *m, in->nrmtmax, in->nrmt, in->spr);
    *out = m;
    return EXS_OK;
}

// Arguments every launch of a call shares: tables, inputs, radial integrals.
int common_args(exs_ctx *c, MtState &m, int lmaxvr, const double *apwfr, const double *lofr, const double *veffmt,
                MtArgs &a, cudaStream_t s)
{
    const int nat = c->natmtot, lmmaxvr = (lmaxvr + 1) * (lmaxvr + 1);
    int rc = upload_tables(c, m, s);
    if (rc != EXS_OK) return rc;
    const size_t nslot = (size_t)lmmaxvr + NSPECIAL;
    MT_CUDA(grow(&m.d_rint, &m.rint_cap, (size_t)nat * nslot * m.nradmax * m.nradmax));
    a = MtArgs{};
    const char *tab = (const char *)m.d_tab;
    a.natmtot = nat;
    a.lmmaxvr = lmmaxvr;
    a.nslot = (int)nslot;
    a.nradmax = m.nradmax;
    a.nrmtmax = m.nrmtmax;
    a.apwordmax = c->apwordmax;
    a.lmaxapw = c->lmaxapw;
    a.nlomax = c->nlomax;
    a.lmmaxmat = (c->lmaxmat + 1) * (c->lmaxmat + 1);
    a.a = c->relativity != EXS_REL_NONE ? 0.5 * ALPHA * ALPHA : 0.0;
    a.species = (const int *)(tab + m.off_species);
    a.nrmt = (const int *)(tab + m.off_nrmt);
    a.nrad = (const int *)(tab + m.off_nrad);
    a.rfun = (const int4 *)(tab + m.off_rfun);
    a.nrow_apw = (const int *)(tab + m.off_napw);
    a.nrow_lo = (const int *)(tab + m.off_nlo);
    a.rows = (const int2 *)(tab + m.off_rows);
    a.maxrows = m.maxrows;
    a.wr = (const double *)(tab + m.off_wr);
    a.apwfr = apwfr;
    a.lofr = lofr;
    a.veffmt = veffmt;
    a.rint = m.d_rint;
    a.gnt_off = (const int *)(tab + m.off_goff);
    a.gnt_lm2 = (const int *)(tab + m.off_glm2);
    a.gnt_val = (const double2 *)(tab + m.off_gval);
    return EXS_OK;
}

// Radial integrals of channel groups g0 .. g0 + ngroups - 1, which fill the
// slots s0 .. s1 - 1.  When the grid would not cover the GPU twice (few
// atoms), the radial range is split over up to 4 blocks per integral and the
// partial sums are added by mt_reduce_kernel.
cudaError_t launch_radial(const MtArgs &a, MtState &m, int g0, int ngroups, int s0, int s1, cudaStream_t s)
{
    MtArgs b = a;
    b.g0 = g0;
    const int T = m.nradmax <= 16 ? 16 : (m.nradmax <= 24 ? 24 : 32);
    const int ntile = (m.nradmax + T - 1) / T;
    const long blocks = (long)ntile * (ntile + 1) / 2 * ngroups * a.natmtot;
    int nsplit = 1;
    int nsm = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    while (nsplit < 4 && blocks * nsplit < 2L * nsm) nsplit++;
    b.nsplit = nsplit;
    if (nsplit > 1) {
        const size_t n = (size_t)nsplit * a.natmtot * m.nradmax * m.nradmax * a.nslot;
        if (n > m.rpart_cap) {
            cudaError_t e = cudaStreamSynchronize(s);   // the old buffer may still be in use
            if (e == cudaSuccess) e = grow(&m.d_rpart, &m.rpart_cap, n);
            if (e != cudaSuccess) return e;
        }
        b.rpart = m.d_rpart;
    }
    const dim3 grid(ntile * (ntile + 1) / 2, ngroups * nsplit, a.natmtot);
    if (T == 16)
        mt_radial_kernel<16><<<grid, 8 * 16, 0, s>>>(b);
    else if (T == 24)
        mt_radial_kernel<24><<<grid, 8 * 24, 0, s>>>(b);
    else
        mt_radial_kernel<32><<<grid, 8 * 32, 0, s>>>(b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || nsplit == 1) return e;
    const size_t total = (size_t)a.natmtot * m.nradmax * m.nradmax * (s1 - s0);
    mt_reduce_kernel<<<(unsigned)std::min<size_t>((total + 255) / 256, 4 * (size_t)nsm), 256, 0, s>>>(b, s0, s1);
    return cudaGetLastError();
}

// hmlint: radial integrals (potential and kinetic channels), angular sums
// into the context's h_a / loa / lolo, then the split-precision slices of
// the new h_a.
int enqueue_hmlint(exs_ctx *c, MtState &m, int lmaxvr, const double *apwfr, const double *lofr,
                   const double *veffmt, bool want_out, cudaStream_t s)
{
    const int nat = c->natmtot, maxaa = c->maxaa, maxnlo = std::max(c->maxnlo, 1);
    MtArgs a;
    int rc = common_args(c, m, lmaxvr, apwfr, lofr, veffmt, a, s);
    if (rc != EXS_OK) return rc;
    MT_CUDA(ensure_dev(&c->d_haa_r, (size_t)nat * c->ldh * c->ldh));
    MT_CUDA(ensure_dev(&c->d_haa_i, (size_t)nat * c->ldh * c->ldh));
    MT_CUDA(ensure_dev(&c->d_loa_r, (size_t)nat * c->ldlo * maxaa));
    MT_CUDA(ensure_dev(&c->d_loa_i, (size_t)nat * c->ldlo * maxaa));
    MT_CUDA(ensure_dev(&c->d_lolo, (size_t)nat * maxnlo * maxnlo));
    const size_t naa = (size_t)maxaa * maxaa * nat, nloa = (size_t)maxnlo * maxaa * nat;
    if (want_out) MT_CUDA(grow(&m.d_out, &m.out_cap, naa + nloa));
    // rows and columns past a species' own block stay zero
    MT_CUDA(cudaMemsetAsync(c->d_haa_r, 0, sizeof(double) * nat * c->ldh * c->ldh, s));
    MT_CUDA(cudaMemsetAsync(c->d_haa_i, 0, sizeof(double) * nat * c->ldh * c->ldh, s));
    MT_CUDA(cudaMemsetAsync(c->d_loa_r, 0, sizeof(double) * nat * c->ldlo * maxaa, s));
    MT_CUDA(cudaMemsetAsync(c->d_loa_i, 0, sizeof(double) * nat * c->ldlo * maxaa, s));
    MT_CUDA(cudaMemsetAsync(c->d_lolo, 0, sizeof(exs_complex) * nat * maxnlo * maxnlo, s));
    if (want_out) MT_CUDA(cudaMemsetAsync(m.d_out, 0, sizeof(exs_complex) * (naa + nloa), s));
    a.haa_r = c->d_haa_r;
    a.haa_i = c->d_haa_i;
    a.ldh = c->ldh;
    a.loa_r = c->d_loa_r;
    a.loa_i = c->d_loa_i;
    a.ldlo = c->ldlo;
    a.maxaa = maxaa;
    a.maxnlo = maxnlo;
    a.lolo = c->d_lolo;
    a.out_aa = want_out ? m.d_out : nullptr;
    a.out_loa = want_out ? m.d_out + naa : nullptr;
    const int ngroup = (a.lmmaxvr + SG - 1) / SG;
    MT_CUDA(launch_radial(a, m, 0, ngroup + 1, 0, a.lmmaxvr + 1, s));   // potential groups + CH_KIN
    mt_angular_kernel<<<dim3((m.maxrows + 31) / 32, (m.maxrows + 7) / 8, nat), 256, 0, s>>>(a);
    MT_CUDA(cudaGetLastError());
    if (c->oz_on() && c->d_xs)
        MT_CUDA(exs::launch_oz_x(c->params(), c->oz_atom_args(), c->oz_sch, s));
    return EXS_OK;
}

// olprad: overlap (and for iora* the h1) channels, then the small arrays
// oalo, ololo (h1aa, h1loa, h1lolo) written into the context's copies.
int enqueue_olprad(exs_ctx *c, MtState &m, int lmaxvr, const double *apwfr, const double *lofr,
                   const double *veffmt, cudaStream_t s)
{
    const int nat = c->natmtot, ao = c->apwordmax, nlo = c->nlomax;
    const bool iora = c->relativity == EXS_REL_IORA;
    MtArgs a;
    int rc = common_args(c, m, lmaxvr, apwfr, lofr, veffmt, a, s);
    if (rc != EXS_OK) return rc;
    MT_CUDA(ensure_dev(&c->d_oalo, (size_t)ao * nlo * nat));
    MT_CUDA(ensure_dev(&c->d_ololo, (size_t)nlo * nlo * nat));
    a.oalo = c->d_oalo;
    a.ololo = c->d_ololo;
    if (iora) {
        MT_CUDA(ensure_dev(&c->d_h1aa, (size_t)ao * ao * (c->lmaxapw + 1) * nat));
        MT_CUDA(ensure_dev(&c->d_h1loa, (size_t)ao * nlo * nat));
        MT_CUDA(ensure_dev(&c->d_h1lolo, (size_t)nlo * nlo * nat));
        a.h1aa = c->d_h1aa;
        a.h1loa = c->d_h1loa;
        a.h1lolo = c->d_h1lolo;
    }
    const int ngroup = (a.lmmaxvr + SG - 1) / SG;
    MT_CUDA(launch_radial(a, m, ngroup + CH_OVL, iora ? 2 : 1, a.lmmaxvr + CH_OVL,
                          a.lmmaxvr + CH_OVL + (iora ? 2 : 1), s));   // CH_OVL (+ CH_H1)
    mt_olprad_kernel<<<nat, 256, 0, s>>>(a);
    MT_CUDA(cudaGetLastError());
    return EXS_OK;
}

// Radial inputs of a host-pointer call copied into the state's device buffer.
int upload_inputs(exs_ctx *c, MtState &m, const exs_mt_radial *in, const double **apwfr, const double **lofr,
                  const double **veffmt, cudaStream_t s)
{
    const int nat = c->natmtot, lmmaxvr = (in->lmaxvr + 1) * (in->lmaxvr + 1);
    const size_t n_apw = (size_t)in->nrmtmax * 2 * c->apwordmax * (c->lmaxapw + 1) * nat;
    const size_t n_lo = in->lofr ? (size_t)in->nrmtmax * 2 * c->nlomax * nat : 0;
    const size_t n_v = (size_t)lmmaxvr * in->nrmtmax * nat;
    MT_CUDA(cudaStreamSynchronize(s));   // the previous call's inputs may still be read
    MT_CUDA(grow(&m.d_in, &m.in_cap, n_apw + n_lo + n_v));
    MT_CUDA(cudaMemcpyAsync(m.d_in, in->apwfr, sizeof(double) * n_apw, cudaMemcpyHostToDevice, s));
    if (n_lo) MT_CUDA(cudaMemcpyAsync(m.d_in + n_apw, in->lofr, sizeof(double) * n_lo, cudaMemcpyHostToDevice, s));
    MT_CUDA(cudaMemcpyAsync(m.d_in + n_apw + n_lo, in->veffmt, sizeof(double) * n_v, cudaMemcpyHostToDevice, s));
    *apwfr = m.d_in;
    *lofr = n_lo ? m.d_in + n_apw : m.d_in;
    *veffmt = m.d_in + n_apw + n_lo;
    return EXS_OK;
}

int copy_out(exs_ctx *c, MtState &m, exs_complex *aa, exs_complex *loa, exs_complex *lolo, cudaStream_t s)
{
    const int nat = c->natmtot, maxaa = c->maxaa, maxnlo = std::max(c->maxnlo, 1);
    const size_t naa = (size_t)maxaa * maxaa * nat, nloa = (size_t)maxnlo * maxaa * nat;
    if (aa) MT_CUDA(cudaMemcpyAsync(aa, m.d_out, sizeof(exs_complex) * naa, cudaMemcpyDeviceToHost, s));
    if (loa) MT_CUDA(cudaMemcpyAsync(loa, m.d_out + naa, sizeof(exs_complex) * nloa, cudaMemcpyDeviceToHost, s));
    if (lolo)
        MT_CUDA(cudaMemcpyAsync(lolo, c->d_lolo, sizeof(exs_complex) * (size_t)maxnlo * maxnlo * nat,
                                cudaMemcpyDeviceToHost, s));
    return EXS_OK;
}

}  // namespace

namespace exs {
void mt_release(exs_ctx *c)
{
    MtState *m = (MtState *)c->mt;
    if (!m) return;
    if (m->d_tab) cudaFree(m->d_tab);
    if (m->d_rint) cudaFree(m->d_rint);
    if (m->d_rpart) cudaFree(m->d_rpart);
    if (m->d_in) cudaFree(m->d_in);
    if (m->d_out) cudaFree(m->d_out);
    delete m;
    c->mt = nullptr;
}
}  // namespace exs

extern "C" {

int exs_hmlint(exs_ctx *c, const exs_mt_radial *in, exs_complex *aa, exs_complex *loa, exs_complex *lolo)
{
    MtState *m = nullptr;
    int rc = prepare(c, in, &m);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const double *apwfr, *lofr, *veffmt;
    rc = upload_inputs(c, *m, in, &apwfr, &lofr, &veffmt, s);
    if (rc != EXS_OK) return rc;
    rc = enqueue_hmlint(c, *m, in->lmaxvr, apwfr, lofr, veffmt, aa || loa, s);
    if (rc != EXS_OK) return rc;
    rc = copy_out(c, *m, aa, loa, lolo, s);
    if (rc != EXS_OK) return rc;
    MT_CUDA(cudaStreamSynchronize(s));
    c->have_mt = true;
    return EXS_OK;
}

int exs_hmlint_device(exs_ctx *c, const exs_mt_radial *in)
{
    MtState *m = nullptr;
    int rc = prepare(c, in, &m);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    rc = enqueue_hmlint(c, *m, in->lmaxvr, in->apwfr, in->lofr ? in->lofr : in->apwfr, in->veffmt, false, c->stream);
    if (rc != EXS_OK) return rc;
    c->have_mt = true;
    return EXS_OK;
}

int exs_olprad(exs_ctx *c, const exs_mt_radial *in, double *oalo, double *ololo, double *h1aa, double *h1loa,
               double *h1lolo)
{
    MtState *m = nullptr;
    int rc = prepare(c, in, &m);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const double *apwfr, *lofr, *veffmt;
    rc = upload_inputs(c, *m, in, &apwfr, &lofr, &veffmt, s);
    if (rc != EXS_OK) return rc;
    rc = enqueue_olprad(c, *m, in->lmaxvr, apwfr, lofr, veffmt, s);
    if (rc != EXS_OK) return rc;
    const int nat = c->natmtot, ao = c->apwordmax, nlo = c->nlomax;
    const bool iora = c->relativity == EXS_REL_IORA;
    if (oalo) MT_CUDA(cudaMemcpyAsync(oalo, c->d_oalo, sizeof(double) * ao * nlo * nat, cudaMemcpyDeviceToHost, s));
    if (ololo) MT_CUDA(cudaMemcpyAsync(ololo, c->d_ololo, sizeof(double) * nlo * nlo * nat, cudaMemcpyDeviceToHost, s));
    if (iora && h1aa)
        MT_CUDA(cudaMemcpyAsync(h1aa, c->d_h1aa, sizeof(double) * ao * ao * (c->lmaxapw + 1) * nat,
                                cudaMemcpyDeviceToHost, s));
    if (iora && h1loa)
        MT_CUDA(cudaMemcpyAsync(h1loa, c->d_h1loa, sizeof(double) * ao * nlo * nat, cudaMemcpyDeviceToHost, s));
    if (iora && h1lolo)
        MT_CUDA(cudaMemcpyAsync(h1lolo, c->d_h1lolo, sizeof(double) * nlo * nlo * nat, cudaMemcpyDeviceToHost, s));
    MT_CUDA(cudaStreamSynchronize(s));
    c->have_olp = true;
    return EXS_OK;
}

int exs_olprad_device(exs_ctx *c, const exs_mt_radial *in)
{
    MtState *m = nullptr;
    int rc = prepare(c, in, &m);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    rc = enqueue_olprad(c, *m, in->lmaxvr, in->apwfr, in->lofr ? in->lofr : in->apwfr, in->veffmt, c->stream);
    if (rc != EXS_OK) return rc;
    c->have_olp = true;
    return EXS_OK;
}

int exs_gauntyry(int l1, int l2, int l3, int m1, int m2, int m3, double *re_im)
{
    if (!re_im || l1 < 0 || l2 < 0 || l3 < 0 || l1 > 50 || l2 > 50 || l3 > 50) return EXS_ERR_ARG;
    LegendreTable t;
    t.build(std::max(l1, std::max(l2, l3)), legendre_points(l1 + l2 + l3));
    gaunt_yry(t, l1, l2, l3, m1, m2, m3, re_im, re_im + 1);
    return EXS_OK;
}

int exs_fderiv_int(int n, const double *x, const double *f, double *result)
{
    if (n < 4 || !x || !f || !result) return EXS_ERR_ARG;
    std::vector<double> scratch(3 * (size_t)n);
    *result = spline_integral(n, x, f, scratch.data());
    return EXS_OK;
}

}  // extern "C"
