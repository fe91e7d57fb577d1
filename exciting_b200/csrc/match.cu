// APW matching coefficients on the device (src/match.f90:83-191).
//
// One thread per (G+k, atom, k-point).  The thread evaluates |G+k|, its
// angles (sphcrd), the structure factor e^{i(G+k).tau_a} (gensfacgp), the
// Bessel derivatives j_l^{(io-1)}(|G+k| R) (sbesseldm) and, l by l, the
// spherical harmonics (genylm's recursion restricted to that l), sets up the
// right-hand sides b_io and solves the small D_l system with the steps of
// zgesv.  Everything is FP64.
//
// Two output layouts:
//   * planes   -- A split into real/imaginary planes [f][G], f = stacked
//                 APW rows (atom, l, m, io), G contiguous (coalesced writes);
//                 the operand layout of the contraction kernels.
//   * apwalm   -- the reference's apwalm(ngkmax, apwordmax, lmmaxapw, natmtot).
#include "exs_internal.cuh"

namespace exs {

// D_l for atom ias (match.f90:136-148) factorised in place; returns info.
__device__ inline int match_dmat(const DevParams &p, int ias, int is, int l, int n, double *d, int *ipiv)
{
    const double *xa = p.spr_tail + (size_t)p.np_tail * is;
    const double rmt = p.rmt[is];
    for (int io2 = 0; io2 < n; io2++) {
        const double *ya = p.apwfr_tail +
            (size_t)p.np_tail * (io2 + (size_t)p.apwordmax * (l + (size_t)(p.lmaxapw + 1) * ias));
        for (int io1 = 0; io1 < n; io1++) d[io1 + n * io2] = polynom(io1, p.np_tail, xa, ya, rmt);
    }
    return lu_factor(n, d, ipiv);
}

// The per-(G, atom) work.  `write(l, m, io, re, im)` stores one coefficient;
// lmax_out is lmaxmat (planes) or lmaxapw (apwalm).
template <class W>
__device__ inline void match_point(const DevParams &p, int ias, double gpc, double theta, double phi,
                                   double sf_re, double sf_im, int lmax_out, W write)
{
    const int is = p.atoms[ias].species;
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * is;
    int omax = 0;
    for (int l = 0; l <= p.lmaxapw; l++) omax = max(omax, apw[l]);
    // djl(l, io) = gpc^(io-1) * j_l^(io-1)(gpc*rmt)   (match.f90:111-121)
    double djl[EXS_APWORD_MAX][EXS_LMAX_APW + 1];
    const double x = gpc * p.rmt[is];
    for (int io = 0; io < omax; io++) sbesseldm(io, p.lmaxapw, x, djl[io]);
    double t1 = 1.0;
    for (int io = 1; io < omax; io++) {
        t1 = t1 * gpc;
        for (int l = 0; l <= p.lmaxapw; l++) djl[io][l] *= t1;
    }
    const double fpso = 12.566370614359172954 / sqrt(p.omega);
    double sn, cs;
    sincos(theta, &sn, &cs);
    // e^{i m phi}, m = 1..lmax_out, once per point (the same values for every l)
    double cmt[EXS_LMAX_APW + 1], smt[EXS_LMAX_APW + 1];
    for (int mm = 1; mm <= lmax_out; mm++) sincos((double)mm * phi, &smt[mm], &cmt[mm]);
    double xm[EXS_LMAX_APW + 1];
    for (int l = 0; l <= lmax_out; l++) {
        const int n = apw[l];
        // D_l of this atom, factorised once per set of SCF inputs (match_dlu_kernel)
        double d[EXS_APWORD_MAX * EXS_APWORD_MAX];
        int ipiv[EXS_APWORD_MAX];
        const double *lu = p.dlu + ((size_t)ias * (p.lmaxapw + 1) + l) * DLU_STRIDE;
        for (int i = 0; i < n * n; i++) d[i] = lu[i];
        for (int i = 0; i < n; i++) ipiv[i] = (int)lu[9 + i];
        const int info = (int)lu[12];
        if (info != 0) atomicOr(p.err, DEV_WARN_SINGULAR);
        // zt2 = fpso * i^l * sfacgp
        double z1r = 0.0, z1i = 0.0;
        switch (l & 3) { case 0: z1r = fpso; break; case 1: z1i = fpso; break; case 2: z1r = -fpso; break; default: z1i = -fpso; }
        const double z2r = z1r * sf_re - z1i * sf_im;
        const double z2i = z1r * sf_im + z1i * sf_re;
        ylm_l(l, sn, cs, xm);
        for (int m = -l; m <= l; m++) {
            // Y_lm as genylm builds it: m > 0: x(m) e^{i m phi};
            // m < 0: (-1)^|m| conj(Y_{l,|m|})
            const int mm = m < 0 ? -m : m;
            double yr, yi;
            if (mm == 0) {
                yr = xm[0]; yi = 0.0;
            } else {
                yr = xm[mm] * cmt[mm]; yi = xm[mm] * smt[mm];
                if (m < 0) { yi = -yi; if (mm & 1) { yr = -yr; yi = -yi; } }
            }
            // b_io = djl(l, io) * zt2 * conj(Y_lm)
            const double wr = z2r * yr + z2i * yi;
            const double wi = z2i * yr - z2r * yi;
            double br[EXS_APWORD_MAX], bi[EXS_APWORD_MAX];
            for (int io = 0; io < n; io++) { br[io] = djl[io][l] * wr; bi[io] = djl[io][l] * wi; }
            if (info == 0) lu_solve(n, d, ipiv, br, bi);
            for (int io = 0; io < n; io++) write(l, m, io, br[io], bi[io]);
        }
    }
}

__global__ void match_planes_kernel(DevParams p, const KDesc *ks)
{
    const KDesc k = ks[blockIdx.z];
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int ias = blockIdx.y;
    if (g >= p.npad) return;
    const AtomDesc at = p.atoms[ias];
    double *ar = k.ar + (size_t)at.apw_off * p.npad + g;
    double *ai = k.ai + (size_t)at.apw_off * p.npad + g;
    if (g >= k.ngp) {
        for (int f = 0; f < at.napw; f++) { ar[(size_t)f * p.npad] = 0.0; ai[(size_t)f * p.npad] = 0.0; }
        return;
    }
    const double v[3] = {k.vgpc[3 * g], k.vgpc[3 * g + 1], k.vgpc[3 * g + 2]};
    double gpc, theta, phi;
    sphcrd(v, &gpc, &theta, &phi);
    double s, c;
    sincos(v[0] * at.pos[0] + v[1] * at.pos[1] + v[2] * at.pos[2], &s, &c);
    int f = 0;
    double amax = 0.0;
    match_point(p, ias, gpc, theta, phi, c, s, p.lmaxmat, [&](int, int, int, double re, double im) {
        ar[(size_t)f * p.npad] = re;
        ai[(size_t)f * p.npad] = im;
        amax = fmax(amax, fmax(fabs(re), fabs(im)));
        f++;
    });
    if (k.oz_scale) atomic_max_nonneg(k.oz_scale + g, amax);   // column maximum for the split-precision path
}

__global__ void match_ref_kernel(DevParams p, int ngp, int ngkmax, const double *gpc, const double *tpgpc,
                                 const exs_complex *sfacgp, exs_complex *apwalm)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int ias = blockIdx.y;
    if (g >= ngp) return;
    const exs_complex sf = sfacgp[g + (size_t)ngkmax * ias];
    const int is = p.atoms[ias].species;
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * is;
    exs_complex *out = apwalm + (size_t)ngkmax * p.apwordmax * p.lmmaxapw * ias + g;
    match_point(p, ias, gpc[g], tpgpc[2 * g], tpgpc[2 * g + 1], sf.re, sf.im, p.lmaxapw,
                [&](int l, int m, int io, double re, double im) {
                    const int lm = l * (l + 1) + m;
                    exs_complex z; z.re = re; z.im = im;
                    out[(size_t)ngkmax * (io + (size_t)p.apwordmax * lm)] = z;
                    if (io == apw[l] - 1)   // orders beyond apword(l) are not set by match: zero them
                        for (int j = apw[l]; j < p.apwordmax; j++) {
                            exs_complex zz; zz.re = 0.0; zz.im = 0.0;
                            out[(size_t)ngkmax * (j + (size_t)p.apwordmax * lm)] = zz;
                        }
                });
}

// apwalm (reference layout) -> A planes of one k-point.
__global__ void apwalm_to_planes_kernel(DevParams p, int ngp, const exs_complex *apwalm, double *ar, double *ai,
                                        double *amax_out)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int ias = blockIdx.y;
    if (g >= p.npad) return;
    const AtomDesc at = p.atoms[ias];
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * at.species;
    int f = at.apw_off;
    double amax = 0.0;
    for (int l = 0; l <= p.lmaxmat; l++)
        for (int m = -l; m <= l; m++) {
            const int lm = l * (l + 1) + m;
            for (int io = 0; io < apw[l]; io++, f++) {
                double re = 0.0, im = 0.0;
                if (g < ngp) {
                    const exs_complex z = apwalm[g + (size_t)p.ngkmax * (io + (size_t)p.apwordmax * (lm + (size_t)p.lmmaxapw * ias))];
                    re = z.re; im = z.im;
                }
                ar[(size_t)f * p.npad + g] = re;
                ai[(size_t)f * p.npad + g] = im;
                amax = fmax(amax, fmax(fabs(re), fabs(im)));
            }
        }
    if (amax_out) atomic_max_nonneg(amax_out + g, amax);
}

// (I + h1aa) A for the IORA overlap (overlapsetup.f90:72-87):
// C(f2) = A(f2) + sum_io1 h1aa(io1, io2, l, ias) A(f1), f = (l, m, io).
__global__ void iora_planes_kernel(DevParams p, const KDesc *ks)
{
    const KDesc k = ks[blockIdx.z];
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int ias = blockIdx.y;
    if (g >= p.npad) return;
    const AtomDesc at = p.atoms[ias];
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * at.species;
    int f = at.apw_off;
    for (int l = 0; l <= p.lmaxmat; l++) {
        const int n = apw[l];
        const double *h1 = p.h1aa + (size_t)p.apwordmax * p.apwordmax * (l + (size_t)(p.lmaxapw + 1) * ias);
        for (int m = -l; m <= l; m++, f += n) {
            for (int io2 = 0; io2 < n; io2++) {
                double re = k.ar[(size_t)(f + io2) * p.npad + g];
                double im = k.ai[(size_t)(f + io2) * p.npad + g];
                for (int io1 = 0; io1 < n; io1++) {
                    const double w = h1[io1 + (size_t)p.apwordmax * io2];
                    re += w * k.ar[(size_t)(f + io1) * p.npad + g];
                    im += w * k.ai[(size_t)(f + io1) * p.npad + g];
                }
                k.cr[(size_t)(f + io2) * p.npad + g] = re;
                k.ci[(size_t)(f + io2) * p.npad + g] = im;
            }
        }
    }
}

static const int MATCH_THREADS = 64;

// LU factors of D_l for every (atom, l <= lmaxapw) (match.f90:136-163):
// one thread per l, one block per atom.
__global__ void match_dlu_kernel(DevParams p, double *dlu)
{
    const int ias = blockIdx.x, l = threadIdx.x;
    if (l > p.lmaxapw) return;
    const int is = p.atoms[ias].species;
    const int n = p.apword[l + (size_t)(p.lmaxapw + 1) * is];
    double d[EXS_APWORD_MAX * EXS_APWORD_MAX];
    int ipiv[EXS_APWORD_MAX];
    const int info = match_dmat(p, ias, is, l, n, d, ipiv);
    double *out = dlu + ((size_t)ias * (p.lmaxapw + 1) + l) * DLU_STRIDE;
    for (int i = 0; i < 9; i++) out[i] = i < n * n ? d[i] : 0.0;
    for (int i = 0; i < 3; i++) out[9 + i] = i < n ? (double)ipiv[i] : 0.0;
    out[12] = (double)info;
}

cudaError_t launch_match_dlu(const DevParams &p, double *dlu, cudaStream_t s)
{
    match_dlu_kernel<<<p.natmtot, 32 * ((p.lmaxapw + 32) / 32), 0, s>>>(p, dlu);
    return cudaGetLastError();
}

cudaError_t launch_match_planes(const DevParams &p, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s)
{
    (void)ngp_max;
    dim3 grid((p.npad + MATCH_THREADS - 1) / MATCH_THREADS, p.natmtot, nk);
    match_planes_kernel<<<grid, MATCH_THREADS, 0, s>>>(p, d_k);
    return cudaGetLastError();
}

cudaError_t launch_match_ref(const DevParams &p, int ngp, int ngkmax, const double *gpc, const double *tpgpc,
                             const exs_complex *sfacgp, exs_complex *apwalm, cudaStream_t s)
{
    if (ngp <= 0) return cudaSuccess;
    dim3 grid((ngp + MATCH_THREADS - 1) / MATCH_THREADS, p.natmtot, 1);
    match_ref_kernel<<<grid, MATCH_THREADS, 0, s>>>(p, ngp, ngkmax, gpc, tpgpc, sfacgp, apwalm);
    return cudaGetLastError();
}

cudaError_t launch_apwalm_to_planes(const DevParams &p, int ngp, const exs_complex *apwalm, double *ar,
                                    double *ai, double *amax, cudaStream_t s)
{
    dim3 grid((p.npad + 127) / 128, p.natmtot, 1);
    apwalm_to_planes_kernel<<<grid, 128, 0, s>>>(p, ngp, apwalm, ar, ai, amax);
    return cudaGetLastError();
}

cudaError_t launch_iora_planes(const DevParams &p, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s)
{
    (void)ngp_max;
    dim3 grid((p.npad + 127) / 128, p.natmtot, nk);
    iora_planes_kernel<<<grid, 128, 0, s>>>(p, d_k);
    return cudaGetLastError();
}

}  // namespace exs
