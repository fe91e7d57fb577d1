/*
 * ORACLE -- test infrastructure only.  A plain-C, FP64 restatement of the
 * reference's per-k-point LAPW H/O setup, used by the tests, by the smoke
 * check and by the benchmark's CPU-baseline leg as the checker.  It is never
 * part of the shipped library and nothing on the product path calls it.
 *
 * Each routine follows the reference Fortran named beside it (paths relative
 * to the exciting source tree).  Arrays use the reference's column-major
 * layout; integer tables keep the reference's 1-based values.
 *
 * The dense zgemm products of hamiltonsetup/overlapsetup/forcek are done in
 * the Python half of the oracle (numpy, OpenBLAS); this file holds the special
 * functions, the matching coefficients, the interstitial gathers and the
 * local-orbital blocks.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <stdlib.h>

typedef double complex zdouble;

#define ORC_FOURPI 12.566370614359172954

/* ---- src/src_lib/factnm.f90:13-88 (only what sbesseldm needs) ---------- */
static double orc_factnm(int n, int m)
{
    static const double f1[24] = {1., 2., 6., 24., 120., 720., 5040., 40320., 362880.,
        3628800., 39916800., 479001600., 6227020800., 87178291200., 1307674368000.,
        20922789888000., 355687428096000., 6402373705728000., 121645100408832000.,
        2432902008176640000., 51090942171709440000., 1124000727777607680000.,
        25852016738884976640000., 620448401733239439360000.};
    static const double f2[38] = {1., 2., 3., 8., 15., 48., 105., 384., 945., 3840.,
        10395., 46080., 135135., 645120., 2027025., 10321920., 34459425., 185794560.,
        654729075., 3715891200., 13749310575., 81749606400., 316234143225.,
        1961990553600., 7905853580625., 51011754393600., 213458046676875.,
        1428329123020800., 6190283353629375., 42849873690624000.,
        191898783962510625., 1371195958099968000., 6332659870762850625.,
        46620662575398912000., 221643095476699771875., 1678343852714360832000.,
        8200794532637891559375., 63777066403145711616000.};
    if (n == 0) return 1.0;
    if (m == 1 && n >= 1 && n <= 24) return f1[n - 1];
    if (m == 2 && n >= 1 && n <= 38) return f2[n - 1];
    double r;
    if (m == 1) {
        r = f1[23];
        for (int i = 25; i <= n; i++) r *= (double)i;
    } else {
        int j = n / m;
        if (n % m == 0) j--;
        r = (double)n;
        for (int i = 1; i <= j; i++) r *= (double)(n - i * m);
    }
    return r;
}

/* x**j for integer j >= 0 by binary powering (Fortran real**integer) */
static double orc_powi(double x, int j)
{
    double r = 1.0;
    while (j > 0) {
        if (j & 1) r *= x;
        x *= x;
        j >>= 1;
    }
    return r;
}

/* ---- src/src_lib/factr.f90 ------------------------------------------- */
static double orc_factr(int n, int d)
{
    double r;
    if (n < d) {
        r = 1.0 / (double)(n + 1);
        for (int i = n + 2; i <= d; i++) r /= (double)i;
    } else if (n == d) {
        r = 1.0;
    } else {
        r = (double)(d + 1);
        for (int i = d + 2; i <= n; i++) r *= (double)i;
    }
    return r;
}

/* ---- src/src_lib/sbessel.f90:48-147 ------------------------------------
 * j_l(x) for l = 0..lmax: series for x < 1e-8, Miller downward recursion from
 * lmax+25 with rescaling for x < lmax, upward recursion otherwise.
 * Returns 0, or -1 for an argument outside the reference's accepted range. */
int orc_sbessel(int lmax, double x, double *jl)
{
    const int lst = 25;
    const double rsc = 1e150, rsci = 1.0 / 1e150;
    if (lmax < 0 || lmax > 50) return -1;
    if (x < 0.0 || x > 1e5) return -1;
    if (x < 1e-8) {
        jl[0] = 1.0;
        double t1 = 1.0, t2 = 1.0;
        for (int l = 1; l <= lmax; l++) {
            t1 = t1 / (double)(2 * l + 1);
            t2 = t2 * x;
            jl[l] = t2 * t1;
        }
        return 0;
    }
    double xi = 1.0 / x;
    if (x < (double)lmax) {
        double j0 = 0.6370354636449841609 * rsci;
        double j1 = 0.3532702964695481204 * rsci;
        double jt;
        for (int l = lmax + lst; l >= lmax + 1; l--) {
            jt = j0 * (double)(2 * l + 1) * xi - j1;
            j1 = j0;
            j0 = jt;
            if (fabs(j0) > rsc) {
                jt *= rsci; j1 *= rsci; j0 *= rsci;
            }
        }
        for (int l = lmax; l >= 0; l--) {
            jt = j0 * (double)(2 * l + 1) * xi - j1;
            j1 = j0;
            j0 = jt;
            if (fabs(j0) > rsc) {
                jt *= rsci; j1 *= rsci; j0 *= rsci;
                for (int k = l + 1; k <= lmax; k++) jl[k] *= rsci;
            }
            jl[l] = j1;
        }
        double t1 = 1.0 / ((jl[0] - x * jl[1]) * cos(x) + x * jl[0] * sin(x));
        for (int l = 0; l <= lmax; l++) jl[l] = t1 * jl[l];
        return 0;
    }
    jl[0] = sin(x) * xi;
    if (lmax == 0) return 0;
    jl[1] = (jl[0] - cos(x)) * xi;
    if (lmax == 1) return 0;
    double j0 = jl[0], j1 = jl[1], jt;
    for (int l = 2; l <= lmax; l++) {
        jt = (double)(2 * l - 1) * j1 * xi - j0;
        j0 = j1;
        j1 = jt;
        jl[l] = j1;
    }
    return 0;
}

/* ---- src/src_lib/sbesseldm.f90:40-130 ----------------------------------
 * m-th derivative of j_l(x), l = 0..lmax (m <= 6, lmax <= 30). */
int orc_sbesseldm(int m, int lmax, double x, double *djl)
{
    const int maxm = 6, maxns = 20;
    if (m < 0 || m > maxm) return -1;
    if (lmax < 0 || lmax > 30) return -1;
    if (x < 0.0 || x > 1e5) return -1;
    if (m == 0) return orc_sbessel(lmax, x, djl);
    if (x > 1.0) {
        double jl[32];
        int a[8], a1[8], b[8], b1[8];
        orc_sbessel(lmax + 1, x, jl);
        for (int l = 0; l <= lmax; l++) {
            for (int i = 1; i <= m + 1; i++) a[i] = 0;
            a[0] = 1;
            for (int i = 0; i <= m + 1; i++) a1[i] = 0;
            for (int i = 1; i <= m; i++) {
                b[0] = 0;
                b1[0] = 0;
                for (int j = 0; j <= i; j++) {
                    b[j + 1] = a[j] * (l - j);
                    b1[j + 1] = -a1[j] * (j + l + 2);
                }
                for (int j = 0; j <= i; j++) {
                    b1[j] = b1[j] - a[j];
                    b[j] = b[j] + a1[j];
                }
                for (int j = 0; j <= i + 1; j++) { a[j] = b[j]; a1[j] = b1[j]; }
            }
            double t1 = 1.0;
            double sum = (double)a[0] * jl[l] + (double)a1[0] * jl[l + 1];
            for (int i = 1; i <= m + 1; i++) {
                t1 = t1 * x;
                sum = sum + ((double)a[i] * jl[l] + (double)a1[i] * jl[l + 1]) / t1;
            }
            djl[l] = sum;
        }
    } else {
        double x2 = x * x;
        for (int l = 0; l <= lmax; l++) {
            int i0 = (m - l + 1) / 2;
            if (i0 < 0) i0 = 0;
            /* Fortran integer division truncates toward zero, as C's does */
            int j = 2 * i0 + l - m;
            double t1 = (j == 0) ? 1.0 : orc_powi(x, j);
            double p2 = orc_powi(-2.0, i0);
            t1 = orc_factr(j + m, j) * t1 / (orc_factnm(i0, 1) * orc_factnm(j + l + m + 1, 2) * p2);
            double sum = t1;
            for (int i = i0 + 1; i <= maxns; i++) {
                j = 2 * i + l;
                t1 = -t1 * (double)((j - 1) * j) * x2
                     / (double)((j - l) * (j - m - 1) * (j - m) * (j + l + 1));
                if (fabs(t1) <= 1e-40) break;
                sum = sum + t1;
            }
            djl[l] = sum;
        }
    }
    return 0;
}

/* ---- src/src_lib/genylm.f90:36-93 --------------------------------------
 * Complex Y_lm with the Condon-Shortley phase, packed lm = l(l+1)+m (0-based),
 * Masters & Richards-Dinger recursion. */
int orc_genylm(int lmax, const double *tp, zdouble *ylm)
{
    if (lmax < 0 || lmax > 50) return -1;
    double x[51];
    zdouble z[51];
    ylm[0] = 0.28209479177387814347;
    if (lmax == 0) return 0;
    double sn = sin(tp[0]), cs = cos(tp[0]);
    for (int m = 1; m <= lmax; m++) {
        double t1 = (double)m * tp[1];
        z[m] = cos(t1) + I * sin(t1);
    }
    for (int l = 1; l <= lmax; l++) {
        x[l] = (l % 2 == 0) ? 1.0 : -1.0;
        double dx = 0.0;
        for (int m = l; m >= 1; m--) {
            double t1 = sqrt((double)((l + m) * (l - m + 1)));
            x[m - 1] = -(sn * dx + (double)(2 * m) * cs * x[m]) / t1;
            dx = sn * x[m] * t1;
        }
        double t1 = sn, sum = 0.0;
        for (int m = 1; m <= l; m++) {
            x[m] = t1 * x[m];
            sum = sum + x[m] * x[m];
            t1 = t1 * sn;
        }
        sum = 2.0 * sum + x[0] * x[0];
        t1 = sqrt((double)(2 * l + 1) / (ORC_FOURPI * sum));
        int lm1 = l * (l + 1), lm2 = lm1;
        ylm[lm1] = t1 * x[0];
        for (int m = 1; m <= l; m++) {
            lm1++;
            lm2--;
            ylm[lm1] = t1 * x[m] * z[m];
            ylm[lm2] = conj(ylm[lm1]);
            if (m % 2 != 0) ylm[lm2] = -ylm[lm2];
        }
    }
    return 0;
}

/* ---- src/src_lib/polynom.f90:11-196 ------------------------------------
 * m-th derivative at x of the polynomial through np points (m >= 0 only;
 * the integral branch m < 0 is not used on this path). */
double orc_polynom(int m, int np, const double *xa, const double *ya, double *c, double x)
{
    double x0, x1, x2, x3, y1, y2, y3, t1, t2, t3, t4, t5, t6, t7, sum;
    switch (np) {
    case 1:
        return (m == 0) ? ya[0] : 0.0;
    case 2:
        c[1] = (ya[1] - ya[0]) / (xa[1] - xa[0]);
        t1 = x - xa[0];
        if (m == 0) return c[1] * t1 + ya[0];
        if (m == 1) return c[1];
        return 0.0;
    case 3:
        x1 = xa[1] - xa[0]; x2 = xa[2] - xa[0];
        y1 = ya[1] - ya[0]; y2 = ya[2] - ya[0];
        t1 = 1.0 / (x1 * x2 * (x2 - x1));
        t2 = x1 * y2; t3 = x2 * y1;
        c[1] = t1 * (x2 * t3 - x1 * t2);
        c[2] = t1 * (t2 - t3);
        t1 = x - xa[0];
        if (m == 0) return ya[0] + t1 * (c[1] + c[2] * t1);
        if (m == 1) return 2.0 * c[2] * t1 + c[1];
        if (m == 2) return 2.0 * c[2];
        return 0.0;
    case 4:
        x1 = xa[1] - xa[0]; x2 = xa[2] - xa[0]; x3 = xa[3] - xa[0];
        y1 = ya[1] - ya[0]; y2 = ya[2] - ya[0]; y3 = ya[3] - ya[0];
        t1 = 1.0 / (x1 * x2 * x3 * (x1 - x2) * (x1 - x3) * (x2 - x3));
        t2 = x1 * x2 * y3; t3 = x2 * x3 * y1; t4 = x3 * x1 * y2;
        t5 = x1 * x1; t6 = x2 * x2; t7 = x3 * x3;
        c[1] = t1 * (t3 * (x3 * t6 - x2 * t7) + t4 * (x1 * t7 - x3 * t5) + t2 * (x2 * t5 - x1 * t6));
        c[2] = t1 * (t3 * (t7 - t6) + t4 * (t5 - t7) + t2 * (t6 - t5));
        c[3] = t1 * (t3 * (x2 - x3) + t4 * (x3 - x1) + t2 * (x1 - x2));
        t1 = x - xa[0];
        if (m == 0) return ya[0] + t1 * (c[1] + t1 * (c[2] + c[3] * t1));
        if (m == 1) return c[1] + t1 * (2.0 * c[2] + 3.0 * c[3] * t1);
        if (m == 2) return 6.0 * c[3] * t1 + 2.0 * c[2];
        if (m == 3) return 6.0 * c[3];
        return 0.0;
    default:
        break;
    }
    if (np <= 0 || m >= np) return 0.0;
    for (int i = 0; i < np; i++) c[i] = ya[i];
    for (int i = 2; i <= np; i++)
        for (int j = np; j >= i; j--)
            c[j - 1] = (c[j - 1] - c[j - 2]) / (xa[j - 1] - xa[j - i]);
    if (m == 0) {
        sum = c[0];
        t1 = 1.0;
        for (int i = 2; i <= np; i++) {
            t1 = t1 * (x - xa[i - 2]);
            sum = sum + c[i - 1] * t1;
        }
        return sum;
    }
    x0 = xa[0];
    for (int j = 1; j <= np - 1; j++)
        for (int i = 1; i <= np - j; i++) {
            int k = np - i;
            c[k - 1] = c[k - 1] + (x0 - xa[k - j]) * c[k];
        }
    for (int j = 1; j <= m; j++)
        for (int i = m + 1; i <= np; i++) c[i - 1] = c[i - 1] * (double)(i - j);
    t1 = c[np - 1];
    t2 = x - x0;
    for (int i = np - 1; i >= m + 1; i--) t1 = t1 * t2 + c[i - 1];
    return t1;
}

/* ---- small dense solve, the steps of LAPACK zgesv for n <= 4 -------------
 * D (n x n, real-valued as the reference's zd) is factored with partial
 * pivoting (largest |d|), the sub-diagonal scaled by the reciprocal of the
 * pivot, then each right-hand side is permuted, forward- and back-substituted
 * (division by the U diagonal).  Returns 0, or k > 0 if U(k,k) is exactly 0,
 * in which case the right-hand sides are left untouched (zgesv's contract). */
int orc_lu_factor(int n, double *d /* n*n col-major, overwritten */, int *ipiv)
{
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(d[k + k * n]);
        for (int i = k + 1; i < n; i++)
            if (fabs(d[i + k * n]) > best) { best = fabs(d[i + k * n]); p = i; }
        ipiv[k] = p;
        if (d[p + k * n] == 0.0) return k + 1;
        if (p != k)
            for (int j = 0; j < n; j++) {
                double t = d[k + j * n]; d[k + j * n] = d[p + j * n]; d[p + j * n] = t;
            }
        double r = 1.0 / d[k + k * n];
        for (int i = k + 1; i < n; i++) d[i + k * n] *= r;
        for (int j = k + 1; j < n; j++)
            for (int i = k + 1; i < n; i++) d[i + j * n] -= d[i + k * n] * d[k + j * n];
    }
    return 0;
}

void orc_lu_solve(int n, const double *d, const int *ipiv, zdouble *b)
{
    for (int k = 0; k < n; k++)
        if (ipiv[k] != k) { zdouble t = b[k]; b[k] = b[ipiv[k]]; b[ipiv[k]] = t; }
    for (int k = 0; k < n; k++)
        for (int i = k + 1; i < n; i++) b[i] -= b[k] * d[i + k * n];
    for (int k = n - 1; k >= 0; k--) {
        b[k] = b[k] / d[k + k * n];
        for (int i = 0; i < k; i++) b[i] -= b[k] * d[i + k * n];
    }
}

/* ---- src/match.f90:83-191 ---------------------------------------------
 * apwalm(ngkmax, apwordmax, lmmaxapw, natmtot).  The last np radial points of
 * the mesh and of the radial functions are passed as tails:
 *   spr_tail(np, nspecies), apwfr_tail(np, apwordmax, 0:lmaxapw, natmtot).
 * Returns the number of (atom, l) pairs whose matching system was singular
 * (the reference prints those and carries on, match.f90:166-175). */
int orc_match(int ngp, int ngkmax, const double *gpc, const double *tpgpc, const zdouble *sfacgp,
              int natmtot, const int *atom_species, int lmaxapw, int apwordmax,
              const int *apword /* (lmaxapw+1, nspecies) */, const double *rmt, double omega,
              int np, const double *spr_tail, const double *apwfr_tail, zdouble *apwalm)
{
    const int lmmaxapw = (lmaxapw + 1) * (lmaxapw + 1);
    const double fpso = ORC_FOURPI / sqrt(omega);
    int nsing = 0;
    zdouble *ylmgp = (zdouble *)malloc(sizeof(zdouble) * lmmaxapw * (ngp > 0 ? ngp : 1));
    double *djl = (double *)malloc(sizeof(double) * (lmaxapw + 1) * apwordmax * (ngp > 0 ? ngp : 1));
    /* spherical harmonics of the G+p vectors (match.f90:93-101) */
#pragma omp parallel for schedule(static)
    for (int igp = 0; igp < ngp; igp++) orc_genylm(lmaxapw, tpgpc + 2 * igp, ylmgp + (size_t)lmmaxapw * igp);
    int last_is = -1;
    for (int ias = 0; ias < natmtot; ias++) {
        const int is = atom_species[ias];
        const int *apw = apword + (size_t)(lmaxapw + 1) * is;
        if (is != last_is) {
            /* Bessel derivatives for this species (match.f90:104-126) */
            int omax = 0;
            for (int l = 0; l <= lmaxapw; l++) if (apw[l] > omax) omax = apw[l];
#pragma omp parallel for schedule(static)
            for (int igp = 0; igp < ngp; igp++) {
                double *dj = djl + (size_t)(lmaxapw + 1) * apwordmax * igp;
                double t1 = gpc[igp] * rmt[is];
                for (int io1 = 1; io1 <= omax; io1++) orc_sbesseldm(io1 - 1, lmaxapw, t1, dj + (lmaxapw + 1) * (io1 - 1));
                t1 = 1.0;
                for (int io1 = 2; io1 <= omax; io1++) {
                    t1 = t1 * gpc[igp];
                    for (int l = 0; l <= lmaxapw; l++) dj[l + (lmaxapw + 1) * (io1 - 1)] *= t1;
                }
            }
            last_is = is;
        }
        for (int l = 0; l <= lmaxapw; l++) {
            /* zt1 = fpso * i^l */
            zdouble zil;
            switch (l % 4) { case 0: zil = 1.0; break; case 1: zil = I; break; case 2: zil = -1.0; break; default: zil = -I; }
            zdouble zt1 = fpso * zil;
            const int n = apw[l];
            double dmat[16];
            int ipiv[4];
            double c[8];
            const double *xa = spr_tail + (size_t)np * is;
            for (int io2 = 0; io2 < n; io2++)
                for (int io1 = 0; io1 < n; io1++) {
                    const double *ya = apwfr_tail + (size_t)np * (io2 + apwordmax * (l + (lmaxapw + 1) * (size_t)ias));
                    dmat[io1 + n * io2] = orc_polynom(io1, np, xa, ya, c, rmt[is]);
                }
            int info = orc_lu_factor(n, dmat, ipiv);
            if (info != 0) nsing++;
#pragma omp parallel for schedule(static)
            for (int igp = 0; igp < ngp; igp++) {
                const double *dj = djl + (size_t)(lmaxapw + 1) * apwordmax * igp;
                zdouble zt2 = zt1 * sfacgp[igp + (size_t)ngkmax * ias];
                for (int m = -l; m <= l; m++) {
                    int lm = l * (l + 1) + m;
                    zdouble b[4];
                    zdouble cy = conj(ylmgp[lm + (size_t)lmmaxapw * igp]);
                    for (int io1 = 0; io1 < n; io1++) b[io1] = dj[l + (lmaxapw + 1) * io1] * zt2 * cy;
                    if (info == 0) orc_lu_solve(n, dmat, ipiv, b);
                    for (int io1 = 0; io1 < n; io1++)
                        apwalm[igp + (size_t)ngkmax * (io1 + (size_t)apwordmax * (lm + (size_t)lmmaxapw * ias))] = b[io1];
                }
            }
        }
    }
    free(ylmgp);
    free(djl);
    return nsing;
}

/* ---- src/src_eigensystem/hmlistln.f90:61-86 and olpistln.f90:53-82 ------
 * Interstitial H and O, added to the upper triangle za(i, j), i <= j
 * (Hermitianmatrix_indexedupdate, modfvsystem.f90:126-143).
 * kinw is meffig (ValenceRelativity /= "none") or cfunig ("none").
 * With h1on (iora*), O also gets 0.5*a2*(vgpc_i.vgpc_j)*m2effig. */
void orc_hmlistln_olpistln(int ngp, const int *igpig, const double *vgpc, int ld,
                           const int *ivg, const int *ivgig, const int *intgv /* (3,2) */, int ngvec,
                           const zdouble *veffig, const zdouble *kinw, const zdouble *cfunig,
                           const zdouble *m2effig, int h1on, zdouble *h, zdouble *o)
{
    const double alpha = 1.0 / 137.03599911, a2 = 0.5 * alpha * alpha;
    const int n1 = intgv[3] - intgv[0] + 1, n2 = intgv[4] - intgv[1] + 1;
#pragma omp parallel for schedule(dynamic, 8)
    for (int j = 0; j < ngp; j++) {
        const int gj = igpig[j] - 1;
        for (int i = 0; i <= j; i++) {
            const int gi = igpig[i] - 1;
            int iv1 = ivg[3 * gi + 0] - ivg[3 * gj + 0];
            int iv2 = ivg[3 * gi + 1] - ivg[3 * gj + 1];
            int iv3 = ivg[3 * gi + 2] - ivg[3 * gj + 2];
            int ig = ivgig[(iv1 - intgv[0]) + n1 * ((iv2 - intgv[1]) + n2 * (iv3 - intgv[2]))];
            if (ig > 0 && ig <= ngvec) {
                double dp = vgpc[3 * i] * vgpc[3 * j] + vgpc[3 * i + 1] * vgpc[3 * j + 1] + vgpc[3 * i + 2] * vgpc[3 * j + 2];
                double t1 = 0.5 * dp;
                if (h) h[i + (size_t)ld * j] += veffig[ig - 1] + t1 * kinw[ig - 1];
                if (o) {
                    if (h1on) o[i + (size_t)ld * j] += (0.5 * a2 * dp) * m2effig[ig - 1] + cfunig[ig - 1];
                    else o[i + (size_t)ld * j] += cfunig[ig - 1];
                }
            }
        }
    }
}

/* ---- src/src_eigensystem/hamiltonoverlapocopy_UL.f90:16-28 --------------
 * za(i+1:, i) = conj(za(i, i+1:)) */
void orc_copy_ul(int n, int ld, zdouble *a)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n - 1; i++)
        for (int j = i + 1; j < n; j++) a[j + (size_t)ld * i] = conj(a[i + (size_t)ld * j]);
}

/* ======================================================================
 * Muffin-tin integrals: hmlint = mt_kin + mt_pot (spin-unpolarised main
 * Hamiltonian), src/src_eigensystem/hmlint.f90:55-57.
 * ==================================================================== */

#define ORC_Y00 0.28209479177387814347

/* ---- src/src_lib/spline.f90:1-80: cubic spline coefficients cf(3, n) ---- */
static void orc_spline(int n, const double *x, const double *f, double *cf, double *w)
{
#define CF(j, i) cf[(j) + 3 * (i)]
    double t1, t2, t3, t4;
    for (int i = 0; i < n - 1; i++) {
        w[i] = 1.0 / (x[i + 1] - x[i]);
        CF(0, i) = w[i] * (f[i + 1] - f[i]);
    }
    CF(1, 0) = 1.0;
    CF(2, 0) = (CF(0, 1) - CF(0, 0)) / (x[2] - x[0]);
    t1 = (x[1] - x[0]) * w[1];
    t2 = t1 * CF(1, 0);
    t3 = 1.0 / (2.0 * (t1 + 1.0));
    CF(1, 1) = t3;
    t4 = 3.0 * (CF(0, 1) - CF(0, 0)) * w[1] - t2 * CF(2, 0);
    CF(2, 1) = t4;
    for (int i = 2; i < n - 1; i++) {
        t1 = (x[i] - x[i - 1]) * w[i];
        t2 = t1 * t3;
        t3 = 1.0 / (2.0 * t1 + 2.0 - t2);
        CF(1, i) = t3;
        t4 = 3.0 * (CF(0, i) - CF(0, i - 1)) * w[i] - t2 * t4;
        CF(2, i) = t4;
    }
    CF(1, n - 1) = 1.0;
    t1 = (CF(0, n - 2) - CF(0, n - 3)) / (x[n - 1] - x[n - 3]);
    CF(2, n - 1) = t1;
    for (int i = n - 2; i >= 1; i--) {
        t1 = CF(2, i) - t1 * CF(1, i + 1);
        CF(2, i) = t1;
    }
    for (int i = 0; i < n; i++) CF(1, i) = CF(1, i) * CF(2, i);
    for (int i = 0; i < n - 1; i++) {
        t1 = 0.3333333333333333333 * (CF(1, i + 1) - CF(1, i)) * w[i];
        CF(2, i) = t1;
        t2 = x[i + 1] - x[i];
        CF(0, i) = CF(0, i) - (CF(1, i) + t1 * t2) * t2;
    }
    t1 = x[n - 1] - x[n - 2];
    CF(0, n - 1) = CF(0, n - 2) + (2.0 * CF(1, n - 2) + 3.0 * CF(2, n - 2) * t1) * t1;
    CF(2, n - 1) = CF(2, n - 2);
#undef CF
}

/* ---- src/src_lib/fderiv.f90, m = -1: the integral from x(1) to x(n) ---- */
double orc_fint(int n, const double *x, const double *f)
{
    double *cf = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    double *w = (double *)malloc(sizeof(double) * (size_t)n);
    orc_spline(n, x, f, cf, w);
    double g = 0.0;
    for (int i = 0; i < n - 1; i++) {
        const double dx = x[i + 1] - x[i];
        g = g + (((0.25 * cf[2 + 3 * i] * dx + 0.3333333333333333333 * cf[1 + 3 * i]) * dx + 0.5 * cf[3 * i]) * dx +
                 f[i]) * dx;
    }
    free(cf);
    free(w);
    return g;
}

/* ---- src/src_lib/wigner3j.f90 --------------------------------------- */
double orc_wigner3j(int j1, int j2, int j3, int m1, int m2, int m3)
{
    if (j1 == 0 && j2 == 0 && j3 == 0) return 1.0;
    const int l1 = j2 - j1 + j3, l2 = j1 - j2 + j3, l3 = j1 + j2 - j3;
    if (m1 + m2 + m3 != 0 || l1 < 0 || l2 < 0 || l3 < 0) return 0.0;
    const int n1 = j1 - m1, n2 = j2 + m2;
    int k1 = 0;
    if (j2 - j3 - m1 > k1) k1 = j2 - j3 - m1;
    if (j1 - j3 + m2 > k1) k1 = j1 - j3 + m2;
    int k2 = l3;
    if (n1 < k2) k2 = n1;
    if (n2 < k2) k2 = n2;
    double sgn = ((k1 + j1 + j2 + m3) % 2 != 0) ? -1.0 : 1.0;
    double sum = 0.0;
    for (int k = k1; k <= k2; k++) {
        const double t1 = sgn * orc_factr(l1, l1 - n2 + k) * orc_factr(l2, l2 - n1 + k) * orc_factr(l3, l3 - k);
        sum = sum + t1 / (orc_factnm(k, 1) * orc_factnm(n1 - k, 1) * orc_factnm(n2 - k, 1));
        sgn = -sgn;
    }
    double t1 = orc_factr(j1 + m1, l1) * orc_factr(j2 + m2, l2) * orc_factr(j3 + m3, l3);
    t1 = t1 * orc_factr(j3 - m3, 1 + j1 + j2 + j3) * orc_factnm(j1 - m1, 1) * orc_factnm(j2 - m2, 1);
    return sum * sqrt(t1);
}

/* ---- src/src_lib/gaunt.f90: integral of conj(Y_l1m1) Y_l2m2 Y_l3m3 ------ */
double orc_gaunt(int l1, int l2, int l3, int m1, int m2, int m3)
{
    if (m1 - m2 - m3 != 0) return 0.0;
    const int j1 = l2 - l1 + l3, j2 = l1 - l2 + l3, j3 = l1 + l2 - l3;
    if (j1 < 0 || j2 < 0 || j3 < 0) return 0.0;
    const int j = l1 + l2 + l3;
    if (j % 2 != 0) return 0.0;
    const int jh = j / 2;
    double t1 = sqrt((double)((2 * l1 + 1) * (2 * l2 + 1) * (2 * l3 + 1)) * orc_factr(j1, j + 1) *
                     orc_factnm(j2, 1) * orc_factnm(j3, 1));
    t1 = t1 * orc_factr(jh, jh - l1) / (orc_factnm(jh - l2, 1) * orc_factnm(jh - l3, 1));
    double g = t1 * ORC_Y00 * orc_wigner3j(l1, l2, l3, -m1, m2, m3);
    if ((m1 + jh) % 2 != 0) g = -g;
    return g;
}

/* ---- src/src_lib/gauntyry.f90: conj(Y_l1m1) R_l2m2 Y_l3m3, R real harmonic */
zdouble orc_gauntyry(int l1, int l2, int l3, int m1, int m2, int m3)
{
    const double c1 = 0.7071067811865475244;
    if (m2 > 0) {
        const double t1 = (m2 % 2 == 0) ? 1.0 : -1.0;
        const double t2 = c1 * (orc_gaunt(l1, l2, l3, m1, m2, m3) + t1 * orc_gaunt(l1, l2, l3, m1, -m2, m3));
        return t2;
    } else if (m2 < 0) {
        const double t1 = ((-m2) % 2 == 0) ? 1.0 : -1.0;
        const double t2 = c1 * (orc_gaunt(l1, l2, l3, m1, m2, m3) - t1 * orc_gaunt(l1, l2, l3, m1, -m2, m3));
        return -t2 * I;
    }
    return orc_gaunt(l1, l2, l3, m1, m2, m3);
}

void orc_gauntyry_re_im(int l1, int l2, int l3, int m1, int m2, int m3, double *re_im)
{
    const zdouble z = orc_gauntyry(l1, l2, l3, m1, m2, m3);
    re_im[0] = creal(z);
    re_im[1] = cimag(z);
}

static int orc_idxlm(int l, int m) { return l * (l + 1) + m; }   /* 0-based */

/* ---- hmlint's main Hamiltonian: mt_kin.f90:70-195 then mt_pot.f90:114-306 ----
 * apwfr(nrmtmax, 2, apwordmax, 0:lmaxapw, natmtot): u and du/dr;
 * lofr(nrmtmax, 2, nlomax, natmtot); veffmt(lmmaxvr, nrmtmax, natmtot) in
 * real spherical harmonics; spr(nrmtmax, nspecies); apword(0:lmaxapw, nspecies);
 * lorbl(nlomax, nspecies).  aa(maxaa, maxaa, natmtot), loa(maxnlo, maxaa,
 * natmtot), lolo(maxnlo, maxnlo, natmtot) are ADDED to (the reference adds
 * to mt_hscf%main, zeroed beforehand by MTInit). */
void orc_hmlint(int natmtot, const int *atom_species, int lmaxapw, int lmaxmat, int lmaxvr, int apwordmax,
                const int *apword, int nlomax, const int *nlorb, const int *lorbl, int nrmtmax, const int *nrmt,
                const double *spr, const double *apwfr, const double *lofr, const double *veffmt, int relativistic,
                int maxaa, int maxnlo, zdouble *aa, zdouble *loa, zdouble *lolo)
{
    const int lmmaxvr = (lmaxvr + 1) * (lmaxvr + 1);
    const double alpha = 1.0 / 137.03599911;
    const double a = relativistic ? 0.5 * alpha * alpha : 0.0;
#define APWFR(ir, d, io, l, ias) \
    apwfr[(ir) + (size_t)nrmtmax * ((d) + 2 * ((io) + (size_t)apwordmax * ((l) + (size_t)(lmaxapw + 1) * (ias))))]
#define LOFR(ir, d, ilo, ias) lofr[(ir) + (size_t)nrmtmax * ((d) + 2 * ((ilo) + (size_t)nlomax * (ias)))]
#define POT(lm, ir, ias) veffmt[(lm) + (size_t)lmmaxvr * ((ir) + (size_t)nrmtmax * (ias))]
#define AA(i, j, ias) aa[(i) + (size_t)maxaa * ((j) + (size_t)maxaa * (ias))]
#define LOA(i, j, ias) loa[(i) + (size_t)maxnlo * ((j) + (size_t)maxaa * (ias))]
#define LOLO(i, j, ias) lolo[(i) + (size_t)maxnlo * ((j) + (size_t)maxnlo * (ias))]
    double *fr = (double *)malloc(sizeof(double) * nrmtmax);
    double *r2 = (double *)malloc(sizeof(double) * nrmtmax);
    double *r2inv = (double *)malloc(sizeof(double) * nrmtmax);
    double *rmtable = (double *)malloc(sizeof(double) * nrmtmax);
    /* Gaunt table gntryy(lm2, lm3, lm1) for lm1, lm3 <= lmmaxmat */
    const int lmmaxmat = (lmaxmat + 1) * (lmaxmat + 1);
    zdouble *gnt = (zdouble *)malloc(sizeof(zdouble) * (size_t)lmmaxvr * lmmaxmat * lmmaxmat);
    for (int l1 = 0; l1 <= lmaxmat; l1++)
        for (int m1 = -l1; m1 <= l1; m1++)
            for (int l3 = 0; l3 <= lmaxmat; l3++)
                for (int m3 = -l3; m3 <= l3; m3++)
                    for (int l2 = 0; l2 <= lmaxvr; l2++)
                        for (int m2 = -l2; m2 <= l2; m2++)
                            gnt[orc_idxlm(l2, m2) + (size_t)lmmaxvr * (orc_idxlm(l3, m3) + (size_t)lmmaxmat * orc_idxlm(l1, m1))] =
                                orc_gauntyry(l1, l2, l3, m1, m2, m3);
#define GNT(lm2, lm3, lm1) gnt[(lm2) + (size_t)lmmaxvr * ((lm3) + (size_t)lmmaxmat * (lm1))]
    /* radial integrals I(lm2, io2, l3, io1, l1) of mt_pot and K(io2, io1, l1) of mt_kin */
    const size_t nint = (size_t)lmmaxvr * apwordmax * (lmaxmat + 1) * apwordmax * (lmaxmat + 1);
    double *hint = (double *)malloc(sizeof(double) * nint);
    double *hkin = (double *)malloc(sizeof(double) * apwordmax * apwordmax * (lmaxmat + 1));
    double *hlo = (double *)malloc(sizeof(double) * (size_t)lmmaxvr * apwordmax * (lmaxmat + 1) * (nlomax > 0 ? nlomax : 1));
    double *hlokin = (double *)malloc(sizeof(double) * apwordmax * (nlomax > 0 ? nlomax : 1));
    double *hll = (double *)malloc(sizeof(double) * (size_t)lmmaxvr * (nlomax > 0 ? nlomax * nlomax : 1));
    double *hllkin = (double *)malloc(sizeof(double) * (nlomax > 0 ? nlomax * nlomax : 1));
#define HINT(lm2, io2, l3, io1, l1) \
    hint[(lm2) + (size_t)lmmaxvr * ((io2) + (size_t)apwordmax * ((l3) + (size_t)(lmaxmat + 1) * ((io1) + (size_t)apwordmax * (l1))))]
#define HLO(lm2, io, l3, ilo) hlo[(lm2) + (size_t)lmmaxvr * ((io) + (size_t)apwordmax * ((l3) + (size_t)(lmaxmat + 1) * (ilo)))]
#define HLL(lm2, i1, i2) hll[(lm2) + (size_t)lmmaxvr * ((i1) + (size_t)nlomax * (i2))]
    for (int ias = 0; ias < natmtot; ias++) {
        const int is = atom_species[ias];
        const int nr = nrmt[is];
        const double *x = spr + (size_t)nrmtmax * is;
        const int *apw = apword + (size_t)(lmaxapw + 1) * is;
        const int nlo = nlorb[is];
        const int *lol = lorbl + (size_t)nlomax * is;
        for (int ir = 0; ir < nr; ir++) {
            r2[ir] = x[ir] * x[ir];
            r2inv[ir] = 1.0 / r2[ir];
            rmtable[ir] = 1.0 / (1.0 - a * POT(0, ir, ias) * ORC_Y00);
        }
        /* ---- mt_kin: radial integrals (mt_kin.f90:71-121) */
        for (int l1 = 0; l1 <= lmaxmat; l1++)
            for (int io1 = 0; io1 < apw[l1]; io1++)
                for (int io2 = 0; io2 < apw[l1]; io2++) {
                    const double ang = (double)(l1 * (l1 + 1));
                    for (int ir = 0; ir < nr; ir++) {
                        const double t1 = APWFR(ir, 0, io1, l1, ias) * APWFR(ir, 0, io2, l1, ias);
                        const double t2 = APWFR(ir, 1, io1, l1, ias) * APWFR(ir, 1, io2, l1, ias);
                        fr[ir] = (0.5 * t2 * rmtable[ir] + 0.5 * ang * t1 * rmtable[ir] * r2inv[ir]) * r2[ir];
                    }
                    hkin[io2 + apwordmax * (io1 + apwordmax * l1)] = orc_fint(nr, x, fr) / ORC_Y00;
                }
        for (int ilo = 0; ilo < nlo; ilo++) {
            const int l1 = lol[ilo];
            for (int io = 0; io < apw[l1]; io++) {
                const double ang = (double)(l1 * (l1 + 1));
                for (int ir = 0; ir < nr; ir++) {
                    const double t1 = APWFR(ir, 0, io, l1, ias) * LOFR(ir, 0, ilo, ias);
                    const double t2 = APWFR(ir, 1, io, l1, ias) * LOFR(ir, 1, ilo, ias);
                    fr[ir] = (0.5 * t2 * rmtable[ir] + 0.5 * ang * t1 * rmtable[ir] * r2inv[ir]) * r2[ir];
                }
                hlokin[io + apwordmax * ilo] = orc_fint(nr, x, fr) / ORC_Y00;
            }
        }
        for (int ilo1 = 0; ilo1 < nlo; ilo1++)
            for (int ilo2 = 0; ilo2 < nlo; ilo2++) {
                if (lol[ilo1] != lol[ilo2]) continue;
                const double ang = (double)(lol[ilo1] * (lol[ilo1] + 1));
                for (int ir = 0; ir < nr; ir++) {
                    const double t1 = LOFR(ir, 0, ilo1, ias) * LOFR(ir, 0, ilo2, ias);
                    const double t2 = LOFR(ir, 1, ilo1, ias) * LOFR(ir, 1, ilo2, ias);
                    fr[ir] = (0.5 * t2 * rmtable[ir] + 0.5 * ang * t1 * rmtable[ir] * r2inv[ir]) * r2[ir];
                }
                hllkin[ilo1 + nlomax * ilo2] = orc_fint(nr, x, fr) / ORC_Y00;
            }
        /* ---- mt_kin: diagonal lm blocks (mt_kin.f90:150-195) */
        {
            int if1 = 0;
            for (int l1 = 0; l1 <= lmaxmat; l1++)
                for (int m1 = -l1; m1 <= l1; m1++) {
                    for (int io1 = 0; io1 < apw[l1]; io1++)
                        for (int io2 = 0; io2 < apw[l1]; io2++)
                            AA(if1 + io1, if1 + io2, ias) += hkin[io2 + apwordmax * (io1 + apwordmax * l1)] * ORC_Y00;
                    if1 += apw[l1];
                }
            if1 = 0;
            for (int ilo = 0; ilo < nlo; ilo++) {
                const int l1 = lol[ilo];
                for (int m1 = -l1; m1 <= l1; m1++) {
                    const int lm1 = orc_idxlm(l1, m1);
                    int if3 = 0;
                    for (int l3 = 0; l3 <= lmaxmat; l3++)
                        for (int m3 = -l3; m3 <= l3; m3++)
                            for (int io = 0; io < apw[l3]; io++) {
                                if (lm1 == orc_idxlm(l3, m3))
                                    LOA(if1, if3, ias) += hlokin[io + apwordmax * ilo] * ORC_Y00;
                                if3++;
                            }
                    if1++;
                }
            }
            if1 = 0;
            for (int ilo1 = 0; ilo1 < nlo; ilo1++)
                for (int m1 = -lol[ilo1]; m1 <= lol[ilo1]; m1++) {
                    const int lm1 = orc_idxlm(lol[ilo1], m1);
                    int if3 = 0;
                    for (int ilo2 = 0; ilo2 < nlo; ilo2++)
                        for (int m3 = -lol[ilo2]; m3 <= lol[ilo2]; m3++) {
                            if (lm1 == orc_idxlm(lol[ilo2], m3))
                                LOLO(if1, if3, ias) += hllkin[ilo1 + nlomax * ilo2] * ORC_Y00;
                            if3++;
                        }
                    if1++;
                }
        }
        /* ---- mt_pot: radial integrals (mt_pot.f90:130-222) */
        for (int l1 = 0; l1 <= lmaxmat; l1++)
            for (int io1 = 0; io1 < apw[l1]; io1++)
                for (int l3 = 0; l3 <= lmaxmat; l3++)
                    for (int io2 = 0; io2 < apw[l3]; io2++)
                        for (int lm2 = 0; lm2 < lmmaxvr; lm2++) {
                            for (int ir = 0; ir < nr; ir++) {
                                const double t1 = APWFR(ir, 0, io1, l1, ias) * APWFR(ir, 0, io2, l3, ias) * r2[ir];
                                fr[ir] = t1 * POT(lm2, ir, ias);
                            }
                            HINT(lm2, io2, l3, io1, l1) = orc_fint(nr, x, fr);
                        }
        for (int ilo = 0; ilo < nlo; ilo++)
            for (int l3 = 0; l3 <= lmaxmat; l3++)
                for (int io = 0; io < apw[l3]; io++)
                    for (int lm2 = 0; lm2 < lmmaxvr; lm2++) {
                        for (int ir = 0; ir < nr; ir++) {
                            const double t1 = LOFR(ir, 0, ilo, ias) * APWFR(ir, 0, io, l3, ias) * r2[ir];
                            fr[ir] = t1 * POT(lm2, ir, ias);
                        }
                        HLO(lm2, io, l3, ilo) = orc_fint(nr, x, fr);
                    }
        for (int ilo1 = 0; ilo1 < nlo; ilo1++)
            for (int ilo2 = 0; ilo2 < nlo; ilo2++)
                for (int lm2 = 0; lm2 < lmmaxvr; lm2++) {
                    for (int ir = 0; ir < nr; ir++) {
                        const double t1 = LOFR(ir, 0, ilo1, ias) * LOFR(ir, 0, ilo2, ias) * r2[ir];
                        fr[ir] = t1 * POT(lm2, ir, ias);
                    }
                    HLL(lm2, ilo1, ilo2) = orc_fint(nr, x, fr);
                }
        /* ---- mt_pot: angular sums over the nonzero Gaunt coefficients, lm2 ascending
         * (mt_pot.f90:232-306, the gntnonz list of init1.f90:575-595) */
        {
            int if1 = 0;
            for (int l1 = 0; l1 <= lmaxmat; l1++)
                for (int m1 = -l1; m1 <= l1; m1++) {
                    const int lm1 = orc_idxlm(l1, m1);
                    for (int io1 = 0; io1 < apw[l1]; io1++) {
                        int if3 = 0;
                        for (int l3 = 0; l3 <= lmaxmat; l3++)
                            for (int m3 = -l3; m3 <= l3; m3++) {
                                const int lm3 = orc_idxlm(l3, m3);
                                for (int io2 = 0; io2 < apw[l3]; io2++) {
                                    zdouble zsum = 0.0;
                                    for (int lm2 = 0; lm2 < lmmaxvr; lm2++) {
                                        const zdouble g = GNT(lm2, lm3, lm1);
                                        if (cabs(g) > 1e-20) zsum = zsum + g * HINT(lm2, io2, l3, io1, l1);
                                    }
                                    AA(if1, if3, ias) += zsum;
                                    if3++;
                                }
                            }
                        if1++;
                    }
                }
            if1 = 0;
            for (int ilo = 0; ilo < nlo; ilo++) {
                const int l1 = lol[ilo];
                for (int m1 = -l1; m1 <= l1; m1++) {
                    const int lm1 = orc_idxlm(l1, m1);
                    int if3 = 0;
                    for (int l3 = 0; l3 <= lmaxmat; l3++)
                        for (int m3 = -l3; m3 <= l3; m3++) {
                            const int lm3 = orc_idxlm(l3, m3);
                            for (int io = 0; io < apw[l3]; io++) {
                                zdouble zsum = 0.0;
                                for (int lm2 = 0; lm2 < lmmaxvr; lm2++) {
                                    const zdouble g = GNT(lm2, lm3, lm1);
                                    if (cabs(g) > 1e-20) zsum = zsum + g * HLO(lm2, io, l3, ilo);
                                }
                                LOA(if1, if3, ias) += zsum;
                                if3++;
                            }
                        }
                    if1++;
                }
            }
            if1 = 0;
            for (int ilo1 = 0; ilo1 < nlo; ilo1++)
                for (int m1 = -lol[ilo1]; m1 <= lol[ilo1]; m1++) {
                    const int lm1 = orc_idxlm(lol[ilo1], m1);
                    int if3 = 0;
                    for (int ilo2 = 0; ilo2 < nlo; ilo2++)
                        for (int m3 = -lol[ilo2]; m3 <= lol[ilo2]; m3++) {
                            const int lm3 = orc_idxlm(lol[ilo2], m3);
                            zdouble zsum = 0.0;
                            for (int lm2 = 0; lm2 < lmmaxvr; lm2++) {
                                const zdouble g = GNT(lm2, lm3, lm1);
                                if (cabs(g) > 1e-20) zsum = zsum + g * HLL(lm2, ilo1, ilo2);
                            }
                            LOLO(if1, if3, ias) += zsum;
                            if3++;
                        }
                    if1++;
                }
        }
    }
    free(fr); free(r2); free(r2inv); free(rmtable); free(gnt); free(hint); free(hkin);
    free(hlo); free(hlokin); free(hll); free(hllkin);
#undef APWFR
#undef LOFR
#undef POT
#undef AA
#undef LOA
#undef LOLO
#undef GNT
#undef HINT
#undef HLO
#undef HLL
}

/* ---- src/src_eigensystem/olprad.f90: overlap radial integrals -------------
 * oalo(apwordmax, nlomax, natmtot), ololo(nlomax, nlomax, natmtot) and, for
 * iora* (iora != 0), h1aa(apwordmax, apwordmax, 0:lmaxapw, natmtot),
 * h1loa(apwordmax, nlomax, natmtot), h1lolo(nlomax, nlomax, natmtot).  The
 * h1 arrays are zeroed first (olprad.f90:11-13); oalo/ololo entries the
 * reference does not visit are left as passed in. */
void orc_olprad(int natmtot, const int *atom_species, int lmaxapw, int lmaxmat, int lmaxvr, int apwordmax,
                const int *apword, int nlomax, const int *nlorb, const int *lorbl, int nrmtmax, const int *nrmt,
                const double *spr, const double *apwfr, const double *lofr, const double *veffmt, int relativistic,
                int iora, double *oalo, double *ololo, double *h1aa, double *h1loa, double *h1lolo)
{
    const int lmmaxvr = (lmaxvr + 1) * (lmaxvr + 1);
    const double alpha = 1.0 / 137.03599911;
    const double a = relativistic ? 0.5 * alpha * alpha : 0.0;
#define APWFR(ir, d, io, l, ias) \
    apwfr[(ir) + (size_t)nrmtmax * ((d) + 2 * ((io) + (size_t)apwordmax * ((l) + (size_t)(lmaxapw + 1) * (ias))))]
#define LOFR(ir, d, ilo, ias) lofr[(ir) + (size_t)nrmtmax * ((d) + 2 * ((ilo) + (size_t)nlomax * (ias)))]
#define POT0(ir, ias) veffmt[(size_t)lmmaxvr * ((ir) + (size_t)nrmtmax * (ias))]
    if (iora) {
        memset(h1aa, 0, sizeof(double) * apwordmax * apwordmax * (lmaxapw + 1) * (size_t)natmtot);
        memset(h1loa, 0, sizeof(double) * apwordmax * nlomax * (size_t)natmtot);
        memset(h1lolo, 0, sizeof(double) * nlomax * nlomax * (size_t)natmtot);
    }
    double *fr = (double *)malloc(sizeof(double) * nrmtmax);
    for (int ias = 0; ias < natmtot; ias++) {
        const int is = atom_species[ias];
        const int nr = nrmt[is];
        const double *x = spr + (size_t)nrmtmax * is;
        const int *apw = apword + (size_t)(lmaxapw + 1) * is;
        const int *lol = lorbl + (size_t)nlomax * is;
        if (iora)
            for (int l = 0; l <= lmaxmat; l++) {
                const double ang = (double)(l * (l + 1));
                for (int io1 = 0; io1 < apw[l]; io1++)
                    for (int io2 = 0; io2 < apw[l]; io2++) {
                        for (int ir = 0; ir < nr; ir++) {
                            const double rm = 1.0 / (1.0 - a * POT0(ir, ias) * ORC_Y00);
                            const double t1 = APWFR(ir, 0, io1, l, ias) * APWFR(ir, 0, io2, l, ias);
                            const double t2 = APWFR(ir, 1, io1, l, ias) * APWFR(ir, 1, io2, l, ias);
                            fr[ir] = a * (0.5 * t2 * rm * rm + 0.5 * ang * t1 * rm * rm / (x[ir] * x[ir])) *
                                     (x[ir] * x[ir]);
                        }
                        h1aa[io1 + (size_t)apwordmax * (io2 + (size_t)apwordmax * (l + (size_t)(lmaxapw + 1) * ias))] =
                            orc_fint(nr, x, fr);
                    }
            }
        for (int ilo = 0; ilo < nlorb[is]; ilo++) {
            const int l = lol[ilo];
            for (int io = 0; io < apw[l]; io++) {
                for (int ir = 0; ir < nr; ir++) fr[ir] = APWFR(ir, 0, io, l, ias) * LOFR(ir, 0, ilo, ias) * (x[ir] * x[ir]);
                oalo[io + (size_t)apwordmax * (ilo + (size_t)nlomax * ias)] = orc_fint(nr, x, fr);
                if (iora) {
                    const double ang = (double)(l * (l + 1));
                    for (int ir = 0; ir < nr; ir++) {
                        const double rm = 1.0 / (1.0 - a * POT0(ir, ias) * ORC_Y00);
                        const double t1 = APWFR(ir, 0, io, l, ias) * LOFR(ir, 0, ilo, ias);
                        const double t2 = APWFR(ir, 1, io, l, ias) * LOFR(ir, 1, ilo, ias);
                        fr[ir] = (a * (0.5 * t2 * rm * rm + 0.5 * ang * t1 * rm * rm / (x[ir] * x[ir]))) * (x[ir] * x[ir]);
                    }
                    h1loa[io + (size_t)apwordmax * (ilo + (size_t)nlomax * ias)] = orc_fint(nr, x, fr);
                }
            }
        }
        for (int ilo1 = 0; ilo1 < nlorb[is]; ilo1++) {
            const int l = lol[ilo1];
            for (int ilo2 = 0; ilo2 < nlorb[is]; ilo2++) {
                if (lol[ilo2] != l) continue;
                for (int ir = 0; ir < nr; ir++)
                    fr[ir] = LOFR(ir, 0, ilo1, ias) * LOFR(ir, 0, ilo2, ias) * (x[ir] * x[ir]);
                ololo[ilo1 + (size_t)nlomax * (ilo2 + (size_t)nlomax * ias)] = orc_fint(nr, x, fr);
                if (iora) {
                    const double ang = (double)(l * (l + 1));
                    for (int ir = 0; ir < nr; ir++) {
                        const double rm = 1.0 / (1.0 - a * POT0(ir, ias) * ORC_Y00);
                        const double t1 = LOFR(ir, 0, ilo1, ias) * LOFR(ir, 0, ilo2, ias);
                        const double t2 = LOFR(ir, 1, ilo1, ias) * LOFR(ir, 1, ilo2, ias);
                        fr[ir] = (a * (0.5 * t2 * rm * rm + 0.5 * ang * t1 * rm * rm / (x[ir] * x[ir]))) * (x[ir] * x[ir]);
                    }
                    h1lolo[ilo1 + (size_t)nlomax * (ilo2 + (size_t)nlomax * ias)] = orc_fint(nr, x, fr);
                }
            }
        }
    }
    free(fr);
#undef APWFR
#undef LOFR
#undef POT0
}

/* ======================================================================
 * Momentum matrix elements of the LAPW+lo basis for real-time TDDFT:
 * pmatrad (src/src_xs/pmatrad.F90) with gradzfmtr (src/src_xs/gradzfmtr.F90)
 * and clebgor (src/src_lib/clebgor.f90).  The basis contraction
 * (genpmatbasisik, src/src_xs/src_rttddft/rttddft_pmat.f90:66-188) is in
 * lapw_oracle.py.
 * ==================================================================== */

/* src/src_lib/clebgor.f90 */
double orc_clebgor(int j1, int j2, int j3, int m1, int m2, int m3)
{
    if (j1 == 0 && j2 == 0 && j3 == 0) return 1.0;
    if (m1 + m2 - m3 != 0 || j2 + j3 < j1 || j1 + j3 < j2 || j1 + j2 < j3) return 0.0;
    double c = sqrt((double)(2 * j3 + 1)) * orc_wigner3j(j1, j2, j3, m1, m2, -m3);
    if ((j1 - j2 + m3) % 2 != 0) c = -c;
    return c;
}

/* src/src_lib/fderiv.f90, m = 1: the first derivative of the spline at the points */
void orc_fderiv1(int n, const double *x, const double *f, double *g)
{
    double *cf = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    double *w = (double *)malloc(sizeof(double) * (size_t)n);
    orc_spline(n, x, f, cf, w);
    for (int i = 0; i < n; i++) g[i] = cf[3 * i];
    free(cf);
    free(w);
}

/* src/src_xs/gradzfmtr.F90: the gradient of f(r) Y_l1m1, expanded in Y_lm2
 * (l2 = l1 +- 1 <= lmax): gfmt(ld1, nr, 3) (x, y, z) */
void orc_gradzfmtr(int lmax, int nr, const double *r, int l1, int m1, int ld1, int ld2, const double *fmt,
                          double *gfmt)
{
    const double s2 = sqrt(2.0);
    double *g1 = (double *)malloc(sizeof(double) * nr);
    for (size_t i = 0; i < (size_t)ld1 * ld2 * 3; i++) gfmt[i] = 0.0;
    orc_fderiv1(nr, r, fmt, g1);
    const double t1 = sqrt((double)(l1 + 1) / (double)(2 * l1 + 1));
    const double t2 = sqrt((double)l1 / (double)(2 * l1 + 1));
#define G(lm, ir, j) gfmt[(lm) + (size_t)ld1 * ((ir) + (size_t)ld2 * (j))]
    int l2 = l1 + 1;
    if (l2 <= lmax)
        for (int m2 = -l2; m2 <= l2; m2++) {
            const int lm2 = l2 * (l2 + 1) + m2;
            const double t3 = orc_clebgor(l2, 1, l1, m2, -1, m1), t4 = orc_clebgor(l2, 1, l1, m2, 0, m1),
                         t5 = orc_clebgor(l2, 1, l1, m2, 1, m1);
            for (int ir = 0; ir < nr; ir++) {
                const double tt2 = t1 * (fmt[ir] * (double)l1 / r[ir] - g1[ir]);
                G(lm2, ir, 0) += ((t3 - t5) / s2) * tt2;
                G(lm2, ir, 1) += ((-t3 - t5) / s2) * tt2;
                G(lm2, ir, 2) += t4 * tt2;
            }
        }
    l2 = l1 - 1;
    if (l2 >= 0)
        for (int m2 = -l2; m2 <= l2; m2++) {
            const int lm2 = l2 * (l2 + 1) + m2;
            const double t3 = orc_clebgor(l2, 1, l1, m2, -1, m1), t4 = orc_clebgor(l2, 1, l1, m2, 0, m1),
                         t5 = orc_clebgor(l2, 1, l1, m2, 1, m1);
            for (int ir = 0; ir < nr; ir++) {
                const double tt2 = t2 * (fmt[ir] * (double)(l1 + 1) / r[ir] + g1[ir]);
                G(lm2, ir, 0) += ((t3 - t5) / s2) * tt2;
                G(lm2, ir, 1) += ((-t3 - t5) / s2) * tt2;
                G(lm2, ir, 2) += t4 * tt2;
            }
        }
#undef G
    free(g1);
}

/* src/src_xs/pmatrad.F90: ripaa(apwordmax, lmmaxapw, apwordmax, lmmaxapw, natmtot, 3),
 * ripalo(apwordmax, lmmaxapw, nlomax, 2 lolmax + 1, natmtot, 3),
 * riploa(nlomax, 2 lolmax + 1, apwordmax, lmmaxapw, natmtot, 3),
 * riplolo(nlomax, 2 lolmax + 1, nlomax, 2 lolmax + 1, natmtot, 3); the m index
 * of a local orbital is stored at m + lolmax.  All outputs are overwritten. */
void orc_pmatrad(int natmtot, const int *atom_species, int lmaxapw, int apwordmax, const int *apword, int nlomax,
                 const int *nlorb, const int *lorbl, int lolmax, int nrmtmax, const int *nrmt, const double *spr,
                 const double *apwfr, const double *lofr, double *ripaa, double *ripalo, double *riploa,
                 double *riplolo)
{
    const int lmmax = (lmaxapw + 1) * (lmaxapw + 1), nm = 2 * lolmax + 1, ao = apwordmax;
    const size_t naa = (size_t)ao * lmmax * ao * lmmax * natmtot, nal = (size_t)ao * lmmax * nlomax * nm * natmtot,
                 nll = (size_t)nlomax * nm * nlomax * nm * natmtot;
    memset(ripaa, 0, sizeof(double) * naa * 3);
    memset(ripalo, 0, sizeof(double) * nal * 3);
    memset(riploa, 0, sizeof(double) * nal * 3);
    memset(riplolo, 0, sizeof(double) * nll * 3);
#define APWFR(ir, io, l, ias) apwfr[(ir) + (size_t)nrmtmax * (2 * ((io) + (size_t)ao * ((l) + (size_t)(lmaxapw + 1) * (ias))))]
#define LOFR(ir, ilo, ias) lofr[(ir) + (size_t)nrmtmax * (2 * ((ilo) + (size_t)nlomax * (ias)))]
    /* dapwfr(lmmax, nrmtmax, 3, apwordmax, lmmax), dlofr(lmmax, nrmtmax, 3, nlomax, nm) */
    const size_t gsz = (size_t)lmmax * nrmtmax * 3;
    double *dapw = (double *)calloc(gsz * ao * lmmax, sizeof(double));
    double *dlo = (double *)calloc(gsz * nlomax * nm, sizeof(double));
    double *fr = (double *)malloc(sizeof(double) * nrmtmax);
#define DAPW(lm1, ir, j, io, lm) dapw[(lm1) + (size_t)lmmax * ((ir) + (size_t)nrmtmax * ((j) + 3 * ((io) + (size_t)ao * (lm))))]
#define DLO(lm1, ir, j, ilo, m) dlo[(lm1) + (size_t)lmmax * ((ir) + (size_t)nrmtmax * ((j) + 3 * ((ilo) + (size_t)nlomax * (m))))]
#define RAA(io1, lm1, io2, lm3, ias, j) \
    ripaa[(io1) + (size_t)ao * ((lm1) + (size_t)lmmax * ((io2) + (size_t)ao * ((lm3) + (size_t)lmmax * ((ias) + (size_t)natmtot * (j)))))]
#define RAL(io1, lm1, ilo, m, ias, j) \
    ripalo[(io1) + (size_t)ao * ((lm1) + (size_t)lmmax * ((ilo) + (size_t)nlomax * ((m) + (size_t)nm * ((ias) + (size_t)natmtot * (j)))))]
#define RLA(ilo, m, io2, lm3, ias, j) \
    riploa[(ilo) + (size_t)nlomax * ((m) + (size_t)nm * ((io2) + (size_t)ao * ((lm3) + (size_t)lmmax * ((ias) + (size_t)natmtot * (j)))))]
#define RLL(i1, m1, i2, m2, ias, j) \
    riplolo[(i1) + (size_t)nlomax * ((m1) + (size_t)nm * ((i2) + (size_t)nlomax * ((m2) + (size_t)nm * ((ias) + (size_t)natmtot * (j)))))]
    for (int ias = 0; ias < natmtot; ias++) {
        const int is = atom_species[ias], nr = nrmt[is];
        const double *r = spr + (size_t)nrmtmax * is;
        const int *apw = apword + (size_t)(lmaxapw + 1) * is;
        const int *lol = lorbl + (size_t)nlomax * is;
        memset(dapw, 0, sizeof(double) * gsz * ao * lmmax);
        memset(dlo, 0, sizeof(double) * gsz * nlomax * nm);
        for (int l1 = 0; l1 <= lmaxapw; l1++)
            for (int m1 = -l1; m1 <= l1; m1++)
                for (int io = 0; io < apw[l1]; io++)
                    orc_gradzfmtr(lmaxapw, nr, r, l1, m1, lmmax, nrmtmax, &APWFR(0, io, l1, ias),
                                  &DAPW(0, 0, 0, io, l1 * (l1 + 1) + m1));
        for (int ilo = 0; ilo < nlorb[is]; ilo++)
            for (int m1 = -lol[ilo]; m1 <= lol[ilo]; m1++)
                orc_gradzfmtr(lmaxapw, nr, r, lol[ilo], m1, lmmax, nrmtmax, &LOFR(0, ilo, ias),
                              &DLO(0, 0, 0, ilo, m1 + lolmax));
        for (int l1 = 0; l1 <= lmaxapw; l1++)
            for (int m1 = -l1; m1 <= l1; m1++) {
                const int lm1 = l1 * (l1 + 1) + m1;
                for (int io1 = 0; io1 < apw[l1]; io1++) {
                    for (int l3 = 0; l3 <= lmaxapw; l3++)
                        for (int m3 = -l3; m3 <= l3; m3++)
                            for (int io2 = 0; io2 < apw[l3]; io2++)
                                for (int j = 0; j < 3; j++) {
                                    const int lm3 = l3 * (l3 + 1) + m3;
                                    for (int ir = 0; ir < nr; ir++)
                                        fr[ir] = r[ir] * r[ir] * APWFR(ir, io1, l1, ias) * DAPW(lm1, ir, j, io2, lm3);
                                    RAA(io1, lm1, io2, lm3, ias, j) = orc_fint(nr, r, fr);
                                }
                    for (int ilo = 0; ilo < nlorb[is]; ilo++)
                        for (int m3 = -lol[ilo]; m3 <= lol[ilo]; m3++)
                            for (int j = 0; j < 3; j++) {
                                for (int ir = 0; ir < nr; ir++)
                                    fr[ir] = r[ir] * r[ir] * APWFR(ir, io1, l1, ias) * DLO(lm1, ir, j, ilo, m3 + lolmax);
                                RAL(io1, lm1, ilo, m3 + lolmax, ias, j) = orc_fint(nr, r, fr);
                            }
                }
            }
        for (int ilo = 0; ilo < nlorb[is]; ilo++) {
            const int l1 = lol[ilo];
            for (int m1 = -l1; m1 <= l1; m1++) {
                const int lm1 = l1 * (l1 + 1) + m1;
                for (int l3 = 0; l3 <= lmaxapw; l3++)
                    for (int m3 = -l3; m3 <= l3; m3++)
                        for (int io2 = 0; io2 < apw[l3]; io2++)
                            for (int j = 0; j < 3; j++) {
                                for (int ir = 0; ir < nr; ir++)
                                    fr[ir] = r[ir] * r[ir] * LOFR(ir, ilo, ias) * DAPW(lm1, ir, j, io2, l3 * (l3 + 1) + m3);
                                RLA(ilo, m1 + lolmax, io2, l3 * (l3 + 1) + m3, ias, j) = orc_fint(nr, r, fr);
                            }
                for (int ilo2 = 0; ilo2 < nlorb[is]; ilo2++)
                    for (int m3 = -lol[ilo2]; m3 <= lol[ilo2]; m3++)
                        for (int j = 0; j < 3; j++) {
                            for (int ir = 0; ir < nr; ir++)
                                fr[ir] = r[ir] * r[ir] * LOFR(ir, ilo, ias) * DLO(lm1, ir, j, ilo2, m3 + lolmax);
                            RLL(ilo, m1 + lolmax, ilo2, m3 + lolmax, ias, j) = orc_fint(nr, r, fr);
                        }
            }
        }
    }
    free(dapw);
    free(dlo);
    free(fr);
#undef APWFR
#undef LOFR
#undef DAPW
#undef DLO
#undef RAA
#undef RAL
#undef RLA
#undef RLL
}
