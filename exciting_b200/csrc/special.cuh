// Device FP64 special functions of the APW matching step.
//
// Each routine follows the reference routine named beside it step by step, so
// that the device values agree with the reference to rounding:
//   exs_sbessel    -- src/src_lib/sbessel.f90:48-147
//   exs_sbesseldm  -- src/src_lib/sbesseldm.f90:40-130
//   exs_ylm_l      -- one l of src/src_lib/genylm.f90:50-92
//   exs_polynom    -- src/src_lib/polynom.f90 (m >= 0 branches)
//   exs_sphcrd     -- src/src_lib/sphcrd.f90:30-56
// sin, cos, sqrt, acos and atan2 are CUDA's own functions.
#pragma once
#include <cuda_runtime.h>

#define EXS_LMAX_APW 14          // compiled limit for lmaxapw
#define EXS_APWORD_MAX 3         // compiled limit for the APW order
#define EXS_NP_MAX 4             // np = max(apwordmax+1, 4) <= 4

namespace exs {

// x**j for integer j >= 0 by binary powering.
__host__ __device__ inline double powi(double x, int j)
{
    double r = 1.0;
    while (j > 0) {
        if (j & 1) r *= x;
        x *= x;
        j >>= 1;
    }
    return r;
}

// src/src_lib/factnm.f90 for the arguments sbesseldm uses (n! and n!!).
__device__ inline double factnm(int n, int m)
{
    if (n <= 0) return 1.0;
    double r = (double)n;
    for (int i = n - m; i > 0; i -= m) r *= (double)i;
    return r;
}

// src/src_lib/factr.f90: n!/d!
__device__ inline double factr(int n, int d)
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

// j_l(x), l = 0..lmax.  Caller guarantees 0 <= lmax <= EXS_LMAX_APW+1.
__device__ inline void sbessel(int lmax, double x, double *jl)
{
    const int lst = 25;
    const double rsc = 1e150, rsci = 1.0 / 1e150;
    if (x < 1e-8) {
        jl[0] = 1.0;
        double t1 = 1.0, t2 = 1.0;
        for (int l = 1; l <= lmax; l++) {
            t1 = t1 / (double)(2 * l + 1);
            t2 = t2 * x;
            jl[l] = t2 * t1;
        }
        return;
    }
    const double xi = 1.0 / x;
    double sn, cs;
    sincos(x, &sn, &cs);
    if (x < (double)lmax) {
        double j0 = 0.6370354636449841609 * rsci;
        double j1 = 0.3532702964695481204 * rsci;
        double jt;
        for (int l = lmax + lst; l >= lmax + 1; l--) {
            jt = j0 * (double)(2 * l + 1) * xi - j1;
            j1 = j0;
            j0 = jt;
            if (fabs(j0) > rsc) { jt *= rsci; j1 *= rsci; j0 *= rsci; }
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
        const double t1 = 1.0 / ((jl[0] - x * jl[1]) * cs + x * jl[0] * sn);
        for (int l = 0; l <= lmax; l++) jl[l] = t1 * jl[l];
        return;
    }
    jl[0] = sn * xi;
    if (lmax == 0) return;
    jl[1] = (jl[0] - cs) * xi;
    if (lmax == 1) return;
    double j0 = jl[0], j1 = jl[1], jt;
    for (int l = 2; l <= lmax; l++) {
        jt = (double)(2 * l - 1) * j1 * xi - j0;
        j0 = j1;
        j1 = jt;
        jl[l] = j1;
    }
}

// m-th derivative of j_l(x), l = 0..lmax (m <= 6).
__device__ inline void sbesseldm(int m, int lmax, double x, double *djl)
{
    if (m == 0) { sbessel(lmax, x, djl); return; }
    const int maxns = 20;
    if (x > 1.0) {
        double jl[EXS_LMAX_APW + 3];
        int a[8], a1[8], b[8], b1[8];
        sbessel(lmax + 1, x, jl);
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
        const double x2 = x * x;
        for (int l = 0; l <= lmax; l++) {
            int i0 = (m - l + 1) / 2;
            if (i0 < 0) i0 = 0;
            int j = 2 * i0 + l - m;
            double t1 = (j == 0) ? 1.0 : powi(x, j);
            const double p2 = powi(-2.0, i0);
            t1 = factr(j + m, j) * t1 / (factnm(i0, 1) * factnm(j + l + m + 1, 2) * p2);
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
}

// Real Masters & Richards-Dinger values of one l: x(m), m = 0..l, already
// multiplied by sin(theta)^m and normalised, i.e. Y_lm = xm[m] * e^{i m phi}
// for m >= 0 (genylm.f90:58-83).  Y_00 = 0.28209479177387814347.
__device__ inline void ylm_l(int l, double sn, double cs, double *xm)
{
    const double fourpi = 12.566370614359172954;
    if (l == 0) { xm[0] = 0.28209479177387814347; return; }
    xm[l] = (l % 2 == 0) ? 1.0 : -1.0;
    double dx = 0.0;
    for (int m = l; m >= 1; m--) {
        const double t1 = sqrt((double)((l + m) * (l - m + 1)));
        xm[m - 1] = -(sn * dx + (double)(2 * m) * cs * xm[m]) / t1;
        dx = sn * xm[m] * t1;
    }
    double t1 = sn, sum = 0.0;
    for (int m = 1; m <= l; m++) {
        xm[m] = t1 * xm[m];
        sum = sum + xm[m] * xm[m];
        t1 = t1 * sn;
    }
    sum = 2.0 * sum + xm[0] * xm[0];
    t1 = sqrt((double)(2 * l + 1) / (fourpi * sum));
    for (int m = 0; m <= l; m++) xm[m] = t1 * xm[m];
}

// m-th derivative of the interpolating polynomial through np <= 4 points.
__device__ inline double polynom(int m, int np, const double *xa, const double *ya, double x)
{
    double x1, x2, x3, y1, y2, y3, t1, t2, t3, t4, t5, t6, t7, c1, c2, c3;
    switch (np) {
    case 1:
        return (m == 0) ? ya[0] : 0.0;
    case 2:
        c1 = (ya[1] - ya[0]) / (xa[1] - xa[0]);
        t1 = x - xa[0];
        if (m == 0) return c1 * t1 + ya[0];
        if (m == 1) return c1;
        return 0.0;
    case 3:
        x1 = xa[1] - xa[0]; x2 = xa[2] - xa[0];
        y1 = ya[1] - ya[0]; y2 = ya[2] - ya[0];
        t1 = 1.0 / (x1 * x2 * (x2 - x1));
        t2 = x1 * y2; t3 = x2 * y1;
        c1 = t1 * (x2 * t3 - x1 * t2);
        c2 = t1 * (t2 - t3);
        t1 = x - xa[0];
        if (m == 0) return ya[0] + t1 * (c1 + c2 * t1);
        if (m == 1) return 2.0 * c2 * t1 + c1;
        if (m == 2) return 2.0 * c2;
        return 0.0;
    default:  // np == 4
        x1 = xa[1] - xa[0]; x2 = xa[2] - xa[0]; x3 = xa[3] - xa[0];
        y1 = ya[1] - ya[0]; y2 = ya[2] - ya[0]; y3 = ya[3] - ya[0];
        t1 = 1.0 / (x1 * x2 * x3 * (x1 - x2) * (x1 - x3) * (x2 - x3));
        t2 = x1 * x2 * y3; t3 = x2 * x3 * y1; t4 = x3 * x1 * y2;
        t5 = x1 * x1; t6 = x2 * x2; t7 = x3 * x3;
        c1 = t1 * (t3 * (x3 * t6 - x2 * t7) + t4 * (x1 * t7 - x3 * t5) + t2 * (x2 * t5 - x1 * t6));
        c2 = t1 * (t3 * (t7 - t6) + t4 * (t5 - t7) + t2 * (t6 - t5));
        c3 = t1 * (t3 * (x2 - x3) + t4 * (x3 - x1) + t2 * (x1 - x2));
        t1 = x - xa[0];
        if (m == 0) return ya[0] + t1 * (c1 + t1 * (c2 + c3 * t1));
        if (m == 1) return c1 + t1 * (2.0 * c2 + 3.0 * c3 * t1);
        if (m == 2) return 6.0 * c3 * t1 + 2.0 * c2;
        if (m == 3) return 6.0 * c3;
        return 0.0;
    }
}

// |v| and (theta, phi) of v (sphcrd.f90:30-56).
__device__ inline void sphcrd(const double v[3], double *r, double *theta, double *phi)
{
    const double twopi = 6.2831853071795864769, eps = 1e-14;
    *r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (*r > eps) {
        double t1 = v[2] / *r;
        t1 = (t1 > 0.0) ? fmin(t1, 1.0) : fmax(t1, -1.0);
        *theta = acos(t1);
        if (fabs(v[0]) > eps || fabs(v[1]) > eps) {
            double p = atan2(v[1], v[0]);
            if (p < 0.0) p += twopi;
            *phi = p;
        } else {
            *phi = 0.0;
        }
    } else {
        *theta = 0.0;
        *phi = 0.0;
    }
}

// In-place LU with partial pivoting of the real n x n matching matrix
// (the steps of LAPACK zgetrf for n <= 4: pivot on the largest |d|, scale
// the column by the reciprocal pivot, rank-1 update).  Returns 0 or k > 0
// when U(k,k) is exactly zero.
__device__ inline int lu_factor(int n, double *d, int *ipiv)
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
                const double t = d[k + j * n]; d[k + j * n] = d[p + j * n]; d[p + j * n] = t;
            }
        const double r = 1.0 / d[k + k * n];
        for (int i = k + 1; i < n; i++) d[i + k * n] *= r;
        for (int j = k + 1; j < n; j++)
            for (int i = k + 1; i < n; i++) d[i + j * n] -= d[i + k * n] * d[k + j * n];
    }
    return 0;
}

// zgetrs steps for one complex right-hand side (re, im held separately).
__device__ inline void lu_solve(int n, const double *d, const int *ipiv, double *br, double *bi)
{
    for (int k = 0; k < n; k++)
        if (ipiv[k] != k) {
            const int p = ipiv[k];
            double t = br[k]; br[k] = br[p]; br[p] = t;
            t = bi[k]; bi[k] = bi[p]; bi[p] = t;
        }
    for (int k = 0; k < n; k++)
        for (int i = k + 1; i < n; i++) { br[i] -= br[k] * d[i + k * n]; bi[i] -= bi[k] * d[i + k * n]; }
    for (int k = n - 1; k >= 0; k--) {
        br[k] = br[k] / d[k + k * n];
        bi[k] = bi[k] / d[k + k * n];
        for (int i = 0; i < k; i++) { br[i] -= br[k] * d[i + k * n]; bi[i] -= bi[k] * d[i + k * n]; }
    }
}

}  // namespace exs
