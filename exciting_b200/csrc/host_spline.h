// Cubic-spline integral and derivative of tabulated radial functions (host
// code of the muffin-tin integral and momentum-matrix generation).
#pragma once
#include <vector>

namespace exs {

// Coefficients of the spline through (x_i, f_i): c_i = f''(x_i)/2 and the
// slopes s_i of the segments, with the end values of c from the second
// divided differences of the first and last three points (the end
// conditions of src/src_lib/spline.f90); forward elimination of the
// tridiagonal rows, then back substitution c_i = (r_i - c_{i+1}) / pivot_i.
inline void spline_curvatures(int n, const double *x, const double *f, double *s, double *piv, double *c)
{
    for (int i = 0; i + 1 < n; i++) s[i] = (f[i + 1] - f[i]) / (x[i + 1] - x[i]);
    c[0] = (s[1] - s[0]) / (x[2] - x[0]);
    c[n - 1] = (s[n - 2] - s[n - 3]) / (x[n - 1] - x[n - 3]);
    double inv_prev = 0.0, rhs_prev = 0.0;
    for (int i = 1; i + 1 < n; i++) {
        const double ratio = (x[i] - x[i - 1]) / (x[i + 1] - x[i]);
        const double rhs = 3.0 * (s[i] - s[i - 1]) / (x[i + 1] - x[i]);
        double r;
        if (i == 1) {
            piv[i] = 1.0 / (2.0 * (ratio + 1.0));
            r = rhs - ratio * c[0];
        } else {
            const double m = ratio * inv_prev;
            piv[i] = 1.0 / (2.0 * ratio + 2.0 - m);
            r = rhs - m * rhs_prev;
        }
        c[i] = r;
        inv_prev = piv[i];
        rhs_prev = r;
    }
    double next = c[n - 1];
    for (int i = n - 2; i >= 1; i--) {
        c[i] = (c[i] - next) * piv[i];
        next = c[i];
    }
}

// Integral from x[0] to x[n-1] of the cubic spline through (x_i, f_i) whose
// end second derivatives are taken from the second divided differences of
// the first and last three points (the end conditions of
// src/src_lib/spline.f90), integrated piecewise as in src/src_lib/fderiv.f90
// (m = -1).  With c_i = f''(x_i)/2 the interior rows read
//   h_{i-1} c_{i-1} + 2 (h_{i-1} + h_i) c_i + h_i c_{i+1} = 3 (s_i - s_{i-1}),
// s_i the slope of segment i; solved by forward elimination and back
// substitution.  Scratch needs 3n doubles.
inline double spline_integral(int n, const double *x, const double *f, double *scratch)
{
    double *s = scratch, *piv = scratch + n, *c = scratch + 2 * n;
    spline_curvatures(n, x, f, s, piv, c);
    double g = 0.0;
    for (int i = 0; i + 1 < n; i++) {
        const double h = x[i + 1] - x[i];
        const double d = (c[i + 1] - c[i]) / (3.0 * h);        // cubic coefficient
        const double b = s[i] - (c[i] + d * h) * h;            // linear coefficient
        g += (((0.25 * d * h + c[i] / 3.0) * h + 0.5 * b) * h + f[i]) * h;
    }
    return g;
}

// Weights w with sum_r w_r f_r = spline_integral(f): the integral applied to
// the unit vectors of the mesh.
inline void spline_weights(int n, const double *x, double *w)
{
    std::vector<double> e(n, 0.0), scratch(3 * (size_t)n);
    for (int j = 0; j < n; j++) {
        e[j] = 1.0;
        w[j] = spline_integral(n, x, e.data(), scratch.data());
        e[j] = 0.0;
    }
}

// First derivative of the spline at the points (fderiv with m = 1,
// src/src_lib/fderiv.f90): the linear coefficient b_i = s_i - (c_i + d_i h) h
// of segment i, and at the last point the derivative of the last segment at
// its end.  Scratch needs 3n doubles.
inline void spline_derivative(int n, const double *x, const double *f, double *g, double *scratch)
{
    double *s = scratch, *piv = scratch + n, *c = scratch + 2 * n;
    spline_curvatures(n, x, f, s, piv, c);
    double d = 0.0, h = 0.0;
    for (int i = 0; i + 1 < n; i++) {
        h = x[i + 1] - x[i];
        d = (c[i + 1] - c[i]) / (3.0 * h);
        g[i] = s[i] - (c[i] + d * h) * h;
    }
    g[n - 1] = g[n - 2] + (2.0 * c[n - 2] + 3.0 * d * h) * h;
}

}  // namespace exs
