// Interstitial H and O element of the APW-APW block, shared by the FP64 and
// the split-precision contraction epilogues.
#pragma once
#include "exs_internal.cuh"

namespace exs {

// Interstitial term of element (i, j), i <= j < ngp (hmlistln.f90:61-86,
// olpistln.f90:53-82).  Returns false when nothing is added.  The tables are
// read-only during every kernel that calls this (read-only data path).
__device__ __forceinline__ bool interstitial(const DevParams &p, int kind, const int *ivi, const int *ivj,
                                             const double *vi, const double *vj, double &zr, double &zi)
{
    const int d0 = ivi[0] - ivj[0] - p.intgv_lo[0];
    const int d1 = ivi[1] - ivj[1] - p.intgv_lo[1];
    const int d2 = ivi[2] - ivj[2] - p.intgv_lo[2];
    if ((unsigned)d0 >= (unsigned)p.intgv_n[0] || (unsigned)d1 >= (unsigned)p.intgv_n[1] ||
        (unsigned)d2 >= (unsigned)p.intgv_n[2]) {
        atomicOr(p.err, DEV_ERR_INDEX);
        return false;
    }
    const int ig = __ldg(p.ivgig + d0 + p.intgv_n[0] * (d1 + p.intgv_n[1] * d2));
    if (ig <= 0 || ig > p.ngvec) return false;
    const double dp = vi[0] * vj[0] + vi[1] * vj[1] + vi[2] * vj[2];
    if (kind == EPI_HAM) {
        const double t1 = 0.5 * dp;
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p.veffig) + ig - 1);
        const double2 w = __ldg(reinterpret_cast<const double2 *>(p.kinw) + ig - 1);
        zr = v.x + t1 * w.x;
        zi = v.y + t1 * w.y;
    } else {
        const double2 cc = __ldg(reinterpret_cast<const double2 *>(p.cfunig) + ig - 1);
        exs_complex c;
        c.re = cc.x;
        c.im = cc.y;
        if (p.relativity == EXS_REL_IORA) {
            const double alpha = 1.0 / 137.03599911, a2 = 0.5 * alpha * alpha;
            const double t1 = 0.5 * a2 * dp;
            const exs_complex w = p.m2effig[ig - 1];
            zr = t1 * w.re + c.re;
            zi = t1 * w.im + c.im;
        } else {
            zr = c.re;
            zi = c.im;
        }
    }
    return true;
}

}  // namespace exs
