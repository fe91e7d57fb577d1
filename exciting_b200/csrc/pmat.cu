// Momentum matrix elements of the LAPW+lo basis for real-time TDDFT on the
// device.  Replaces Obtain_Pmat_LAPWLOBasis
// (src/src_xs/src_rttddft/rttddft_pmat.f90:22-64): the radial-angular
// integrals of pmatrad (src/src_xs/pmatrad.F90, with the gradient of
// gradzfmtr, src/src_xs/gradzfmtr.F90), then per k-point genpmatbasisik
// (:66-188).
//
// The gradient of u(r) Y_lm has components only in Y_{l+-1, m+q}, q = -1..1,
// so every integral <phi_1 Y_1 | d/dx_j | phi_2 Y_2> is one angular
// coefficient times one of two radial integrals per pair of radial
// functions; the host builds these small per-atom matrices (R for APW-APW,
// RL for APW-lo, RLA for lo-APW, RLL for lo-lo).  Per k-point and direction
// the device then forms
//   P^T = sum_atoms A R^T A^H  (+ the lo blocks)
// with cuBLAS ZGEMMs (plain library GEMMs: this runs once per propagation),
// and one tiled kernel transposes P^T, multiplies the x and z components by
// -i (:170-171) and adds (k+G_j)_x Theta(G_i - G_j) (:173-184), writing
// straight into the momentum matrices that exs_rttddft_updateham reads.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "exs_internal.cuh"
#include "host_spline.h"

namespace {

int pfail(exs_ctx *c, int code, const std::string &msg)
{
    if (c) c->last_error = msg;
    return code;
}

#define PM_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return pfail(c, EXS_ERR_CUDA, std::string(#call ": ") + \
                                                                 cudaGetErrorString(e_)); \
    } while (0)
#define PM_BLAS(call)                                                                                  \
    do {                                                                                               \
        cublasStatus_t e_ = (call);                                                                    \
        if (e_ != CUBLAS_STATUS_SUCCESS) return pfail(c, EXS_ERR_CUDA, std::string(#call " failed")); \
    } while (0)

// <l2 m2; 1 q | l m> for l = l2 +- 1: the vector-coupling coefficients of
// an angular momentum with a unit one, in their closed forms (j = l2,
// M = m = m2 + q).
double cg_unit(int l2, int m2, int q, int l, int m)
{
    if (m2 + q != m || std::abs(m2) > l2 || std::abs(m) > l || l2 < 0) return 0.0;
    const double j = l2, M = m;
    if (l == l2 + 1) {
        if (q == 1) return std::sqrt((j + M) * (j + M + 1) / ((2 * j + 1) * (2 * j + 2)));
        if (q == 0) return std::sqrt((j - M + 1) * (j + M + 1) / ((2 * j + 1) * (j + 1)));
        return std::sqrt((j - M) * (j - M + 1) / ((2 * j + 1) * (2 * j + 2)));
    }
    if (l == l2 - 1) {
        if (q == 1) return std::sqrt((j - M) * (j - M + 1) / (2 * j * (2 * j + 1)));
        if (q == 0) return -std::sqrt((j - M) * (j + M) / (j * (2 * j + 1)));
        return std::sqrt((j + M + 1) * (j + M) / (2 * j * (2 * j + 1)));
    }
    return 0.0;
}

// Cartesian coefficient (x, y, z) of Y_{l2 m2} in the gradient of u Y_lm
// (gradzfmtr.F90:27-70; the y entry is -i d/dy).
double grad_coef(int j, int l2, int m2, int l, int m)
{
    const double t3 = cg_unit(l2, m2, -1, l, m), t4 = cg_unit(l2, m2, 0, l, m), t5 = cg_unit(l2, m2, 1, l, m);
    if (j == 0) return (t3 - t5) / std::sqrt(2.0);
    if (j == 1) return (-t3 - t5) / std::sqrt(2.0);
    return t4;
}

struct Fun {          // a radial function of one atom
    int l;
    const double *u;  // u(r) on the species mesh
};

// Per-atom matrices of one call, complex (real values), column-major.
struct AtomMats {
    int F = 0, L = 0;                 // APW functions (l <= lmaxapw), lo functions
    std::vector<int> col_io, col_lm;  // APW function f -> (io, lm)
    std::vector<int> lo_pos;          // lo function c -> position within the atom's lo block
    std::vector<exs_complex> R[3], RL[3], RLA[3], RLLt[3];
};

void build_atom(const exs_ctx *c, const exs_mt_radial *in, int ias, const std::vector<double> &w, AtomMats &a)
{
    const int is = c->atom_species[ias], nr = in->nrmt[is], nrmtmax = in->nrmtmax;
    const int lmaxapw = c->lmaxapw, ao = c->apwordmax, nlomax = c->nlomax;
    const double *r = in->spr + (size_t)nrmtmax * is;
    const int *apw = c->apword.data() + (size_t)(lmaxapw + 1) * is;
    // functions in the order l, m, io (APW) and the atom's lo block order
    std::vector<Fun> fa, fl;
    std::vector<int> fa_m, fl_m;
    for (int l = 0; l <= lmaxapw; l++)
        for (int m = -l; m <= l; m++)
            for (int io = 0; io < apw[l]; io++) {
                a.col_io.push_back(io);
                a.col_lm.push_back(l * (l + 1) + m);
                fa.push_back(Fun{l, in->apwfr + (size_t)nrmtmax * 2 * (io + (size_t)ao * (l + (size_t)(lmaxapw + 1) * ias))});
                fa_m.push_back(m);
            }
    const exs::AtomDesc &at = c->atoms[ias];
    const int nlo = c->nlorb[is];
    for (int ilo = 0; ilo < nlo; ilo++) {
        const int l = c->lorbl[ilo + (size_t)nlomax * is];
        for (int m = -l; m <= l; m++) {
            const int g = c->idxlo[(l * (l + 1) + m) + (size_t)c->lolmmax * (ilo + (size_t)nlomax * ias)] - 1;
            a.lo_pos.push_back(g - at.lo_off);
            fl.push_back(Fun{l, in->lofr + (size_t)nrmtmax * 2 * (ilo + (size_t)nlomax * ias)});
            fl_m.push_back(m);
        }
    }
    a.F = (int)fa.size();
    a.L = (int)fl.size();
    // radial parts of the gradient of each distinct radial function:
    // tp = t1 (u l / r - u') (component l + 1), tm = t2 (u (l+1) / r + u') (l - 1)
    struct Rad {
        std::vector<double> tp, tm;
    };
    auto radial = [&](const Fun &f) {
        Rad q;
        std::vector<double> du(nr), scratch(3 * (size_t)nr);
        exs::spline_derivative(nr, r, f.u, du.data(), scratch.data());
        const double t1 = std::sqrt((double)(f.l + 1) / (2 * f.l + 1)), t2 = std::sqrt((double)f.l / (2 * f.l + 1));
        q.tp.resize(nr);
        q.tm.resize(nr);
        for (int i = 0; i < nr; i++) {
            q.tp[i] = t1 * (f.u[i] * (double)f.l / r[i] - du[i]);
            q.tm[i] = t2 * (f.u[i] * (double)(f.l + 1) / r[i] + du[i]);
        }
        return q;
    };
    std::vector<Rad> ra(fa.size()), rl(fl.size());
    for (size_t i = 0; i < fa.size(); i++) ra[i] = radial(fa[i]);
    for (size_t i = 0; i < fl.size(); i++) rl[i] = radial(fl[i]);
    // <phi_1 Y_{l1 m1} | d_j | phi_2 Y_{l2 m2}> = coef_j(l1 m1; l2 m2) int r^2 phi_1 t(phi_2)
    auto elem = [&](const Fun &f1, int m1, const Fun &f2, int m2, const Rad &q2, double *out3) {
        out3[0] = out3[1] = out3[2] = 0.0;
        const std::vector<double> *t = nullptr;
        if (f1.l == f2.l + 1 && f1.l <= lmaxapw) t = &q2.tp;
        else if (f1.l == f2.l - 1) t = &q2.tm;
        if (!t || std::abs(m1 - m2) > 1) return;
        double integ = 0.0;
        for (int i = 0; i < nr; i++) integ += w[i] * (r[i] * r[i] * f1.u[i] * (*t)[i]);
        for (int j = 0; j < 3; j++) out3[j] = grad_coef(j, f1.l, m1, f2.l, m2) * integ;
    };
    const int F = a.F, L = a.L;
    for (int j = 0; j < 3; j++) {
        a.R[j].assign((size_t)F * F, exs_complex{0, 0});
        a.RL[j].assign((size_t)F * L, exs_complex{0, 0});
        a.RLA[j].assign((size_t)L * F, exs_complex{0, 0});
        a.RLLt[j].assign((size_t)L * L, exs_complex{0, 0});
    }
    double v[3];
    for (int f1 = 0; f1 < F; f1++)
        for (int f2 = 0; f2 < F; f2++) {
            elem(fa[f1], fa_m[f1], fa[f2], fa_m[f2], ra[f2], v);
            for (int j = 0; j < 3; j++) a.R[j][f1 + (size_t)F * f2].re = v[j];
        }
    for (int f1 = 0; f1 < F; f1++)
        for (int c2 = 0; c2 < L; c2++) {   // ripalo: APW row, lo column (pmatrad.F90:84-104)
            elem(fa[f1], fa_m[f1], fl[c2], fl_m[c2], rl[c2], v);
            for (int j = 0; j < 3; j++) a.RL[j][f1 + (size_t)F * a.lo_pos[c2]].re = v[j];
        }
    for (int c1 = 0; c1 < L; c1++) {
        for (int f2 = 0; f2 < F; f2++) {   // riploa: lo row, APW column (:105-125)
            elem(fl[c1], fl_m[c1], fa[f2], fa_m[f2], ra[f2], v);
            for (int j = 0; j < 3; j++) a.RLA[j][a.lo_pos[c1] + (size_t)L * f2].re = v[j];
        }
        for (int c2 = 0; c2 < L; c2++) {   // riplolo (:126-145), stored transposed
            elem(fl[c1], fl_m[c1], fl[c2], fl_m[c2], rl[c2], v);
            for (int j = 0; j < 3; j++) a.RLLt[j][a.lo_pos[c2] + (size_t)L * a.lo_pos[c1]].re = v[j];
        }
    }
}

struct PmArgs {
    int ngp, nmat, comp;
    const exs_complex *q;        // P^T of this component, (nmat, nmat)
    exs_complex *p;              // P, (nmat, nmat)
    const int *igpig;            // (ngp) 1-based G indices
    const double *vgpc;          // (3, ngp)
};

// grid (ceil(nmat/32), ceil(nmat/32)), 32 x 8 threads: P(i, j) = fac Q(j, i)
// + [i, j < ngp] vgpc(comp, j) cfunig(G_i - G_j), fac = -i for x and z.
__global__ void __launch_bounds__(256) pm_finish_kernel(exs::DevParams p, PmArgs a)
{
    __shared__ double2 tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += 8) {           // Q(j0 + k, i0 + tx) ... read Q column i0+k
        const int jj = j0 + tx, ii = i0 + k;
        double2 v = make_double2(0.0, 0.0);
        if (jj < a.nmat && ii < a.nmat) v = reinterpret_cast<const double2 *>(a.q)[jj + (size_t)a.nmat * ii];
        tile[k][tx] = v;                          // tile[i - i0][j - j0] = Q(j, i)
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int i = i0 + tx, j = j0 + k;
        if (i >= a.nmat || j >= a.nmat) continue;
        double2 v = tile[tx][k];
        if (a.comp != 1) v = make_double2(v.y, -v.x);   // -i (x + iy) = y - ix
        if (i < a.ngp && j < a.ngp) {
            const int gi = a.igpig[i] - 1, gj = a.igpig[j] - 1;
            bool ok = gi >= 0 && gi < p.ngrtot && gj >= 0 && gj < p.ngrtot;
            int ig = 0;
            if (ok) {
                const int d0 = p.ivg[3 * gi] - p.ivg[3 * gj] - p.intgv_lo[0];
                const int d1 = p.ivg[3 * gi + 1] - p.ivg[3 * gj + 1] - p.intgv_lo[1];
                const int d2 = p.ivg[3 * gi + 2] - p.ivg[3 * gj + 2] - p.intgv_lo[2];
                ok = (unsigned)d0 < (unsigned)p.intgv_n[0] && (unsigned)d1 < (unsigned)p.intgv_n[1] &&
                     (unsigned)d2 < (unsigned)p.intgv_n[2];
                if (ok) ig = p.ivgig[d0 + p.intgv_n[0] * (d1 + p.intgv_n[1] * d2)];
                ok = ok && ig > 0 && ig <= p.ngvec;
            }
            if (!ok) {
                atomicOr(p.err, exs::DEV_ERR_INDEX);
            } else {
                const double vj = a.vgpc[3 * j + a.comp];
                const double2 th = reinterpret_cast<const double2 *>(p.cfunig)[ig - 1];
                v.x += vj * th.x;
                v.y += vj * th.y;
            }
        }
        reinterpret_cast<double2 *>(a.p)[i + (size_t)a.nmat * j] = v;
    }
}

struct PmState {
    cublasHandle_t blas = nullptr;
    exs_complex *d_mats = nullptr;   // the per-atom matrices of the call
    size_t mats_cap = 0;
    exs_complex *d_a = nullptr;      // matching coefficients of one k-point, compact per atom
    size_t a_cap = 0;
    exs_complex *d_t = nullptr;      // A R^T of one atom
    size_t t_cap = 0;
    exs_complex *d_q = nullptr;      // P^T of one component
    size_t q_cap = 0;
    int *d_ig = nullptr;
    double *d_vg = nullptr;
    size_t ig_cap = 0, vg_cap = 0;
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

}  // namespace

namespace exs {
void pm_release(exs_ctx *c)
{
    PmState *m = (PmState *)c->pm;
    if (!m) return;
    if (m->blas) cublasDestroy(m->blas);
    void *ps[] = {m->d_mats, m->d_a, m->d_t, m->d_q, m->d_ig, m->d_vg};
    for (void *q : ps)
        if (q) cudaFree(q);
    delete m;
    c->pm = nullptr;
}
}  // namespace exs

extern "C" {

int exs_rttddft_genpmat(exs_ctx *c, int nk, const int *ngp, const int *igpig, const double *vgpc,
                        const exs_complex *const *apwalm, const exs_mt_radial *in, exs_complex *const *pmat, int ld)
{
    if (!c || !in || nk < 0 || (nk > 0 && (!ngp || !igpig || !vgpc || !apwalm)))
        return pfail(c, EXS_ERR_ARG, "exs_rttddft_genpmat: bad argument");
    if (!in->nrmt || !in->spr || !in->apwfr || (c->nlotot > 0 && !in->lofr))
        return pfail(c, EXS_ERR_ARG, "exs_rttddft_genpmat: missing radial functions");
    if (!c->have_inputs) return pfail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    if (nk > c->max_batch) return pfail(c, EXS_ERR_SIZE, "nk exceeds max_batch");
    for (int is = 0; is < c->nspecies; is++)
        if (in->nrmt[is] < 4 || in->nrmt[is] > in->nrmtmax)
            return pfail(c, EXS_ERR_SIZE, "exs_rttddft_genpmat: nrmt outside 4..nrmtmax");
    std::vector<int> nmat(nk);
    for (int k = 0; k < nk; k++) {
        if (ngp[k] <= 0 || ngp[k] > c->ngkmax || !apwalm[k]) return pfail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax");
        nmat[k] = ngp[k] + c->nlotot;
        if (pmat && pmat[k] && ld < nmat[k]) return pfail(c, EXS_ERR_SIZE, "ld < nmat");
    }
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    if (!c->pm) c->pm = new PmState;
    PmState &m = *(PmState *)c->pm;
    if (!m.blas) {
        PM_BLAS(cublasCreate(&m.blas));
    }
    PM_BLAS(cublasSetStream(m.blas, s));
    PM_CUDA(cudaStreamSynchronize(s));
    PM_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));

    // ---- per-atom matrices (host), uploaded once for all k-points
    const int nat = c->natmtot;
    std::vector<AtomMats> mats(nat);
    std::vector<std::vector<double>> wsp(c->nspecies);
    for (int is = 0; is < c->nspecies; is++) {
        wsp[is].assign(in->nrmt[is], 0.0);
        exs::spline_weights(in->nrmt[is], in->spr + (size_t)in->nrmtmax * is, wsp[is].data());
    }
    std::vector<size_t> moff(nat);
    size_t mtot = 0;
    int Fmax = 0;
    for (int a = 0; a < nat; a++) {
        build_atom(c, in, a, wsp[c->atom_species[a]], mats[a]);
        const AtomMats &x = mats[a];
        moff[a] = mtot;
        mtot += 3 * ((size_t)x.F * x.F + 2 * (size_t)x.F * x.L + (size_t)x.L * x.L);
        Fmax = std::max(Fmax, x.F);
    }
    PM_CUDA(grow(&m.d_mats, &m.mats_cap, mtot));
    {
        std::vector<exs_complex> h(mtot);
        for (int a = 0; a < nat; a++) {
            const AtomMats &x = mats[a];
            size_t o = moff[a];
            for (int j = 0; j < 3; j++) {
                for (const auto *v : {&x.R[j], &x.RL[j], &x.RLA[j], &x.RLLt[j]}) {
                    std::copy(v->begin(), v->end(), h.begin() + o);
                    o += v->size();
                }
            }
        }
        PM_CUDA(cudaMemcpyAsync(m.d_mats, h.data(), sizeof(exs_complex) * mtot, cudaMemcpyHostToDevice, s));
        PM_CUDA(cudaStreamSynchronize(s));
    }

    // ---- registered momentum matrices: (nmat, nmat, 3) per k-point
    exs_complex *d_p = nullptr;
    std::vector<size_t> poff(nk);
    int rc = exs::rt_reserve_pmat(c, nk, nmat.data(), &d_p, poff.data());
    if (rc != EXS_OK) return rc;

    size_t amax = 0, qmax = 0;
    int Ftot = 0;
    for (int a = 0; a < nat; a++) Ftot += mats[a].F;
    for (int k = 0; k < nk; k++) {
        amax = std::max(amax, (size_t)ngp[k] * Ftot);
        qmax = std::max(qmax, (size_t)nmat[k] * nmat[k]);
    }
    PM_CUDA(grow(&m.d_a, &m.a_cap, amax));
    PM_CUDA(grow(&m.d_t, &m.t_cap, (size_t)c->ngkmax * std::max(Fmax, 1)));
    PM_CUDA(grow(&m.d_q, &m.q_cap, qmax));
    PM_CUDA(grow(&m.d_ig, &m.ig_cap, (size_t)c->ngkmax));
    PM_CUDA(grow(&m.d_vg, &m.vg_cap, 3 * (size_t)c->ngkmax));

    const exs::DevParams dp = c->params();
    const int lmmaxapw = (c->lmaxapw + 1) * (c->lmaxapw + 1);
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    std::vector<exs_complex> hA;
    for (int k = 0; k < nk; k++) {
        const int ng = ngp[k], n = nmat[k];
        // matching coefficients of the atoms' APW functions, (ng, F_a) per atom
        hA.assign((size_t)ng * Ftot, exs_complex{0, 0});
        std::vector<size_t> aoff(nat);
        size_t o = 0;
        for (int a = 0; a < nat; a++) {
            aoff[a] = o;
            const AtomMats &x = mats[a];
            for (int f = 0; f < x.F; f++) {
                const exs_complex *src =
                    apwalm[k] + (size_t)c->ngkmax * (x.col_io[f] + (size_t)c->apwordmax * (x.col_lm[f] + (size_t)lmmaxapw * a));
                std::memcpy(hA.data() + o + (size_t)ng * f, src, sizeof(exs_complex) * ng);
            }
            o += (size_t)ng * x.F;
        }
        PM_CUDA(cudaMemcpyAsync(m.d_a, hA.data(), sizeof(exs_complex) * hA.size(), cudaMemcpyHostToDevice, s));
        PM_CUDA(cudaMemcpyAsync(m.d_ig, igpig + (size_t)c->ngkmax * k, sizeof(int) * ng, cudaMemcpyHostToDevice, s));
        PM_CUDA(cudaMemcpyAsync(m.d_vg, vgpc + 3 * (size_t)c->ngkmax * k, sizeof(double) * 3 * ng,
                                cudaMemcpyHostToDevice, s));
        auto Z = [](const exs_complex *p) { return reinterpret_cast<const cuDoubleComplex *>(p); };
        auto W = [](exs_complex *p) { return reinterpret_cast<cuDoubleComplex *>(p); };
        for (int j = 0; j < 3; j++) {
            PM_CUDA(cudaMemsetAsync(m.d_q, 0, sizeof(exs_complex) * (size_t)n * n, s));
            for (int a = 0; a < nat; a++) {
                const AtomMats &x = mats[a];
                if (x.F == 0) continue;
                const exs_complex *A = m.d_a + aoff[a];
                size_t mo = moff[a];
                for (int jj = 0; jj < j; jj++) mo += (size_t)x.F * x.F + 2 * (size_t)x.F * x.L + (size_t)x.L * x.L;
                const exs_complex *R = m.d_mats + mo, *RL = R + (size_t)x.F * x.F, *RLA = RL + (size_t)x.F * x.L,
                                  *RLLt = RLA + (size_t)x.L * x.F;
                // T = A R^T (ng x F); Q(0:ng, 0:ng) += T A^H
                PM_BLAS(cublasZgemm(m.blas, CUBLAS_OP_N, CUBLAS_OP_T, ng, x.F, x.F, &one, Z(A), ng, Z(R), x.F, &zero,
                                    W(m.d_t), ng));
                PM_BLAS(cublasZgemm(m.blas, CUBLAS_OP_N, CUBLAS_OP_C, ng, ng, x.F, &one, Z(m.d_t), ng, Z(A), ng, &one,
                                    W(m.d_q), n));
                if (x.L > 0) {
                    const int r0 = ng + c->atoms[a].lo_off;
                    // Q(lo rows, 0:ng) += RL^T A^H (P's APW-lo columns, transposed)
                    PM_BLAS(cublasZgemm(m.blas, CUBLAS_OP_T, CUBLAS_OP_C, x.L, ng, x.F, &one, Z(RL), x.F, Z(A), ng,
                                        &one, W(m.d_q + r0), n));
                    // Q(0:ng, lo columns) += A RLA^T (P's lo-APW rows, transposed)
                    PM_BLAS(cublasZgemm(m.blas, CUBLAS_OP_N, CUBLAS_OP_T, ng, x.L, x.F, &one, Z(A), ng, Z(RLA), x.L,
                                        &one, W(m.d_q + (size_t)n * r0), n));
                    // Q(lo, lo) = RLL^T (P's lo-lo block, set)
                    PM_CUDA(cudaMemcpy2DAsync(m.d_q + r0 + (size_t)n * r0, sizeof(exs_complex) * n, RLLt,
                                              sizeof(exs_complex) * x.L, sizeof(exs_complex) * x.L, x.L,
                                              cudaMemcpyDeviceToDevice, s));
                }
            }
            PmArgs pa{ng, n, j, m.d_q, d_p + poff[k] + (size_t)j * n * n, m.d_ig, m.d_vg};
            pm_finish_kernel<<<dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, s>>>(dp, pa);
            PM_CUDA(cudaGetLastError());
        }
        if (pmat && pmat[k])
            for (int j = 0; j < 3; j++)
                PM_CUDA(cudaMemcpy2DAsync(pmat[k] + (size_t)j * ld * ld, sizeof(exs_complex) * ld,
                                          d_p + poff[k] + (size_t)j * n * n, sizeof(exs_complex) * n,
                                          sizeof(exs_complex) * n, n, cudaMemcpyDeviceToHost, s));
        PM_CUDA(cudaStreamSynchronize(s));   // hA is reused for the next k-point
    }
    return exs_synchronize(c);
}

int exs_clebgor_unit(int l2, int m2, int q, int l, int m, double *value)
{
    if (!value) return EXS_ERR_ARG;
    *value = cg_unit(l2, m2, q, l, m);
    return EXS_OK;
}

}  // extern "C"
