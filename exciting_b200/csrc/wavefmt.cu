// Muffin-tin wavefunction coefficients of the first-variational states on
// the device: the consumer of the matching coefficients that the density
// (rhovalk.f90:119-142) and the LDA+U density matrix (gendmatmt.f90, after
// match at :72) call per state and atom.  Replaces the loop of
//   call wavefmt(lrstp, lmax, is, ia, ngp, apwalm, evecfv(:, ist), ld, wfmt)
// (src/wavefmt.f90:13-124) over all atoms and states:
//   wfmt(lm, ir) = sum_io [sum_G evecfv(G) apwalm(G, io, lm, ias)] u_{io,l}(r_ir)
//                + sum_ilo evecfv(ngp + idxlo(lm, ilo, ias)) v_ilo(r_ir)  (l_ilo = l)
// on the radial points ir = 1, 1 + lrstp, ... of the atom's mesh
// (src/wavefmt.f90:82-121, wavefmt_add :126-174).
//
// The G sums for all (io, lm, atom) and states are one complex product
// C = apwalm(1:ngp, :)^T evecfv(1:ngp, :) (no conjugation: zdotu), a plain
// library GEMM (cuBLAS ZGEMM); one kernel then expands C and the
// local-orbital coefficients on the radial functions, one thread per
// (lm, radial point) of an (atom, state).  wavefmt_add skips constants below
// 1e-14 in magnitude (:152-170); the device adds every term, which differs
// from the skipped ones by less than 1e-14 |u|.
#include <cublas_v2.h>

#include <algorithm>
#include <string>

#include "exs_internal.cuh"

namespace {

int wfail(exs_ctx *c, int code, const std::string &msg)
{
    if (c) c->last_error = msg;
    return code;
}

#define WF_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return wfail(c, EXS_ERR_CUDA, std::string(#call ": ") + \
                                                                 cudaGetErrorString(e_)); \
    } while (0)
#define WF_BLAS(call)                                                                                  \
    do {                                                                                               \
        cublasStatus_t e_ = (call);                                                                    \
        if (e_ != CUBLAS_STATUS_SUCCESS) return wfail(c, EXS_ERR_CUDA, std::string(#call " failed")); \
    } while (0)

struct WfState {
    cublasHandle_t blas = nullptr;
    exs_complex *d_alm = nullptr;    // apwalm(ngkmax, apwordmax, lmmaxapw, natmtot)
    size_t alm_cap = 0;
    exs_complex *d_ev = nullptr;     // evecfv(nmat, nst)
    size_t ev_cap = 0;
    exs_complex *d_c = nullptr;      // C(apwordmax * lmmaxapw * natmtot, nst)
    size_t c_cap = 0;
    double *d_fr = nullptr;          // apwfr, then lofr
    size_t fr_cap = 0;
    int *d_nrmt = nullptr;           // nspecies
    size_t nrmt_cap = 0;
    exs_complex *d_out = nullptr;    // wfmt(ld, nrc, natmtot, nst)
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

struct WfArgs {
    int ngp, nmat, nst, lrstp, lmax, ld, nrc, nrmtmax;
    const exs_complex *c;        // (apwordmax * lmmaxapw * natmtot, nst)
    const exs_complex *ev;       // (nmat, nst)
    const double *apwfr;         // (nrmtmax, 2, apwordmax, lmaxapw + 1, natmtot)
    const double *lofr;          // (nrmtmax, 2, nlomax, natmtot) or null
    const int *nrmt;             // nspecies
    exs_complex *out;            // (ld, nrc, natmtot, nst)
};

// One block per (atom, state) and range of radial points; threads over
// (lm, radial point) with lm fastest, so a warp writes consecutive lm of one
// point (the layout of wfmt(ld, nr)).
__global__ void wavefmt_kernel(exs::DevParams p, WfArgs a)
{
    const int ias = blockIdx.y, ist = blockIdx.z;
    const int is = p.atoms[ias].species;
    const int nr = (a.nrmt[is] - 1) / a.lrstp + 1;
    const int lmmax = (a.lmax + 1) * (a.lmax + 1);
    const int *apw = p.apword + (size_t)(p.lmaxapw + 1) * is;
    const size_t M = (size_t)p.apwordmax * p.lmmaxapw * p.natmtot;
    exs_complex *out = a.out + (size_t)a.ld * a.nrc * (ias + (size_t)p.natmtot * ist);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.ld * a.nrc; t += gridDim.x * blockDim.x) {
        const int lm = t % a.ld, ir = t / a.ld;
        double re = 0.0, im = 0.0;
        if (lm < lmmax && ir < nr) {
            int l = 0;
            while ((l + 1) * (l + 1) <= lm) l++;
            const size_t r = (size_t)ir * a.lrstp;
            for (int io = 0; io < apw[l]; io++) {
                const exs_complex z = a.c[io + (size_t)p.apwordmax * (lm + (size_t)p.lmmaxapw * ias) + M * ist];
                const double u =
                    a.apwfr[r + (size_t)a.nrmtmax * 2 * (io + (size_t)p.apwordmax * (l + (size_t)(p.lmaxapw + 1) * ias))];
                re += z.re * u;
                im += z.im * u;
            }
            if (a.lofr) {
                const int nlo = p.nlorb[is];
                for (int ilo = 0; ilo < nlo; ilo++) {
                    if (p.lorbl[ilo + (size_t)p.nlomax * is] != l) continue;
                    const int idx = p.idxlo[lm + (size_t)p.lolmmax * (ilo + (size_t)p.nlomax * ias)];
                    const int row = a.ngp + idx - 1;
                    if (idx < 1 || row >= a.nmat) {
                        atomicOr(p.err, exs::DEV_ERR_INDEX);
                        continue;
                    }
                    const exs_complex z = a.ev[row + (size_t)a.nmat * ist];
                    const double v = a.lofr[r + (size_t)a.nrmtmax * 2 * (ilo + (size_t)p.nlomax * ias)];
                    re += z.re * v;
                    im += z.im * v;
                }
            }
        }
        exs_complex o;
        o.re = re;
        o.im = im;
        out[t] = o;
    }
}

}  // namespace

namespace exs {
void wf_release(exs_ctx *c)
{
    WfState *m = (WfState *)c->wf;
    if (!m) return;
    if (m->blas) cublasDestroy(m->blas);
    void *ps[] = {m->d_alm, m->d_ev, m->d_c, m->d_fr, m->d_nrmt, m->d_out};
    for (void *q : ps)
        if (q) cudaFree(q);
    delete m;
    c->wf = nullptr;
}
}  // namespace exs

extern "C" {

int exs_wavefmt(exs_ctx *c, int ngp, const exs_complex *apwalm, int nst, const exs_complex *evecfv, int ldv,
                int lrstp, int lmax, const exs_mt_radial *in, int ld, exs_complex *wfmt)
{
    if (!c || !apwalm || !evecfv || !in || !wfmt || nst < 0)
        return wfail(c, EXS_ERR_ARG, "exs_wavefmt: bad argument");
    if (!in->nrmt || !in->apwfr || (c->nlotot > 0 && !in->lofr))
        return wfail(c, EXS_ERR_ARG, "exs_wavefmt: missing radial functions");
    if (!c->have_inputs) return wfail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    if (lmax < 0 || lmax > c->lmaxapw) return wfail(c, EXS_ERR_ARG, "exs_wavefmt: lmax outside 0..lmaxapw");
    if (lrstp < 1) return wfail(c, EXS_ERR_ARG, "exs_wavefmt: lrstp < 1");
    if (ngp < 1 || ngp > c->ngkmax) return wfail(c, EXS_ERR_SIZE, "exs_wavefmt: ngp outside 1..ngkmax");
    const int nmat = ngp + c->nlotot;
    if (ldv < nmat) return wfail(c, EXS_ERR_SIZE, "exs_wavefmt: ldv < nmat");
    if (ld < (lmax + 1) * (lmax + 1)) return wfail(c, EXS_ERR_SIZE, "exs_wavefmt: ld < (lmax + 1)^2");
    for (int is = 0; is < c->nspecies; is++)
        if (in->nrmt[is] < 1 || in->nrmt[is] > in->nrmtmax)
            return wfail(c, EXS_ERR_SIZE, "exs_wavefmt: nrmt outside 1..nrmtmax");
    if (nst == 0) return EXS_OK;
    const int nrc = (in->nrmtmax - 1) / lrstp + 1;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    if (!c->wf) c->wf = new WfState;
    WfState &m = *(WfState *)c->wf;
    if (!m.blas) WF_BLAS(cublasCreate(&m.blas));
    WF_BLAS(cublasSetStream(m.blas, s));
    WF_CUDA(cudaStreamSynchronize(s));
    WF_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));

    const int nat = c->natmtot, nsp = c->nspecies;
    const size_t lmmax = (size_t)(c->lmaxapw + 1) * (c->lmaxapw + 1);
    const size_t M = (size_t)c->apwordmax * lmmax * nat;
    const size_t nfr = (size_t)in->nrmtmax * 2 * c->apwordmax * (c->lmaxapw + 1) * nat;
    const size_t nlo = c->nlotot > 0 ? (size_t)in->nrmtmax * 2 * c->nlomax * nat : 0;
    const size_t nout = (size_t)ld * nrc * nat * nst;
    WF_CUDA(grow(&m.d_alm, &m.alm_cap, (size_t)c->ngkmax * M));
    WF_CUDA(grow(&m.d_ev, &m.ev_cap, (size_t)nmat * nst));
    WF_CUDA(grow(&m.d_c, &m.c_cap, M * nst));
    WF_CUDA(grow(&m.d_fr, &m.fr_cap, nfr + nlo));
    WF_CUDA(grow(&m.d_nrmt, &m.nrmt_cap, (size_t)nsp));
    WF_CUDA(grow(&m.d_out, &m.out_cap, nout));
    // uploads: the first ngp rows of each apwalm column, the nmat rows of each state
    WF_CUDA(cudaMemcpy2DAsync(m.d_alm, sizeof(exs_complex) * c->ngkmax, apwalm, sizeof(exs_complex) * c->ngkmax,
                              sizeof(exs_complex) * ngp, M, cudaMemcpyHostToDevice, s));
    WF_CUDA(cudaMemcpy2DAsync(m.d_ev, sizeof(exs_complex) * nmat, evecfv, sizeof(exs_complex) * ldv,
                              sizeof(exs_complex) * nmat, nst, cudaMemcpyHostToDevice, s));
    WF_CUDA(cudaMemcpyAsync(m.d_fr, in->apwfr, sizeof(double) * nfr, cudaMemcpyHostToDevice, s));
    if (nlo) WF_CUDA(cudaMemcpyAsync(m.d_fr + nfr, in->lofr, sizeof(double) * nlo, cudaMemcpyHostToDevice, s));
    WF_CUDA(cudaMemcpyAsync(m.d_nrmt, in->nrmt, sizeof(int) * nsp, cudaMemcpyHostToDevice, s));
    // C = apwalm(1:ngp, :)^T evecfv(1:ngp, :)   (the zdotu of src/wavefmt.f90:100)
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    WF_BLAS(cublasZgemm(m.blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)M, nst, ngp, &one,
                        reinterpret_cast<const cuDoubleComplex *>(m.d_alm), c->ngkmax,
                        reinterpret_cast<const cuDoubleComplex *>(m.d_ev), nmat, &zero,
                        reinterpret_cast<cuDoubleComplex *>(m.d_c), (int)M));
    WfArgs a{};
    a.ngp = ngp; a.nmat = nmat; a.nst = nst; a.lrstp = lrstp; a.lmax = lmax; a.ld = ld; a.nrc = nrc;
    a.nrmtmax = in->nrmtmax;
    a.c = m.d_c; a.ev = m.d_ev; a.apwfr = m.d_fr; a.lofr = nlo ? m.d_fr + nfr : nullptr; a.nrmt = m.d_nrmt;
    a.out = m.d_out;
    const int per = ld * nrc;
    const dim3 grid((unsigned)std::min(64, (per + 255) / 256), (unsigned)nat, (unsigned)nst);
    wavefmt_kernel<<<grid, 256, 0, s>>>(c->params(), a);
    WF_CUDA(cudaGetLastError());
    WF_CUDA(cudaMemcpyAsync(wfmt, m.d_out, sizeof(exs_complex) * nout, cudaMemcpyDeviceToHost, s));
    return exs_synchronize(c);
}

}  // extern "C"
