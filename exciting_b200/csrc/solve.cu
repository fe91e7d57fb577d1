// The consumer of the setup: the first-variational generalized eigenproblem
// H x = e O x solved on the device, so that H and O never cross PCIe.
// Replaces solvewithlapack (src/src_eigensystem/modfvsystem.f90:585-720),
// which asks LAPACK zhegvx for the eigenvalues IL = 1 .. IU = nstfv and their
// vectors; here cuSOLVER's zhegvdx (the library routine for the dense
// Hermitian-definite problem) with the same index range, upper triangles.
#include <cusolverDn.h>

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "exs_internal.cuh"

namespace {

int sfail(exs_ctx *c, int code, const char *msg)
{
    if (c) c->last_error = msg;
    return code;
}

// One solver lane: a cuSOLVER handle on its own stream with its work space.
// Solves of different k-points run on different lanes at the same time (a
// single dense solve of order ~1000 leaves most of the GPU idle).
struct SolveLane {
    cusolverDnHandle_t h = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t done = nullptr;
    void *work = nullptr;
    size_t lwork = 0;
    double *w = nullptr;
    size_t wn = 0;
    int *info = nullptr;
};

struct SolverState {
    std::vector<SolveLane> lanes;
};

constexpr int SOLVE_LANES = 8;

int lanes_reserve(exs_ctx *c, int nl)
{
    SolverState *st = (SolverState *)c->solver;
    if (!st) {
        st = new SolverState;
        c->solver = st;
    }
    while ((int)st->lanes.size() < nl) {
        SolveLane l;
        if (cusolverDnCreate(&l.h) != CUSOLVER_STATUS_SUCCESS) return sfail(c, EXS_ERR_CUDA, "cusolverDnCreate failed");
        if (cudaStreamCreateWithFlags(&l.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc((void **)&l.info, sizeof(int)) != cudaSuccess) {
            cusolverDnDestroy(l.h);
            return sfail(c, EXS_ERR_CUDA, "solver lane");
        }
        if (cusolverDnSetStream(l.h, l.s) != CUSOLVER_STATUS_SUCCESS)
            return sfail(c, EXS_ERR_CUDA, "cusolverDnSetStream failed");
        st->lanes.push_back(l);
    }
    if (!c->pool) {
        const unsigned hc = std::thread::hardware_concurrency();
        c->pool = new exs::HostPool((int)std::max(1u, std::min(hc, 32u)) - 1);
    }
    return EXS_OK;
}

// Work space of a lane for one solve of order n (grown on demand).  Returns
// EXS_OK or an error code; no context state is written (lanes run on
// several host threads).
int lane_reserve(SolveLane &l, int n, int nstfv, const exs_complex *a, const exs_complex *b, bool vectors)
{
    int lwork = 0, meig = 0;
    if (cusolverDnZhegvdx_bufferSize(l.h, CUSOLVER_EIG_TYPE_1,
                                     vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_RANGE_I,
                                     CUBLAS_FILL_MODE_UPPER, n, (const cuDoubleComplex *)a, n,
                                     (const cuDoubleComplex *)b, n, 0.0, 0.0, 1, nstfv, &meig, nullptr,
                                     &lwork) != CUSOLVER_STATUS_SUCCESS)
        return EXS_ERR_CUDA;
    if ((size_t)lwork > l.lwork) {
        if (l.work) cudaFree(l.work);
        l.work = nullptr;
        l.lwork = 0;
        if (cudaMalloc(&l.work, sizeof(cuDoubleComplex) * (size_t)lwork) != cudaSuccess) return EXS_ERR_NOMEM;
        l.lwork = (size_t)lwork;
    }
    if ((size_t)n > l.wn) {
        if (l.w) cudaFree(l.w);
        l.w = nullptr;
        l.wn = 0;
        if (cudaMalloc((void **)&l.w, sizeof(double) * (size_t)n) != cudaSuccess) return EXS_ERR_NOMEM;
        l.wn = (size_t)n;
    }
    return EXS_OK;
}

// Solve one problem in place on a lane: the first nstfv columns of a become
// the eigenvectors (leading dimension n), l.w[0 .. nstfv) the values; then
// copy them to the caller's arrays on the lane's stream.  evec = NULL: the
// values only (no vectors are formed: a far smaller work space).
int lane_solve(SolveLane &l, int n, exs_complex *a, exs_complex *b, int nstfv, double *eval, exs_complex *evec,
               int ldv)
{
    const bool vectors = evec != nullptr;
    int rc = lane_reserve(l, n, nstfv, a, b, vectors);
    if (rc != EXS_OK) return rc;
    int meig = 0;
    if (cusolverDnZhegvdx(l.h, CUSOLVER_EIG_TYPE_1, vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR,
                          CUSOLVER_EIG_RANGE_I,
                          CUBLAS_FILL_MODE_UPPER, n, (cuDoubleComplex *)a, n, (cuDoubleComplex *)b, n, 0.0, 0.0, 1,
                          nstfv, &meig, l.w, (cuDoubleComplex *)l.work, (int)l.lwork,
                          l.info) != CUSOLVER_STATUS_SUCCESS)
        return EXS_ERR_CUDA;
    int info = 0;
    if (cudaMemcpyAsync(&info, l.info, sizeof(int), cudaMemcpyDeviceToHost, l.s) != cudaSuccess ||
        cudaStreamSynchronize(l.s) != cudaSuccess)
        return EXS_ERR_CUDA;
    if (info != 0 || meig < nstfv) return EXS_ERR_ARG;
    if (cudaMemcpyAsync(eval, l.w, sizeof(double) * nstfv, cudaMemcpyDeviceToDevice, l.s) != cudaSuccess)
        return EXS_ERR_CUDA;
    if (vectors && cudaMemcpy2DAsync(evec, sizeof(exs_complex) * ldv, a, sizeof(exs_complex) * n,
                                     sizeof(exs_complex) * n, nstfv, cudaMemcpyDeviceToDevice, l.s) != cudaSuccess)
        return EXS_ERR_CUDA;
    return EXS_OK;
}

}  // namespace

namespace exs {

void solver_release(exs_ctx *c)
{
    SolverState *st = (SolverState *)c->solver;
    if (!st) return;
    for (SolveLane &l : st->lanes) {
        if (l.h) cusolverDnDestroy(l.h);
        if (l.s) cudaStreamDestroy(l.s);
        if (l.done) cudaEventDestroy(l.done);
        if (l.work) cudaFree(l.work);
        if (l.w) cudaFree(l.w);
        if (l.info) cudaFree(l.info);
    }
    delete st;
    c->solver = nullptr;
}

}  // namespace exs

extern "C" {

int exs_solve_batched_device(exs_ctx *c, int nk, const int *nmat, exs_complex *const *h_dev,
                             exs_complex *const *o_dev, int nstfv, double *evalfv_dev,
                             exs_complex *const *evecfv_dev, int ldv)
{
    if (!c || nk < 0 || (nk > 0 && (!nmat || !h_dev || !o_dev || !evalfv_dev)) || nstfv <= 0)
        return sfail(c, EXS_ERR_ARG, "exs_solve_batched_device: bad argument");
    for (int k = 0; k < nk; k++)
        if (nmat[k] <= 0 || nstfv > nmat[k] || !h_dev[k] || !o_dev[k] ||
            (evecfv_dev && (ldv < nmat[k] || !evecfv_dev[k])))
            return sfail(c, EXS_ERR_SIZE, "nmat, nstfv or ldv out of range");
    if (nk == 0) return EXS_OK;
    cudaSetDevice(c->device);
    const int nl = std::min(nk, SOLVE_LANES);
    int rc = lanes_reserve(c, nl);
    if (rc != EXS_OK) return rc;
    SolverState *st = (SolverState *)c->solver;
    // the lanes start after the work already queued on the context's stream
    if (cudaEventRecord(c->ev[7], c->stream) != cudaSuccess) return sfail(c, EXS_ERR_CUDA, "event record");
    for (int l = 0; l < nl; l++)
        if (cudaStreamWaitEvent(st->lanes[l].s, c->ev[7], 0) != cudaSuccess)
            return sfail(c, EXS_ERR_CUDA, "stream wait");
    std::vector<int> lrc(nl, EXS_OK);
    c->pool->parallel_for(nl, [&](int l) {
        cudaSetDevice(c->device);
        SolveLane &ln = st->lanes[l];
        for (int k = l; k < nk && lrc[l] == EXS_OK; k += nl)
            lrc[l] = lane_solve(ln, nmat[k], h_dev[k], o_dev[k], nstfv, evalfv_dev + (size_t)nstfv * k,
                                evecfv_dev ? evecfv_dev[k] : nullptr, ldv);
        if (cudaEventRecord(ln.done, ln.s) != cudaSuccess && lrc[l] == EXS_OK) lrc[l] = EXS_ERR_CUDA;
    });
    for (int l = 0; l < nl; l++) {   // the context's stream continues after every lane
        if (lrc[l] == EXS_OK && cudaStreamWaitEvent(c->stream, st->lanes[l].done, 0) != cudaSuccess)
            lrc[l] = EXS_ERR_CUDA;
    }
    for (int l = 0; l < nl; l++) cudaStreamSynchronize(st->lanes[l].s);
    for (int l = 0; l < nl; l++) {
        if (lrc[l] == EXS_ERR_ARG) return sfail(c, EXS_ERR_ARG, "zhegvdx did not converge or O is not positive definite");
        if (lrc[l] == EXS_ERR_NOMEM) return sfail(c, EXS_ERR_NOMEM, "solver work space");
        if (lrc[l] != EXS_OK) return sfail(c, EXS_ERR_CUDA, "cuSOLVER call failed");
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return sfail(c, EXS_ERR_CUDA, "synchronize");
    return EXS_OK;
}

}  // extern "C"
