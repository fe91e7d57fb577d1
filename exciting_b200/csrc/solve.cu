// The consumer of the setup: the first-variational generalized eigenproblem
// H x = e O x solved on the device, so that H and O never cross PCIe.
// Replaces solvewithlapack (src/src_eigensystem/modfvsystem.f90:585-720),
// which asks LAPACK zhegvx for the eigenvalues IL = 1 .. IU = nstfv and their
// vectors; here cuSOLVER's zhegvdx (the library routine for the dense
// Hermitian-definite problem) with the same index range, upper triangles.
#include <cusolverDn.h>

#include <algorithm>
#include <cstring>

#include "exs_internal.cuh"

namespace {

int sfail(exs_ctx *c, int code, const char *msg)
{
    if (c) c->last_error = msg;
    return code;
}

// Work space for one solve of order n (grown on demand, kept in the context).
int solve_reserve(exs_ctx *c, int n, int nstfv, const exs_complex *a, const exs_complex *b)
{
    if (!c->solver) {
        cusolverDnHandle_t h = nullptr;
        if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return sfail(c, EXS_ERR_CUDA, "cusolverDnCreate failed");
        c->solver = h;
    }
    cusolverDnHandle_t h = (cusolverDnHandle_t)c->solver;
    if (cusolverDnSetStream(h, c->stream) != CUSOLVER_STATUS_SUCCESS)
        return sfail(c, EXS_ERR_CUDA, "cusolverDnSetStream failed");
    int lwork = 0, meig = 0;
    if (cusolverDnZhegvdx_bufferSize(h, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                                     CUBLAS_FILL_MODE_UPPER, n, (const cuDoubleComplex *)a, n,
                                     (const cuDoubleComplex *)b, n, 0.0, 0.0, 1, nstfv, &meig, nullptr,
                                     &lwork) != CUSOLVER_STATUS_SUCCESS)
        return sfail(c, EXS_ERR_CUDA, "cusolverDnZhegvdx_bufferSize failed");
    if ((size_t)lwork > c->solve_lwork) {
        if (c->d_solve_work) cudaFree(c->d_solve_work);
        c->d_solve_work = nullptr;
        c->solve_lwork = 0;
        if (cudaMalloc(&c->d_solve_work, sizeof(cuDoubleComplex) * (size_t)lwork) != cudaSuccess)
            return sfail(c, EXS_ERR_NOMEM, "solver work space");
        c->solve_lwork = (size_t)lwork;
    }
    if ((size_t)n > c->solve_n) {
        if (c->d_solve_w) cudaFree(c->d_solve_w);
        c->d_solve_w = nullptr;
        c->solve_n = 0;
        if (cudaMalloc((void **)&c->d_solve_w, sizeof(double) * (size_t)n) != cudaSuccess)
            return sfail(c, EXS_ERR_NOMEM, "solver eigenvalue space");
        c->solve_n = (size_t)n;
    }
    if (!c->d_solve_info && cudaMalloc((void **)&c->d_solve_info, sizeof(int)) != cudaSuccess)
        return sfail(c, EXS_ERR_NOMEM, "solver info");
    return EXS_OK;
}

// Solve one problem in place: on return the first nstfv columns of a hold
// the eigenvectors (leading dimension n), d_solve_w[0 .. nstfv) the values.
int solve_one(exs_ctx *c, int n, exs_complex *a, exs_complex *b, int nstfv)
{
    int rc = solve_reserve(c, n, nstfv, a, b);
    if (rc != EXS_OK) return rc;
    cusolverDnHandle_t h = (cusolverDnHandle_t)c->solver;
    int meig = 0;
    const cusolverStatus_t st = cusolverDnZhegvdx(
        h, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_UPPER, n,
        (cuDoubleComplex *)a, n, (cuDoubleComplex *)b, n, 0.0, 0.0, 1, nstfv, &meig, c->d_solve_w,
        (cuDoubleComplex *)c->d_solve_work, (int)c->solve_lwork, c->d_solve_info);
    if (st != CUSOLVER_STATUS_SUCCESS) return sfail(c, EXS_ERR_CUDA, "cusolverDnZhegvdx failed");
    int info = 0;
    if (cudaMemcpyAsync(&info, c->d_solve_info, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return sfail(c, EXS_ERR_CUDA, "solver status read");
    if (info != 0 || meig < nstfv)
        return sfail(c, EXS_ERR_ARG, "zhegvdx did not converge or O is not positive definite");
    return EXS_OK;
}

}  // namespace

namespace exs {

void solver_release(exs_ctx *c)
{
    if (c->solver) cusolverDnDestroy((cusolverDnHandle_t)c->solver);
    if (c->d_solve_work) cudaFree(c->d_solve_work);
    if (c->d_solve_w) cudaFree(c->d_solve_w);
    if (c->d_solve_info) cudaFree(c->d_solve_info);
    c->solver = nullptr;
    c->d_solve_work = nullptr;
    c->d_solve_w = nullptr;
    c->d_solve_info = nullptr;
}

}  // namespace exs

extern "C" {

int exs_solve_batched_device(exs_ctx *c, int nk, const int *nmat, exs_complex *const *h_dev,
                             exs_complex *const *o_dev, int nstfv, double *evalfv_dev,
                             exs_complex *const *evecfv_dev, int ldv)
{
    if (!c || nk < 0 || (nk > 0 && (!nmat || !h_dev || !o_dev || !evalfv_dev || !evecfv_dev)) || nstfv <= 0)
        return sfail(c, EXS_ERR_ARG, "exs_solve_batched_device: bad argument");
    cudaSetDevice(c->device);
    for (int k = 0; k < nk; k++) {
        const int n = nmat[k];
        if (n <= 0 || nstfv > n || ldv < n || !h_dev[k] || !o_dev[k] || !evecfv_dev[k])
            return sfail(c, EXS_ERR_SIZE, "nmat, nstfv or ldv out of range");
        int rc = solve_one(c, n, h_dev[k], o_dev[k], nstfv);
        if (rc != EXS_OK) return rc;
        if (cudaMemcpyAsync(evalfv_dev + (size_t)nstfv * k, c->d_solve_w, sizeof(double) * nstfv,
                            cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess ||
            cudaMemcpy2DAsync(evecfv_dev[k], sizeof(exs_complex) * ldv, h_dev[k], sizeof(exs_complex) * n,
                              sizeof(exs_complex) * n, nstfv, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
            return sfail(c, EXS_ERR_CUDA, "eigenpair copy");
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return sfail(c, EXS_ERR_CUDA, "synchronize");
    return EXS_OK;
}

}  // extern "C"
