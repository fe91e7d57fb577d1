// Real-time TDDFT Hamiltonian update on the device.  Replaces the k-loop of
// UpdateHam (src/src_xs/src_rttddft/rttddft_hamiltonianoverlap.f90:40-106):
// per k-point the module's own hamsetup/overlapsetup (:108-190, :191-330)
// rebuild H and O from the stored matching coefficients with the same
// muffin-tin, APW-lo, lo-lo and interstitial blocks as the ground-state
// setup, then
//   ham_time = H + (|A|^2 / 2c^2) O + (A_1/c) P_1 + (A_2/c) P_2 + (A_3/c) P_3
// (:95-100), A the total vector potential and P the momentum matrix
// elements (pmat).  Here the batched setup computes H and O on the device
// and one memory-bound kernel applies the combination; P stays resident on
// the device for the whole propagation (it does not change in time).
#include <algorithm>
#include <string>
#include <vector>

#include "exs_internal.cuh"

namespace {

// speed of light in atomic units, as src/constants/physical_constants.f90:41-50
constexpr double C0 = 299792458.0, T0 = 2.418884326509e-17, A0 = 0.52917721067e-10;
constexpr double C_AU = C0 * T0 / A0;

int rfail(exs_ctx *c, int code, const std::string &msg)
{
    if (c) c->last_error = msg;
    return code;
}

#define RT_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return rfail(c, EXS_ERR_CUDA, std::string(#call ": ") + \
                                                                 cudaGetErrorString(e_)); \
    } while (0)

constexpr int RT_MAXK = 32;   // k-points per combine launch (kernel parameter block)

struct RtBatch {
    int n;
    double fact, ca[3];
    long nmat[RT_MAXK];
    exs_complex *h[RT_MAXK];
    const exs_complex *o[RT_MAXK];
    const exs_complex *p[RT_MAXK];   // (nmat, nmat, 3)
};

// grid (blocks per matrix, k), 256 threads: H <- H + fact O + sum_i ca_i P_i
// element by element, the terms added left to right as the reference writes
// them.  Reads 5 and writes 1 complex per element: HBM-bound.
__global__ void __launch_bounds__(256) rt_combine_kernel(RtBatch b)
{
    const int k = blockIdx.y;
    const long n = b.nmat[k];
    const size_t total = (size_t)n * n;
    const double2 *o = (const double2 *)b.o[k];
    const double2 *p = (const double2 *)b.p[k];
    double2 *h = (double2 *)b.h[k];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const double2 hv = h[i], ov = o[i], p1 = p[i], p2 = p[total + i], p3 = p[2 * total + i];
        double re = __dadd_rn(hv.x, __dmul_rn(b.fact, ov.x));
        double im = __dadd_rn(hv.y, __dmul_rn(b.fact, ov.y));
        re = __dadd_rn(re, __dmul_rn(b.ca[0], p1.x));
        im = __dadd_rn(im, __dmul_rn(b.ca[0], p1.y));
        re = __dadd_rn(re, __dmul_rn(b.ca[1], p2.x));
        im = __dadd_rn(im, __dmul_rn(b.ca[1], p2.y));
        re = __dadd_rn(re, __dmul_rn(b.ca[2], p3.x));
        im = __dadd_rn(im, __dmul_rn(b.ca[2], p3.y));
        h[i] = make_double2(re, im);
    }
}

struct RtState {
    // momentum matrix elements of the registered k-points, (nmat, nmat, 3) each
    exs_complex *d_p = nullptr;
    size_t p_cap = 0;
    std::vector<size_t> p_off;
    std::vector<int> p_nmat;
    // work space of the host-pointer call
    exs_complex *d_h = nullptr, *d_o = nullptr, *d_o2 = nullptr;
    size_t ho_cap = 0, o2_cap = 0;
    int *d_ig = nullptr;
    double *d_vg = nullptr;
    size_t kv_cap = 0;
    // device time of the last combination (CUDA events around its launches)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
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

RtState *state(exs_ctx *c)
{
    if (!c->rt) c->rt = new RtState;
    return (RtState *)c->rt;
}

double field_fact(const double *atot) { return (atot[0] * atot[0] + atot[1] * atot[1] + atot[2] * atot[2]) / (2.0 * C_AU * C_AU); }

int launch_combine(exs_ctx *c, int nk, const int *nmat, exs_complex *const *h, const exs_complex *const *o,
                   const exs_complex *const *p, const double *atot, cudaStream_t s)
{
    for (int k0 = 0; k0 < nk; k0 += RT_MAXK) {
        RtBatch b{};
        b.n = std::min(RT_MAXK, nk - k0);
        b.fact = field_fact(atot);
        for (int i = 0; i < 3; i++) b.ca[i] = atot[i] / C_AU;
        long nmax = 0;
        for (int k = 0; k < b.n; k++) {
            b.nmat[k] = nmat[k0 + k];
            b.h[k] = h[k0 + k];
            b.o[k] = o[k0 + k];
            b.p[k] = p[k0 + k];
            nmax = std::max(nmax, b.nmat[k]);
        }
        const size_t total = (size_t)nmax * nmax;
        const unsigned gx = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 8);
        rt_combine_kernel<<<dim3(gx, b.n), 256, 0, s>>>(b);
        RT_CUDA(cudaGetLastError());
    }
    return EXS_OK;
}

}  // namespace

namespace exs {
// Storage for the momentum matrices of nk k-points, (nmat_k, nmat_k, 3)
// each, registered as exs_rttddft_set_pmat registers them; returns the
// device base and the per-k-point element offsets.
int rt_reserve_pmat(exs_ctx *c, int nk, const int *nmat, exs_complex **d_p, size_t *off)
{
    RtState *r = state(c);
    RT_CUDA(cudaStreamSynchronize(c->stream));
    r->p_off.assign(nk, 0);
    r->p_nmat.assign(nmat, nmat + nk);
    size_t tot = 0;
    for (int k = 0; k < nk; k++) {
        r->p_off[k] = off[k] = tot;
        tot += 3 * (size_t)nmat[k] * nmat[k];
    }
    RT_CUDA(grow(&r->d_p, &r->p_cap, tot));
    *d_p = r->d_p;
    return EXS_OK;
}

// Device milliseconds of the last combination (0 if none); waits for it.
double rt_combine_ms(exs_ctx *c)
{
    RtState *r = (RtState *)c->rt;
    if (!r || !r->timed) return 0.0;
    float ms = 0.f;
    if (cudaEventSynchronize(r->ev1) != cudaSuccess || cudaEventElapsedTime(&ms, r->ev0, r->ev1) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0.0;
    }
    return ms;
}

void rt_release(exs_ctx *c)
{
    RtState *r = (RtState *)c->rt;
    if (!r) return;
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    void *ps[] = {r->d_p, r->d_h, r->d_o, r->d_o2, r->d_ig, r->d_vg};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete r;
    c->rt = nullptr;
}
}  // namespace exs

extern "C" {

int exs_rttddft_set_pmat(exs_ctx *c, int nk, const int *nmat, const exs_complex *const *pmat, int ld)
{
    if (!c || nk < 0 || (nk > 0 && (!nmat || !pmat))) return rfail(c, EXS_ERR_ARG, "exs_rttddft_set_pmat: bad argument");
    if (nk > c->max_batch) return rfail(c, EXS_ERR_SIZE, "exs_rttddft_set_pmat: nk exceeds max_batch");
    for (int k = 0; k < nk; k++)
        if (nmat[k] <= 0 || nmat[k] > c->ngkmax + c->nlotot || ld < nmat[k] || !pmat[k])
            return rfail(c, EXS_ERR_SIZE, "exs_rttddft_set_pmat: nmat outside 1..ngkmax+nlotot or ld < nmat");
    cudaSetDevice(c->device);
    RtState *r = state(c);
    cudaStream_t s = c->stream;
    RT_CUDA(cudaStreamSynchronize(s));
    r->p_off.assign(nk, 0);
    r->p_nmat.assign(nmat, nmat + nk);
    size_t tot = 0;
    for (int k = 0; k < nk; k++) {
        r->p_off[k] = tot;
        tot += 3 * (size_t)nmat[k] * nmat[k];
    }
    RT_CUDA(grow(&r->d_p, &r->p_cap, tot));
    for (int k = 0; k < nk; k++)
        for (int i = 0; i < 3; i++)   // pmat(1:nmat, 1:nmat, i) of a (ld, ld, 3) array
            RT_CUDA(cudaMemcpy2DAsync(r->d_p + r->p_off[k] + (size_t)i * nmat[k] * nmat[k], sizeof(exs_complex) * nmat[k],
                                      pmat[k] + (size_t)i * ld * ld, sizeof(exs_complex) * ld,
                                      sizeof(exs_complex) * nmat[k], nmat[k], cudaMemcpyHostToDevice, s));
    RT_CUDA(cudaStreamSynchronize(s));
    return EXS_OK;
}

int exs_rttddft_updateham_device(exs_ctx *c, int nk, const int *ngp_host, const int *igpig_dev,
                                 const double *vgpc_dev, const double *atot, int calculate_overlap,
                                 exs_complex *const *pmat_dev, exs_complex *const *h_dev, exs_complex *const *o_dev)
{
    if (!c || !atot || nk < 0 || (nk > 0 && (!ngp_host || !pmat_dev || !h_dev || !o_dev)))
        return rfail(c, EXS_ERR_ARG, "exs_rttddft_updateham_device: bad argument");
    if (nk > c->max_batch) return rfail(c, EXS_ERR_SIZE, "nk exceeds max_batch");
    cudaSetDevice(c->device);
    RtState *r = state(c);
    std::vector<int> nmat(nk);
    for (int k = 0; k < nk; k++) {
        if (!pmat_dev[k]) return rfail(c, EXS_ERR_ARG, "exs_rttddft_updateham_device: null pmat");
        nmat[k] = ngp_host[k] + c->nlotot;
    }
    // with calculate_overlap = 0 the caller's o_dev is the overlap to use: the
    // setup writes its O into scratch instead
    std::vector<exs_complex *> o_setup(o_dev, o_dev + nk);
    if (!calculate_overlap) {
        size_t need = 0;
        for (int k = 0; k < nk; k++) need = std::max(need, (size_t)nmat[k] * nmat[k]);
        if (need * nk > r->o2_cap) {
            RT_CUDA(cudaStreamSynchronize(c->stream));   // the old scratch may still be written
            RT_CUDA(grow(&r->d_o2, &r->o2_cap, need * nk));
        }
        for (int k = 0; k < nk; k++) o_setup[k] = r->d_o2 + (size_t)k * need;
    }
    int rc = exs_setup_batched_device(c, nk, ngp_host, igpig_dev, vgpc_dev, h_dev, o_setup.data());
    if (rc != EXS_OK) return rc;
    std::vector<const exs_complex *> oc(o_dev, o_dev + nk), pc(pmat_dev, pmat_dev + nk);
    if (!r->ev0) {
        RT_CUDA(cudaEventCreate(&r->ev0));
        RT_CUDA(cudaEventCreate(&r->ev1));
    }
    RT_CUDA(cudaEventRecord(r->ev0, c->stream));
    rc = launch_combine(c, nk, nmat.data(), h_dev, oc.data(), pc.data(), atot, c->stream);
    if (rc != EXS_OK) return rc;
    RT_CUDA(cudaEventRecord(r->ev1, c->stream));
    r->timed = true;
    return EXS_OK;
}

int exs_rttddft_updateham(exs_ctx *c, int nk, const int *ngp, const int *igpig, const double *vgpc,
                          const double *atot, int calculate_overlap, exs_complex *const *ham,
                          exs_complex *const *overlap, int ld)
{
    if (!c || !atot || nk < 0 || (nk > 0 && (!ngp || !igpig || !vgpc || !ham || !overlap)))
        return rfail(c, EXS_ERR_ARG, "exs_rttddft_updateham: bad argument");
    if (nk > c->max_batch) return rfail(c, EXS_ERR_SIZE, "nk exceeds max_batch");
    RtState *r = state(c);
    if ((int)r->p_nmat.size() < nk) return rfail(c, EXS_ERR_STATE, "exs_rttddft_set_pmat has not registered nk k-points");
    std::vector<int> nmat(nk);
    for (int k = 0; k < nk; k++) {
        if (ngp[k] <= 0 || ngp[k] > c->ngkmax) return rfail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax");
        nmat[k] = ngp[k] + c->nlotot;
        if (nmat[k] != r->p_nmat[k]) return rfail(c, EXS_ERR_SIZE, "nmat differs from the registered pmat");
        if (ld < nmat[k] || !ham[k] || !overlap[k]) return rfail(c, EXS_ERR_SIZE, "ld < nmat or null output");
    }
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    RT_CUDA(cudaStreamSynchronize(s));
    size_t tot = 0;
    std::vector<size_t> off(nk);
    for (int k = 0; k < nk; k++) {
        off[k] = tot;
        tot += (size_t)nmat[k] * nmat[k];
    }
    if (tot > r->ho_cap) {
        size_t cap = 0;
        RT_CUDA(grow(&r->d_h, &cap, tot));
        cap = 0;
        RT_CUDA(grow(&r->d_o, &cap, tot));
        r->ho_cap = tot;
    }
    const size_t nkv = (size_t)c->ngkmax * nk;
    if (nkv > r->kv_cap) {
        size_t cap = 0;
        RT_CUDA(grow(&r->d_ig, &cap, nkv));
        cap = 0;
        RT_CUDA(grow(&r->d_vg, &cap, 3 * nkv));
        r->kv_cap = nkv;
    }
    RT_CUDA(cudaMemcpyAsync(r->d_ig, igpig, sizeof(int) * nkv, cudaMemcpyHostToDevice, s));
    RT_CUDA(cudaMemcpyAsync(r->d_vg, vgpc, sizeof(double) * 3 * nkv, cudaMemcpyHostToDevice, s));
    std::vector<exs_complex *> hp(nk), op(nk), pp(nk);
    for (int k = 0; k < nk; k++) {
        hp[k] = r->d_h + off[k];
        op[k] = r->d_o + off[k];
        pp[k] = r->d_p + r->p_off[k];
        if (!calculate_overlap)   // the overlap of an earlier call, as the reference keeps it
            RT_CUDA(cudaMemcpy2DAsync(op[k], sizeof(exs_complex) * nmat[k], overlap[k], sizeof(exs_complex) * ld,
                                      sizeof(exs_complex) * nmat[k], nmat[k], cudaMemcpyHostToDevice, s));
    }
    int rc = exs_rttddft_updateham_device(c, nk, ngp, r->d_ig, r->d_vg, atot, calculate_overlap, pp.data(),
                                          hp.data(), op.data());
    if (rc != EXS_OK) return rc;
    for (int k = 0; k < nk; k++) {
        RT_CUDA(cudaMemcpy2DAsync(ham[k], sizeof(exs_complex) * ld, hp[k], sizeof(exs_complex) * nmat[k],
                                  sizeof(exs_complex) * nmat[k], nmat[k], cudaMemcpyDeviceToHost, s));
        if (calculate_overlap)
            RT_CUDA(cudaMemcpy2DAsync(overlap[k], sizeof(exs_complex) * ld, op[k], sizeof(exs_complex) * nmat[k],
                                      sizeof(exs_complex) * nmat[k], nmat[k], cudaMemcpyDeviceToHost, s));
    }
    return exs_synchronize(c);
}

}  // extern "C"
