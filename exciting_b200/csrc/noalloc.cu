// exs_mt_contract_noalloc: the muffin-tin APW-APW contraction for callers
// that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not safe --
// inside a stream-ordered region of a host framework that forbids
// allocation, under a memory pool that owns the whole device, or in a
// plug-in whose host application has already reserved every byte it may
// use.  Such a caller owns its inputs and outputs but cannot create a
// context (exs_ctx_create allocates its work space).
//
// This entry point therefore keeps its work space -- the planar copies of
// the matching coefficients and of the MT integrals, the products h_a A_a,
// the two N x N products and the tile tables of the grouped product -- in
// one file-scope device array of EXS_NOALLOC_SCRATCH_BYTES (32 MiB).  Every
// GPU that loads the library holds that array until the process exits.
// Problems whose work space does not fit are rejected with EXS_ERR_SIZE.
//
// The array is shared by all calls and keeps the previous call's contents;
// each call rewrites every part it reads (padding included).  Two calls
// whose work overlaps on the GPU (different streams, or different host
// threads) race on the array and give wrong results: serialise them.
//
// Host code cannot use the array's name as a device address; on the first
// call on each device (with that device current) the address is looked up
// with cudaGetSymbolAddress and cached.  That first call should therefore
// come before any stream capture.
#include <cstring>
#include <mutex>
#include <vector>

#include "exs_internal.cuh"

#define EXS_NOALLOC_SCRATCH_BYTES (32u << 20)
#define EXS_NOALLOC_MAX_DEVICES 64

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[EXS_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[EXS_NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device.
cudaError_t noalloc_scratch(unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= EXS_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = (unsigned char *)p;
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

// apwi(maxaa, ngp, natmtot) -> A planes [K][np]; rows beyond K and columns
// beyond ngp are written as zero.
__global__ void na_pack_a(int natmtot, int maxaa, const int *off, const int *napw, int K, int Kp, int ngp, int np,
                          const exs_complex *apwi, double *ar, double *ai)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;                 // stacked row 0..Kp-1
    if (g >= np || f >= Kp) return;
    double re = 0.0, im = 0.0;
    if (f < K && g < ngp) {
        int ias = 0;
        while (ias + 1 < natmtot && f >= off[ias + 1]) ias++;
        const int fl = f - off[ias];
        if (fl < napw[ias]) {
            const exs_complex z = apwi[fl + (size_t)maxaa * (g + (size_t)ngp * ias)];
            re = z.re;
            im = z.im;
        }
    }
    ar[(size_t)f * np + g] = re;
    ai[(size_t)f * np + g] = im;
}

// aa(maxaa, maxaa, natmtot) -> planar [ias][f'][f] with leading dimension ldh.
__global__ void na_pack_h(int natmtot, int maxaa, int ldh, const exs_complex *aa, double *hr, double *hi)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int f2 = blockIdx.y;
    const int ias = blockIdx.z;
    if (f >= ldh || f2 >= ldh) return;
    double re = 0.0, im = 0.0;
    if (f < maxaa && f2 < maxaa) {
        const exs_complex z = aa[f + (size_t)maxaa * (f2 + (size_t)maxaa * ias)];
        re = z.re;
        im = z.im;
    }
    hr[f + (size_t)ldh * (f2 + (size_t)ldh * ias)] = re;
    hi[f + (size_t)ldh * (f2 + (size_t)ldh * ias)] = im;
}

// Upper triangle of the planar products -> full Hermitian za(ld, ngp).
__global__ void na_store_hermitian(int ngp, int np, const double *cr, const double *ci, exs_complex *z, int ld)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= ngp || i > j || j >= ngp) return;
    const double re = cr[(size_t)i * np + j], im = ci[(size_t)i * np + j];
    exs_complex v;
    v.re = re;
    v.im = im;
    z[(size_t)i + (size_t)ld * j] = v;
    if (i < j) {
        v.im = -im;
        z[(size_t)j + (size_t)ld * i] = v;
    }
}

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" int exs_mt_contract_noalloc(int natmtot, int maxaa, const int *napw, int ngp, const exs_complex *apwi,
                                       const exs_complex *aa, exs_complex *h, exs_complex *o, int ld, void *stream)
{
    using namespace exs;
    if (natmtot <= 0 || maxaa <= 0 || ngp <= 0 || ld < ngp || !napw || !apwi || !aa || !h || !o) return EXS_ERR_ARG;
    const cudaStream_t s = (cudaStream_t)stream;
    // ---- layout of the work space inside the scratch array
    std::vector<int> off(natmtot), na(natmtot);
    int K = 0;
    for (int a = 0; a < natmtot; a++) {
        if (napw[a] < 0 || napw[a] > maxaa) return EXS_ERR_ARG;
        off[a] = K;
        na[a] = napw[a];
        K += napw[a];
    }
    if (K == 0) return EXS_ERR_ARG;
    const int Kp = (K + 15) / 16 * 16;
    const int np = (ngp + 63) / 64 * 64;
    const int ldh = (maxaa + 7) / 8 * 8;
    const int ntile = np / 64;
    std::vector<GemmProb> probs;
    std::vector<TileWork> work_ha, work_main;
    const size_t plane = (size_t)Kp * np;
    size_t o_ints = 0;
    size_t o_tab = al256(o_ints + sizeof(int) * 2 * (size_t)natmtot);
    // problem table sized below; planes follow the tables
    const size_t nprob = (size_t)natmtot + 2;
    size_t nwork_ha = 0;
    for (int a = 0; a < natmtot; a++) nwork_ha += (size_t)((na[a] + 63) / 64) * ntile;
    const size_t nwork_main = 2 * (size_t)ntile * ntile;
    const size_t o_work = al256(o_tab + sizeof(GemmProb) * nprob);
    const size_t o_planes = al256(o_work + sizeof(TileWork) * (nwork_ha + nwork_main));
    const size_t n_doubles = 4 * plane + 2 * (size_t)natmtot * ldh * ldh + 4 * (size_t)ngp * np;
    const size_t need = o_planes + sizeof(double) * n_doubles;
    if (need > EXS_NOALLOC_SCRATCH_BYTES) return EXS_ERR_SIZE;

    unsigned char *base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess) return EXS_ERR_CUDA;
    int *d_off = (int *)(base + o_ints);
    int *d_napw = d_off + natmtot;
    GemmProb *d_probs = (GemmProb *)(base + o_tab);
    TileWork *d_work = (TileWork *)(base + o_work);
    double *ar = (double *)(base + o_planes);
    double *ai = ar + plane;
    double *br = ai + plane;
    double *bi = br + plane;
    double *hr = bi + plane;
    double *hi = hr + (size_t)natmtot * ldh * ldh;
    double *Hr = hi + (size_t)natmtot * ldh * ldh;
    double *Hi = Hr + (size_t)ngp * np;
    double *Or = Hi + (size_t)ngp * np;
    double *Oi = Or + (size_t)ngp * np;

    // ---- grouped-product tables (the same kernel as the context path)
    for (int a = 0; a < natmtot; a++) {           // B_a = h_a A_a
        GemmProb P{};
        P.xr = hr + (size_t)a * ldh * ldh; P.xi = hi + (size_t)a * ldh * ldh; P.ldx = ldh;
        P.yr = ar + (size_t)off[a] * np; P.yi = ai + (size_t)off[a] * np; P.ldy = np;
        P.M = na[a]; P.N = np; P.K = na[a]; P.conjx = 0;
        P.outr = br + (size_t)off[a] * np; P.outi = bi + (size_t)off[a] * np; P.ldo = np;
        const int pi = (int)probs.size();
        probs.push_back(P);
        for (int tm = 0; tm < (na[a] + 63) / 64; tm++)
            for (int tn = 0; tn < ntile; tn++) work_ha.push_back({pi, tm, tn});
    }
    for (int which = 0; which < 2; which++) {    // H = A^H B, O = A^H A
        GemmProb P{};
        P.xr = ar; P.xi = ai; P.ldx = np;
        P.yr = which == 0 ? br : ar; P.yi = which == 0 ? bi : ai; P.ldy = np;
        P.M = ngp; P.N = ngp; P.K = K; P.conjx = 1;
        P.outr = which == 0 ? Hr : Or; P.outi = which == 0 ? Hi : Oi; P.ldo = np;
        const int pi = (int)probs.size();
        probs.push_back(P);
        for (int tm = 0; tm < ntile; tm++)
            for (int tn = tm; tn < ntile; tn++) work_main.push_back({pi, tm, tn});
    }
    std::vector<int> ints(2 * (size_t)natmtot);
    for (int a = 0; a < natmtot; a++) { ints[a] = off[a]; ints[natmtot + a] = na[a]; }
    cudaError_t e = cudaMemcpyAsync(d_off, ints.data(), sizeof(int) * ints.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_probs, probs.data(), sizeof(GemmProb) * probs.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_work, work_ha.data(), sizeof(TileWork) * work_ha.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_work + work_ha.size(), work_main.data(), sizeof(TileWork) * work_main.size(),
                            cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return EXS_ERR_CUDA;

    // ---- pack, contract, store
    na_pack_a<<<dim3(np / 64, Kp), 64, 0, s>>>(natmtot, maxaa, d_off, d_napw, K, Kp, ngp, np, apwi, ar, ai);
    na_pack_h<<<dim3((ldh + 63) / 64, ldh, natmtot), 64, 0, s>>>(natmtot, maxaa, ldh, aa, hr, hi);
    if ((e = cudaGetLastError()) != cudaSuccess) return EXS_ERR_CUDA;
    const DevParams none{};
    e = launch_gemm_kind(EPI_PLANAR, none, d_probs, d_work, (int)work_ha.size(), nullptr, s);
    if (e == cudaSuccess)
        e = launch_gemm_kind(EPI_PLANAR, none, d_probs, d_work + work_ha.size(), (int)work_main.size(), nullptr, s);
    if (e != cudaSuccess) return EXS_ERR_CUDA;
    na_store_hermitian<<<dim3((ngp + 127) / 128, ngp), 128, 0, s>>>(ngp, np, Hr, Hi, h, ld);
    na_store_hermitian<<<dim3((ngp + 127) / 128, ngp), 128, 0, s>>>(ngp, np, Or, Oi, o, ld);
    if ((e = cudaGetLastError()) != cudaSuccess) return EXS_ERR_CUDA;
    return EXS_OK;
}
