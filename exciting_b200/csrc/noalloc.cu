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
// each call rewrites every part it reads (padding included), its tables
// included: they are written on the device by kernels that receive the
// per-atom sizes as launch arguments, so no host buffer is copied.  Two
// calls whose work overlaps on the GPU (different streams, or different
// host threads) race on the array and give wrong results: serialise them.
//
// Host code cannot use the array's name as a device address; on the first
// call on each device (with that device current) the address is looked up
// with cudaGetSymbolAddress and cached.  That first call should therefore
// come before any stream capture.  cudaDeviceReset destroys the array with
// the context, so the cached address is stale afterwards: this entry point
// is not for processes that reset a device and go on using it.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "exs_internal.cuh"

#define EXS_NOALLOC_SCRATCH_BYTES (32u << 20)
#define EXS_NOALLOC_MAX_DEVICES 64

namespace {

using exs::GemmProb;
using exs::TileWork;

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

// The grouped-product tables on the device.  Per-atom entries come in
// chunks of NA_CHUNK atoms whose sizes, row offsets and first work entries
// travel as launch arguments: problem a is B_a = h_a A_a with tiles
// (a, tm, tn), tm < ceil(napw / 64), tn < ntile, from entry wbase on.
constexpr int NA_CHUNK = 256;

struct NaBase {
    double *ar, *ai, *br, *bi, *hr, *hi, *Hr, *Hi, *Or, *Oi;
    int natmtot, ldh, np, ngp, K, ntile;
};

struct NaChunk {
    int a0, count;
    int off[NA_CHUNK], napw[NA_CHUNK], wbase[NA_CHUNK];
};

__global__ void na_atom_tables(const __grid_constant__ NaBase b, const __grid_constant__ NaChunk c, int *d_off,
                               int *d_napw, GemmProb *probs, TileWork *work)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= c.count) return;
    const int a = c.a0 + t, na = c.napw[t], off = c.off[t];
    d_off[a] = off;
    d_napw[a] = na;
    GemmProb P{};
    P.xr = b.hr + (size_t)a * b.ldh * b.ldh;
    P.xi = b.hi + (size_t)a * b.ldh * b.ldh;
    P.ldx = b.ldh;
    P.yr = b.ar + (size_t)off * b.np;
    P.yi = b.ai + (size_t)off * b.np;
    P.ldy = b.np;
    P.M = na;
    P.N = b.np;
    P.K = na;
    P.conjx = 0;
    P.outr = b.br + (size_t)off * b.np;
    P.outi = b.bi + (size_t)off * b.np;
    P.ldo = b.np;
    probs[a] = P;
    int w = c.wbase[t];
    for (int tm = 0; tm < (na + 63) / 64; tm++)
        for (int tn = 0; tn < b.ntile; tn++) work[w++] = TileWork{a, tm, tn};
}

// The two main problems (H = A^H B, O = A^H A) and their upper tiles, from
// entry nwork_ha on: entry q < T = ntile (ntile + 1) / 2 of problem `which`
// is the q-th (tm, tn >= tm) pair in row order.
__global__ void na_main_tables(const __grid_constant__ NaBase b, int nwork_ha, GemmProb *probs, TileWork *work)
{
    const int T = b.ntile * (b.ntile + 1) / 2;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < 2) {
        GemmProb P{};
        P.xr = b.ar;
        P.xi = b.ai;
        P.ldx = b.np;
        P.yr = q == 0 ? b.br : b.ar;
        P.yi = q == 0 ? b.bi : b.ai;
        P.ldy = b.np;
        P.M = b.ngp;
        P.N = b.ngp;
        P.K = b.K;
        P.conjx = 1;
        P.outr = q == 0 ? b.Hr : b.Or;
        P.outi = q == 0 ? b.Hi : b.Oi;
        P.ldo = b.np;
        probs[b.natmtot + q] = P;
    }
    if (q >= 2 * T) return;
    const int which = q / T;
    int r = q - which * T, tm = 0;
    while (r >= b.ntile - tm) {
        r -= b.ntile - tm;
        tm++;
    }
    work[nwork_ha + q] = TileWork{b.natmtot + which, tm, tm + r};
}

// apwi(maxaa, ngp, natmtot) -> A planes [K][np]; rows beyond K and columns
// beyond ngp are written as zero.  The atom of row f is found by a binary
// search of the row offsets (the same for the whole block).
__global__ void na_pack_a(int natmtot, int maxaa, const int *off, const int *napw, int K, int Kp, int ngp, int np,
                          const exs_complex *apwi, double *ar, double *ai)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;                 // stacked row 0..Kp-1
    if (g >= np || f >= Kp) return;
    double re = 0.0, im = 0.0;
    if (f < K && g < ngp) {
        int lo = 0, hi = natmtot - 1;         // the last atom with off <= f
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (off[mid] <= f)
                lo = mid;
            else
                hi = mid - 1;
        }
        const int ias = lo;
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
    const size_t plane = (size_t)Kp * np;
    size_t o_ints = 0;
    size_t o_tab = al256(o_ints + sizeof(int) * 2 * (size_t)natmtot);
    // problem table sized below; planes follow the tables
    const size_t nprob = (size_t)natmtot + 2;
    size_t nwork_ha = 0;
    for (int a = 0; a < natmtot; a++) nwork_ha += (size_t)((na[a] + 63) / 64) * ntile;
    const size_t nwork_main = (size_t)ntile * (ntile + 1);      // the upper tiles of H and of O
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

    // ---- grouped-product tables (the same kernel as the context path), written on the device
    NaBase nb{};
    nb.ar = ar; nb.ai = ai; nb.br = br; nb.bi = bi; nb.hr = hr; nb.hi = hi;
    nb.Hr = Hr; nb.Hi = Hi; nb.Or = Or; nb.Oi = Oi;
    nb.natmtot = natmtot; nb.ldh = ldh; nb.np = np; nb.ngp = ngp; nb.K = K; nb.ntile = ntile;
    cudaError_t e = cudaSuccess;
    size_t wnext = 0;
    for (int a0 = 0; a0 < natmtot && e == cudaSuccess; a0 += NA_CHUNK) {
        NaChunk ch{};
        ch.a0 = a0;
        ch.count = std::min(NA_CHUNK, natmtot - a0);
        for (int t = 0; t < ch.count; t++) {
            ch.off[t] = off[a0 + t];
            ch.napw[t] = na[a0 + t];
            ch.wbase[t] = (int)wnext;
            wnext += (size_t)((na[a0 + t] + 63) / 64) * ntile;
        }
        na_atom_tables<<<(ch.count + 127) / 128, 128, 0, s>>>(nb, ch, d_off, d_napw, d_probs, d_work);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        na_main_tables<<<(unsigned)((nwork_main + 127) / 128), 128, 0, s>>>(nb, (int)nwork_ha, d_probs, d_work);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return EXS_ERR_CUDA;

    // ---- pack, contract, store
    na_pack_a<<<dim3(np / 64, Kp), 64, 0, s>>>(natmtot, maxaa, d_off, d_napw, K, Kp, ngp, np, apwi, ar, ai);
    na_pack_h<<<dim3((ldh + 63) / 64, ldh, natmtot), 64, 0, s>>>(natmtot, maxaa, ldh, aa, hr, hi);
    if ((e = cudaGetLastError()) != cudaSuccess) return EXS_ERR_CUDA;
    const DevParams none{};
    e = launch_gemm_kind(EPI_PLANAR, none, d_probs, d_work, (int)nwork_ha, nullptr, s);
    if (e == cudaSuccess)
        e = launch_gemm_kind(EPI_PLANAR, none, d_probs, d_work + nwork_ha, (int)nwork_main, nullptr, s);
    if (e != cudaSuccess) return EXS_ERR_CUDA;
    na_store_hermitian<<<dim3((ngp + 127) / 128, ngp), 128, 0, s>>>(ngp, np, Hr, Hi, h, ld);
    na_store_hermitian<<<dim3((ngp + 127) / 128, ngp), 128, 0, s>>>(ngp, np, Or, Oi, o, ld);
    if ((e = cudaGetLastError()) != cudaSuccess) return EXS_ERR_CUDA;
    return EXS_OK;
}
