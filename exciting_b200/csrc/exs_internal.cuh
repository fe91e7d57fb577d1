// Internal definitions shared by the CUDA translation units of libexciting_b200.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/exciting_b200.h"
#include "host_pool.h"
#include "special.cuh"

namespace exs {

// Device error flags (bit set), read back after each public call.
enum : int {
    DEV_ERR_INDEX = 1,   // ivgig lookup outside the box
    DEV_WARN_SINGULAR = 2,
    DEV_ERR_TIMEOUT = 4,  // a bounded wait in a kernel expired
};

// A kernel attribute (such as the dynamic shared memory size) is a setting of
// the current device: set it once per device, bit d of `done` recording
// device d (devices past 63 set it on every call).  Host threads that race
// both set it, which is harmless.
template <class F>
inline cudaError_t once_per_device(std::atomic<unsigned long long> &done, F set)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = set();
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// Pipeline configurations of the split-precision kernel.
constexpr int OZ_NCFG = 32;
// Modes of the split-precision kernel: H/O tiles, per-atom products (h_a A, loa A).
enum : int { OZ_HO = 0, OZ_ATOM = 1 };

// Per-atom operands of the split-precision kernel (h_a and loa, their slices).
struct OzAtomArgs {
    const double *hr, *hi;       // h_a planar [ias][f'][f], leading dim ldh
    const double *lr, *li;       // loa planar [ias][f][r], leading dim ldlo
    int ldh, ldlo, maxaa;
    int nfb;                     // 64-row blocks of h_a rows (ceil(maxaa / 64)); blocks nfb.. hold the lo rows
    int nxb;                     // blocks per atom (nfb + ceil(maxnlo / 64))
    int lw;                      // window bytes per row (multiple of 128)
    int8_t *xs;                  // slices [atom][slice][block][re, im][64][lw]
    double *xsig;                // row scales [atom][block][64]
};
static_assert(OZ_NCFG == EXS_OZ_NCONFIG, "public configuration count");

// The arithmetic of the split-precision contraction.
//   slices (mod = 0): n int8 slices of 7 bits per operand, pairs s + t <= n + 1,
//     folded diagonal by diagonal in FP64 (seg / segx pairs per exact int32
//     segment for the H/O and the per-atom tiles);
//   moduli (mod = 1): every column of A and B scaled by a power of two above
//     its 2-norm and rounded to integers (b bits: the scaled column has norm
//     <= 2^b; bx for the h_a / loa rows, scaled by their row norms), stored
//     as residues modulo n pairwise coprime odd moduli p[m] (int8 in
//     [-127, 127]); one int8 product per modulus.  By the Cauchy-Schwarz
//     inequality an H/O product obeys |X| <= 2^(2b) (1 + eps)^2 with
//     2^(2b + 2) <= M, and its residues are recombined by 96-bit constants
//     c96 (residue tiles, oz_res_kernel / oz_crt_kernel): exact but for
//     2^-64 M.  A per-atom product (|X| <= 2^(b + bx) (1 + eps)^2) is folded in
//     the kernel into a 64-bit sum t += (v mod p[m]) c[m] (mod 2^64) with
//     c[m] = round(2^(64+h) y_m / p[m]) mod 2^64 and 2^(b + bx + h + 2) <= M,
//     so that t / 2^64 = 2^h X / M (mod 1) and t read as a signed integer is
//     exact but for the rounding of the constants (sum |r| / 2 units of
//     2^-(64+h) M; the h >= 5 headroom bits divide it by 2^h); the value is t
//     times finx.  fin is the same factor for the H/O products folded in the
//     64-bit form (2^(2b + h + 2) <= M does not hold for the plan's b: only
//     the per-atom products use the fold).
constexpr int OZ_MAX_MODULI = 16;
struct OzScheme {
    int mod, n, seg, segx, b, bx, h;
    long long wait;                    // limit of the pipeline waits in cycles (0: OZ_WAIT_CYCLES)
    double fin, finx;
    int p[OZ_MAX_MODULI];
    int mg[OZ_MAX_MODULI];             // round(2^32 / p): quotient estimate by a multiply-high
    float fp[OZ_MAX_MODULI], finv[OZ_MAX_MODULI];  // p and 1/p in FP32 (the split kernels)
    float fc[3][OZ_MAX_MODULI];        // 2^13, 2^26, 2^39 mod p
    unsigned long long c[OZ_MAX_MODULI];
    // the H/O products (residue tiles): C_m = round(2^96 y_m / p_m) in 32-bit
    // words (low first); the recombination reads the 64 bits below the top
    // crt_shift bits of the 96-bit sum (the bits that |X| <= 2^2b leaves as
    // sign copies when M is far above 2^2b), exact but for 2^-(64+crt_shift) M;
    // fin96 = M 2^-(64+crt_shift) 2^-2b
    unsigned c96[3][OZ_MAX_MODULI];
    int crt_shift;
    double fin96;
};

// atomicMax for non-negative doubles: their IEEE bit patterns order like
// unsigned integers.
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
    atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

// One atom's place in the device layouts.
struct AtomDesc {
    int species;
    int apw_off;     // first row of this atom in the stacked APW rows (A, B planes)
    int napw;        // m_a: APW rows of this atom (l <= lmaxmat)
    int lo_off;      // first row of this atom inside the lo block (0-based), -1 if none
    int losize;      // lo rows of this atom
    int oz_x0;       // split precision: apw_off rounded down to 16 (start of the atom's K window)
    int oz_nch;      // split precision: 128-byte K chunks of the window (apw_off - oz_x0 + napw)
    double pos[3];   // atposc
};

// Per-k-point descriptor of a batched call (device copy).
struct KDesc {
    int ngp;
    int nmat;
    const int *igpig;        // (ngkmax) device, 1-based G indices
    const double *vgpc;      // (3, ngkmax) device
    exs_complex *h;          // (nmat, nmat) device, column-major
    exs_complex *o;
    double *ar, *ai;         // A planes  [Kpad][npad]
    double *br, *bi;         // B = blockdiag(h_a) A planes
    double *cr, *ci;         // (I + h1) A planes (iora* only) else == ar/ai
    int8_t *oz_slices;       // split-precision path: int8 slices of this slot [S][4 arrays][npad][kp8]
    double *oz_scale;        // split-precision path: column bounds of A and B [2][npad] (maxima with slices,
                             // 2-norms with moduli; the scale is the power of two above; null: FP64 path)
    int oz_slot;             // split-precision path: slot index in the slice tensor maps
};

// Constant per-context device parameters passed by value to kernels.
// Per (atom, l) entry of DevParams::dlu: the n x n LU factors of D_l
// (n <= EXS_APWORD_MAX = 3), the pivots and the factorisation's info.
constexpr int DLU_STRIDE = 13;

struct DevParams {
    int natmtot, lmaxapw, lmaxmat, apwordmax, lmmaxapw, np_tail;
    int ngkmax, npad, K, Kpad;
    int nlotot, maxnlo, nlomax, lolmmax;
    int ngvec, ngrtot;
    int intgv_lo[3], intgv_n[3];
    int relativity;
    double omega;
    const AtomDesc *atoms;       // natmtot
    const int *apword;           // (lmaxapw+1, nspecies)
    const double *rmt;           // nspecies
    const double *spr_tail;      // (np, nspecies)
    const double *apwfr_tail;    // (np, apwordmax, lmaxapw+1, natmtot)
    const int *ivg;              // (3, ngrtot)
    const int *ivgig;            // box
    const exs_complex *veffig;   // ngvec
    const exs_complex *kinw;     // ngvec (meffig or cfunig)
    const exs_complex *cfunig;   // ngvec
    const exs_complex *m2effig;  // ngvec or null
    const exs_complex *lolo;     // (maxnlo, maxnlo, natmtot)
    const double *ololo;         // (nlomax, nlomax, natmtot)
    const double *h1lolo;        // (nlomax, nlomax, natmtot) or null
    const double *oalo;          // (apwordmax, nlomax, natmtot)
    const double *h1loa;         // or null
    const double *h1aa;          // (apwordmax, apwordmax, lmaxapw+1, natmtot) or null
    const int *idxlo;            // (lolmmax, nlomax, natmtot), 1-based values
    const int *lorbl;            // (nlomax, nspecies)
    const int *nlorb;            // nspecies
    const double *dlu;           // LU factors of D_l per (atom, l): [ias][l][DLU_STRIDE]
    int *err;                    // device error flags
};

enum EpiKind { EPI_PLANAR = 0, EPI_HAM = 1, EPI_OVL = 2, EPI_LOROWS = 3 };

// One complex product C = op(X) Y of a grouped launch, X stored [k][m],
// Y stored [k][n], real and imaginary planes apart.
struct GemmProb {
    const double *xr, *xi;
    long ldx;
    const double *yr, *yi;
    long ldy;
    int M, N, K;
    int conjx;
    double *outr, *outi;   // EPI_PLANAR output [m][n]
    long ldo;
    exs_complex *z;        // EPI_HAM / EPI_OVL / EPI_LOROWS: za(ldz, *)
    long ldz;
    int row0;              // EPI_LOROWS: za row of m = 0
    int kidx;              // k-point of this problem (interstitial tables)
    double *colmax;        // EPI_PLANAR: column maxima of |out| raised atomically (split precision), or null
};

struct TileWork {
    int prob, tm, tn;
};

struct GemmTables {
    std::vector<GemmProb> probs[4];
    std::vector<TileWork> work[4];
};

}  // namespace exs

// Host-side context.
struct exs_ctx {
    // configuration
    int natmtot = 0, nspecies = 0, lmaxapw = 0, lmaxmat = 0, apwordmax = 0, nlomax = 0;
    std::vector<int> atom_species, apword, nlorb, lorbl;
    std::vector<double> rmt, atposc, bvec;
    double omega = 0.0;
    int ngkmax = 0, ngrtot = 0, ngvec = 0, relativity = 0, np_tail = 4, max_batch = 1;
    int intgv[6] = {0, 0, 0, 0, 0, 0};
    // derived
    int maxaa = 0, maxnlo = 0, nlotot = 0, lolmmax = 1, lolmax = 0;
    std::vector<int> idxlo, losize;
    std::vector<exs::AtomDesc> atoms;
    int K = 0, Kpad = 0, npad = 0, nmatmax = 0;
    int ldh = 0, ldlo = 0;       // leading dims of the planar h_a and loa copies
    // device tables
    exs::AtomDesc *d_atoms = nullptr;
    int *d_apword = nullptr, *d_ivg = nullptr, *d_ivgig = nullptr, *d_idxlo = nullptr;
    int *d_lorbl = nullptr, *d_nlorb = nullptr;
    double *d_rmt = nullptr;
    // SCF inputs
    bool have_inputs = false;
    double *d_haa_r = nullptr, *d_haa_i = nullptr;   // [ias][f'][f] ld ldh
    double *d_loa_r = nullptr, *d_loa_i = nullptr;   // [ias][f][r] ld ldlo
    exs_complex *d_lolo = nullptr;
    double *d_oalo = nullptr, *d_ololo = nullptr, *d_h1aa = nullptr, *d_h1loa = nullptr, *d_h1lolo = nullptr;
    exs_complex *d_veffig = nullptr, *d_kinw = nullptr, *d_cfunig = nullptr, *d_m2effig = nullptr;
    double *d_spr_tail = nullptr, *d_apwfr_tail = nullptr;
    double *d_dlu = nullptr;         // LU factors of the matching systems D_l (from the tails)
    // work space (max_batch slots)
    size_t plane = 0;            // Kpad * npad doubles per plane
    double *d_work = nullptr;    // A, B (and C) planes for all slots
    int nplanes = 4;
    exs_complex *d_ho = nullptr; // H and O of all slots (host-facing calls)
    int *d_igpig = nullptr;
    double *d_vgpc = nullptr;
    int *d_err = nullptr;
    // per-call tables (k descriptors, grouped-GEMM problems and tiles):
    // packed in pinned host memory, uploaded with one copy
    void *h_tables = nullptr, *d_tables = nullptr;
    size_t tables_bytes = 0;
    cudaEvent_t tables_free = nullptr;   // recorded after the upload
    exs::GemmTables gt;
    // pinned staging for host-facing calls
    int *h_igpig_pinned = nullptr;
    double *h_vgpc_pinned = nullptr;
    // host-pointer batched path: packed upper triangles, two group slots
    int host_copy_mode = EXS_COPY_AUTO;
    exs_complex *d_pack[2] = {nullptr, nullptr}, *h_pack[2] = {nullptr, nullptr};
    size_t pack_elems = 0;               // capacity of each slot
    void *h_packdesc[2] = {nullptr, nullptr}, *d_packdesc[2] = {nullptr, nullptr};
    size_t packdesc_cap = 0;             // descriptors per slot
    cudaEvent_t ev_d2h[2] = {};
    exs::HostPool *pool = nullptr;
    // device eigen-solve: solver lanes (cuSOLVER handles, streams, work space)
    void *solver = nullptr;
    double *d_eval = nullptr;            // eigenpairs of the host-pointer solve call
    exs_complex *d_evec = nullptr;
    size_t eval_cap = 0, evec_cap = 0;
    // muffin-tin integral generation (mtint.cu): tables, Gaunt list, work space
    void *mt = nullptr;
    bool have_mt = false;                // h_a, loa, lolo on the device came from exs_hmlint
    bool have_olp = false;               // oalo, ololo (h1*) on the device came from exs_olprad
    // real-time TDDFT Hamiltonian update (rttddft.cu): momentum matrices, work space
    void *rt = nullptr;
    void *pm = nullptr;                  // momentum-matrix generation (pmat.cu)
    void *wf = nullptr;                  // muffin-tin wavefunction coefficients (wavefmt.cu)
    // match-only buffers
    double *d_match_in = nullptr;      // gpc, tpgpc (ngkmax*3 doubles)
    exs_complex *d_match_sf = nullptr; // sfacgp (ngkmax, natmtot)
    exs_complex *d_apwalm = nullptr;   // (ngkmax, apwordmax, lmmaxapw, natmtot)
    // IBS force / adjoint work space (grown on demand)
    void *fk_dev = nullptr;
    size_t fk_bytes = 0;
    void *fk_tab_h = nullptr, *fk_tab_d = nullptr;
    void *fk_dh = nullptr;                 // dL/dh_a of the adjoint (maxaa, maxaa, natmtot), kept between calls
    size_t fk_dh_bytes = 0;
    size_t fk_tab_hbytes = 0, fk_tab_dbytes = 0;
    // precision
    int prec_mode = EXS_PREC_FP64;
    int slices = 7;              // slices or moduli of the split-precision modes
    exs::OzScheme oz_sch{};      // their arithmetic
    long long oz_wait = 0;       // limit of their pipeline waits in cycles (0: the default)
    bool oz_on() const { return prec_mode == EXS_PREC_OZAKI_INT8 || prec_mode == EXS_PREC_OZAKI_MOD; }
    int kp8 = 0;                 // K rounded up to 256 (int8 slice rows)
    int oz_seg = 0;              // slice pairs per exact int32 segment
    int8_t *d_oz = nullptr;      // int8 slices of all slots
    double *d_ozscale = nullptr; // column scales of all slots
    size_t oz_slot_bytes = 0;
    CUtensorMap oz_mapA[exs::OZ_NCFG], oz_mapB[exs::OZ_NCFG];   // TMA views of d_oz per pipeline configuration
    CUtensorMap oz_mapB2[exs::OZ_NCFG];                            // half-B views (two-SM tiles)
    CUtensorMap oz_mapB64;                                         // B operand of the 128 x 64 residue tiles
    CUtensorMap oz_mapB64h;                                        // one CTA's half of it in the 256 x 64 pairs
    uint8_t *d_res = nullptr;                                      // residue tiles of the modular H/O products
    int *d_pace = nullptr;                                         // pacing of the persistent pair kernel
    size_t res_bytes = 0;
    int oz_cfg = 0;                   // pipeline configuration of the split-precision kernel
    // per-atom products of the split-precision path (h_a A, loa A)
    int8_t *d_xs = nullptr;           // slices of h_a and loa
    double *d_xsig = nullptr;         // their row scales
    int oz_lw = 0, oz_nfb = 0, oz_nxb = 0, oz_xseg = 0;
    CUtensorMap oz_mapArow, oz_mapX;
    exs::OzAtomArgs oz_atom_args() const;
    unsigned gen = 0;                 // bumped when device buffers that captured graphs use are replaced
    std::map<std::tuple<int, int, int, int>, int> oz_tuned;   // (prec, npad, K, slices) -> configuration
    // runtime
    int device = 0;
    cudaStream_t stream = nullptr;      // stream the work runs on
    cudaStream_t own_stream = nullptr;  // the context's own stream
    cudaStream_t copy_stream = nullptr; // device-to-host copies of the host-facing calls
    cudaStream_t copy_stream2 = nullptr; // a second copy engine's share (the overlaps of direct copies)
    cudaEvent_t ev_copy2 = nullptr;
    cudaEvent_t ev_group[2] = {};
    cudaEvent_t ev[8] = {};
    double last_t[5] = {0, 0, 0, 0, 0};
    bool timed = false;          // ev[0..4] recorded by the last setup call
    std::string last_error;

    exs::DevParams params() const;
};

// Launch helpers implemented in the .cu files.
namespace exs {
cudaError_t launch_match_planes(const DevParams &p, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s);
cudaError_t launch_match_dlu(const DevParams &p, double *dlu, cudaStream_t s);
cudaError_t launch_match_ref(const DevParams &p, int ngp, int ngkmax, const double *gpc, const double *tpgpc,
                             const exs_complex *sfacgp, exs_complex *apwalm, cudaStream_t s);
cudaError_t launch_apwalm_to_planes(const DevParams &p, int ngp, const exs_complex *apwalm, double *ar,
                                    double *ai, double *amax, cudaStream_t s);
cudaError_t launch_iora_planes(const DevParams &p, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s);
cudaError_t launch_lolo_blocks(const DevParams &p, const KDesc *d_k, int nk, cudaStream_t s);
cudaError_t launch_olp_apwlo(const DevParams &p, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s);
// Grouped FP64 GEMM stages (setup_f64.cu)
void build_gemm_tables(const exs_ctx *c, const std::vector<KDesc> &ks, GemmTables &t);
cudaError_t launch_gemm_kind(int kind, const DevParams &p, const void *d_probs, const void *d_work, int nwork,
                             const KDesc *d_k, cudaStream_t s);
// Device eigen-solve (solve.cu)
void solver_release(exs_ctx *c);
// Muffin-tin integral generation (mtint.cu)
void mt_release(exs_ctx *c);
// Real-time TDDFT Hamiltonian update (rttddft.cu)
void rt_release(exs_ctx *c);
int rt_reserve_pmat(exs_ctx *c, int nk, const int *nmat, exs_complex **d_p, size_t *off);
double rt_combine_ms(exs_ctx *c);
// Momentum-matrix generation (pmat.cu)
void pm_release(exs_ctx *c);
void wf_release(exs_ctx *c);
// Stand-alone interstitial gather (interstitial.cu)
cudaError_t launch_interstitial(const DevParams &p, int which, const KDesc *d_k, int nk, int ngp_max, cudaStream_t s);
// Split-precision contraction (ozaki.cu)
cudaError_t launch_oz_split(const DevParams &p, const KDesc *d_k, int nk, const OzScheme &sch, int kp8, int which,
                            cudaStream_t s);
cudaError_t launch_oz_x(const DevParams &p, const OzAtomArgs &xa, const OzScheme &sch, cudaStream_t s);
cudaError_t launch_oz_colnorm(const DevParams &p, const KDesc *d_k, int nk, int which, int norm, cudaStream_t s);
cudaError_t launch_oz_res(int cfg, const CUtensorMap *mapA, const CUtensorMap *mapB32, const CUtensorMap *mapB64,
                          const CUtensorMap *mapB64h, const DevParams &p, const KDesc *d_k, const void *d_tiles,
                          int ntiles, const OzScheme &sch, int kp8, uint8_t *res, int *pace, cudaStream_t s);
int oz_res_cols(int cfg);
int oz_res_rows(int cfg);
size_t oz_pace_bytes();
size_t oz_res_tile_bytes(int n, int cfg);
bool make_oz_b64_map(void *base, size_t nss, int npad, int kp8, int narr, CUtensorMap *mapB64, CUtensorMap *mapB64h);
cudaError_t launch_oz_atom(int cfg, const CUtensorMap *mapArow, const CUtensorMap *mapX, const DevParams &p,
                           const KDesc *d_k, const void *d_tiles, int ntiles, const OzScheme &sch, int kp8,
                           const OzAtomArgs &xa, cudaStream_t s);
bool make_oz_atom_maps(void *base, size_t nss, int npad, int kp8, int narr, void *xbase, size_t xgroups, int lw,
                       CUtensorMap *mapArow, CUtensorMap *mapX);
cudaError_t launch_oz_mma(int cfg, const CUtensorMap *mapA, const CUtensorMap *mapB, const DevParams &p,
                          const KDesc *d_k, const void *d_tiles, int ntiles, const OzScheme &sch, int kp8,
                          cudaStream_t s);
bool make_oz_tensor_maps(void *base, size_t nss, int npad, int kp8, int kch, int narr, CUtensorMap *mapA,
                         CUtensorMap *mapB, CUtensorMap *mapB2);
extern const int OZ_CFG_KCH[OZ_NCFG], OZ_CFG_NST[OZ_NCFG];
int oz_kpad(int K);
size_t oz_slot_bytes(int S, int npad, int kp8, int narr);
int oz_seg_pairs(int S, int kp8);
int oz_mod_plan(int n, int K, int kx, OzScheme *sch);
}  // namespace exs
