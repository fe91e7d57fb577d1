/*
 * exciting_b200 -- C-ABI of the B200 (sm_100a) per-k-point LAPW H/O setup.
 *
 * Drop-in for the reference's (exciting) per-k-point first-variational
 * Hamiltonian/overlap setup path.  Every array argument follows the
 * reference's Fortran declaration: column-major, complex(8) as two
 * interleaved doubles, integer index tables with their 1-based values.
 * All pointers are HOST pointers unless the entry point says "_device".
 *
 * Return codes: 0 success, > 0 warning (the call completed), < 0 error
 * (the outputs are undefined; exs_last_error() gives the text).
 */
#ifndef EXCITING_B200_H
#define EXCITING_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct exs_complex { double re, im; } exs_complex;   /* Fortran complex(8) */
typedef struct exs_ctx exs_ctx;

enum {
    EXS_OK = 0,
    EXS_WARN_SINGULAR = 1,   /* a matching system D_l was singular (match.f90:166-175) */
    EXS_ERR_ARG = -1,        /* bad argument (null pointer, negative size, ...) */
    EXS_ERR_CUDA = -2,       /* a CUDA runtime call failed */
    EXS_ERR_SIZE = -3,       /* a size above the compiled limits or the context's maxima */
    EXS_ERR_INDEX = -4,      /* a G-G' difference fell outside the ivgig box */
    EXS_ERR_STATE = -5,      /* exs_set_scf_inputs has not been called */
    EXS_ERR_NOMEM = -6,      /* a device allocation failed */
    EXS_ERR_TIMEOUT = -7     /* a bounded wait inside a tensor-core kernel expired; the kernel gave up
                                cleanly (its copies and products drained) and the context stays usable */
};

enum { EXS_REL_NONE = 0, EXS_REL_ZORA = 1, EXS_REL_IORA = 2 };   /* ValenceRelativity */
enum { EXS_PREC_FP64 = 0, EXS_PREC_OZAKI_INT8 = 1, EXS_PREC_OZAKI_MOD = 2 };   /* MT contraction path */

/* Per-run description: what init0/init1 leave in the reference's modules. */
typedef struct exs_config {
    int natmtot, nspecies;
    const int *atom_species;  /* (natmtot) 0-based species of atom ias; atoms grouped by species (idxas order) */
    int lmaxapw, lmaxmat;     /* input%groundstate%lmaxapw, lmaxmat */
    int apwordmax;
    const int *apword;        /* apword(0:lmaxapw, nspecies) */
    int nlomax;
    const int *nlorb;         /* nlorb(nspecies) */
    const int *lorbl;         /* lorbl(nlomax, nspecies) */
    const double *rmt;        /* rmt(nspecies) */
    double omega;             /* unit-cell volume */
    const double *atposc;     /* atposc(3, natmtot), Cartesian */
    const double *bvec;       /* bvec(3,3), reciprocal lattice vectors as columns */
    int ngkmax;               /* maximum number of G+k over all k */
    int ngrtot, ngvec;
    const int *intgv;         /* intgv(3,2): inclusive integer box of ivgig */
    const int *ivg;           /* ivg(3, ngrtot) */
    const int *ivgig;         /* ivgig(intgv(1,1):intgv(1,2), ..., ...) */
    int relativity;           /* EXS_REL_* (input%groundstate%ValenceRelativity) */
    int np_tail;              /* max(apwordmax+1, 4) radial points used by match (match.f90:87) */
    int max_batch;            /* most k-points handed to one batched call (>= 1) */
} exs_config;

/* Per-SCF-iteration inputs (what scf_cycle recomputes before the k-loop). */
typedef struct exs_scf_inputs {
    const exs_complex *mt_aa;    /* mt_hscf%main%aa(maxaa, maxaa, natmtot) */
    const exs_complex *mt_loa;   /* mt_hscf%main%loa(maxnlo, maxaa, natmtot) (may be NULL if no lo) */
    const exs_complex *mt_lolo;  /* mt_hscf%main%lolo(maxnlo, maxnlo, natmtot) */
    const double *oalo;          /* oalo(apwordmax, nlomax, natmtot) */
    const double *ololo;         /* ololo(nlomax, nlomax, natmtot) */
    const double *h1aa;          /* h1aa(apwordmax, apwordmax, 0:lmaxapw, natmtot), iora* only, else NULL */
    const double *h1loa;         /* h1loa(apwordmax, nlomax, natmtot), iora* only, else NULL */
    const double *h1lolo;        /* h1lolo(nlomax, nlomax, natmtot), iora* only, else NULL */
    const exs_complex *veffig;   /* veffig(ngvec) */
    const exs_complex *meffig;   /* meffig(ngvec), relativity /= none, else NULL */
    const exs_complex *cfunig;   /* cfunig(ngrtot) (only the first ngvec are read) */
    const exs_complex *m2effig;  /* m2effig(ngvec), iora* only, else NULL */
    const double *spr_tail;      /* spr(nrmt-np+1:nrmt, nspecies) */
    const double *apwfr_tail;    /* apwfr(nrmt-np+1:nrmt, 1, 1:apwordmax, 0:lmaxapw, natmtot) */
} exs_scf_inputs;

/* Inputs of the muffin-tin integral generation (exs_hmlint): the full
 * radial functions and the effective potential of the current SCF
 * iteration, in the reference's layouts. */
typedef struct exs_mt_radial {
    int lmaxvr;                  /* potential expanded in real harmonics up to lmaxvr */
    int nrmtmax;                 /* leading dimension of the radial arrays */
    const int *nrmt;             /* nrmt(nspecies): radial points per species (HOST, >= 4) */
    const double *spr;           /* spr(nrmtmax, nspecies): radial meshes (HOST) */
    const double *apwfr;         /* apwfr(nrmtmax, 2, apwordmax, 0:lmaxapw, natmtot): u and du/dr */
    const double *lofr;          /* lofr(nrmtmax, 2, nlomax, natmtot): v and dv/dr (NULL if no lo) */
    const double *veffmt;        /* veffmt(lmmaxvr, nrmtmax, natmtot), lmmaxvr = (lmaxvr+1)^2 */
} exs_mt_radial;

/* Create a context on the current CUDA device: validates the basis, builds
 * maxaa (MaxAPWs, mod_eigensystem.F90:151-184), losize/maxnlo (MTInitAll,
 * :194-235) and idxlo (genidxlo.f90), uploads the G-vector tables and sizes
 * the device work space for max_batch k-points of ngkmax G+k each. */
int exs_ctx_create(const exs_config *cfg, exs_ctx **out);
int exs_ctx_destroy(exs_ctx *ctx);
const char *exs_last_error(const exs_ctx *ctx);

/* Sizes the context derived: maxaa, maxnlo, nlotot (so a caller can size za). */
int exs_ctx_sizes(const exs_ctx *ctx, int *maxaa, int *maxnlo, int *nlotot);

/* Upload the per-SCF-iteration inputs (copied; the caller may free them).
 * mt_aa = NULL (with mt_loa, mt_lolo ignored) keeps the muffin-tin integrals
 * that exs_hmlint left on the device, oalo = NULL (with ololo and h1*
 * ignored) the overlap integrals of exs_olprad; EXS_ERR_ARG if that call
 * has not run. */
int exs_set_scf_inputs(exs_ctx *ctx, const exs_scf_inputs *in);

/* Replaces  call hmlint  (src/src_eigensystem/hmlint.f90:53-55: mt_kin then
 * mt_pot, the spin-unpolarised mt_hscf%main): the muffin-tin Hamiltonian
 * integrals of every atom,
 *   aa(maxaa, maxaa, natmtot), loa(maxnlo, maxaa, natmtot),
 *   lolo(maxnlo, maxnlo, natmtot)
 * (as the reference leaves them in arrays MTInit zeroed; alo is the plain
 * transpose of loa, mt_pot.f90:285), computed on the device from the radial
 * functions and potential in *in (host arrays) and installed as the
 * context's h_a for the following setups.  aa, loa, lolo: optional HOST
 * outputs (NULL: not copied).  The scalar-relativistic kinetic factor
 * 1/(1 - a V_00 Y00), a = alpha^2/2, applies when the context's relativity
 * is not "none" (ValenceRelativity /= 'none', mt_kin.f90:55-59).
 * Synchronous. */
int exs_hmlint(exs_ctx *ctx, const exs_mt_radial *in, exs_complex *aa, exs_complex *loa,
               exs_complex *lolo);
/* The same with apwfr, lofr, veffmt DEVICE arrays (nrmt, spr stay on the
 * host); enqueued on the context's stream, no host outputs. */
int exs_hmlint_device(exs_ctx *ctx, const exs_mt_radial *in);
/* Replaces  call olprad  (src/src_eigensystem/olprad.f90, called before
 * hmlint in scf_cycle.f90:207): the overlap radial integrals
 *   oalo(apwordmax, nlomax, natmtot) = int u_{l,io} v_ilo r^2 (l = lorbl(ilo)),
 *   ololo(nlomax, nlomax, natmtot)   = int v_ilo1 v_ilo2 r^2 (equal l, else 0),
 * and for iora* h1aa(apwordmax, apwordmax, 0:lmaxapw, natmtot), h1loa,
 * h1lolo (olprad.f90:30-44, :58-69, :78-90), computed on the device from
 * *in and installed for the following setups.  Host outputs optional (NULL:
 * not copied; the h1 arrays are written only for iora*).  Synchronous. */
int exs_olprad(exs_ctx *ctx, const exs_mt_radial *in, double *oalo, double *ololo, double *h1aa,
               double *h1loa, double *h1lolo);
/* The same with apwfr, lofr, veffmt DEVICE arrays; enqueued, no outputs. */
int exs_olprad_device(exs_ctx *ctx, const exs_mt_radial *in);
/* Host utilities of the integral generation, callable without a GPU:
 * gauntyry (src/src_lib/gauntyry.f90) -> re_im[2]; the spline integral
 * fderiv(-1, n, x, f, g, cf) g(n) (src/src_lib/fderiv.f90), n >= 4. */
int exs_gauntyry(int l1, int l2, int l3, int m1, int m2, int m3, double *re_im);
int exs_fderiv_int(int n, const double *x, const double *f, double *result);

/* Select the MT contraction arithmetic: EXS_PREC_FP64 (native FP64),
 * EXS_PREC_OZAKI_INT8 with `slices` int8 slices per operand (3..9), or
 * EXS_PREC_OZAKI_MOD: the operands as integers modulo `slices` pairwise
 * coprime odd moduli (6..16; 0 = the fewest that keep 41 + log2(K)/2 bits
 * per 2-norm-scaled operand column for this context's K), one int8 product
 * per modulus, recombined by the Chinese remainder theorem.  No reference counterpart (the reference's
 * contraction is zgemm in FP64). */
int exs_set_precision(exs_ctx *ctx, int mode, int slices);

/* The modular plan exs_set_precision(EXS_PREC_OZAKI_MOD, n) would use for a
 * contraction length K (2K products per real sum) and per-atom windows of
 * kx rows: the moduli p[0..n-1], the constants
 * c[m] = round(2^(64+h) y_m / p_m) mod 2^64 with y_m = (M / p_m)^-1 mod p_m,
 * M = prod p, the bits b of the A and B columns (scaled to 2-norm <= 2^b),
 * bx of the h_a / loa rows (likewise) and the headroom h of the 64-bit
 * recombination (2^(2b + h + 2) <= M and 2^(b + bx + h + 2) <= M).  n = 0
 * picks n as exs_set_precision does; *n_out receives it.  Any output pointer
 * may be NULL.  Host only. */
int exs_ozaki_moduli(int n, int K, int kx, int *n_out, int *p, unsigned long long *c, int *b, int *bx,
                     int *h);

/* Replaces  call match(ngp, gpc, tpgpc, sfacgp, apwalm)   (src/match.f90:13).
 *   gpc(ngkmax), tpgpc(2, ngkmax), sfacgp(ngkmax, natmtot)  in;
 *   apwalm(ngkmax, apwordmax, lmmaxapw, natmtot)              out.
 * Returns EXS_WARN_SINGULAR if some D_l was singular; as the reference, the
 * unsolved right-hand sides are then returned for that (atom, l). */
int exs_match(exs_ctx *ctx, int ngp, const double *gpc, const double *tpgpc,
              const exs_complex *sfacgp, exs_complex *apwalm);

/* Replaces  call hamiltonandoverlapsetup(system, ngp, apwalm, igpig, vgpc)
 * (src/src_eigensystem/hamiltonandoverlapsetup.f90:8), equivalently the live
 * pair  call hamiltonsetup(...); call overlapsetup(...)  (src/seceqnfv.f90:76-77)
 * on the zeroed matrices newsystem allocates.
 *   igpig(ngkmax), vgpc(3, ngkmax) in; apwalm in, or NULL to compute the
 *   matching coefficients on the device from vgpc;
 *   h, o: za(nmat, nmat) with nmat = ngp + nlotot, OVERWRITTEN with the full
 *   Hermitian matrices (upper triangle as set up, lower = conjugate, as
 *   hamiltonoverlapocopy_UL leaves them). */
int exs_hamiltonandoverlapsetup(exs_ctx *ctx, int ngp, const exs_complex *apwalm,
                                const int *igpig, const double *vgpc,
                                exs_complex *h, exs_complex *o);

/* The whole k-point list of one SCF iteration in one call (the reference's
 * k-loop over seceqn, scf_cycle.f90:237-278): nk <= max_batch k-points;
 *   ngp(nk); igpig(ngkmax, nk); vgpc(3, ngkmax, nk);
 *   h[ik], o[ik]: za(nmat_k, nmat_k), nmat_k = ngp(ik) + nlotot (host). */
int exs_setup_batched(exs_ctx *ctx, int nk, const int *ngp, const int *igpig,
                      const double *vgpc, exs_complex *const *h, exs_complex *const *o);

/* Same with every array already in device memory (h, o: nk device pointers
 * in a host array).  Asynchronous on the context's stream; exs_synchronize
 * waits for it. */
int exs_setup_batched_device(exs_ctx *ctx, int nk, const int *ngp_host,
                             const int *igpig_dev, const double *vgpc_dev,
                             exs_complex *const *h_dev, exs_complex *const *o_dev);
int exs_synchronize(exs_ctx *ctx);

/* How exs_setup_batched / exs_hamiltonandoverlapsetup bring H and O to the
 * host (no counterpart in the reference; results are identical):
 *   EXS_COPY_DIRECT  full matrices copied into the caller's arrays (fast
 *                    when those are pinned, e.g. cudaHostRegister'ed);
 *   EXS_COPY_PACKED  upper triangles packed on the device, half the bytes
 *                    over PCIe into pinned staging, full matrices rebuilt on
 *                    host threads (any caller memory);
 *   EXS_COPY_UPPER   per block of 64 columns only the rows down to the
 *                    block's last column copied into the caller's arrays
 *                    (the upper triangle and the diagonal blocks, ~55 % of
 *                    the bytes), the rest filled on host threads by
 *                    conjugate transposes inside the same array (pinned
 *                    caller memory);
 *   EXS_COPY_AUTO    DIRECT when every output array is pinned, else PACKED
 *                    (default). */
#define EXS_COPY_AUTO 0
#define EXS_COPY_DIRECT 1
#define EXS_COPY_PACKED 2
#define EXS_COPY_UPPER 3
int exs_set_host_copy_mode(exs_ctx *ctx, int mode);

/* The interstitial blocks alone: replaces
 *   call hmlistln(hamilton, ngp, igpig, vgpc)  (src/src_eigensystem/hmlistln.f90:13)
 *   call olpistln(overlap, ngp, igpig, vgpc)   (src/src_eigensystem/olpistln.f90:13)
 * ADDING to the upper triangle za(i, j), i <= j < ngp, of za(ld, *) as the
 * reference does (Hermitianmatrix_indexedupdate, modfvsystem.f90:126-143):
 * V(ig) + 1/2 (k+G_i).(k+G_j) W(ig) for H, Theta(ig) (+ the iora* term) for
 * O, ig = ivgig(ivg(:,igpig(i)) - ivg(:,igpig(j))).  Host arrays,
 * synchronous; ld <= nmatmax.  (exs_hamiltonandoverlapsetup already
 * includes these terms.) */
int exs_hmlistln(exs_ctx *ctx, int ngp, const int *igpig, const double *vgpc, exs_complex *h, int ld);
int exs_olpistln(exs_ctx *ctx, int ngp, const int *igpig, const double *vgpc, exs_complex *o, int ld);
/* Same on device arrays: which = 1 (H), 2 (O) or 3 (both); asynchronous on
 * the context's stream, exs_synchronize waits. */
int exs_interstitial_device(exs_ctx *ctx, int which, int ngp, const int *igpig_dev,
                            const double *vgpc_dev, exs_complex *h_dev, exs_complex *o_dev, int ld);
/* nk k-points in one launch: igpig_dev(ngkmax, nk), vgpc_dev(3, ngkmax, nk),
 * h_dev[k], o_dev[k] with leading dimensions ld[k] (host arrays of device
 * pointers / sizes). */
int exs_interstitial_batched_device(exs_ctx *ctx, int which, int nk, const int *ngp_host,
                                    const int *igpig_dev, const double *vgpc_dev,
                                    exs_complex *const *h_dev, exs_complex *const *o_dev,
                                    const int *ld_host);

/* The consumer of the setup on the device: replaces
 *   call solvewithlapack(system, nstfv, evecfv, evalfv)
 *   (src/src_eigensystem/modfvsystem.f90:585-720, LAPACK zhegvx for the
 *   eigenvalues IL = 1 .. IU = nstfv of H x = e O x and their vectors)
 * by cuSOLVER zhegvdx with the same index range on the upper triangles.
 * Device form: h_dev[k], o_dev[k] (nmat_k x nmat_k, destroyed),
 * evalfv_dev(nstfv, nk), evecfv_dev[k] (ldv, nstfv); evecfv_dev = NULL
 * computes the eigenvalues only (no vectors: a much smaller work space, as
 * needed for nmat of tens of thousands).  Synchronous.
 * EXS_ERR_ARG if O is not positive definite or the solver does not
 * converge. */
int exs_solve_batched_device(exs_ctx *ctx, int nk, const int *nmat_host, exs_complex *const *h_dev,
                             exs_complex *const *o_dev, int nstfv, double *evalfv_dev,
                             exs_complex *const *evecfv_dev, int ldv);
/* Setup and solve for host callers: H and O stay on the device, only the
 * eigenpairs come back.  Arguments as exs_setup_batched; evalfv(nstfv, nk),
 * evecfv(ldv, nstfv, nk) host arrays (the reference's evecfv(nmatmax, nstfv)
 * per k-point with ldv = nmatmax).  Synchronous. */
int exs_setup_and_solve_batched(exs_ctx *ctx, int nk, const int *ngp, const int *igpig,
                                const double *vgpc, int nstfv, double *evalfv, exs_complex *evecfv,
                                int ldv);

/* Real-time TDDFT (src/src_xs/src_rttddft/rttddft_hamiltonianoverlap.f90,
 * UpdateHam :40-106).  exs_rttddft_set_pmat registers the momentum matrix
 * elements pmat(1:nmat, 1:nmat, 1:3, ik) of nk k-points (host arrays of
 * leading dimension ld, each the start of an (ld, ld, 3) block) and keeps a
 * device copy for the whole propagation.  exs_rttddft_updateham then
 * replaces the k-loop of UpdateHam (:80-101): per k-point H and O of the
 * current SCF inputs (its hamsetup / overlapsetup, the ground-state
 * blocks), and
 *   ham[ik] = H + (|atot|^2 / (2 c^2)) O + sum_i (atot(i) / c) pmat(:,:,i)
 * with c the speed of light in atomic units (physical_constants.f90:50).
 * calculate_overlap /= 0: overlap[ik] receives the new O, which enters the
 * sum; = 0: overlap[ik] is read as the overlap to use (the reference keeps
 * the array of an earlier step).  ham, overlap: nk host pointers to
 * (ld, ld) arrays (the reference's ham_time(:,:,ik), overlap(:,:,ik) with
 * ld = nmatmax); ngp, igpig, vgpc as exs_setup_batched.  Synchronous. */
int exs_rttddft_set_pmat(exs_ctx *ctx, int nk, const int *nmat, const exs_complex *const *pmat, int ld);
int exs_rttddft_updateham(exs_ctx *ctx, int nk, const int *ngp, const int *igpig, const double *vgpc,
                          const double *atot, int calculate_overlap, exs_complex *const *ham,
                          exs_complex *const *overlap, int ld);
/* The same on device arrays: pmat_dev[ik] (nmat, nmat, 3), h_dev[ik],
 * o_dev[ik] (nmat, nmat); igpig_dev, vgpc_dev as exs_setup_batched_device.
 * Asynchronous on the context's stream. */
int exs_rttddft_updateham_device(exs_ctx *ctx, int nk, const int *ngp_host, const int *igpig_dev,
                                 const double *vgpc_dev, const double *atot, int calculate_overlap,
                                 exs_complex *const *pmat_dev, exs_complex *const *h_dev,
                                 exs_complex *const *o_dev);

/* Replaces Obtain_Pmat_LAPWLOBasis (src/src_xs/src_rttddft/rttddft_pmat.f90:
 * 22-64: pmatrad, then genpmatbasisik per k-point): the momentum matrix
 * elements pmat(1:nmat, 1:nmat, 1:3) of nk k-points, -i<phi|d/dx_j|phi'> in
 * the LAPW+lo basis with the interstitial (k+G')_j Theta(G - G') term,
 * computed on the device and registered for exs_rttddft_updateham as
 * exs_rttddft_set_pmat registers them.  apwalm[ik]: HOST matching
 * coefficients (ngkmax, apwordmax, lmmaxapw, natmtot) of the k-point (as
 * exs_match returns them); *in: the radial functions apwfr, lofr on the
 * meshes spr, nrmt (host; lmaxvr and veffmt unused); ngp, igpig, vgpc as
 * exs_setup_batched.  pmat: NULL, or nk HOST pointers (entries may be NULL)
 * to (ld, ld, 3) arrays that receive a copy.  Synchronous. */
int exs_rttddft_genpmat(exs_ctx *ctx, int nk, const int *ngp, const int *igpig, const double *vgpc,
                        const exs_complex *const *apwalm, const exs_mt_radial *in,
                        exs_complex *const *pmat, int ld);
/* Host utility of the above, callable without a GPU: the vector-coupling
 * coefficient <l2 m2; 1 q | l m> for l = l2 +- 1 (clebgor(l2, 1, l, m2, q, m),
 * src/src_lib/clebgor.f90, as gradzfmtr uses it), else 0. */
int exs_clebgor_unit(int l2, int m2, int q, int l, int m, double *value);

/* Replaces the loop of  call wavefmt(lrstp, lmax, is, ia, ngp, apwalm,
 * evecfv(:, ist), ld, wfmt)  (src/wavefmt.f90:13) over every atom and nst
 * states, as rhovalk.f90:119-142 and gendmatmt.f90 call it after match:
 *   apwalm(ngkmax, apwordmax, lmmaxapw, natmtot) HOST, as exs_match returns
 *     it (rows 1..ngp used);
 *   evecfv(ldv, nst) HOST, rows 1..nmat (nmat = ngp + nlotot);
 *   *in: apwfr(nrmtmax, 2, apwordmax, 0:lmaxapw, natmtot) and, with local
 *     orbitals, lofr(nrmtmax, 2, nlomax, natmtot), nrmt(nspecies) (HOST;
 *     spr, lmaxvr and veffmt unused);
 *   wfmt(ld, nrc, natmtot, nst) HOST out, nrc = (nrmtmax - 1) / lrstp + 1:
 *     wfmt(lm, ir, ias, ist) for lm < (lmax + 1)^2 and the points
 *     ir < (nrmt(is) - 1) / lrstp + 1 of the atom's species, as wavefmt
 *     writes wfmt(lm, ir); zero elsewhere.
 * lmax <= lmaxapw (the reference stops otherwise), ld >= (lmax + 1)^2.
 * The G sums are one cuBLAS ZGEMM, the radial expansion one kernel.
 * Synchronous. */
int exs_wavefmt(exs_ctx *ctx, int ngp, const exs_complex *apwalm, int nst, const exs_complex *evecfv, int ldv,
                int lrstp, int lmax, const exs_mt_radial *in, int ld, exs_complex *wfmt);

/* Autotuner (no counterpart in the reference): runs the batch described as
 * for exs_setup_batched_device once per kernel configuration of the active
 * precision mode (for the split-precision contraction: K chunks per
 * pipeline stage and stage count), times each on the device and keeps the
 * fastest for this (precision, padded N_G+k, APW rows, slices); a later
 * exs_set_precision with the same shape reuses the choice.  Overwrites the
 * outputs h_dev/o_dev with valid results.  *choice (may be NULL) receives
 * the configuration index.  Synchronous. */
int exs_autotune(exs_ctx *ctx, int nk, const int *ngp_host, const int *igpig_dev,
                 const double *vgpc_dev, exs_complex *const *h_dev,
                 exs_complex *const *o_dev, int *choice);

/* Selects the split-precision kernel configuration by index
 * (0 .. EXS_OZ_NCONFIG-1) instead of the autotuner's choice: bit 0 picks the
 * pipeline shape of the H/O tiles (slices: two 96 KB stages or four 48 KB
 * stages; moduli: 128 x 64 or 128 x 32 residue tiles), bit 1 a persistent
 * launch (one block per SM walking the tiles) of the H/O tiles instead of
 * one block per tile, bit 2 the same for the per-atom products (h_a A,
 * APW-lo rows), bit 3 two-SM H/O tiles (a pair of blocks computes 256 x 32,
 * or 256 x 64 residue tiles with moduli, with the B operand split between
 * them; with slices bit 1 is then ignored, with moduli bit 0 is ignored and
 * bit 1 makes the pairs persistent, one cluster per SM pair), bit 4 the products
 * h_a A and the APW-lo rows of H in native FP64 (DMMA) instead of int8
 * slices (bit 2 is then ignored; only the H/O contraction stays split).
 * Configurations with the same bit 4 give bit-identical results; the two
 * arithmetics for h_a A agree to FP64 rounding.  Until the autotuner or
 * this call chooses, exs_set_precision sets 0 for slices and 10 (persistent
 * two-SM residue tiles) for moduli. */
#define EXS_OZ_NCONFIG 32
int exs_set_kernel_config(exs_ctx *ctx, int config);

/* CUDA graph of one batched device setup (no counterpart in the reference):
 * the launches of exs_setup_batched_device for exactly these k-point sizes
 * and device buffers, captured once and replayed by exs_graph_launch on the
 * context's current stream (exs_synchronize waits and reports device
 * errors).  The contents of igpig_dev/vgpc_dev and the SCF inputs
 * (exs_set_scf_inputs overwrites them in place) may change between launches;
 * the sizes and buffers may not.  exs_set_precision invalidates the graph
 * (exs_graph_launch then returns EXS_ERR_STATE).  exs_graph_create runs the
 * setup once before capturing.  Phase timings are not recorded. */
typedef struct exs_graph exs_graph;
int exs_graph_create(exs_ctx *ctx, int nk, const int *ngp_host, const int *igpig_dev,
                     const double *vgpc_dev, exs_complex *const *h_dev,
                     exs_complex *const *o_dev, exs_graph **out);
int exs_graph_launch(exs_graph *graph);
void exs_graph_destroy(exs_graph *graph);

/* One graph over several contexts: the batched device setup of nk[i]
 * k-points of context ctx[i] (arguments per context as for
 * exs_setup_batched_device), for the uneven-size batch of independent cells
 * (one context per cell).  The contexts' launches are captured on up to 32
 * concurrent branches; the graph is launched on ctx[0]'s stream.
 * exs_graph_synchronize waits for it and returns the worst status of all
 * contexts (device error flags included); it also serves single-context
 * graphs. */
int exs_graph_create_multi(int nctx, exs_ctx *const *ctx, const int *nk, const int *const *ngp_host,
                           const int *const *igpig_dev, const double *const *vgpc_dev,
                           exs_complex *const *const *h_dev, exs_complex *const *const *o_dev,
                           exs_graph **out);
int exs_graph_synchronize(exs_graph *graph);

/* Replaces the IBS part of  call forcek(ik, ffacg)  (src/forcek.f90:13) for
 * one k-point without second variation:
 *   igpig(ngkmax), vgpc(3, ngkmax), evecfv(nmatmax, nstfv) (leading dim ldv),
 *   evalfv(nstfv), occsv(nstfv), wkpt(ik);
 *   ffacg(ngvec, nspecies) (genffacg), vgc(3, ngvec);
 *   forceibs(3, natmtot) is ACCUMULATED into, as the reference does. */
int exs_forcek(exs_ctx *ctx, int ngp, const int *igpig, const double *vgpc,
               int nstfv, const exs_complex *evecfv, int ldv, const double *evalfv,
               const double *occsv, double wkpt, const double *ffacg, const double *vgc,
               double *forceibs);

/* Adjoint of the setup for L = sum_n w_n c_n^H (H - eps_n O) c_n with the
 * weighted factors given (no counterpart routine in the reference; it
 * generalises forcek.f90): c(ldv, nst) with nmat = ngp + nlotot rows,
 * w(nst), eps(nst); ffacg(ngvec, nspecies), vgc(3, ngvec) as for exs_forcek.
 * Outputs (overwritten): dtau(3, natmtot) = dL/dtau (= -F_IBS);
 * dveffig(ngvec) (may be NULL): for any perturbation with
 * dV(-G) = conj dV(G), dL = sum_g dveffig(g) dV(g);
 * dh(maxaa, maxaa, natmtot) (may be NULL): dL = sum dh(f,f',a) d aa(f,f',a)
 * for Hermitian perturbations of mt_hscf%main%aa. */
int exs_adjoint(exs_ctx *ctx, int ngp, const int *igpig, const double *vgpc, int nst,
                const exs_complex *c, int ldv, const double *w, const double *eps,
                const double *ffacg, const double *vgc, double *dtau,
                exs_complex *dveffig, exs_complex *dh);

/* Index map that sorts a(1 + inc*(i-1)), i = 1..n, ascending: the heapsort
 * of sort_index_1d_real (src/sorting.f90:74-117) step for step, so that
 * elements of equal value come out in the reference's order (the heapsort is
 * not stable).  idx(n) receives 1-based indices.  Host only; used to number
 * the G-vectors by length as gengvec does (src/gengvec.f90:73-74). */
int exs_sort_index_1d(int n, const double *a, int inc, int *idx);

/* Limit, in SM clock cycles, of every wait of the split-precision
 * kernels' pipelines (a producer on a free stage, the tensor core on a
 * filled one, the epilogue on finished products); 0 restores the default
 * of 2e9 (about one second).  A wait that runs out makes the kernel give up
 * cleanly and the call return EXS_ERR_TIMEOUT; the context stays usable.
 * Graphs captured before the call keep their old limit (they are
 * invalidated: exs_graph_launch returns EXS_ERR_STATE).  No counterpart in
 * the reference (failure detection of the device pipeline). */
int exs_set_wait_limit(exs_ctx *ctx, long long cycles);

/* Run the context's work on a caller-owned CUDA stream (a cudaStream_t
 * passed as void*); NULL returns to the context's own stream. */
int exs_set_stream(exs_ctx *ctx, void *stream);

/* Device time of the phases of the last setup call, milliseconds:
 * t[0] match, t[1] h_a A, t[2] MT contraction + interstitial, t[3] lo blocks, t[4] total;
 * with n > 5, t[5] the field/momentum combination of the last RT-TDDFT update. */
int exs_last_timings(exs_ctx *ctx, double *t, int n);

/* For callers that cannot allocate device memory (no exs_ctx: creating one
 * allocates).  No counterpart in the reference: it is the APW-APW muffin-tin
 * block of hamiltonsetup/overlapsetup without the interstitial term, on
 * caller-owned DEVICE arrays, with all work space in one 32 MiB static
 * device array inside this library (held by every GPU that loads it):
 *   apwi(maxaa, ngp, natmtot): each atom's matching coefficients in the
 *     reference's row order (l, m, io) (hamiltonsetup.f90:59-71), zero past
 *     napw[ias] rows;  aa(maxaa, maxaa, natmtot): mt_hscf%main%aa;
 *   napw: HOST array (natmtot) of APW rows per atom;
 *   h, o: za(ld, ngp) outputs, H = sum_a apwi^H aa apwi and O = sum_a
 *     apwi^H apwi as full Hermitian matrices (lower = conjugate of upper).
 * Allocates nothing; EXS_ERR_SIZE when the work space exceeds 32 MiB.  The
 * first call on a device looks up the array's device address (make it
 * before any stream capture); cudaDeviceReset destroys the array, so do not
 * call it again on a device after resetting it.  Calls share the array:
 * calls that overlap on the GPU race, so serialise them.  stream: a
 * cudaStream_t, or NULL. */
int exs_mt_contract_noalloc(int natmtot, int maxaa, const int *napw, int ngp,
                            const exs_complex *apwi, const exs_complex *aa,
                            exs_complex *h, exs_complex *o, int ld, void *stream);

#ifdef __cplusplus
}
#endif
#endif
