// C-ABI of libexciting_b200: context, input upload, and the entry points that
// replace the reference's match / hamiltonandoverlapsetup calls.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "exs_internal.cuh"

using exs::AtomDesc;
using exs::DevParams;
using exs::KDesc;

namespace {

int fail(exs_ctx *c, int code, const std::string &msg)
{
    if (c) c->last_error = msg;
    return code;
}

int cuda_fail(exs_ctx *c, cudaError_t e, const char *where)
{
    return fail(c, EXS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define EXS_CUDA(call)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call);  \
    } while (0)

template <class T>
cudaError_t dalloc(T **p, size_t n)
{
    *p = nullptr;
    if (n == 0) return cudaSuccess;
    return cudaMalloc((void **)p, n * sizeof(T));
}

// Copy n elements to the device array *p, allocating it on first use (the
// sizes of every array uploaded more than once are fixed per context, so a
// later upload reuses the allocation and captured graphs stay valid).
template <class T>
cudaError_t upload(T **p, const T *h, size_t n, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    if (!*p) {
        cudaError_t e = dalloc(p, n);
        if (e != cudaSuccess) return e;
    }
    return cudaMemcpyAsync(*p, h, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace

exs::OzAtomArgs exs_ctx::oz_atom_args() const
{
    exs::OzAtomArgs a{};
    a.hr = d_haa_r;
    a.hi = d_haa_i;
    a.lr = d_loa_r;
    a.li = d_loa_i;
    a.ldh = ldh;
    a.ldlo = ldlo;
    a.maxaa = maxaa;
    a.nfb = oz_nfb;
    a.nxb = oz_nxb;
    a.lw = oz_lw;
    a.xs = d_xs;
    a.xsig = d_xsig;
    return a;
}

exs::DevParams exs_ctx::params() const
{
    DevParams p{};
    p.natmtot = natmtot;
    p.lmaxapw = lmaxapw;
    p.lmaxmat = lmaxmat;
    p.apwordmax = apwordmax;
    p.lmmaxapw = (lmaxapw + 1) * (lmaxapw + 1);
    p.np_tail = np_tail;
    p.ngkmax = ngkmax;
    p.npad = npad;
    p.K = K;
    p.Kpad = Kpad;
    p.nlotot = nlotot;
    p.maxnlo = maxnlo;
    p.nlomax = nlomax;
    p.lolmmax = lolmmax;
    p.ngvec = ngvec;
    p.ngrtot = ngrtot;
    for (int i = 0; i < 3; i++) {
        p.intgv_lo[i] = intgv[i];
        p.intgv_n[i] = intgv[3 + i] - intgv[i] + 1;
    }
    p.relativity = relativity;
    p.omega = omega;
    p.atoms = d_atoms;
    p.apword = d_apword;
    p.rmt = d_rmt;
    p.spr_tail = d_spr_tail;
    p.apwfr_tail = d_apwfr_tail;
    p.ivg = d_ivg;
    p.ivgig = d_ivgig;
    p.veffig = d_veffig;
    p.kinw = d_kinw;
    p.cfunig = d_cfunig;
    p.m2effig = d_m2effig;
    p.lolo = d_lolo;
    p.ololo = d_ololo;
    p.h1lolo = d_h1lolo;
    p.oalo = d_oalo;
    p.h1loa = d_h1loa;
    p.h1aa = d_h1aa;
    p.idxlo = d_idxlo;
    p.lorbl = d_lorbl;
    p.nlorb = d_nlorb;
    p.dlu = d_dlu;
    p.err = d_err;
    return p;
}

extern "C" {

const char *exs_last_error(const exs_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int exs_ctx_sizes(const exs_ctx *c, int *maxaa, int *maxnlo, int *nlotot)
{
    if (!c) return EXS_ERR_ARG;
    if (maxaa) *maxaa = c->maxaa;
    if (maxnlo) *maxnlo = c->maxnlo;
    if (nlotot) *nlotot = c->nlotot;
    return EXS_OK;
}

int exs_ctx_destroy(exs_ctx *c)
{
    if (!c) return EXS_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *dev[] = {c->d_atoms, c->d_apword, c->d_ivg, c->d_ivgig, c->d_idxlo, c->d_lorbl, c->d_nlorb, c->d_rmt,
                   c->d_haa_r, c->d_haa_i, c->d_loa_r, c->d_loa_i, c->d_lolo, c->d_oalo, c->d_ololo, c->d_h1aa,
                   c->d_h1loa, c->d_h1lolo, c->d_veffig, c->d_kinw, c->d_cfunig, c->d_m2effig, c->d_spr_tail,
                   c->d_apwfr_tail, c->d_dlu, c->d_work, c->d_ho, c->d_igpig, c->d_vgpc, c->d_err, c->d_tables,
                   c->d_match_in, c->d_match_sf, c->d_apwalm};
    for (void *p : dev)
        if (p) cudaFree(p);
    if (c->d_oz) cudaFree(c->d_oz);
    if (c->d_res) cudaFree(c->d_res);
    if (c->d_pace) cudaFree(c->d_pace);
    if (c->d_ozscale) cudaFree(c->d_ozscale);
    if (c->d_xs) cudaFree(c->d_xs);
    if (c->d_xsig) cudaFree(c->d_xsig);
    if (c->fk_dev) cudaFree(c->fk_dev);
    if (c->fk_tab_d) cudaFree(c->fk_tab_d);
    if (c->fk_dh) cudaFree(c->fk_dh);
    if (c->fk_tab_h) cudaFreeHost(c->fk_tab_h);
    if (c->h_tables) cudaFreeHost(c->h_tables);
    if (c->h_igpig_pinned) cudaFreeHost(c->h_igpig_pinned);
    if (c->h_vgpc_pinned) cudaFreeHost(c->h_vgpc_pinned);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->tables_free) cudaEventDestroy(c->tables_free);
    for (auto &e : c->ev_group)
        if (e) cudaEventDestroy(e);
    for (int q = 0; q < 2; q++) {
        if (c->ev_d2h[q]) cudaEventDestroy(c->ev_d2h[q]);
        if (c->d_pack[q]) cudaFree(c->d_pack[q]);
        if (c->h_pack[q]) cudaFreeHost(c->h_pack[q]);
        if (c->d_packdesc[q]) cudaFree(c->d_packdesc[q]);
        if (c->h_packdesc[q]) cudaFreeHost(c->h_packdesc[q]);
    }
    delete c->pool;
    exs::solver_release(c);
    exs::mt_release(c);
    exs::rt_release(c);
    exs::pm_release(c);
    exs::wf_release(c);
    if (c->d_eval) cudaFree(c->d_eval);
    if (c->d_evec) cudaFree(c->d_evec);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->copy_stream2) cudaStreamDestroy(c->copy_stream2);
    if (c->ev_copy2) cudaEventDestroy(c->ev_copy2);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return EXS_OK;
}

int exs_ctx_create(const exs_config *cfg, exs_ctx **out)
{
    if (!out) return EXS_ERR_ARG;
    *out = nullptr;
    if (!cfg || !cfg->atom_species || !cfg->apword || !cfg->rmt || !cfg->atposc || !cfg->bvec || !cfg->intgv ||
        !cfg->ivg || !cfg->ivgig)
        return EXS_ERR_ARG;
    if (cfg->natmtot <= 0 || cfg->nspecies <= 0 || cfg->ngkmax <= 0 || cfg->ngrtot <= 0 || cfg->ngvec <= 0 ||
        cfg->ngvec > cfg->ngrtot || cfg->max_batch <= 0)
        return EXS_ERR_ARG;
    if (cfg->lmaxapw < 0 || cfg->lmaxapw > EXS_LMAX_APW || cfg->lmaxmat < 0 || cfg->lmaxmat > cfg->lmaxapw)
        return EXS_ERR_SIZE;
    if (cfg->apwordmax < 1 || cfg->apwordmax > EXS_APWORD_MAX) return EXS_ERR_SIZE;
    if (cfg->np_tail != std::max(cfg->apwordmax + 1, 4)) return EXS_ERR_ARG;
    if (cfg->relativity < EXS_REL_NONE || cfg->relativity > EXS_REL_IORA) return EXS_ERR_ARG;

    exs_ctx *c = new (std::nothrow) exs_ctx();
    if (!c) return EXS_ERR_NOMEM;
    cudaGetDevice(&c->device);
    c->natmtot = cfg->natmtot;
    c->nspecies = cfg->nspecies;
    c->lmaxapw = cfg->lmaxapw;
    c->lmaxmat = cfg->lmaxmat;
    c->apwordmax = cfg->apwordmax;
    c->nlomax = std::max(cfg->nlomax, 1);
    c->omega = cfg->omega;
    c->ngkmax = cfg->ngkmax;
    c->ngrtot = cfg->ngrtot;
    c->ngvec = cfg->ngvec;
    c->relativity = cfg->relativity;
    c->np_tail = cfg->np_tail;
    c->max_batch = cfg->max_batch;
    std::memcpy(c->intgv, cfg->intgv, sizeof(c->intgv));
    c->atom_species.assign(cfg->atom_species, cfg->atom_species + c->natmtot);
    c->apword.assign(cfg->apword, cfg->apword + (size_t)(c->lmaxapw + 1) * c->nspecies);
    c->nlorb.assign(c->nspecies, 0);
    if (cfg->nlorb) c->nlorb.assign(cfg->nlorb, cfg->nlorb + c->nspecies);
    c->lorbl.assign((size_t)c->nlomax * c->nspecies, 0);
    if (cfg->lorbl && cfg->nlomax > 0) c->lorbl.assign(cfg->lorbl, cfg->lorbl + (size_t)cfg->nlomax * c->nspecies);
    c->rmt.assign(cfg->rmt, cfg->rmt + c->nspecies);
    c->atposc.assign(cfg->atposc, cfg->atposc + 3 * (size_t)c->natmtot);
    c->bvec.assign(cfg->bvec, cfg->bvec + 9);

    // ---- validation of the basis description
    for (int ias = 0; ias < c->natmtot; ias++) {
        const int s = c->atom_species[ias];
        if (s < 0 || s >= c->nspecies || (ias > 0 && s < c->atom_species[ias - 1])) {
            exs_ctx_destroy(c);
            return EXS_ERR_ARG;  // atoms must be grouped by species (idxas order)
        }
    }
    for (int is = 0; is < c->nspecies; is++) {
        for (int l = 0; l <= c->lmaxapw; l++) {
            const int a = c->apword[l + (size_t)(c->lmaxapw + 1) * is];
            if (a < 1 || a > c->apwordmax) { exs_ctx_destroy(c); return EXS_ERR_ARG; }
        }
        if (c->nlorb[is] < 0 || c->nlorb[is] > c->nlomax) { exs_ctx_destroy(c); return EXS_ERR_ARG; }
        for (int ilo = 0; ilo < c->nlorb[is]; ilo++) {
            const int l = c->lorbl[ilo + (size_t)c->nlomax * is];
            if (l < 0 || l > c->lmaxmat) { exs_ctx_destroy(c); return EXS_ERR_SIZE; }
            c->lolmax = std::max(c->lolmax, l);
        }
    }
    for (int i = 0; i < 3; i++)
        if (c->intgv[3 + i] < c->intgv[i]) { exs_ctx_destroy(c); return EXS_ERR_ARG; }
    const long nbox = (long)(c->intgv[3] - c->intgv[0] + 1) * (c->intgv[4] - c->intgv[1] + 1) * (c->intgv[5] - c->intgv[2] + 1);

    // ---- MaxAPWs, genidxlo, MTInitAll
    auto napw_species = [&](int is) {
        int n = 0;
        for (int l = 0; l <= c->lmaxmat; l++) n += (2 * l + 1) * c->apword[l + (size_t)(c->lmaxapw + 1) * is];
        return n;
    };
    c->maxaa = 0;
    for (int is = 0; is < c->nspecies; is++) c->maxaa = std::max(c->maxaa, napw_species(is));
    c->lolmmax = (c->lolmax + 1) * (c->lolmax + 1);
    c->idxlo.assign((size_t)c->lolmmax * c->nlomax * c->natmtot, 0);
    int i = 0;
    for (int is = 0; is < c->nspecies; is++)
        for (int ias = 0; ias < c->natmtot; ias++) {
            if (c->atom_species[ias] != is) continue;
            for (int ilo = 0; ilo < c->nlorb[is]; ilo++) {
                const int l = c->lorbl[ilo + (size_t)c->nlomax * is];
                for (int m = -l; m <= l; m++) {
                    i++;
                    c->idxlo[(l * (l + 1) + m) + (size_t)c->lolmmax * (ilo + (size_t)c->nlomax * ias)] = i;
                }
            }
        }
    c->nlotot = i;
    c->losize.assign(c->nspecies, 0);
    c->maxnlo = 0;
    for (int is = 0; is < c->nspecies; is++) {
        int n = 0;
        for (int ilo = 0; ilo < c->nlorb[is]; ilo++) n += 2 * c->lorbl[ilo + (size_t)c->nlomax * is] + 1;
        c->losize[is] = n;
        c->maxnlo = std::max(c->maxnlo, n);
    }
    c->atoms.resize(c->natmtot);
    int off = 0;
    for (int ias = 0; ias < c->natmtot; ias++) {
        AtomDesc &a = c->atoms[ias];
        const int is = c->atom_species[ias];
        a.species = is;
        a.apw_off = off;
        a.napw = napw_species(is);
        off += a.napw;
        a.losize = c->losize[is];
        if (c->nlorb[is] > 0) {
            const int l = c->lorbl[(size_t)c->nlomax * is];
            a.lo_off = c->idxlo[(l * (l + 1) - l) + (size_t)c->lolmmax * ((size_t)c->nlomax * ias)] - 1;
        } else {
            a.lo_off = -1;
        }
        for (int k = 0; k < 3; k++) a.pos[k] = c->atposc[3 * (size_t)ias + k];
        a.oz_x0 = a.apw_off & ~15;
        a.oz_nch = (a.apw_off - a.oz_x0 + a.napw + 127) / 128;
    }
    c->K = off;
    c->Kpad = round_up(c->K, 16);
    c->npad = round_up(c->ngkmax, 64);
    c->nmatmax = c->ngkmax + c->nlotot;
    c->ldh = round_up(c->maxaa, 8);
    c->ldlo = round_up(std::max(c->maxnlo, 1), 2);
    c->nplanes = (c->relativity == EXS_REL_IORA) ? 6 : 4;
    c->plane = (size_t)c->Kpad * c->npad;

    // ---- device objects
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        exs_ctx_destroy(c);
        return EXS_ERR_CUDA;
    }
    c->stream = c->own_stream;
    if ((e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->copy_stream2, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_copy2, cudaEventDisableTiming)) != cudaSuccess) {
        exs_ctx_destroy(c);
        return EXS_ERR_CUDA;
    }
    cudaEventCreateWithFlags(&c->ev_group[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_group[1], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_d2h[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_d2h[1], cudaEventDisableTiming);
    for (auto &ev : c->ev) cudaEventCreate(&ev);
    cudaEventCreateWithFlags(&c->tables_free, cudaEventDisableTiming);
    cudaStream_t s = c->stream;
    e = upload(&c->d_atoms, c->atoms.data(), c->atoms.size(), s);
    if (e == cudaSuccess) e = upload(&c->d_apword, c->apword.data(), c->apword.size(), s);
    if (e == cudaSuccess) e = upload(&c->d_ivg, cfg->ivg, 3 * (size_t)c->ngrtot, s);
    if (e == cudaSuccess) e = upload(&c->d_ivgig, cfg->ivgig, (size_t)nbox, s);
    if (e == cudaSuccess) e = upload(&c->d_idxlo, c->idxlo.data(), c->idxlo.size(), s);
    if (e == cudaSuccess) e = upload(&c->d_lorbl, c->lorbl.data(), c->lorbl.size(), s);
    if (e == cudaSuccess) e = upload(&c->d_nlorb, c->nlorb.data(), c->nlorb.size(), s);
    if (e == cudaSuccess) e = upload(&c->d_rmt, c->rmt.data(), c->rmt.size(), s);
    if (e == cudaSuccess) e = dalloc(&c->d_err, 4);
    if (e == cudaSuccess) e = dalloc(&c->d_work, c->plane * c->nplanes * c->max_batch);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_work, 0, c->plane * c->nplanes * c->max_batch * sizeof(double), s);
    if (e == cudaSuccess) e = dalloc(&c->d_ho, 2 * (size_t)c->nmatmax * c->nmatmax * c->max_batch);
    if (e == cudaSuccess) e = dalloc(&c->d_igpig, (size_t)c->ngkmax * c->max_batch);
    if (e == cudaSuccess) e = dalloc(&c->d_vgpc, 3 * (size_t)c->ngkmax * c->max_batch);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_igpig_pinned, sizeof(int) * (size_t)c->ngkmax * c->max_batch);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_vgpc_pinned, sizeof(double) * 3 * (size_t)c->ngkmax * c->max_batch);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? EXS_ERR_NOMEM : EXS_ERR_CUDA;
        exs_ctx_destroy(c);
        return code;
    }
    *out = c;
    return EXS_OK;
}

int exs_set_precision(exs_ctx *c, int mode, int slices)
{
    if (!c) return EXS_ERR_ARG;
    c->gen++;   // graphs captured before this call are no longer valid
    if (mode == EXS_PREC_FP64) {
        c->prec_mode = mode;
        return EXS_OK;
    }
    if (mode != EXS_PREC_OZAKI_INT8 && mode != EXS_PREC_OZAKI_MOD)
        return fail(c, EXS_ERR_ARG, "unknown precision mode");
    if (mode == EXS_PREC_OZAKI_INT8 && (slices < 3 || slices > 9))
        return fail(c, EXS_ERR_ARG, "slices must be in 3..9");
    if (mode == EXS_PREC_OZAKI_MOD && slices != 0 && (slices < 6 || slices > exs::OZ_MAX_MODULI))
        return fail(c, EXS_ERR_ARG, "moduli must be 0 (automatic) or in 6..16");
    const int kp8 = exs::oz_kpad(c->K);
    exs::OzScheme sch{};
    if (mode == EXS_PREC_OZAKI_MOD) {
        if (exs::oz_mod_plan(slices, c->K, std::max(1, c->maxaa), &sch) != 0)
            return fail(c, EXS_ERR_SIZE, "no modular plan for this K (K <= 65536, at least 8 bits per operand)");
        slices = sch.n;
    } else {
        sch.n = slices;
        sch.seg = exs::oz_seg_pairs(slices, kp8);
        if (sch.seg < 1) return fail(c, EXS_ERR_SIZE, "K too large for exact int32 accumulation of one slice pair");
    }
    const int seg = sch.seg;
    cudaSetDevice(c->device);
    EXS_CUDA(cudaStreamSynchronize(c->stream));
    const int narr = c->relativity == EXS_REL_IORA ? 6 : 4;    // + Cr, Ci: O = A^H (I + h1aa) A
    const size_t slot = exs::oz_slot_bytes(slices, c->npad, kp8, narr);
    if (c->d_oz) { cudaFree(c->d_oz); c->d_oz = nullptr; }
    if (c->d_res) { cudaFree(c->d_res); c->d_res = nullptr; c->res_bytes = 0; }
    if (c->d_pace) { cudaFree(c->d_pace); c->d_pace = nullptr; }
    if (c->d_ozscale) { cudaFree(c->d_ozscale); c->d_ozscale = nullptr; }
    if (c->d_xs) { cudaFree(c->d_xs); c->d_xs = nullptr; }
    if (c->d_xsig) { cudaFree(c->d_xsig); c->d_xsig = nullptr; }
    // per-atom operands: windows of 128-byte chunks, 64-row blocks of h_a and lo rows
    int nch = 1;
    for (const AtomDesc &a : c->atoms) nch = std::max(nch, a.oz_nch);
    c->oz_lw = 128 * nch;
    c->oz_nfb = (c->maxaa + 63) / 64;
    c->oz_nxb = c->oz_nfb + (c->maxnlo + 63) / 64;
    c->oz_xseg = mode == EXS_PREC_OZAKI_MOD ? 1 : exs::oz_seg_pairs(slices, c->oz_lw);
    sch.segx = c->oz_xseg;
    const size_t xgroups = (size_t)c->natmtot * slices * c->oz_nxb;
    // moduli: the residue tiles of the H/O products of a whole batch, for
    // either tile width (the upper tiles of ngkmax G+k per k-point)
    size_t res = 0;
    if (mode == EXS_PREC_OZAKI_MOD)
        for (int q : {0, 1, 8}) {
            const int bj = exs::oz_res_cols(q), bi = exs::oz_res_rows(q);
            size_t tiles = 0;      // 128-row residue tiles
            for (int ib = 0; ib < (c->ngkmax + bi - 1) / bi; ib++)
                for (int jb = 0; jb < (c->ngkmax + bj - 1) / bj; jb++)
                    if (jb * bj + bj - 1 >= ib * bi) tiles += bi / 128;
            res = std::max(res, tiles * exs::oz_res_tile_bytes(slices, q) * c->max_batch);
        }
    cudaError_t e = cudaMalloc((void **)&c->d_oz, slot * c->max_batch);
    if (e == cudaSuccess && res > 0) {
        e = cudaMalloc((void **)&c->d_res, res);
        if (e == cudaSuccess) c->res_bytes = res;
        if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_pace, exs::oz_pace_bytes());
    }
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_ozscale, sizeof(double) * 3 * c->npad * c->max_batch);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_xs, xgroups * 128 * c->oz_lw);
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_xsig, sizeof(double) * c->natmtot * c->oz_nxb * 64);
    if (e != cudaSuccess || c->oz_xseg < 1) {
        c->prec_mode = EXS_PREC_FP64;
        return fail(c, e != cudaSuccess ? EXS_ERR_NOMEM : EXS_ERR_SIZE, "split-precision work space");
    }
    c->kp8 = kp8;
    c->oz_seg = seg;
    c->oz_slot_bytes = slot;
    // the slices of all slots: (slot x slice) groups of 4 arrays x npad rows x kp8 bytes
    const size_t nss = (size_t)slices * c->max_batch;
    bool maps_ok = true;
    for (int q = 0; q < exs::OZ_NCFG; q++)
        maps_ok = maps_ok && exs::make_oz_tensor_maps(c->d_oz, nss, c->npad, kp8, exs::OZ_CFG_KCH[q], narr,
                                                      &c->oz_mapA[q], &c->oz_mapB[q], &c->oz_mapB2[q]);
    maps_ok = maps_ok && exs::make_oz_atom_maps(c->d_oz, nss, c->npad, kp8, narr, c->d_xs, xgroups, c->oz_lw,
                                                &c->oz_mapArow, &c->oz_mapX);
    maps_ok = maps_ok && exs::make_oz_b64_map(c->d_oz, nss, c->npad, kp8, narr, &c->oz_mapB64, &c->oz_mapB64h);
    if (!maps_ok) {
        cudaFree(c->d_oz); c->d_oz = nullptr;
        cudaFree(c->d_ozscale); c->d_ozscale = nullptr;
        c->prec_mode = EXS_PREC_FP64;
        return fail(c, EXS_ERR_CUDA, "cuTensorMapEncodeTiled failed for the slice array");
    }
    c->slices = slices;
    sch.wait = c->oz_wait;
    c->oz_sch = sch;
    c->prec_mode = mode;
    if (c->have_inputs) {   // slices of the current h_a and loa
        EXS_CUDA(exs::launch_oz_x(c->params(), c->oz_atom_args(), c->oz_sch, c->stream));
        EXS_CUDA(cudaStreamSynchronize(c->stream));
    }
    {   // a configuration the autotuner chose earlier for this shape; else, with moduli, the paced
        // persistent two-SM residue tiles (1.5x the 128 x 64 tiles on the 216-atom cell)
        auto it = c->oz_tuned.find(std::make_tuple((int)mode, c->npad, c->K, slices));
        c->oz_cfg = it != c->oz_tuned.end() ? it->second : (mode == EXS_PREC_OZAKI_MOD ? 10 : 0);
    }
    return EXS_OK;
}

int exs_set_scf_inputs(exs_ctx *c, const exs_scf_inputs *in)
{
    if (!c || !in || !in->veffig || !in->cfunig || !in->spr_tail || !in->apwfr_tail)
        return fail(c, EXS_ERR_ARG, "exs_set_scf_inputs: missing input array");
    // oalo = NULL keeps the overlap radial integrals (and h1*) exs_olprad left on the device
    const bool keep_olp = !in->oalo;
    if (keep_olp && !c->have_olp)
        return fail(c, EXS_ERR_ARG, "exs_set_scf_inputs: oalo is NULL and exs_olprad has not run");
    if (!keep_olp && !in->ololo) return fail(c, EXS_ERR_ARG, "exs_set_scf_inputs: missing ololo");
    // mt_aa = NULL keeps the muffin-tin integrals exs_hmlint left on the device
    const bool keep_mt = !in->mt_aa;
    if (keep_mt && !c->have_mt)
        return fail(c, EXS_ERR_ARG, "exs_set_scf_inputs: mt_aa is NULL and exs_hmlint has not run");
    if (!keep_mt && c->nlotot > 0 && (!in->mt_loa || !in->mt_lolo)) return fail(c, EXS_ERR_ARG, "missing loa/lolo");
    if (c->relativity != EXS_REL_NONE && !in->meffig) return fail(c, EXS_ERR_ARG, "missing meffig");
    if (c->relativity == EXS_REL_IORA && (!in->m2effig || (!keep_olp && (!in->h1aa || !in->h1loa || !in->h1lolo))))
        return fail(c, EXS_ERR_ARG, "missing iora* inputs");
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    EXS_CUDA(cudaStreamSynchronize(s));
    // a new SCF iteration overwrites the previous inputs in place
    c->have_inputs = false;
    const int nat = c->natmtot, maxaa = c->maxaa, maxnlo = std::max(c->maxnlo, 1);
    // h_a: aa(f, f', ias) -> planar [ias][f'][f] with leading dim ldh
    if (!keep_mt) {
        std::vector<double> re((size_t)nat * c->ldh * c->ldh, 0.0), im(re.size(), 0.0);
        for (int ias = 0; ias < nat; ias++)
            for (int f2 = 0; f2 < maxaa; f2++)
                for (int f1 = 0; f1 < maxaa; f1++) {
                    const exs_complex z = in->mt_aa[f1 + (size_t)maxaa * (f2 + (size_t)maxaa * ias)];
                    re[f1 + (size_t)c->ldh * (f2 + (size_t)c->ldh * ias)] = z.re;
                    im[f1 + (size_t)c->ldh * (f2 + (size_t)c->ldh * ias)] = z.im;
                }
        EXS_CUDA(upload(&c->d_haa_r, re.data(), re.size(), s));
        EXS_CUDA(upload(&c->d_haa_i, im.data(), im.size(), s));
        EXS_CUDA(cudaStreamSynchronize(s));
    }
    // loa(r, f, ias) -> planar [ias][f][r] with leading dim ldlo
    if (!keep_mt) {
        std::vector<double> re((size_t)nat * c->ldlo * maxaa, 0.0), im(re.size(), 0.0);
        if (in->mt_loa)
            for (int ias = 0; ias < nat; ias++)
                for (int f = 0; f < maxaa; f++)
                    for (int r = 0; r < c->maxnlo; r++) {
                        const exs_complex z = in->mt_loa[r + (size_t)maxnlo * (f + (size_t)maxaa * ias)];
                        re[r + (size_t)c->ldlo * (f + (size_t)maxaa * ias)] = z.re;
                        im[r + (size_t)c->ldlo * (f + (size_t)maxaa * ias)] = z.im;
                    }
        EXS_CUDA(upload(&c->d_loa_r, re.data(), re.size(), s));
        EXS_CUDA(upload(&c->d_loa_i, im.data(), im.size(), s));
        EXS_CUDA(cudaStreamSynchronize(s));
    }
    if (!keep_mt) {
        std::vector<exs_complex> zero_lolo;
        const exs_complex *lolo = in->mt_lolo;
        if (!lolo) { zero_lolo.assign((size_t)maxnlo * maxnlo * nat, exs_complex{0, 0}); lolo = zero_lolo.data(); }
        EXS_CUDA(upload(&c->d_lolo, lolo, (size_t)maxnlo * maxnlo * nat, s));
        EXS_CUDA(cudaStreamSynchronize(s));
        c->have_mt = false;
    }
    if (!keep_olp) {
        EXS_CUDA(upload(&c->d_oalo, in->oalo, (size_t)c->apwordmax * c->nlomax * nat, s));
        EXS_CUDA(upload(&c->d_ololo, in->ololo, (size_t)c->nlomax * c->nlomax * nat, s));
        if (c->relativity == EXS_REL_IORA) {
            EXS_CUDA(upload(&c->d_h1aa, in->h1aa, (size_t)c->apwordmax * c->apwordmax * (c->lmaxapw + 1) * nat, s));
            EXS_CUDA(upload(&c->d_h1loa, in->h1loa, (size_t)c->apwordmax * c->nlomax * nat, s));
            EXS_CUDA(upload(&c->d_h1lolo, in->h1lolo, (size_t)c->nlomax * c->nlomax * nat, s));
        }
        EXS_CUDA(cudaStreamSynchronize(s));
        c->have_olp = false;
    }
    if (c->relativity == EXS_REL_IORA) EXS_CUDA(upload(&c->d_m2effig, in->m2effig, (size_t)c->ngvec, s));
    EXS_CUDA(upload(&c->d_veffig, in->veffig, (size_t)c->ngvec, s));
    EXS_CUDA(upload(&c->d_cfunig, in->cfunig, (size_t)c->ngvec, s));
    EXS_CUDA(upload(&c->d_kinw, c->relativity == EXS_REL_NONE ? in->cfunig : in->meffig, (size_t)c->ngvec, s));
    EXS_CUDA(upload(&c->d_spr_tail, in->spr_tail, (size_t)c->np_tail * c->nspecies, s));
    EXS_CUDA(upload(&c->d_apwfr_tail, in->apwfr_tail,
                    (size_t)c->np_tail * c->apwordmax * (c->lmaxapw + 1) * nat, s));
    // the matching systems D_l depend only on the tails: factorised once here
    if (!c->d_dlu) EXS_CUDA(dalloc(&c->d_dlu, (size_t)nat * (c->lmaxapw + 1) * exs::DLU_STRIDE));
    EXS_CUDA(exs::launch_match_dlu(c->params(), c->d_dlu, s));
    if (c->oz_on())   // slices of the new h_a and loa, in place
        EXS_CUDA(exs::launch_oz_x(c->params(), c->oz_atom_args(), c->oz_sch, s));
    EXS_CUDA(cudaStreamSynchronize(s));
    c->have_inputs = true;
    return EXS_OK;
}

int exs_synchronize(exs_ctx *c)
{
    if (!c) return EXS_ERR_ARG;
    cudaSetDevice(c->device);
    EXS_CUDA(cudaStreamSynchronize(c->stream));
    int err = 0;
    EXS_CUDA(cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (c->timed) {   // phase events were recorded by the last setup call
        for (int i = 0; i < 4; i++) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]) == cudaSuccess) c->last_t[i] = ms;
        }
        float tot = 0.f;
        if (cudaEventElapsedTime(&tot, c->ev[0], c->ev[4]) == cudaSuccess) c->last_t[4] = tot;
        c->timed = false;
        (void)cudaGetLastError();   // an event query must not leave a sticky error for the next call
    }
    if (err & exs::DEV_ERR_INDEX)
        return fail(c, EXS_ERR_INDEX, "a G-G' difference fell outside the ivgig box");
    if (err & exs::DEV_ERR_TIMEOUT)
        return fail(c, EXS_ERR_TIMEOUT, "a tensor-core pipeline wait expired (the kernel gave up and drained)");
    if (err & exs::DEV_WARN_SINGULAR) {
        c->last_error = "a matching system D_l was singular (match.f90:166-175)";
        return EXS_WARN_SINGULAR;
    }
    return EXS_OK;
}

int exs_set_wait_limit(exs_ctx *c, long long cycles)
{
    if (!c) return EXS_ERR_ARG;
    if (cycles < 0) return fail(c, EXS_ERR_ARG, "negative wait limit");
    c->gen++;   // captured graphs carry the old limit
    c->oz_wait = cycles;
    c->oz_sch.wait = cycles;
    return EXS_OK;
}

int exs_set_stream(exs_ctx *c, void *stream)
{
    if (!c) return EXS_ERR_ARG;
    cudaSetDevice(c->device);
    EXS_CUDA(cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return EXS_OK;
}

int exs_last_timings(exs_ctx *c, double *t, int n)
{
    if (!c || !t) return EXS_ERR_ARG;
    for (int i = 0; i < n && i < 5; i++) t[i] = c->last_t[i];
    if (n > 5) t[5] = exs::rt_combine_ms(c);
    return EXS_OK;
}

int exs_match(exs_ctx *c, int ngp, const double *gpc, const double *tpgpc, const exs_complex *sfacgp,
              exs_complex *apwalm)
{
    if (!c || !gpc || !tpgpc || !sfacgp || !apwalm) return fail(c, EXS_ERR_ARG, "exs_match: null argument");
    if (ngp < 0 || ngp > c->ngkmax) return fail(c, EXS_ERR_SIZE, "exs_match: ngp outside 0..ngkmax");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const int lmmax = (c->lmaxapw + 1) * (c->lmaxapw + 1);
    const size_t nalm = (size_t)c->ngkmax * c->apwordmax * lmmax * c->natmtot;
    if (!c->d_apwalm) {
        EXS_CUDA(dalloc(&c->d_apwalm, nalm));
        EXS_CUDA(dalloc(&c->d_match_in, 3 * (size_t)c->ngkmax));
        EXS_CUDA(dalloc(&c->d_match_sf, (size_t)c->ngkmax * c->natmtot));
    }
    if (ngp == 0) return EXS_OK;
    EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
    EXS_CUDA(cudaMemcpyAsync(c->d_match_in, gpc, sizeof(double) * ngp, cudaMemcpyHostToDevice, s));
    EXS_CUDA(cudaMemcpyAsync(c->d_match_in + c->ngkmax, tpgpc, sizeof(double) * 2 * ngp, cudaMemcpyHostToDevice, s));
    EXS_CUDA(cudaMemcpy2DAsync(c->d_match_sf, sizeof(exs_complex) * c->ngkmax, sfacgp, sizeof(exs_complex) * c->ngkmax,
                               sizeof(exs_complex) * ngp, c->natmtot, cudaMemcpyHostToDevice, s));
    (void)cudaGetLastError();
    EXS_CUDA(cudaEventRecord(c->ev[0], s));
    EXS_CUDA(exs::launch_match_ref(c->params(), ngp, c->ngkmax, c->d_match_in, c->d_match_in + c->ngkmax,
                                   c->d_match_sf, c->d_apwalm, s));
    for (int i = 1; i <= 4; i++) EXS_CUDA(cudaEventRecord(c->ev[i], s));
    c->timed = true;
    // only the first ngp rows of each column are defined by match
    EXS_CUDA(cudaMemcpy2DAsync(apwalm, sizeof(exs_complex) * c->ngkmax, c->d_apwalm, sizeof(exs_complex) * c->ngkmax,
                               sizeof(exs_complex) * ngp, nalm / c->ngkmax, cudaMemcpyDeviceToHost, s));
    return exs_synchronize(c);
}

}  // extern "C"

// ---------------------------------------------------------------- setup pipeline
namespace {

// Pack the k descriptors and the grouped-GEMM tables into the pinned staging
// buffer, upload them with one copy and return the device addresses.
struct Uploaded {
    const KDesc *d_k;
    const void *d_probs[4];
    const void *d_work[4];
    int nwork[4];
    const void *d_oztiles;
    int noztiles;
    const void *d_ozatiles;   // per-atom tiles of the split-precision path
    int nozatiles;
};

// Upper tiles (128 rows x 32 columns, 256 x 32 for the two-SM tiles with ib
// counting pairs of 128-row blocks, 128 x 32, 128 x 64 or 256 x 64 for the
// residue tiles of the modular mode) of the split-precision contraction, in
// groups of `group` row blocks x `gcols` column blocks (gcols 0: `group`;
// row blocks outer, then column blocks, inside a group row blocks outer
// again): the tiles that run at the same time (one
// CTA per SM) then read about `group` row blocks of A and `group` column
// blocks of B instead of one row block and ~148 column blocks, so the L2
// serves the shared operand chunks and HBM streams each block about
// (number of groups in its row or column) times instead of once per tile
// row.  group = 1 is the plain row-major order.
void oz_tiles(const std::vector<KDesc> &ks, std::vector<int> &t, int rows, int cols, int group = 1, int gcols = 0)
{
    t.clear();
    if (gcols <= 0) gcols = group;
    for (size_t k = 0; k < ks.size(); k++) {
        const int n = ks[k].ngp;
        const int nib = (n + rows - 1) / rows, njb = (n + cols - 1) / cols;
        for (int gi = 0; gi < nib; gi += group)
            for (int gj = 0; gj < njb; gj += gcols)
                for (int ib = gi; ib < std::min(nib, gi + group); ib++)
                    for (int jb = gj; jb < std::min(njb, gj + gcols); jb++)
                        if (jb * cols + cols - 1 >= ib * rows) {
                            t.push_back((int)k);
                            t.push_back(ib);
                            t.push_back(jb);
                        }
    }
}

// Per-atom tiles {k, atom, G block of 128, row block of 64} of the
// split-precision path: h_a A (row blocks 0..nfb-1) and the APW-lo rows
// (blocks nfb..).
void oz_atom_tiles(const exs_ctx *c, const std::vector<KDesc> &ks, std::vector<int> &t)
{
    for (size_t k = 0; k < ks.size(); k++)
        for (int ias = 0; ias < c->natmtot; ias++) {
            const AtomDesc &a = c->atoms[ias];
            for (int ib = 0; ib < (ks[k].ngp + 127) / 128; ib++) {
                for (int xb = 0; xb < (a.napw + 63) / 64; xb++) {
                    t.push_back((int)k); t.push_back(ias); t.push_back(ib); t.push_back(xb);
                }
                for (int lb = 0; lb < (a.losize + 63) / 64; lb++) {
                    t.push_back((int)k); t.push_back(ias); t.push_back(ib); t.push_back(c->oz_nfb + lb);
                }
            }
        }
}

// Layout of the packed tables (byte offsets from the start of the buffer).
struct TableLayout {
    size_t k, probs[4], work[4], oz, oza, total;
    int nwork[4], noz, noza;
};

void pack_tables(exs_ctx *c, const std::vector<KDesc> &ks, std::vector<int> &ozt, TableLayout &L)
{
    exs::build_gemm_tables(c, ks, c->gt);
    ozt.clear();
    std::vector<int> ozat;
    if (c->oz_on()) {
        if (c->oz_sch.mod && (c->oz_cfg & 8)) {   // 256-row pairs, grouped 6 x 12, as two 128-row tiles each
            std::vector<int> pairs;
            oz_tiles(ks, pairs, 256, 64, 6, 12);
            for (size_t t = 0; t < pairs.size(); t += 3)
                for (int r = 0; r < 2; r++) {
                    ozt.push_back(pairs[t]);
                    ozt.push_back(2 * pairs[t + 1] + r);
                    ozt.push_back(pairs[t + 2]);
                }
        } else if (c->oz_sch.mod)   // grouped 12 x 12 (about one wave of 148 CTAs)
            oz_tiles(ks, ozt, 128, exs::oz_res_cols(c->oz_cfg), 12);
        else
            oz_tiles(ks, ozt, (c->oz_cfg & 8) ? 256 : 128, 32);
        oz_atom_tiles(c, ks, ozat);
    }
    L.noz = (int)(ozt.size() / 3);
    L.noza = (int)(ozat.size() / 4);
    ozt.insert(ozt.end(), ozat.begin(), ozat.end());   // HO tiles, then the per-atom tiles
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t off = 0;
    L.k = off;
    off += al(ks.size() * sizeof(KDesc));
    for (int q = 0; q < 4; q++) {
        L.probs[q] = off;
        off += al(c->gt.probs[q].size() * sizeof(exs::GemmProb));
        L.work[q] = off;
        off += al(c->gt.work[q].size() * sizeof(exs::TileWork));
        L.nwork[q] = (int)c->gt.work[q].size();
    }
    L.oz = off;
    L.oza = off + sizeof(int) * 3 * (size_t)L.noz;
    off += al(ozt.size() * sizeof(int));
    L.total = off;
}

void write_tables(const exs_ctx *c, const std::vector<KDesc> &ks, const std::vector<int> &ozt, const TableLayout &L,
                  char *h)
{
    std::memcpy(h + L.k, ks.data(), ks.size() * sizeof(KDesc));
    for (int q = 0; q < 4; q++) {
        if (!c->gt.probs[q].empty())
            std::memcpy(h + L.probs[q], c->gt.probs[q].data(), c->gt.probs[q].size() * sizeof(exs::GemmProb));
        if (!c->gt.work[q].empty())
            std::memcpy(h + L.work[q], c->gt.work[q].data(), c->gt.work[q].size() * sizeof(exs::TileWork));
    }
    if (!ozt.empty()) std::memcpy(h + L.oz, ozt.data(), ozt.size() * sizeof(int));
}

Uploaded device_view(const TableLayout &L, char *d)
{
    Uploaded u{};
    u.d_k = (const KDesc *)(d + L.k);
    for (int q = 0; q < 4; q++) {
        u.d_probs[q] = d + L.probs[q];
        u.d_work[q] = d + L.work[q];
        u.nwork[q] = L.nwork[q];
    }
    u.d_oztiles = d + L.oz;
    u.noztiles = L.noz;
    u.d_ozatiles = d + L.oza;
    u.nozatiles = L.noza;
    return u;
}

int upload_tables(exs_ctx *c, const std::vector<KDesc> &ks, Uploaded &u)
{
    std::vector<int> ozt;
    TableLayout L;
    pack_tables(c, ks, ozt, L);
    // the previous upload must have left the staging buffer
    EXS_CUDA(cudaEventSynchronize(c->tables_free));
    if (L.total > c->tables_bytes) {
        if (c->h_tables) cudaFreeHost(c->h_tables);
        if (c->d_tables) cudaFree(c->d_tables);
        c->h_tables = c->d_tables = nullptr;
        c->tables_bytes = 0;
        const size_t cap = L.total * 2;
        EXS_CUDA(cudaMallocHost(&c->h_tables, cap));
        EXS_CUDA(cudaMalloc(&c->d_tables, cap));
        c->tables_bytes = cap;
    }
    write_tables(c, ks, ozt, L, (char *)c->h_tables);
    u = device_view(L, (char *)c->d_tables);
    EXS_CUDA(cudaMemcpyAsync(c->d_tables, c->h_tables, L.total, cudaMemcpyHostToDevice, c->stream));
    EXS_CUDA(cudaEventRecord(c->tables_free, c->stream));
    return EXS_OK;
}

// Only the k descriptors, through the same staging buffer as upload_tables.
int upload_kdesc(exs_ctx *c, const std::vector<KDesc> &ks, Uploaded &u)
{
    const size_t need = ks.size() * sizeof(KDesc);
    EXS_CUDA(cudaEventSynchronize(c->tables_free));
    if (need > c->tables_bytes) {
        if (c->h_tables) cudaFreeHost(c->h_tables);
        if (c->d_tables) cudaFree(c->d_tables);
        c->h_tables = c->d_tables = nullptr;
        c->tables_bytes = 0;
        EXS_CUDA(cudaMallocHost(&c->h_tables, need * 2));
        EXS_CUDA(cudaMalloc(&c->d_tables, need * 2));
        c->tables_bytes = need * 2;
    }
    std::memcpy(c->h_tables, ks.data(), need);
    u = Uploaded{};
    u.d_k = (const KDesc *)c->d_tables;
    EXS_CUDA(cudaMemcpyAsync(c->d_tables, c->h_tables, need, cudaMemcpyHostToDevice, c->stream));
    EXS_CUDA(cudaEventRecord(c->tables_free, c->stream));
    return EXS_OK;
}

// Zero the column maxima that the A and B producers raise (split-precision
// path only; the slots of one call are contiguous).
cudaError_t oz_reset_maxima(exs_ctx *c, const std::vector<KDesc> &ks, cudaStream_t s)
{
    if (!c->oz_on() || ks.empty()) return cudaSuccess;
    double *lo = ks[0].oz_scale, *hi = ks[0].oz_scale;
    for (const KDesc &k : ks) {
        lo = std::min(lo, k.oz_scale);
        hi = std::max(hi, k.oz_scale);
    }
    return cudaMemsetAsync(lo, 0, sizeof(double) * ((size_t)(hi - lo) + 3 * (size_t)c->npad), s);
}

// Enqueue the whole setup for the k descriptors in ks (device arrays filled)
// with the tables already on the device (u).  If have_planes, the A planes
// are already in place (apwalm given).  With timed, the phase events
// ev[0..4] are recorded (not while a graph is being captured).
int enqueue_setup(exs_ctx *c, const std::vector<KDesc> &ks, const Uploaded &u, bool have_planes, bool timed)
{
    cudaStream_t s = c->stream;
    const DevParams p = c->params();
    int ngp_max = 0;
    for (auto &k : ks) ngp_max = std::max(ngp_max, k.ngp);
#define EXS_EV(i) \
    if (timed) EXS_CUDA(cudaEventRecord(c->ev[i], s))
    EXS_EV(0);
    if (!have_planes) EXS_CUDA(oz_reset_maxima(c, ks, s));
    if (!have_planes) EXS_CUDA(exs::launch_match_planes(p, u.d_k, (int)ks.size(), ngp_max, s));
    if (c->relativity == EXS_REL_IORA) EXS_CUDA(exs::launch_iora_planes(p, u.d_k, (int)ks.size(), ngp_max, s));
    EXS_EV(1);
    const bool oz = c->oz_on();
    if (oz && c->relativity == EXS_REL_IORA) {
        // C = (I + h1aa) A, the right operand of O: its column bound (maximum or 2-norm), then its slices
        EXS_CUDA(exs::launch_oz_colnorm(p, u.d_k, (int)ks.size(), 2, c->oz_sch.mod, s));
        EXS_CUDA(exs::launch_oz_split(p, u.d_k, (int)ks.size(), c->oz_sch, c->kp8, 2, s));
    }
    // configuration bit 4: B = h_a A and the APW-lo rows in native FP64 even
    // when the H/O contraction is split
    const bool b64 = !oz || (c->oz_cfg & 16);
    // moduli: the columns are scaled by their 2-norms (over the maxima the producers raised)
    const bool norms = oz && c->oz_sch.mod;
    if (oz) {
        // slices of A; B = h_a A and the APW-lo rows of H from the slices of h_a and loa
        if (norms) EXS_CUDA(exs::launch_oz_colnorm(p, u.d_k, (int)ks.size(), 0, 1, s));
        EXS_CUDA(exs::launch_oz_split(p, u.d_k, (int)ks.size(), c->oz_sch, c->kp8, 0, s));
        if (!b64)
            EXS_CUDA(exs::launch_oz_atom(c->oz_cfg, &c->oz_mapArow, &c->oz_mapX, p, u.d_k, u.d_ozatiles,
                                         u.nozatiles, c->oz_sch, c->kp8, c->oz_atom_args(), s));
    }
    if (b64) {
        EXS_CUDA(exs::launch_gemm_kind(exs::EPI_PLANAR, p, u.d_probs[exs::EPI_PLANAR], u.d_work[exs::EPI_PLANAR],
                                       u.nwork[exs::EPI_PLANAR], u.d_k, s));
    }
    EXS_EV(2);
    if (oz) {
        if (norms) EXS_CUDA(exs::launch_oz_colnorm(p, u.d_k, (int)ks.size(), 1, 1, s));
        EXS_CUDA(exs::launch_oz_split(p, u.d_k, (int)ks.size(), c->oz_sch, c->kp8, 1, s));
        const int q = c->oz_cfg;
        if (c->oz_sch.mod)   // residue tiles (one K chunk per stage: the maps of configuration 1), then the CRT
            EXS_CUDA(exs::launch_oz_res(q, &c->oz_mapA[1], &c->oz_mapB[1], &c->oz_mapB64, &c->oz_mapB64h, p, u.d_k,
                                        u.d_oztiles, u.noztiles, c->oz_sch, c->kp8, c->d_res, c->d_pace, s));
        else
            EXS_CUDA(exs::launch_oz_mma(q, &c->oz_mapA[q], (q & 8) ? &c->oz_mapB2[q] : &c->oz_mapB[q], p, u.d_k,
                                        u.d_oztiles, u.noztiles, c->oz_sch, c->kp8, s));
    } else {
        EXS_CUDA(exs::launch_gemm_kind(exs::EPI_HAM, p, u.d_probs[exs::EPI_HAM], u.d_work[exs::EPI_HAM],
                                       u.nwork[exs::EPI_HAM], u.d_k, s));
        EXS_CUDA(exs::launch_gemm_kind(exs::EPI_OVL, p, u.d_probs[exs::EPI_OVL], u.d_work[exs::EPI_OVL],
                                       u.nwork[exs::EPI_OVL], u.d_k, s));
    }
    EXS_EV(3);
    if (b64)
        EXS_CUDA(exs::launch_gemm_kind(exs::EPI_LOROWS, p, u.d_probs[exs::EPI_LOROWS], u.d_work[exs::EPI_LOROWS],
                                       u.nwork[exs::EPI_LOROWS], u.d_k, s));
    EXS_CUDA(exs::launch_olp_apwlo(p, u.d_k, (int)ks.size(), ngp_max, s));
    EXS_CUDA(exs::launch_lolo_blocks(p, u.d_k, (int)ks.size(), s));
    EXS_EV(4);
#undef EXS_EV
    if (timed) c->timed = true;
    return EXS_OK;
}

int run_setup(exs_ctx *c, std::vector<KDesc> &ks, bool have_planes)
{
    (void)cudaGetLastError();   // launch checks below read the last error: start clean
    Uploaded u{};
    int rc = upload_tables(c, ks, u);
    if (rc != EXS_OK) return rc;
    return enqueue_setup(c, ks, u, have_planes, true);
}

KDesc slot_desc(exs_ctx *c, int slot, int ngp, const int *d_igpig, const double *d_vgpc, exs_complex *h, exs_complex *o)
{
    KDesc k{};
    k.ngp = ngp;
    k.nmat = ngp + c->nlotot;
    k.igpig = d_igpig;
    k.vgpc = d_vgpc;
    k.h = h;
    k.o = o;
    double *w = c->d_work + (size_t)slot * c->nplanes * c->plane;
    k.ar = w;
    k.ai = w + c->plane;
    k.br = w + 2 * c->plane;
    k.bi = w + 3 * c->plane;
    if (c->relativity == EXS_REL_IORA) {
        k.cr = w + 4 * c->plane;
        k.ci = w + 5 * c->plane;
    } else {
        k.cr = k.ar;
        k.ci = k.ai;
    }
    k.oz_slices = c->d_oz ? c->d_oz + (size_t)slot * c->oz_slot_bytes : nullptr;
    const bool oz = c->oz_on() && c->d_ozscale;
    k.oz_scale = oz ? c->d_ozscale + (size_t)slot * 3 * c->npad : nullptr;
    k.oz_slot = slot;
    return k;
}

// Checks and k descriptors of the device-pointer entry points.
int device_batch(exs_ctx *c, int nk, const int *ngp, const int *igpig_dev, const double *vgpc_dev,
                 exs_complex *const *h_dev, exs_complex *const *o_dev, std::vector<KDesc> &ks)
{
    if (!c || nk < 0 || (nk > 0 && (!ngp || !igpig_dev || !vgpc_dev || !h_dev || !o_dev)))
        return fail(c, EXS_ERR_ARG, "bad argument");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    if (nk > c->max_batch) return fail(c, EXS_ERR_SIZE, "nk exceeds max_batch");
    for (int k = 0; k < nk; k++)
        if (ngp[k] <= 0 || ngp[k] > c->ngkmax || !h_dev[k] || !o_dev[k])
            return fail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax or null output");
    ks.clear();
    for (int k = 0; k < nk; k++)
        ks.push_back(slot_desc(c, k, ngp[k], igpig_dev + (size_t)c->ngkmax * k, vgpc_dev + 3 * (size_t)c->ngkmax * k,
                               h_dev[k], o_dev[k]));
    return EXS_OK;
}

}  // namespace

struct exs_graph {
    std::vector<exs_ctx *> cs;        // cs[0]'s stream is the one the graph is launched on
    std::vector<unsigned> gens;
    std::vector<void *> tables;       // per context, owned by the graph
    std::vector<cudaStream_t> branches;
    std::vector<cudaEvent_t> events;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" {

int exs_autotune(exs_ctx *c, int nk, const int *ngp, const int *igpig_dev, const double *vgpc_dev,
                 exs_complex *const *h_dev, exs_complex *const *o_dev, int *choice)
{
    std::vector<KDesc> ks;
    int rc = device_batch(c, nk, ngp, igpig_dev, vgpc_dev, h_dev, o_dev, ks);
    if (rc != EXS_OK) return rc;
    if (choice) *choice = 0;
    if (nk == 0) return EXS_OK;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    if (!c->oz_on()) {   // one configuration only: just run it
        EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
        rc = run_setup(c, ks, false);
        return rc < 0 ? rc : exs_synchronize(c);
    }
    (void)cudaGetLastError();
    constexpr int REPS = 3;
    float best = 0.f;
    int best_q = 0;
    for (int q = 0; q < exs::OZ_NCFG; q++) {
        if ((q & 8) && (q & 2) && !c->oz_sch.mod) continue;   // the slices' two-SM tiles have no persistent form
        if ((q & 8) && c->oz_sch.mod && (q & 1)) continue;   // moduli: the two-SM residue tiles are 64 wide
        if ((q & 16) && (q & 4)) continue;  // no per-atom int8 kernel to make persistent
        c->oz_cfg = q;
        Uploaded u{};                        // the tile list depends on the configuration
        rc = upload_tables(c, ks, u);
        if (rc != EXS_OK) return rc;
        EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
        rc = enqueue_setup(c, ks, u, false, false);      // warm-up
        if (rc < 0) return rc;
        EXS_CUDA(cudaEventRecord(c->ev[5], s));
        for (int r = 0; r < REPS; r++) {
            rc = enqueue_setup(c, ks, u, false, false);
            if (rc < 0) return rc;
        }
        EXS_CUDA(cudaEventRecord(c->ev[6], s));
        rc = exs_synchronize(c);
        if (rc < 0) return rc;
        float ms = 0.f;
        EXS_CUDA(cudaEventElapsedTime(&ms, c->ev[5], c->ev[6]));
        if (q == 0 || ms < best) {
            best = ms;
            best_q = q;
        }
    }
    c->oz_cfg = best_q;
    c->oz_tuned[std::make_tuple((int)c->prec_mode, c->npad, c->K, c->slices)] = best_q;
    if (choice) *choice = best_q;
    // the outputs hold the last configuration's results: leave the chosen one's
    EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
    rc = run_setup(c, ks, false);
    return rc < 0 ? rc : exs_synchronize(c);
}

int exs_set_kernel_config(exs_ctx *c, int cfg)
{
    if (!c) return EXS_ERR_ARG;
    if (cfg < 0 || cfg >= exs::OZ_NCFG) return fail(c, EXS_ERR_ARG, "kernel configuration out of range");
    c->oz_cfg = cfg;
    return EXS_OK;
}

}  // extern "C"

namespace {

void graph_free(exs_graph *G)
{
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    for (void *t : G->tables)
        if (t) cudaFree(t);
    for (cudaStream_t b : G->branches) cudaStreamDestroy(b);
    for (cudaEvent_t e : G->events) cudaEventDestroy(e);
    delete G;
}

// Capture the batched setups of one or more contexts into one graph.  With
// several contexts each one's launches go to one of up to 32 branch streams
// forked from the first context's stream, so independent cells run
// concurrently when the graph is replayed.
int graph_capture(const std::vector<exs_ctx *> &cs, std::vector<std::vector<KDesc>> &kss, exs_graph **out)
{
    exs_ctx *c0 = cs[0];
    exs_graph *G = new exs_graph;
    G->cs = cs;
    auto bail = [&](int code) {
        graph_free(G);
        return code;
    };
    std::vector<Uploaded> us(cs.size());
    for (size_t i = 0; i < cs.size(); i++) {   // tables owned by the graph, then one plain run
        exs_ctx *c = cs[i];
        G->gens.push_back(c->gen);
        std::vector<int> ozt;
        TableLayout L;
        pack_tables(c, kss[i], ozt, L);
        std::vector<char> h(L.total);
        write_tables(c, kss[i], ozt, L, h.data());
        void *d = nullptr;
        if (cudaMalloc(&d, L.total) != cudaSuccess) return bail(fail(c, EXS_ERR_NOMEM, "graph tables"));
        G->tables.push_back(d);
        if (cudaMemcpy(d, h.data(), L.total, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(fail(c, EXS_ERR_CUDA, "graph tables upload"));
        us[i] = device_view(L, (char *)d);
        // kernel attributes are set on first launch, outside any capture
        if (cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream) != cudaSuccess)
            return bail(fail(c, EXS_ERR_CUDA, "memset"));
        int rc = enqueue_setup(c, kss[i], us[i], false, false);
        if (rc < 0) return bail(rc);
        rc = exs_synchronize(c);
        if (rc < 0) return bail(rc);
    }
    const int nb = cs.size() > 1 ? (int)std::min<size_t>(cs.size(), 32) : 0;
    for (int b = 0; b < nb; b++) {
        cudaStream_t st;
        cudaEvent_t ev;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(c0, EXS_ERR_CUDA, "branch stream"));
        G->branches.push_back(st);
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(c0, EXS_ERR_CUDA, "branch event"));
        G->events.push_back(ev);
    }
    cudaEvent_t fork = nullptr;
    if (nb > 0) {
        if (cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(c0, EXS_ERR_CUDA, "fork event"));
        G->events.push_back(fork);
    }
    cudaStream_t origin = c0->stream;
    if (cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return bail(fail(c0, EXS_ERR_CUDA, "cudaStreamBeginCapture"));
    int rc = EXS_OK;
    if (nb > 0 && cudaEventRecord(fork, origin) != cudaSuccess) rc = EXS_ERR_CUDA;
    for (int b = 0; b < nb && rc == EXS_OK; b++)
        if (cudaStreamWaitEvent(G->branches[b], fork, 0) != cudaSuccess) rc = EXS_ERR_CUDA;
    for (size_t i = 0; i < cs.size() && rc == EXS_OK; i++) {
        exs_ctx *c = cs[i];
        cudaStream_t own = c->stream;
        if (nb > 0) c->stream = G->branches[i % nb];
        if (cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream) != cudaSuccess) rc = EXS_ERR_CUDA;
        if (rc == EXS_OK) rc = enqueue_setup(c, kss[i], us[i], false, false);
        c->stream = own;
    }
    for (int b = 0; b < nb && rc == EXS_OK; b++)
        if (cudaEventRecord(G->events[b], G->branches[b]) != cudaSuccess ||
            cudaStreamWaitEvent(origin, G->events[b], 0) != cudaSuccess)
            rc = EXS_ERR_CUDA;
    cudaError_t ee = cudaStreamEndCapture(origin, &G->graph);
    if (rc < 0 || ee != cudaSuccess) return bail(rc < 0 ? rc : fail(c0, EXS_ERR_CUDA, "cudaStreamEndCapture"));
    if (cudaGraphInstantiate(&G->exec, G->graph, 0) != cudaSuccess)
        return bail(fail(c0, EXS_ERR_CUDA, "cudaGraphInstantiate"));
    *out = G;
    return EXS_OK;
}

}  // namespace

extern "C" {

int exs_graph_create(exs_ctx *c, int nk, const int *ngp, const int *igpig_dev, const double *vgpc_dev,
                     exs_complex *const *h_dev, exs_complex *const *o_dev, exs_graph **out)
{
    if (!out) return fail(c, EXS_ERR_ARG, "exs_graph_create: null output");
    *out = nullptr;
    std::vector<std::vector<KDesc>> kss(1);
    int rc = device_batch(c, nk, ngp, igpig_dev, vgpc_dev, h_dev, o_dev, kss[0]);
    if (rc != EXS_OK) return rc;
    if (nk == 0) return fail(c, EXS_ERR_SIZE, "exs_graph_create: empty batch");
    cudaSetDevice(c->device);
    (void)cudaGetLastError();
    return graph_capture({c}, kss, out);
}

int exs_graph_create_multi(int nctx, exs_ctx *const *ctx, const int *nk, const int *const *ngp,
                           const int *const *igpig_dev, const double *const *vgpc_dev,
                           exs_complex *const *const *h_dev, exs_complex *const *const *o_dev, exs_graph **out)
{
    if (!out || nctx <= 0 || !ctx || !nk || !ngp || !igpig_dev || !vgpc_dev || !h_dev || !o_dev)
        return EXS_ERR_ARG;
    *out = nullptr;
    std::vector<exs_ctx *> cs(ctx, ctx + nctx);
    std::vector<std::vector<KDesc>> kss(nctx);
    for (int i = 0; i < nctx; i++) {
        if (!cs[i] || cs[i]->device != cs[0]->device) return EXS_ERR_ARG;
        int rc = device_batch(cs[i], nk[i], ngp[i], igpig_dev[i], vgpc_dev[i], h_dev[i], o_dev[i], kss[i]);
        if (rc != EXS_OK) return rc;
        if (nk[i] == 0) return fail(cs[i], EXS_ERR_SIZE, "exs_graph_create_multi: empty batch");
    }
    cudaSetDevice(cs[0]->device);
    (void)cudaGetLastError();
    return graph_capture(cs, kss, out);
}

int exs_graph_launch(exs_graph *G)
{
    if (!G) return EXS_ERR_ARG;
    for (size_t i = 0; i < G->cs.size(); i++)
        if (G->gens[i] != G->cs[i]->gen)
            return fail(G->cs[i], EXS_ERR_STATE, "graph captured before the last exs_set_precision");
    exs_ctx *c = G->cs[0];
    cudaSetDevice(c->device);
    EXS_CUDA(cudaGraphLaunch(G->exec, c->stream));
    for (exs_ctx *x : G->cs) x->timed = false;
    return EXS_OK;
}

int exs_graph_synchronize(exs_graph *G)
{
    if (!G) return EXS_ERR_ARG;
    int worst = EXS_OK;
    for (exs_ctx *c : G->cs) {   // the first waits for the graph; each reports its own device flags
        const int rc = exs_synchronize(c);
        if (rc < 0) return rc;
        if (rc > worst) worst = rc;
    }
    return worst;
}

void exs_graph_destroy(exs_graph *G)
{
    if (!G) return;
    cudaSetDevice(G->cs[0]->device);
    graph_free(G);
}

int exs_interstitial_batched_device(exs_ctx *c, int which, int nk, const int *ngp, const int *igpig_dev,
                                    const double *vgpc_dev, exs_complex *const *h_dev, exs_complex *const *o_dev,
                                    const int *ld)
{
    if (!c || which < 1 || which > 3 || nk < 0 || (nk > 0 && (!ngp || !igpig_dev || !vgpc_dev || !ld)) ||
        ((which & 1) && nk > 0 && !h_dev) || ((which & 2) && nk > 0 && !o_dev))
        return fail(c, EXS_ERR_ARG, "exs_interstitial_batched_device: bad argument");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    std::vector<KDesc> ks(nk);
    int ngp_max = 0;
    for (int k = 0; k < nk; k++) {
        if (ngp[k] <= 0 || ngp[k] > c->ngkmax || ld[k] < ngp[k] || ((which & 1) && !h_dev[k]) ||
            ((which & 2) && !o_dev[k]))
            return fail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax, ld < ngp or null matrix");
        KDesc &d = ks[k];
        d = KDesc{};
        d.ngp = ngp[k];
        d.nmat = ld[k];
        d.igpig = igpig_dev + (size_t)c->ngkmax * k;
        d.vgpc = vgpc_dev + 3 * (size_t)c->ngkmax * k;
        d.h = (which & 1) ? h_dev[k] : nullptr;
        d.o = (which & 2) ? o_dev[k] : nullptr;
        ngp_max = std::max(ngp_max, ngp[k]);
    }
    if (nk == 0) return EXS_OK;
    cudaSetDevice(c->device);
    (void)cudaGetLastError();
    // the descriptors travel through the context's table buffer (same staging rules as the setup)
    Uploaded u{};
    int rc = upload_kdesc(c, ks, u);
    if (rc != EXS_OK) return rc;
    EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    EXS_CUDA(exs::launch_interstitial(c->params(), which, u.d_k, nk, ngp_max, c->stream));
    c->timed = false;
    return EXS_OK;
}

int exs_interstitial_device(exs_ctx *c, int which, int ngp, const int *igpig_dev, const double *vgpc_dev,
                            exs_complex *h_dev, exs_complex *o_dev, int ld)
{
    exs_complex *hh[1] = {h_dev}, *oo[1] = {o_dev};
    return exs_interstitial_batched_device(c, which, 1, &ngp, igpig_dev, vgpc_dev, hh, oo, &ld);
}

}  // extern "C"

namespace {

// Host-array form: za(1:ngp, 1:ngp) (leading dimension ld) through the
// context's H/O buffer of slot 0.
int host_interstitial(exs_ctx *c, int which, int ngp, const int *igpig, const double *vgpc, exs_complex *z, int ld)
{
    if (!c || !igpig || !vgpc || !z) return fail(c, EXS_ERR_ARG, "hmlistln/olpistln: null argument");
    if (ngp <= 0 || ngp > c->ngkmax || ld < ngp || ld > c->nmatmax)
        return fail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax or ld outside ngp..nmatmax");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    for (int i = 0; i < ngp; i++)
        if (igpig[i] < 1 || igpig[i] > c->ngrtot) return fail(c, EXS_ERR_INDEX, "igpig entry outside 1..ngrtot");
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    EXS_CUDA(cudaStreamSynchronize(s));
    const size_t bytes = sizeof(exs_complex) * (size_t)ld * ngp;
    EXS_CUDA(cudaMemcpyAsync(c->d_igpig, igpig, sizeof(int) * ngp, cudaMemcpyHostToDevice, s));
    EXS_CUDA(cudaMemcpyAsync(c->d_vgpc, vgpc, sizeof(double) * 3 * ngp, cudaMemcpyHostToDevice, s));
    EXS_CUDA(cudaMemcpyAsync(c->d_ho, z, bytes, cudaMemcpyHostToDevice, s));
    int rc = exs_interstitial_device(c, which, ngp, c->d_igpig, c->d_vgpc, which == 1 ? c->d_ho : nullptr,
                                     which == 2 ? c->d_ho : nullptr, ld);
    if (rc < 0) return rc;
    EXS_CUDA(cudaMemcpyAsync(z, c->d_ho, bytes, cudaMemcpyDeviceToHost, s));
    return exs_synchronize(c);
}

}  // namespace

extern "C" {

int exs_hmlistln(exs_ctx *c, int ngp, const int *igpig, const double *vgpc, exs_complex *h, int ld)
{
    return host_interstitial(c, 1, ngp, igpig, vgpc, h, ld);
}

int exs_olpistln(exs_ctx *c, int ngp, const int *igpig, const double *vgpc, exs_complex *o, int ld)
{
    return host_interstitial(c, 2, ngp, igpig, vgpc, o, ld);
}

int exs_setup_batched_device(exs_ctx *c, int nk, const int *ngp, const int *igpig_dev, const double *vgpc_dev,
                             exs_complex *const *h_dev, exs_complex *const *o_dev)
{
    std::vector<KDesc> ks;
    int rc = device_batch(c, nk, ngp, igpig_dev, vgpc_dev, h_dev, o_dev, ks);
    if (rc != EXS_OK) return rc;
    cudaSetDevice(c->device);
    EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    if (nk == 0) return EXS_OK;
    return run_setup(c, ks, false);
}

int exs_set_host_copy_mode(exs_ctx *c, int mode)
{
    if (!c) return EXS_ERR_ARG;
    if (mode < EXS_COPY_AUTO || mode > EXS_COPY_UPPER) return fail(c, EXS_ERR_ARG, "unknown host copy mode");
    c->host_copy_mode = mode;
    return EXS_OK;
}

}  // extern "C"

namespace {

// One matrix of a packed transfer: the upper triangle (i <= j) of the
// column-major n x n matrix src, column after column, at element offset off.
struct PackDesc {
    const exs_complex *src;
    long n;
    size_t off;
};

__global__ void pack_upper_kernel(const PackDesc *pd, exs_complex *out)
{
    const PackDesc d = pd[blockIdx.y];
    for (long j = blockIdx.x; j < d.n; j += gridDim.x) {
        exs_complex *o = out + d.off + (size_t)j * (j + 1) / 2;
        const exs_complex *z = d.src + (size_t)d.n * j;
        for (long i = threadIdx.x; i <= j; i += blockDim.x) o[i] = z[i];
    }
}

// Full Hermitian z (n x n, column-major) from its packed upper triangle p,
// columns [c0, c1): the upper part is a copy per column, the lower part
// (rows r > c) the conjugate of p read row by row in 64-row blocks.
void unpack_columns(const exs_complex *p, exs_complex *z, long n, long c0, long c1)
{
    for (long j = c0; j < c1; j++) std::memcpy(z + n * j, p + (size_t)j * (j + 1) / 2, sizeof(exs_complex) * (j + 1));
    for (long r0 = c0 + 1; r0 < n; r0 += 64) {
        const long r1 = std::min(n, r0 + 64);
        for (long r = r0; r < r1; r++) {
            const exs_complex *pr = p + (size_t)r * (r + 1) / 2;     // row r of the upper part: p[.. + c], c <= r
            const long ce = std::min(c1, r);
            for (long cc = c0; cc < ce; cc++) {
                exs_complex v = pr[cc];
                v.im = -v.im;
                z[r + n * cc] = v;
            }
        }
    }
}

// Rows c0+64 .. n-1 of columns c0 .. c0+63 of the Hermitian z (n x n,
// column-major) from its upper part: z(r, c) = conj(z(c, r)), in 64 x 64
// tiles (each source column segment z(c0 .. c0+63, r) is contiguous).
void fill_lower_block(exs_complex *z, long n, long c0)
{
    const long c1 = std::min(n, c0 + 64);
    for (long r0 = c0 + 64; r0 < n; r0 += 64) {
        const long r1 = std::min(n, r0 + 64);
        for (long c = c0; c < c1; c++) {
            exs_complex *dst = z + n * c;
            for (long r = r0; r < r1; r++) {
                exs_complex v = z[c + n * r];
                v.im = -v.im;
                dst[r] = v;
            }
        }
    }
}

bool host_pinned(const void *ptr)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Grow the two packed-transfer slots to hold `elems` elements and `ndesc`
// descriptors each.
int pack_reserve(exs_ctx *c, size_t elems, size_t ndesc)
{
    if (elems > c->pack_elems) {
        for (int q = 0; q < 2; q++) {
            if (c->d_pack[q]) cudaFree(c->d_pack[q]);
            if (c->h_pack[q]) cudaFreeHost(c->h_pack[q]);
            c->d_pack[q] = c->h_pack[q] = nullptr;
        }
        c->pack_elems = 0;
        for (int q = 0; q < 2; q++) {
            EXS_CUDA(cudaMalloc((void **)&c->d_pack[q], sizeof(exs_complex) * elems));
            EXS_CUDA(cudaMallocHost((void **)&c->h_pack[q], sizeof(exs_complex) * elems));
        }
        c->pack_elems = elems;
    }
    if (ndesc > c->packdesc_cap) {
        for (int q = 0; q < 2; q++) {
            if (c->d_packdesc[q]) cudaFree(c->d_packdesc[q]);
            if (c->h_packdesc[q]) cudaFreeHost(c->h_packdesc[q]);
            c->d_packdesc[q] = c->h_packdesc[q] = nullptr;
        }
        c->packdesc_cap = 0;
        for (int q = 0; q < 2; q++) {
            EXS_CUDA(cudaMalloc(&c->d_packdesc[q], sizeof(PackDesc) * ndesc));
            EXS_CUDA(cudaMallocHost(&c->h_packdesc[q], sizeof(PackDesc) * ndesc));
        }
        c->packdesc_cap = ndesc;
    }
    if (!c->pool) {
        const unsigned hc = std::thread::hardware_concurrency();
        c->pool = new exs::HostPool((int)std::max(1u, std::min(hc, 32u)) - 1);
    }
    return EXS_OK;
}

}  // namespace

extern "C" {

int exs_setup_batched(exs_ctx *c, int nk, const int *ngp, const int *igpig, const double *vgpc,
                      exs_complex *const *h, exs_complex *const *o)
{
    if (!c || nk < 0 || (nk > 0 && (!ngp || !igpig || !vgpc || !h || !o)))
        return fail(c, EXS_ERR_ARG, "exs_setup_batched: bad argument");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    for (int k = 0; k < nk; k++) {
        if (ngp[k] <= 0 || ngp[k] > c->ngkmax || !h[k] || !o[k])
            return fail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax or null output");
        for (int i = 0; i < ngp[k]; i++) {
            const int g = igpig[(size_t)c->ngkmax * k + i];
            if (g < 1 || g > c->ngrtot) return fail(c, EXS_ERR_INDEX, "igpig entry outside 1..ngrtot");
        }
    }
    cudaSetDevice(c->device);
    bool packed = c->host_copy_mode == EXS_COPY_PACKED;
    const bool upper = c->host_copy_mode == EXS_COPY_UPPER;
    if (c->host_copy_mode == EXS_COPY_AUTO) {
        packed = false;
        for (int k = 0; k < nk && !packed; k++) packed = !host_pinned(h[k]) || !host_pinned(o[k]);
    }
    cudaStream_t s = c->stream;
    int worst = EXS_OK;
    for (int k0 = 0; k0 < nk; k0 += c->max_batch) {
        const int nb = std::min(c->max_batch, nk - k0);
        EXS_CUDA(cudaStreamSynchronize(s));
        EXS_CUDA(cudaStreamSynchronize(c->copy_stream));
        std::memcpy(c->h_igpig_pinned, igpig + (size_t)c->ngkmax * k0, sizeof(int) * (size_t)c->ngkmax * nb);
        std::memcpy(c->h_vgpc_pinned, vgpc + 3 * (size_t)c->ngkmax * k0, sizeof(double) * 3 * (size_t)c->ngkmax * nb);
        EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
        EXS_CUDA(cudaMemcpyAsync(c->d_igpig, c->h_igpig_pinned, sizeof(int) * (size_t)c->ngkmax * nb,
                                 cudaMemcpyHostToDevice, s));
        EXS_CUDA(cudaMemcpyAsync(c->d_vgpc, c->h_vgpc_pinned, sizeof(double) * 3 * (size_t)c->ngkmax * nb,
                                 cudaMemcpyHostToDevice, s));
        std::vector<KDesc> all;
        for (int k = 0; k < nb; k++) {
            exs_complex *dh = c->d_ho + (size_t)2 * k * c->nmatmax * c->nmatmax;
            exs_complex *dob = dh + (size_t)c->nmatmax * c->nmatmax;
            all.push_back(slot_desc(c, k, ngp[k0 + k], c->d_igpig + (size_t)c->ngkmax * k,
                                    c->d_vgpc + 3 * (size_t)c->ngkmax * k, dh, dob));
        }
        // Groups of k-points: the device-to-host copies of group g run on the
        // copy stream while group g+1 is set up on the compute stream.
        const int ngroups = nb >= 8 ? 4 : (nb >= 2 ? 2 : 1);
        const int per = (nb + ngroups - 1) / ngroups;
        const int G = (nb + per - 1) / per;
        auto group = [&](int g) {
            const int a = g * per, e = std::min(nb, a + per);
            return std::vector<KDesc>(all.begin() + a, all.begin() + e);
        };
        if (upper && !c->pool) {
            const unsigned hc = std::thread::hardware_concurrency();
            c->pool = new exs::HostPool((int)std::max(1u, std::min(hc, 32u)) - 1);
        }
        if (packed) {   // room for the largest group (2 matrices per k)
            size_t need = 0;
            for (int g = 0; g < G; g++) {
                size_t el = 0;
                for (const KDesc &k : group(g)) el += 2 * ((size_t)k.nmat * (k.nmat + 1) / 2);
                need = std::max(need, el);
            }
            int rc = pack_reserve(c, need, 2 * (size_t)per);
            if (rc < 0) return rc;
        }
        // enqueue group g: its setup, and for the packed transfer its pack
        // kernel; then the event that the copy stream waits for
        auto enqueue = [&](int g) -> int {
            std::vector<KDesc> cur = group(g);
            int rc = run_setup(c, cur, false);
            if (rc < 0) return rc;
            if (packed) {
                PackDesc *pd = (PackDesc *)c->h_packdesc[g & 1];
                size_t off = 0;
                for (size_t q = 0; q < cur.size(); q++) {
                    const size_t t = (size_t)cur[q].nmat * (cur[q].nmat + 1) / 2;
                    pd[2 * q] = PackDesc{cur[q].h, cur[q].nmat, off};
                    pd[2 * q + 1] = PackDesc{cur[q].o, cur[q].nmat, off + t};
                    off += 2 * t;
                }
                EXS_CUDA(cudaMemcpyAsync(c->d_packdesc[g & 1], pd, sizeof(PackDesc) * 2 * cur.size(),
                                         cudaMemcpyHostToDevice, s));
                pack_upper_kernel<<<dim3(512, (unsigned)(2 * cur.size())), 256, 0, s>>>(
                    (const PackDesc *)c->d_packdesc[g & 1], c->d_pack[g & 1]);
                EXS_CUDA(cudaGetLastError());
            }
            EXS_CUDA(cudaEventRecord(c->ev_group[g & 1], s));
            return EXS_OK;
        };
        // the device-to-host copies of group g on the copy stream
        auto copy_out = [&](int g) -> int {
            std::vector<KDesc> cur = group(g);
            EXS_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_group[g & 1], 0));
            if (packed) {
                size_t el = 0;
                for (const KDesc &k : cur) el += 2 * ((size_t)k.nmat * (k.nmat + 1) / 2);
                EXS_CUDA(cudaMemcpyAsync(c->h_pack[g & 1], c->d_pack[g & 1], sizeof(exs_complex) * el,
                                         cudaMemcpyDeviceToHost, c->copy_stream));
            } else if (upper) {   // rows 0 .. j0+63 of each block of 64 columns
                for (size_t q = 0; q < cur.size(); q++) {
                    const int kk = k0 + g * per + (int)q;
                    const long n = cur[q].nmat;
                    const size_t pitch = sizeof(exs_complex) * n;
                    for (int w = 0; w < 2; w++) {
                        const exs_complex *src = w == 0 ? cur[q].h : cur[q].o;
                        exs_complex *dst = w == 0 ? h[kk] : o[kk];
                        for (long j0 = 0; j0 < n; j0 += 64) {
                            const long rows = std::min(n, j0 + 64), cols = std::min(n, j0 + 64) - j0;
                            EXS_CUDA(cudaMemcpy2DAsync(dst + n * j0, pitch, src + n * j0, pitch,
                                                       sizeof(exs_complex) * rows, cols, cudaMemcpyDeviceToHost,
                                                       c->copy_stream));
                        }
                    }
                }
            } else {
                // H on one copy stream, O on a second one (two copy engines)
                EXS_CUDA(cudaStreamWaitEvent(c->copy_stream2, c->ev_group[g & 1], 0));
                for (size_t q = 0; q < cur.size(); q++) {
                    const int kk = k0 + g * per + (int)q;
                    const size_t bytes = sizeof(exs_complex) * (size_t)cur[q].nmat * cur[q].nmat;
                    EXS_CUDA(cudaMemcpyAsync(h[kk], cur[q].h, bytes, cudaMemcpyDeviceToHost, c->copy_stream));
                    EXS_CUDA(cudaMemcpyAsync(o[kk], cur[q].o, bytes, cudaMemcpyDeviceToHost, c->copy_stream2));
                }
                EXS_CUDA(cudaEventRecord(c->ev_copy2, c->copy_stream2));
                EXS_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_copy2, 0));
            }
            EXS_CUDA(cudaEventRecord(c->ev_d2h[g & 1], c->copy_stream));
            return EXS_OK;
        };
        // the lower parts of group g filled from the copied upper parts
        auto fill = [&](int g) -> int {
            EXS_CUDA(cudaEventSynchronize(c->ev_d2h[g & 1]));
            std::vector<KDesc> cur = group(g);
            struct Task {
                exs_complex *z;
                long n, c0;
            };
            std::vector<Task> tasks;
            for (size_t q = 0; q < cur.size(); q++) {
                const int kk = k0 + g * per + (int)q;
                for (int w = 0; w < 2; w++)
                    for (long c0 = 0; c0 + 64 < cur[q].nmat; c0 += 64)
                        tasks.push_back(Task{w == 0 ? h[kk] : o[kk], cur[q].nmat, c0});
            }
            c->pool->parallel_for((int)tasks.size(), [&](int i) { fill_lower_block(tasks[i].z, tasks[i].n, tasks[i].c0); });
            return EXS_OK;
        };
        // the full matrices of group g rebuilt on the host threads
        auto unpack = [&](int g) -> int {
            EXS_CUDA(cudaEventSynchronize(c->ev_d2h[g & 1]));
            std::vector<KDesc> cur = group(g);
            struct Task {
                const exs_complex *p;
                exs_complex *z;
                long n, c0, c1;
            };
            std::vector<Task> tasks;
            size_t off = 0;
            for (size_t q = 0; q < cur.size(); q++) {
                const int kk = k0 + g * per + (int)q;
                const long n = cur[q].nmat;
                const size_t t = (size_t)n * (n + 1) / 2;
                for (int w = 0; w < 2; w++) {
                    const exs_complex *pm = c->h_pack[g & 1] + off + w * t;
                    exs_complex *z = w == 0 ? h[kk] : o[kk];
                    for (long c0 = 0; c0 < n; c0 += 64) tasks.push_back(Task{pm, z, n, c0, std::min(n, c0 + 64)});
                }
                off += 2 * t;
            }
            c->pool->parallel_for((int)tasks.size(), [&](int i) {
                const Task &t = tasks[i];
                unpack_columns(t.p, t.z, t.n, t.c0, t.c1);
            });
            return EXS_OK;
        };
        int rc = enqueue(0);
        if (rc < 0) return rc;
        rc = copy_out(0);
        if (rc < 0) return rc;
        for (int g = 0; g < G; g++) {
            if (g + 1 < G) {   // the next group's setup goes ahead of this group's host work
                rc = enqueue(g + 1);
                if (rc < 0) return rc;
            }
            if (packed) {
                // slot (g+1)&1 was last unpacked in iteration g-1: its copy may start now
                if (g + 1 < G && (rc = copy_out(g + 1)) < 0) return rc;
                if ((rc = unpack(g)) < 0) return rc;
            } else if (upper) {
                if (g + 1 < G && (rc = copy_out(g + 1)) < 0) return rc;
                if ((rc = fill(g)) < 0) return rc;
            } else if (g + 1 < G && (rc = copy_out(g + 1)) < 0) {
                return rc;
            }
        }
        EXS_CUDA(cudaStreamSynchronize(c->copy_stream));
        rc = exs_synchronize(c);
        if (rc < 0) return rc;
        if (rc > worst) worst = rc;
    }
    return worst;
}

int exs_setup_and_solve_batched(exs_ctx *c, int nk, const int *ngp, const int *igpig, const double *vgpc, int nstfv,
                                double *evalfv, exs_complex *evecfv, int ldv)
{
    if (!c || nk < 0 || nstfv <= 0 || (nk > 0 && (!ngp || !igpig || !vgpc || !evalfv || !evecfv)))
        return fail(c, EXS_ERR_ARG, "exs_setup_and_solve_batched: bad argument");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    for (int k = 0; k < nk; k++) {
        if (ngp[k] <= 0 || ngp[k] > c->ngkmax) return fail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax");
        if (ldv < ngp[k] + c->nlotot || nstfv > ngp[k] + c->nlotot)
            return fail(c, EXS_ERR_SIZE, "ldv < nmat or nstfv > nmat");
        for (int i = 0; i < ngp[k]; i++) {
            const int g = igpig[(size_t)c->ngkmax * k + i];
            if (g < 1 || g > c->ngrtot) return fail(c, EXS_ERR_INDEX, "igpig entry outside 1..ngrtot");
        }
    }
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const size_t nev = (size_t)nstfv * c->max_batch, nvec = (size_t)ldv * nstfv * c->max_batch;
    if (nev > c->eval_cap) {
        if (c->d_eval) cudaFree(c->d_eval);
        c->d_eval = nullptr;
        c->eval_cap = 0;
        EXS_CUDA(cudaMalloc((void **)&c->d_eval, sizeof(double) * nev));
        c->eval_cap = nev;
    }
    if (nvec > c->evec_cap) {
        if (c->d_evec) cudaFree(c->d_evec);
        c->d_evec = nullptr;
        c->evec_cap = 0;
        EXS_CUDA(cudaMalloc((void **)&c->d_evec, sizeof(exs_complex) * nvec));
        c->evec_cap = nvec;
    }
    int worst = EXS_OK;
    for (int k0 = 0; k0 < nk; k0 += c->max_batch) {
        const int nb = std::min(c->max_batch, nk - k0);
        EXS_CUDA(cudaStreamSynchronize(s));
        std::memcpy(c->h_igpig_pinned, igpig + (size_t)c->ngkmax * k0, sizeof(int) * (size_t)c->ngkmax * nb);
        std::memcpy(c->h_vgpc_pinned, vgpc + 3 * (size_t)c->ngkmax * k0, sizeof(double) * 3 * (size_t)c->ngkmax * nb);
        EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
        EXS_CUDA(cudaMemcpyAsync(c->d_igpig, c->h_igpig_pinned, sizeof(int) * (size_t)c->ngkmax * nb,
                                 cudaMemcpyHostToDevice, s));
        EXS_CUDA(cudaMemcpyAsync(c->d_vgpc, c->h_vgpc_pinned, sizeof(double) * 3 * (size_t)c->ngkmax * nb,
                                 cudaMemcpyHostToDevice, s));
        std::vector<KDesc> ks;
        std::vector<int> nmat(nb);
        std::vector<exs_complex *> hp(nb), op(nb), vp(nb);
        for (int k = 0; k < nb; k++) {
            exs_complex *dh = c->d_ho + (size_t)2 * k * c->nmatmax * c->nmatmax;
            exs_complex *dob = dh + (size_t)c->nmatmax * c->nmatmax;
            ks.push_back(slot_desc(c, k, ngp[k0 + k], c->d_igpig + (size_t)c->ngkmax * k,
                                   c->d_vgpc + 3 * (size_t)c->ngkmax * k, dh, dob));
            nmat[k] = ks.back().nmat;
            hp[k] = dh;
            op[k] = dob;
            vp[k] = c->d_evec + (size_t)ldv * nstfv * k;
        }
        int rc = run_setup(c, ks, false);
        if (rc < 0) return rc;
        rc = exs_synchronize(c);
        if (rc < 0) return rc;
        if (rc > worst) worst = rc;
        rc = exs_solve_batched_device(c, nb, nmat.data(), hp.data(), op.data(), nstfv, c->d_eval, vp.data(), ldv);
        if (rc < 0) return rc;
        EXS_CUDA(cudaMemcpyAsync(evalfv + (size_t)nstfv * k0, c->d_eval, sizeof(double) * nstfv * nb,
                                 cudaMemcpyDeviceToHost, s));
        EXS_CUDA(cudaMemcpyAsync(evecfv + (size_t)ldv * nstfv * k0, c->d_evec, sizeof(exs_complex) * ldv * nstfv * nb,
                                 cudaMemcpyDeviceToHost, s));
        EXS_CUDA(cudaStreamSynchronize(s));
    }
    return worst;
}

int exs_hamiltonandoverlapsetup(exs_ctx *c, int ngp, const exs_complex *apwalm, const int *igpig,
                                const double *vgpc, exs_complex *h, exs_complex *o)
{
    if (!c || !igpig || !vgpc || !h || !o) return fail(c, EXS_ERR_ARG, "exs_hamiltonandoverlapsetup: null argument");
    if (ngp <= 0 || ngp > c->ngkmax) return fail(c, EXS_ERR_SIZE, "ngp outside 1..ngkmax");
    if (!c->have_inputs) return fail(c, EXS_ERR_STATE, "exs_set_scf_inputs has not been called");
    if (!apwalm) {
        exs_complex *hh[1] = {h}, *oo[1] = {o};
        // single k-point: the batched path with nk = 1 (igpig/vgpc carry ngkmax rows)
        std::vector<int> ig((size_t)c->ngkmax, 0);
        std::vector<double> vg(3 * (size_t)c->ngkmax, 0.0);
        std::memcpy(ig.data(), igpig, sizeof(int) * ngp);
        std::memcpy(vg.data(), vgpc, sizeof(double) * 3 * ngp);
        return exs_setup_batched(c, 1, &ngp, ig.data(), vg.data(), hh, oo);
    }
    for (int i = 0; i < ngp; i++)
        if (igpig[i] < 1 || igpig[i] > c->ngrtot) return fail(c, EXS_ERR_INDEX, "igpig entry outside 1..ngrtot");
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    EXS_CUDA(cudaStreamSynchronize(s));
    const int lmmax = (c->lmaxapw + 1) * (c->lmaxapw + 1);
    const size_t nalm = (size_t)c->ngkmax * c->apwordmax * lmmax * c->natmtot;
    if (!c->d_apwalm) {
        EXS_CUDA(dalloc(&c->d_apwalm, nalm));
        EXS_CUDA(dalloc(&c->d_match_in, 3 * (size_t)c->ngkmax));
        EXS_CUDA(dalloc(&c->d_match_sf, (size_t)c->ngkmax * c->natmtot));
    }
    EXS_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
    EXS_CUDA(cudaMemcpy2DAsync(c->d_apwalm, sizeof(exs_complex) * c->ngkmax, apwalm, sizeof(exs_complex) * c->ngkmax,
                               sizeof(exs_complex) * ngp, nalm / c->ngkmax, cudaMemcpyHostToDevice, s));
    EXS_CUDA(cudaMemcpyAsync(c->d_igpig, igpig, sizeof(int) * ngp, cudaMemcpyHostToDevice, s));
    EXS_CUDA(cudaMemcpyAsync(c->d_vgpc, vgpc, sizeof(double) * 3 * ngp, cudaMemcpyHostToDevice, s));
    std::vector<KDesc> ks;
    ks.push_back(slot_desc(c, 0, ngp, c->d_igpig, c->d_vgpc, c->d_ho, c->d_ho + (size_t)c->nmatmax * c->nmatmax));
    EXS_CUDA(oz_reset_maxima(c, ks, s));
    EXS_CUDA(exs::launch_apwalm_to_planes(c->params(), ngp, c->d_apwalm, ks[0].ar, ks[0].ai, ks[0].oz_scale, s));
    int rc = run_setup(c, ks, true);
    if (rc < 0) return rc;
    const size_t bytes = sizeof(exs_complex) * (size_t)ks[0].nmat * ks[0].nmat;
    EXS_CUDA(cudaMemcpyAsync(h, ks[0].h, bytes, cudaMemcpyDeviceToHost, s));
    EXS_CUDA(cudaMemcpyAsync(o, ks[0].o, bytes, cudaMemcpyDeviceToHost, s));
    return exs_synchronize(c);
}

// sort_index_1d_real (src/sorting.f90:74-117): the heapsort's sift-down
// with 1-based positions l (heap build) and k (extraction), comparing
// a(inc (idx - 1) + 1) with strict "<" as the reference does.
int exs_sort_index_1d(int n, const double *a, int inc, int *idx)
{
    if (n < 0 || (n > 0 && (!a || !idx)) || inc < 1) return EXS_ERR_ARG;
    if (n == 0) return EXS_OK;
    auto key = [&](int m) { return a[(size_t)inc * (m - 1)]; };
    int *ix = idx - 1;                         // ix[1..n]
    for (int i = 1; i <= n; i++) ix[i] = i;
    if (n == 1) return EXS_OK;
    int l = n / 2 + 1, k = n;
    while (true) {
        int m;
        if (l > 1) {
            l = l - 1;
            m = ix[l];
        } else {
            m = ix[k];
            ix[k] = ix[1];
            k = k - 1;
            if (k == 1) {
                ix[1] = m;
                break;
            }
        }
        int i = l, j = l + l;
        while (j <= k) {
            if (j < k && key(ix[j]) < key(ix[j + 1])) j = j + 1;
            if (key(m) < key(ix[j])) {
                ix[i] = ix[j];
                i = j;
                j = j + j;
            } else {
                j = k + 1;
            }
        }
        ix[i] = m;
    }
    return EXS_OK;
}

}  // extern "C"
