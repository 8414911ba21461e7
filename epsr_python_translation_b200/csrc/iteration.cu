// iteration.cu -- one EPSR iteration of the pair path on one box, driven from native code.
//
// The iteration body of runepsr17 (epsr_standalone_rev3.py:1235-1842) restricted to this
// path, in its order: the cell list (:1259), fmolec1 (:1265), ntimes molfit cycles
// (:1280-1318), atogen (:1397), gensq (:1400), the per-data-set differences of ptgnsq
// (:3844-3867), press (:1842 -> ato_manipulation_rev4.py:3903), fit_expansion for every
// data set (ptgnsq :3936), optionally the EP refinement that follows the fits (ptgnsq
// :3948-3962 and generate_ep :4014, then the packed tables of the next iteration's energies),
// the running averages sumsq and sumgr (:1611-1642) and stog of the simulated S(Q) (:1987).  Every stage is the C ABI
// routine of that name, launched on the caller's stream from this thread, so a host that
// advances many boxes on many threads does no per-launch work in an interpreter.  Host
// reads happen where the routines need them (the cell list's region size, store and
// capacity counts, the fit's per-set scalars).
#include <string.h>

#include "common.cuh"

using namespace epsr;

namespace {

inline int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }

int cell_dims(const epsr_iteration_t *it, int32_t dims[4]) {
    return epsr_cell_dims(it->nmolcell, it->box->nmol, it->lat6, dims);
}

void mark(const epsr_iteration_t *it, int stage, int end, cudaStream_t s) {
    void *ev = it->stage_events[2 * stage + end];
    if (ev) cudaEventRecord((cudaEvent_t)ev, s);
}

}  // namespace

extern "C" int64_t epsr_iteration_scratch_bytes(const epsr_iteration_t *it) {
    if (!it || !it->box) return -1;
    int32_t dims[4];
    if (cell_dims(it, dims)) return -1;
    const epsr_box_t *b = it->box;
    const int ldq = it->nq + 1;
    int64_t n = epsr_fmolec1_scratch_bytes(b->nmol, dims[3], it->store_m);
    n = imax64(n, epsr_molfit_scratch_bytes(b->nmol, b->natom, it->store_m));
    n = imax64(n, epsr_atogen_scratch_bytes(b->nmol, b->natom, b->nmoltype, b->ntype));
    n = imax64(n, epsr_press_scratch_bytes(b->nmol, it->store_m));
    n = imax64(n, epsr_fit_expansion_batch_scratch_bytes(it->ndata, it->nq, it->nterms));
    n = imax64(n, epsr_stog_scratch_bytes(b->npairs, ldq));
    if (it->intra > 0) n = imax64(n, epsr_molfit_shake_scratch_bytes(b->nmol, b->natom));
    return n;
}

extern "C" int epsr_iteration_step(const epsr_iteration_t *it, epsr_iteration_report_t *rep, void *stream) {
    if (!it || !rep || !it->box || !it->mc || !it->scratch) {
        epsr_set_error("epsr_iteration_step: null pointer");
        return EPSR_ERR_ARG;
    }
    const int64_t need = epsr_iteration_scratch_bytes(it);
    if (need < 0 || it->scratch_bytes < need) {
        epsr_set_error("epsr_iteration_step: scratch too small (%lld < %lld bytes)", (long long)it->scratch_bytes,
                       (long long)need);
        return EPSR_ERR_CAPACITY;
    }
    const epsr_box_t *b = it->box;
    if (it->intra > 0 && (!it->intra_model || !it->faddbs || !it->eintra_work || !it->nmovei)) {
        epsr_set_error("epsr_iteration_step: intramolecular cycles need intra_model, faddbs, eintra_work, nmovei");
        return EPSR_ERR_ARG;
    }
    if (it->refine && (b->izcut != b->npt2 || !it->pcoefp || !it->irefpcof_host || !it->efacp || !it->cwtpot ||
                       !it->expgr || !it->wfac || !it->ecoul || !it->ecoul1 || !it->xavs || !it->xavs1 ||
                       !it->xavtot || !it->xavtot1 || !it->ep_pwtold || !it->potfac || !it->ep_result || !it->tab ||
                       it->tab != b->tab)) {
        epsr_set_error("epsr_iteration_step: EP refinement needs its buffers, tab == box->tab and izcut == npt2 "
                       "(izcut %d, npt2 %d)", b->izcut, b->npt2);
        return EPSR_ERR_ARG;
    }
    memset(rep, 0, sizeof(*rep));
    cudaStream_t s = (cudaStream_t)stream;
    int rc;

    // ---- cell list (initialise_cellneighbourlist)
    mark(it, 0, 0, s);
    epsr_cells_t cells;
    memset(&cells, 0, sizeof(cells));
    cells.molcellno = it->cell_molcellno;
    cells.cell_start = it->cell_start;
    cells.cell_mols = it->cell_mols;
    cells.offsets = it->cell_offsets;
    rc = epsr_cell_list(b->xadd, b->yadd, b->zadd, b->nmol, it->nmolcell, it->rmax, it->lat6, it->lat9, &cells,
                        it->cell_scratch, it->cell_scratch_n, stream);
    if (rc) return rc;
    rep->nnbrefmax = cells.nnbrefmax;
    if (cells.nnbrefmax > it->store_m) {   // nothing of the box has changed yet
        epsr_set_error("epsr_iteration_step: region size %d exceeds the store's %d slots per molecule",
                       cells.nnbrefmax, it->store_m);
        return EPSR_ERR_CAPACITY;
    }
    mark(it, 0, 1, s);

    // ---- fmolec1: the pair store
    mark(it, 1, 0, s);
    epsr_store_t store;
    store.nnbrefmax = cells.nnbrefmax;
    store.capacity = it->store_capacity;
    store.nergpairm = it->nergpairm;
    store.molergpair = it->molergpair;
    store.ergpairref = it->ergpairref;
    store.ergpair = it->ergpair;
    store.nergpair = it->nergpair;
    store.mirror = it->mirror;
    const float *eintra = it->eintra;
    if (it->intra_model) {   // the intramolecular energies of the box's model, as fmolec1 forms them
        rc = epsr_en_mole_intra(b, it->intra_model, it->eintra_work, stream);
        if (rc) return rc;
        eintra = it->eintra_work;
    }
    rc = epsr_fmolec1(b, &cells, eintra, &store, it->scratch, it->scratch_bytes, it->strict, rep->ftest, stream);
    if (rc) return rc;
    mark(it, 1, 1, s);

    // ---- molfit cycles (runepsr17 :1313-1345): molfit's branch by nisum, and after an
    // intramolecular cycle the centres put back in the box and the pair store rebuilt
    mark(it, 2, 0, s);
    epsr_mc_t *mc = it->mc;
    mc->strict = it->strict;
    mc->cos_override = nullptr;
    int32_t nisum = it->nisum;
    for (int t = 0; t < it->ntimes; ++t) {
        if (it->intra > 0 && nisum >= it->intra) {
            rc = epsr_molfit_shake(b, &store, mc, it->intra_model, it->stepmi, it->nmovei, it->faddbs, it->scratch,
                                   it->scratch_bytes, stream);
            if (rc) return rc;
            nisum = 1;
            rc = epsr_minimage_centres(b, stream);
            if (rc) return rc;
            rc = epsr_en_mole_intra(b, it->intra_model, it->eintra_work, stream);
            if (rc) return rc;
            rc = epsr_fmolec1(b, &cells, it->eintra_work, &store, it->scratch, it->scratch_bytes, it->strict,
                              rep->ftest, stream);
            if (rc) return rc;
        } else {
            mc->rotcycle = it->rotfreq > 0 && nisum % it->rotfreq == 0;   // molfit.py:295
            rc = epsr_molfit(b, &cells, &store, mc, it->scratch, it->scratch_bytes, stream);
            if (rc) return rc;
            nisum += 1;
        }
    }
    rep->nisum = nisum;
    mark(it, 2, 1, s);

    // ---- atogen: the partial g(r) histograms
    mark(it, 3, 0, s);
    EPSR_CUDA(cudaMemsetAsync(it->wav, 0, sizeof(float) * 2 * (size_t)b->npairs * it->ldw, s));
    EPSR_CUDA(cudaMemsetAsync(it->potex, 0, sizeof(float) * (size_t)b->npairs, s));
    int32_t ngr = it->ngrsamples;
    rc = epsr_atogen(b, it->npt1, it->sizefactor, it->dmax, it->rminex, it->cfrac, it->ycoh, it->n1extr, it->n2extr,
                     it->natomr, &ngr, mc->ran1, it->wav, it->ldw, it->potex, it->counts, it->scratch,
                     it->scratch_bytes, stream);
    if (rc) return rc;
    rep->ngrsamples = ngr;
    rep->pair_updates = epsr_atogen_last_pair_updates();
    mark(it, 3, 1, s);

    // ---- gensq and the data-set differences the fit works on
    mark(it, 4, 0, s);
    const int ldq = it->nq + 1;
    rc = epsr_gensq(it->nq, b->npairs, it->npt1, it->wav, it->ldw, it->foqols, it->foqols_sj, it->foqols_si, it->ycoh,
                    it->n2extr, it->natomsphere, it->sofq, stream);
    if (rc) return rc;
    const float *inter = it->sofq + (size_t)b->npairs * ldq;   // intermolecular S(Q) per pair
    rc = epsr_ptgnsq_difference(it->ndata, b->npairs, it->nq, it->data, it->cwt, inter, nullptr, nullptr, nullptr,
                                nullptr, 0.0f, nullptr, nullptr, it->dt, stream);
    if (rc) return rc;
    mark(it, 4, 1, s);

    // ---- press
    mark(it, 5, 0, s);
    rc = epsr_press(b, &store, it->npt1, it->scratch, it->scratch_bytes, it->strict, rep->press, stream);
    if (rc) return rc;
    mark(it, 5, 1, s);

    // ---- fit_expansion for every data set, one launch
    mark(it, 6, 0, s);
    for (int d = 0; d < it->ndata; ++d)   // stepr carries over; acceptr, rejrat, chisq start at 0
        for (int k = 1; k < 4; ++k) it->fit_scal_host[4 * d + k] = 0.0f;
    EPSR_CUDA(cudaMemsetAsync(it->fit_wt, 0, sizeof(float) * (size_t)it->ndata * (it->nterms + 1), s));
    EPSR_CUDA(cudaMemsetAsync(it->fit_yout, 0, sizeof(float) * (size_t)it->ndata * ldq, s));
    rc = epsr_fit_expansion_batch(it->ndata, it->dt, it->expr, it->fit_yout, it->fit_wt, it->fit_wtold,
                                  it->fit_scal_host, 1, it->nq, it->ncfirst, it->nterms, it->nits, it->nfreq, mc->ran1,
                                  it->scratch, it->scratch_bytes, it->strict, it->fit_trials_host, stream);
    if (rc) return rc;
    mark(it, 6, 1, s);

    // ---- EP refinement: ptgnsq's coefficient increment, generate_ep(.false.), the packed tables
    mark(it, 7, 0, s);
    if (it->refine) {
        rc = epsr_ep_update(it->ndata, b->npairs, it->nterms, it->pcoefp, it->nsets, it->ldc, it->irefpcof_host,
                            it->efacp, it->cwtpot, it->fit_wtold, it->nterms + 1, it->pfact, stream);
        if (rc) return rc;
        rc = epsr_generate_ep(b->npairs, b->ld - 1, b->npt2, it->nterms, it->expgr, it->pcoefp, it->nsets, it->ldc,
                              it->irefpcof_host, it->dmax, b->xstar, it->wfac, it->ecoul, it->xavs, it->xavs1,
                              it->xavtot, it->xavtot1, b->ld, it->ep_pwtold, it->absolute_energy, it->erequnit,
                              it->ereqstep, it->potfacamp, it->potfac, 0, it->ep_result, stream);
        if (rc) return rc;
        rc = epsr_pack_tables(b->npairs, b->ld, it->xavs, it->xavs1, it->ecoul, it->ecoul1, it->tab, stream);
        if (rc) return rc;
    }
    mark(it, 7, 1, s);

    // ---- running averages of S(Q) and g(r) (runepsr17 :1611-1642)
    mark(it, 8, 0, s);
    if (it->nsum < 1) {
        epsr_set_error("epsr_iteration_step: nsum %d < 1", it->nsum);
        return EPSR_ERR_ARG;
    }
    const double fc1 = (double)(1.0f / (float)it->nsum);
    const double fc2 = (double)(float)(it->nsum - 1) * fc1;
    rc = epsr_sumsq(it->nq, b->npairs, it->sofq, ldq, fc1, fc2, it->soqintra, it->soqinter, it->sq2intra,
                    it->sq2inter, stream);
    if (rc) return rc;
    rc = epsr_sumgr(it->npt1, b->npairs, it->wav, it->ldw, it->ycoh, fc1, fc2, it->gorintra, it->gorinter,
                    it->gr2intra, it->gr2inter, it->entsig, stream);
    if (rc) return rc;
    mark(it, 8, 1, s);

    // ---- stog of the simulated intermolecular S(Q)
    mark(it, 9, 0, s);
    rc = epsr_stog(it->rho, it->q, ldq, inter, it->r, it->nr, b->npairs, it->nqmin, it->nqmax, it->xwt, it->gofr,
                   it->scratch, it->scratch_bytes, stream);
    if (rc) return rc;
    mark(it, 9, 1, s);
    return EPSR_OK;
}
