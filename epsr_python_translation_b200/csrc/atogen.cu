// atogen.cu -- pair-distance histograms (atogen ato_manipulation_rev4.py:3640-3899).
//
// (1) origin selection: one ran1 draw per candidate molecule (the reference always draws,
//     :3765), then the sequential sampling rule (draw < probaccept, or the molecule type not
//     yet sampled, or a type rarer than probaccept);
// (2) intramolecular bins (nint, +2 per pair, :3696-3725);
// (3) intermolecular all-pairs: blocks take a tile of target atoms staged in shared memory
//     and a chunk of origin atoms (one per thread); counts go to a block-private shared
//     histogram per pair type, merged into global 64-bit counts by atomics; close contacts
//     (potex) are counted alongside;
// (4) normalisation in float32 exactly as the reference (counts are exact integers; the
//     reference's float accumulation equals them while a bin stays below 2^24).

#include "common.cuh"

namespace epsr {

struct AgDev {
    Lattice L;
    int nmol, natom, ntype, npairs, nmoltype, npt1, ldw, full;
    const int32_t *naf, *nato, *mtype, *npairref;
    const float4 *pos;
    const float *xa, *ya, *za;
    float stepcl, sizefactor, dmax;
    const float *rminex;
};

// (1) selection.  draws: one ran1 value per candidate im in [im1, im2] (:3765).  The rule
// "u < probaccept or type not yet sampled or type fraction < probaccept" is sequential only
// through "not yet sampled", which holds exactly for the first candidate of each type; so the
// selection is a parallel filter followed by an ordered compaction (one block).  It also
// returns the per-type atom counts of the sampled molecules (csampled, exact integers like the
// reference's float sums of 1.0), the origin-atom prefix and the pair-update count.
__device__ __forceinline__ int ag_bscan(int v, int *total) {
    __shared__ int ws[32];
    __shared__ int wp[33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0;
        for (int w = 0; w < nw; ++w) {
            wp[w] = a;
            a += ws[w];
        }
        wp[32] = a;
    }
    __syncthreads();
    const int r = wp[wid] + incl - v;
    *total = wp[32];
    __syncthreads();
    return r;
}

__global__ void ag_select_kernel(AgDev A, const float *draws, int im1, int im2, float probaccept,
                                 const int32_t *itype, int32_t *origins, int32_t *prefix, int32_t *counts_out,
                                 float *csampled, long long *pairs_out) {
    __shared__ int first[64];
    __shared__ int cntt[64];
    __shared__ int catoms[64];
    __shared__ unsigned long long spairs;
    const int tid = threadIdx.x;
    for (int t = tid; t < 64; t += blockDim.x) {
        first[t] = 0x7fffffff;
        cntt[t] = 0;
        catoms[t] = 0;
    }
    if (tid == 0) spairs = 0ull;
    __syncthreads();
    for (int m = tid; m < A.nmol; m += blockDim.x) atomicAdd(&cntt[A.mtype[m]], 1);
    for (int im = im1 + tid; im <= im2; im += blockDim.x) atomicMin(&first[A.mtype[im]], im);
    if (A.full && tid == 0) {
        const int m = A.nmol - 1;
        for (int a = A.naf[m]; a < A.naf[m] + A.nato[m]; ++a) atomicAdd(&catoms[itype[a]], 1);
    }
    __syncthreads();
    int carry = 0, acarry = 0;
    unsigned long long mypairs = 0ull;
    for (int base = im1; base <= im2; base += blockDim.x) {
        const int im = base + tid;
        int sel = 0, na = 0;
        if (im <= im2) {
            const int mt = A.mtype[im];
            const float frac = __fdiv_rn((float)cntt[mt], (float)A.nmol);  // molfraction (:3753-3756)
            sel = draws[im - im1] < probaccept || first[mt] == im || frac < probaccept;
            if (sel) {
                na = A.nato[im];
                for (int a = A.naf[im]; a < A.naf[im] + na; ++a) atomicAdd(&catoms[itype[a]], 1);
                const long long tgt = A.full ? (long long)(A.natom - A.naf[im] - na) : (long long)(A.natom - na);
                mypairs += (unsigned long long)((long long)na * tgt);
            }
        }
        int tot, atot;
        const int pos = carry + ag_bscan(sel, &tot);
        const int apos = acarry + ag_bscan(na, &atot);
        if (sel) {
            origins[pos] = im;
            prefix[pos] = apos;
        }
        carry += tot;
        acarry += atot;
    }
    atomicAdd(&spairs, mypairs);
    __syncthreads();
    for (int t = tid; t < A.ntype; t += blockDim.x) csampled[t] = (float)catoms[t];
    if (tid == 0) {
        counts_out[0] = carry;   // sampled molecules
        counts_out[1] = acarry;  // origin atoms
        *pairs_out = (long long)spairs;
    }
}

// (2) intramolecular pairs
__global__ void ag_intra_kernel(AgDev A, const int32_t *itype, unsigned long long *counts, long long *pairs_out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= A.nmol) return;
    const int a0 = A.naf[m], n = A.nato[m];
    if (n <= 1) return;
    long long np = 0;
    for (int ia = a0; ia < a0 + n - 1; ++ia) {
        for (int ja = ia + 1; ja < a0 + n; ++ja) {
            const int icref = A.npairref[itype[ia] * A.ntype + itype[ja]];
            float xx = __fmul_rn(__fsub_rn(A.xa[ia], A.xa[ja]), A.sizefactor);
            float yy = __fmul_rn(__fsub_rn(A.ya[ia], A.ya[ja]), A.sizefactor);
            float zz = __fmul_rn(__fsub_rn(A.za[ia], A.za[ja]), A.sizefactor);
            const float d = dist_f(A.L, xx, yy, zz);
            const int iz1 = nint_i(__fdiv_rn(d, A.stepcl)) + 2;
            if (iz1 > 1 && iz1 <= A.npt1) atomicAdd(counts + (size_t)icref * A.ldw + iz1, 1ull);
            ++np;
        }
    }
    atomicAdd((unsigned long long *)pairs_out, (unsigned long long)np);
}

// origin atoms of the selected molecules: (atom, molecule) pairs in selection order
__global__ void ag_origin_atoms_kernel(AgDev A, const int32_t *origins, const int32_t *norigin, const int32_t *prefix,
                                       int2 *oatoms) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *norigin) return;
    const int im = origins[k];
    for (int q = 0; q < A.nato[im]; ++q) oatoms[prefix[k] + q] = make_int2(A.naf[im] + q, im);
}

// (3) intermolecular all-pairs
constexpr int AG_THREADS = 256;

__global__ void __launch_bounds__(AG_THREADS) ag_inter_kernel(AgDev A, const int2 *oatoms, const int32_t *noatoms_p,
                                                              const int32_t *molof, int tile,
                                                              unsigned long long *counts, unsigned long long *potex) {
    extern __shared__ unsigned char sm[];
    const int nbins = A.npairs * A.ldw;
    unsigned int *hist = (unsigned int *)sm;
    unsigned int *hpot = hist + nbins;
    // the float4 tile must start on a 16-byte boundary
    const size_t tp_off = ((sizeof(unsigned int) * ((size_t)nbins + A.npairs)) + 15) & ~(size_t)15;
    float4 *tp = (float4 *)(sm + tp_off);
    int *tm = (int *)(tp + tile);
    const int noatoms = *noatoms_p;
    const int t0 = blockIdx.x * tile;
    const int tn = min(tile, A.natom - t0);
    const int obase = blockIdx.y * AG_THREADS;
    if (obase >= noatoms || tn <= 0) return;
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) hist[i] = 0;
    for (int i = threadIdx.x; i < A.npairs; i += blockDim.x) hpot[i] = 0;
    for (int i = threadIdx.x; i < tn; i += blockDim.x) {
        tp[i] = A.pos[t0 + i];
        tm[i] = molof[t0 + i];
    }
    __syncthreads();
    const int k = obase + threadIdx.x;
    if (k < noatoms) {
        const int2 oa = oatoms[k];
        const float4 p1 = A.pos[oa.x];
        const int im = oa.y;
        const int it = __float_as_int(p1.w);
        const int *pr = A.npairref + it * A.ntype;
        for (int q = 0; q < tn; ++q) {
            const int jm = tm[q];
            const bool use = A.full ? (jm > im) : (jm != im);
            if (!use) continue;
            const float4 p2 = tp[q];
            const int icref = __ldg(pr + __float_as_int(p2.w));
            // xx = x1 - x2 (ato_manipulation_rev4.py:3798)
            const float d = dist_f(A.L, __fsub_rn(p1.x, p2.x), __fsub_rn(p1.y, p2.y), __fsub_rn(p1.z, p2.z));
            const int iz1 = nint_i(__fdiv_rn(d, A.stepcl)) + 2;
            if (iz1 > 1 && iz1 <= A.npt1) atomicAdd(hist + icref * A.ldw + iz1, 1u);
            if (__fmul_rn(d, A.dmax) < fabsf(__ldg(A.rminex + icref))) atomicAdd(hpot + icref, 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (hist[i]) atomicAdd(counts + (size_t)A.npairs * A.ldw + i, (unsigned long long)hist[i]);
    for (int i = threadIdx.x; i < A.npairs; i += blockDim.x)
        if (hpot[i]) atomicAdd(potex + i, (unsigned long long)hpot[i]);
}

__global__ void ag_molof_kernel(AgDev A, int32_t *molof) {
    const int m = blockIdx.x;
    for (int a = A.naf[m] + threadIdx.x; a < A.naf[m] + A.nato[m]; a += blockDim.x) molof[a] = m;
}

// (4) normalisation (:3857-3897)
__global__ void ag_norm_kernel(AgDev A, const unsigned long long *counts, const unsigned long long *potc,
                               const float *csampled, const float *cfrac, const int32_t *n1extr,
                               const int32_t *n2extr, int natomr, float addwav, const float *ycoh, float *wav,
                               float *potex) {
    const int ic = blockIdx.x;
    const int it = n1extr[ic], jt = n2extr[ic];
    float cprod = __fmul_rn(__fmul_rn(cfrac[it], cfrac[jt]), (float)natomr);
    float cprod2 = __fmul_rn(csampled[it], cfrac[jt]);
    if (it != jt) {
        cprod = __fmul_rn(cprod, 2.0f);
        cprod2 = __fadd_rn(cprod2, __fmul_rn(csampled[jt], cfrac[it]));
    }
    float *w1 = wav + (size_t)ic * A.ldw;
    float *w2 = wav + (size_t)(A.npairs + ic) * A.ldw;
    const unsigned long long *c1 = counts + (size_t)ic * A.ldw;
    const unsigned long long *c2 = counts + (size_t)(A.npairs + ic) * A.ldw;
    for (int iz = 1 + threadIdx.x; iz <= A.npt1; iz += blockDim.x) {
        const float v1 = (float)(2ull * c1[iz]);
        const float v2 = __fmul_rn((float)c2[iz], addwav);
        w1[iz] = cprod > 0.0f ? __fdiv_rn(v1, cprod) : 0.0f;
        w2[iz] = cprod2 > 0.0f ? __fdiv_rn(v2, cprod2) : ycoh[iz];
    }
    if (threadIdx.x == 0 && cprod2 > 0.0f) potex[ic] = __fdiv_rn(__fmul_rn((float)potc[ic], cfrac[jt]), cprod2);
    else if (threadIdx.x == 0) potex[ic] = (float)potc[ic];
}

}  // namespace epsr

using namespace epsr;

static thread_local long long g_last_pairs = 0;

static inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int64_t epsr_atogen_scratch_bytes(int32_t nmol, int32_t natom, int32_t nmoltype, int32_t ntype) {
    (void)nmoltype;
    size_t b = 0;
    b += al256(sizeof(float) * nmol);          // draws
    b += al256(sizeof(int32_t) * nmol);        // origins
    b += al256(sizeof(int32_t) * nmol);        // prefix
    b += al256(sizeof(int2) * natom);          // origin atoms
    b += al256(sizeof(int32_t) * natom);       // molecule of atom
    b += al256(sizeof(float) * (ntype + 1));   // csampled
    b += al256(sizeof(int32_t) * 8);           // norigin, noatoms
    b += al256(sizeof(long long) * 2);         // pair counters
    return (int64_t)b;
}

extern "C" int64_t epsr_atogen_last_pair_updates(void) { return g_last_pairs; }

extern "C" int epsr_atogen(const epsr_box_t *box, int32_t npt1, float sizefactor, float dmax, const float *rminex,
                           const float *cfrac, const float *ycoh, const int32_t *n1extr, const int32_t *n2extr,
                           int32_t natomr, int32_t *ngrsamples_io, int32_t *ran1, float *wav, int32_t ldw,
                           float *potex, unsigned long long *counts, void *scratch, int64_t scratch_bytes,
                           void *stream) {
    if (!box || !rminex || !cfrac || !ycoh || !n1extr || !n2extr || !ngrsamples_io || !ran1 || !wav || !potex ||
        !counts || !scratch) {
        epsr_set_error("epsr_atogen: null pointer");
        return EPSR_ERR_ARG;
    }
    const int nmol = box->nmol, natom = box->natom;
    if (npt1 + 1 > ldw || ldw > box->ld + 4096) {
        epsr_set_error("epsr_atogen: ldw %d must be >= npt1+1 (%d)", ldw, npt1 + 1);
        return EPSR_ERR_ARG;
    }
    if (box->nmoltype > 64) {
        epsr_set_error("epsr_atogen: at most 64 molecule types");
        return EPSR_ERR_UNSUPPORTED;
    }
    // refused before any device work: a rejected call leaves the counts and the ran1 state as given
    if (box->ntype > 64) {
        epsr_set_error("epsr_atogen: at most 64 atom types");
        return EPSR_ERR_UNSUPPORTED;
    }
    if (scratch_bytes < epsr_atogen_scratch_bytes(nmol, natom, box->nmoltype, box->ntype)) {
        epsr_set_error("epsr_atogen: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += al256(bytes);
        return (void *)r;
    };
    float *draws = (float *)take(sizeof(float) * nmol);
    int32_t *origins = (int32_t *)take(sizeof(int32_t) * nmol);
    int32_t *prefix = (int32_t *)take(sizeof(int32_t) * nmol);
    int2 *oatoms = (int2 *)take(sizeof(int2) * natom);
    int32_t *molof = (int32_t *)take(sizeof(int32_t) * natom);
    float *csampled = (float *)take(sizeof(float) * (box->ntype + 1));
    int32_t *misc = (int32_t *)take(sizeof(int32_t) * 8);
    long long *pairc = (long long *)take(sizeof(long long) * 2);

    int ngr = *ngrsamples_io;
    if (ngr <= 0) ngr = 1000;
    if (ngr > nmol) ngr = nmol;
    const float probaccept = (float)ngr / (float)nmol;
    const int full = probaccept >= 1.0f;
    const int im1 = 0, im2 = full ? nmol - 2 : nmol - 1;
    const float addwav = full ? 2.0f : 1.0f;

    AgDev A;
    A.L.cubic = box->cubic;
    A.L.alatx = box->lat[0];
    A.L.blatx = box->lat[1];
    A.L.clatx = box->lat[2];
    A.L.blaty = box->lat[3];
    A.L.claty = box->lat[4];
    A.L.clatz = box->lat[5];
    A.nmol = nmol;
    A.natom = natom;
    A.ntype = box->ntype;
    A.npairs = box->npairs;
    A.nmoltype = box->nmoltype;
    A.npt1 = npt1;
    A.ldw = ldw;
    A.full = full;
    A.naf = box->naf;
    A.nato = box->nato;
    A.mtype = box->mtype;
    A.npairref = box->npairref;
    A.pos = (const float4 *)box->pos;
    A.xa = box->xa;
    A.ya = box->ya;
    A.za = box->za;
    A.stepcl = box->stepcl;
    A.sizefactor = sizefactor;
    A.dmax = dmax;
    A.rminex = rminex;

    const size_t nbins = (size_t)box->npairs * ldw;
    EPSR_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * (2 * nbins + box->npairs), s));
    EPSR_CUDA(cudaMemsetAsync(pairc, 0, sizeof(long long) * 2, s));
    int rc = epsr_box_positions(box, stream);
    if (rc) return rc;
    const int ncand = im2 - im1 + 1;
    if (ncand > 0) {
        rc = epsr_ran1_fill(ran1, draws, ncand, stream);
        if (rc) return rc;
    }
    ag_select_kernel<<<1, 1024, 0, s>>>(A, draws, im1, im2, probaccept, box->itype, origins, prefix, misc, csampled,
                                         pairc);
    ag_intra_kernel<<<(nmol + 127) / 128, 128, 0, s>>>(A, box->itype, counts, pairc + 1);
    ag_molof_kernel<<<nmol, 32, 0, s>>>(A, molof);
    ag_origin_atoms_kernel<<<(nmol + 127) / 128, 128, 0, s>>>(A, origins, misc, prefix, oatoms);
    EPSR_CUDA(cudaGetLastError());
    int32_t hmisc[2];
    EPSR_D2H(hmisc, misc, sizeof(hmisc), s);
    const int noatoms = hmisc[1];
    // tile of target atoms: enough blocks to fill the GPU several times over
    int tile = 1024;
    const int ychunks = (noatoms + AG_THREADS - 1) / AG_THREADS;
    while (tile > 128 && (long long)ychunks * ((natom + tile - 1) / tile) < 4 * 148) tile >>= 1;
    const size_t tp_off = ((sizeof(unsigned int) * (nbins + box->npairs)) + 15) & ~(size_t)15;
    const size_t shm = tp_off + (sizeof(float4) + sizeof(int)) * tile;
    if (shm > 220 * 1024) {
        epsr_set_error("epsr_atogen: histogram of %zu bins does not fit in shared memory", nbins);
        return EPSR_ERR_UNSUPPORTED;
    }
    if (shm > 48 * 1024)
        EPSR_SMEM_OPTIN(ag_inter_kernel);
    if (noatoms > 0) {
        dim3 grid((natom + tile - 1) / tile, ychunks);
        EPSR_TIMED("ag_inter_kernel", s, ag_inter_kernel<<<grid, AG_THREADS, shm, s>>>(A, oatoms, misc + 1, molof, tile, counts, counts + 2 * nbins));
    }
    ag_norm_kernel<<<box->npairs, 256, 0, s>>>(A, counts, counts + 2 * nbins, csampled, cfrac, n1extr, n2extr, natomr,
                                                addwav, ycoh, wav, potex);
    EPSR_CUDA(cudaGetLastError());
    long long hp[2];
    EPSR_D2H(hp, pairc, sizeof(hp), s);
    g_last_pairs = hp[0] + hp[1];
    *ngrsamples_io = ngr;
    return EPSR_OK;
}

// ----------------------------------------------------------------- allocation-free variant
// Some callers cannot hand this library device buffers: a host whose device memory is owned
// by another allocator (a caching pool that must not be bypassed, or a host process that
// reserves its whole budget up front), or a plain C/Fortran/ctypes caller with no device
// allocator at all.  epsr_atogen_noalloc needs only the inputs and outputs: its working
// memory and histogram counts live in one file-scope device array, sized for the reference's
// own limits (50,000 molecules, 150,000 atoms) and at most 2^19 histogram entries.
namespace {
constexpr int64_t NOALLOC_MAX_NMOL = 50000;
constexpr int64_t NOALLOC_MAX_NATOM = 150000;
constexpr int64_t NOALLOC_MAX_COUNTS = 1 << 19;   // 2*npairs*ldw + npairs
constexpr int64_t NOALLOC_COUNTS_BYTES = NOALLOC_MAX_COUNTS * 8;
constexpr int64_t NOALLOC_WORK_BYTES = 4 << 20;   // >= epsr_atogen_scratch_bytes at the maxima
static __device__ __align__(256) unsigned char g_atogen_noalloc[NOALLOC_COUNTS_BYTES + NOALLOC_WORK_BYTES];
}  // namespace

extern "C" int epsr_atogen_noalloc(const epsr_box_t *box, int32_t npt1, float sizefactor, float dmax,
                                   const float *rminex, const float *cfrac, const float *ycoh, const int32_t *n1extr,
                                   const int32_t *n2extr, int32_t natomr, int32_t *ngrsamples_io, int32_t *ran1,
                                   float *wav, int32_t ldw, float *potex, void *stream) {
    if (!box) {
        epsr_set_error("epsr_atogen_noalloc: null box");
        return EPSR_ERR_ARG;
    }
    const int64_t ncounts = 2 * (int64_t)box->npairs * ldw + box->npairs;
    if (box->nmol > NOALLOC_MAX_NMOL || box->natom > NOALLOC_MAX_NATOM || ncounts > NOALLOC_MAX_COUNTS) {
        epsr_set_error("epsr_atogen_noalloc: box exceeds the built-in working memory (at most %lld molecules, %lld "
                       "atoms, %lld histogram entries 2*npairs*ldw+npairs; got %d, %d, %lld) -- use epsr_atogen",
                       (long long)NOALLOC_MAX_NMOL, (long long)NOALLOC_MAX_NATOM, (long long)NOALLOC_MAX_COUNTS,
                       box->nmol, box->natom, (long long)ncounts);
        return EPSR_ERR_CAPACITY;
    }
    const int64_t need = epsr_atogen_scratch_bytes(box->nmol, box->natom, box->nmoltype, box->ntype);
    if (need > NOALLOC_WORK_BYTES) {
        epsr_set_error("epsr_atogen_noalloc: working memory %lld bytes exceeds %lld", (long long)need,
                       (long long)NOALLOC_WORK_BYTES);
        return EPSR_ERR_CAPACITY;
    }
    // The device address of the array in the current device's context.  It is looked up on
    // every call (a cheap host query) rather than cached, so a context that was re-created
    // (after cudaDeviceReset) is served at its own address.
    void *base = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress(&base, g_atogen_noalloc);
        if (e != cudaSuccess) return epsr_cuda_check(e, "cudaGetSymbolAddress(g_atogen_noalloc)");
    }
    unsigned long long *counts = (unsigned long long *)base;  // zeroed inside epsr_atogen
    void *work = (unsigned char *)base + NOALLOC_COUNTS_BYTES;
    return epsr_atogen(box, npt1, sizefactor, dmax, rminex, cfrac, ycoh, n1extr, n2extr, natomr, ngrsamples_io, ran1,
                       wav, ldw, potex, counts, work, NOALLOC_WORK_BYTES, stream);
}
