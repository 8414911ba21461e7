// store.cu -- fmolec1 (ato_manipulation_rev4.py:2374-2528): the pair-energy store.
//
// The reference walks cells in order and, for every molecule im of a cell, evaluates
// en_mole_pair(im, jm) for the molecules jm > im of the cell's neighbour region, storing
// the nonzero ones from the region's second entry on (the store loop increments before
// use, :2466-2474).  Store index g numbers the intramolecular entries first (molecule
// order, nonzero only) and then the pairs in (visit position, region index) order; each
// molecule's row lists its entries in increasing g (set_ergpair ergpairreference.py:103).
//
// Device plan: (1) region lists per cell; (2) per visit position, count nonzero pairs;
// (3) scans give every pair its g; (4) rewrite pairs at g and append (g, partner) to both
// molecules' rows; (5) sort each row by g.  Pair energies are evaluated once, in the
// reference's operation order (so the store is bit-identical), by the counting pass, which
// keeps them for the writing pass in an nmol x nnbrefmax buffer.
#include <math.h>

#include "common.cuh"

namespace epsr {

constexpr int FM_THREADS = 256;   // threads of a visit position's CTA (its region entries)
constexpr int FM_MAXAT = 64;      // atom-count buckets of the evaluation list (larger share the last)

struct BoxDev {
    Lattice L;
    Tables T;
    const int32_t *naf, *nato, *itype, *npairref;
    const float4 *pos;
    int ntype;
};

__device__ __forceinline__ float en_mole_pair_dev(const BoxDev &B, int im, int jm) {
    float sume = 0.0f;
    const int a0 = B.naf[im], a1 = a0 + B.nato[im];
    const int b0 = B.naf[jm], b1 = b0 + B.nato[jm];
    for (int ia = a0; ia < a1; ++ia) {
        const float4 p1 = B.pos[ia];
        const int it = __float_as_int(p1.w);
        for (int ja = b0; ja < b1; ++ja) {
            const float4 p2 = B.pos[ja];
            const int icref = __ldg(B.npairref + it * B.ntype + __float_as_int(p2.w));
            sume = __fadd_rn(sume, pair_energy(B.L, B.T, p1, p2, icref));
        }
    }
    return sume;
}

__device__ __forceinline__ int fold(int x, int n) {
    while (x < 0) x += n;
    while (x >= n) x -= n;
    return x;
}

// Block-wide exclusive scan (<= 32 warps); *total = block sum.
__device__ __forceinline__ int bscan(int v, int *total) {
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
    int r = wp[wid] + incl - v;
    *total = wp[32];
    __syncthreads();
    return r;
}

// (1) region list of every cell (make_neighbour_list_from_cells cellneighbourlist.py:187)
__global__ void region_build_kernel(const int32_t *start, const int32_t *mols, const int32_t *offsets, int noff,
                                    int na, int nb, int nc, int M, int32_t *reg, int32_t *nn, int32_t *err) {
    extern __shared__ int32_t sh[];  // [2*noff]: cell, prefix
    const int c0 = blockIdx.x;
    const int icc = c0 / (na * nb);
    const int ibb = (c0 - icc * na * nb) / na;
    const int iaa = c0 - na * (ibb + nb * icc);
    int carry = 0;
    for (int base = 0; base < noff; base += blockDim.x) {
        int k = base + threadIdx.x;
        int cnt = 0, cell = 0;
        if (k < noff) {
            int a = fold(iaa + offsets[3 * k], na), b = fold(ibb + offsets[3 * k + 1], nb),
                c = fold(icc + offsets[3 * k + 2], nc);
            cell = a + na * (b + nb * c);
            cnt = start[cell + 1] - start[cell];
        }
        int tot;
        int pre = bscan(cnt, &tot);
        if (k < noff) {
            sh[2 * k] = cell;
            sh[2 * k + 1] = carry + pre;
        }
        carry += tot;
    }
    __syncthreads();
    if (carry > M) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    if (threadIdx.x == 0) nn[c0] = carry;
    for (int k = threadIdx.x; k < noff; k += blockDim.x) {
        const int cell = sh[2 * k], p0 = sh[2 * k + 1];
        const int s = start[cell], e = start[cell + 1];
        for (int q = s; q < e; ++q) reg[(size_t)c0 * M + p0 + (q - s)] = mols[q];
    }
}

struct Prefilter {
    int on;
    float cut;          // (izcut-1)*stepcl with margin, box units
    const float *rad;   // [nmol] molecule radius (box units)
    const float *xadd, *yadd, *zadd;
};

__device__ __forceinline__ bool far_apart(const Prefilter &P, int im, int jm) {
    if (!P.on) return false;
    float xd = P.xadd[jm] - P.xadd[im], yd = P.yadd[jm] - P.yadd[im], zd = P.zadd[jm] - P.zadd[im];
    xd -= rintf(xd);
    yd -= rintf(yd);
    zd -= rintf(zd);
    float d = sqrtf(xd * xd + yd * yd + zd * zd);
    return d - P.rad[im] - P.rad[jm] > P.cut;
}

// (2) the pair energies of each visit position's region entries (0 where not evaluated),
// and the count of nonzero ones
__global__ void __launch_bounds__(FM_THREADS) fm_count_kernel(BoxDev B, Prefilter P, const int32_t *visit,
                                                              const int32_t *molcellno, const int32_t *reg,
                                                              const int32_t *nn, int M, float *ebuf, int32_t *cnt) {
    extern __shared__ int list[];   // [M] region entries to evaluate, by partner atom count
    __shared__ int bk[FM_MAXAT + 2];
    const int v = blockIdx.x;
    const int im = visit[v];
    const int c = molcellno[im] - 1;
    const int n = nn[c];
    for (int i = threadIdx.x; i < FM_MAXAT + 2; i += blockDim.x) bk[i] = 0;
    __syncthreads();
    // entries evaluated: partner later in molecule order and not certainly beyond the cutoff;
    // the others store 0.  Listing them by the partner's atom count gives the lanes of a warp
    // loops of the same length.
    auto nb_of = [&](int inn) -> int {
        const int jm = reg[(size_t)c * M + inn];
        return (jm > im && !far_apart(P, im, jm)) ? min(B.nato[jm], FM_MAXAT) : 0;
    };
    for (int inn = 1 + threadIdx.x; inn < n; inn += blockDim.x) {
        const int nb = nb_of(inn);
        if (nb > 0) atomicAdd(&bk[nb], 1);
        else ebuf[(size_t)v * M + inn] = 0.0f;
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // bk[b] -> first list position of atom count b; bk[FM_MAXAT+1] = total
        int a = 0;
        for (int b = 0; b <= FM_MAXAT; ++b) {
            const int t = bk[b];
            bk[b] = a;
            a += t;
        }
        bk[FM_MAXAT + 1] = a;
    }
    __syncthreads();
    for (int inn = 1 + threadIdx.x; inn < n; inn += blockDim.x) {
        const int nb = nb_of(inn);
        if (nb > 0) list[atomicAdd(&bk[nb], 1)] = inn;
    }
    __syncthreads();
    const int total = bk[FM_MAXAT + 1];
    int mine = 0;
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int inn = list[q];
        const float e = en_mole_pair_dev(B, im, reg[(size_t)c * M + inn]);
        ebuf[(size_t)v * M + inn] = e;
        if (e != 0.0f) ++mine;
    }
    int tot;
    bscan(mine, &tot);
    if (threadIdx.x == 0) cnt[v] = tot;
}

// (3) exclusive scan over visit positions / molecules (single block)
__global__ void scan1_kernel(const int32_t *in, int n, int32_t *out, int flag_nonzero_float, const float *fin) {
    int carry = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = 0;
        if (i < n) v = flag_nonzero_float ? (fin[i] != 0.0f ? 1 : 0) : in[i];
        int tot;
        int pre = bscan(v, &tot);
        if (i < n) out[i] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// intramolecular entries: slot 0 of molecules with nonzero intra energy
__global__ void fm_intra_kernel(const float *eintra, const int32_t *iidx, int nmol, int M, float *ergpair,
                                int32_t *rowcnt, int32_t *molergpair, int32_t *ergpairref) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    if (eintra[m] != 0.0f) {
        const int g = iidx[m];
        ergpair[g] = eintra[m];
        molergpair[(size_t)m * M] = m;
        ergpairref[(size_t)m * M] = g;
        rowcnt[m] = 1;
    } else {
        rowcnt[m] = 0;
    }
}

// (4) write the pairs at their store index and append to both rows (unordered)
__global__ void __launch_bounds__(FM_THREADS) fm_write_kernel(const int32_t *visit, const int32_t *molcellno,
                                                              const int32_t *reg, const int32_t *nn, int M,
                                                              const float *ebuf, const int32_t *off, int nintra,
                                                              float *ergpair, int32_t *rowcnt, int32_t *molergpair,
                                                              int32_t *ergpairref, int32_t *err) {
    const int v = blockIdx.x;
    const int im = visit[v];
    const int c = molcellno[im] - 1;
    const int n = nn[c];
    int carry = 0;
    for (int base = 1; base < n; base += blockDim.x) {
        const int inn = base + threadIdx.x;
        float e = 0.0f;
        int jm = -1, flag = 0;
        if (inn < n) {
            jm = reg[(size_t)c * M + inn];
            e = ebuf[(size_t)v * M + inn];
            flag = e != 0.0f;
        }
        int tot;
        const int rank = carry + bscan(flag, &tot);
        if (flag) {
            const int g = nintra + off[v] + rank;
            ergpair[g] = e;
            int s1 = atomicAdd(rowcnt + im, 1);
            int s2 = atomicAdd(rowcnt + jm, 1);
            if (s1 < M && s2 < M) {
                molergpair[(size_t)im * M + s1] = jm;
                ergpairref[(size_t)im * M + s1] = g;
                molergpair[(size_t)jm * M + s2] = im;
                ergpairref[(size_t)jm * M + s2] = g;
            } else {
                atomicExch(err, 2);
            }
        }
        carry += tot;
    }
}

// (5) sort each molecule's row by store index; refs become 1-based
__global__ void fm_sort_kernel(int M, const int32_t *rowcnt, int32_t *nergpairm, int32_t *molergpair,
                               int32_t *ergpairref, int cap_pow2) {
    extern __shared__ int32_t sk[];  // keys [cap], vals [cap]
    const int m = blockIdx.x;
    const int n = min(rowcnt[m], M);
    int32_t *key = sk, *val = sk + cap_pow2;
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    for (int i = threadIdx.x; i < np2; i += blockDim.x) {
        if (i < n) {
            key[i] = ergpairref[(size_t)m * M + i];
            val[i] = molergpair[(size_t)m * M + i];
        } else {
            key[i] = 0x7fffffff;
            val[i] = -1;
        }
    }
    __syncthreads();
    for (int k = 2; k <= np2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    bool up = (i & k) == 0;
                    int a = key[i], b = key[ixj];
                    if ((a > b) == up) {
                        key[i] = b;
                        key[ixj] = a;
                        int t = val[i];
                        val[i] = val[ixj];
                        val[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        ergpairref[(size_t)m * M + i] = key[i] + 1;
        molergpair[(size_t)m * M + i] = val[i];
    }
    if (threadIdx.x == 0) nergpairm[m] = n;
}

// mirror index: the two entries that reference one energy slot point at each other
__global__ void mirror_claim_kernel(int nmol, int M, const int32_t *nergpairm, const int32_t *ergpairref,
                                    int32_t *owners) {
    const int m = blockIdx.x;
    const int n = nergpairm[m];
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const int e = m * M + s;
        const int r = ergpairref[e] - 1;
        if (atomicCAS(owners + 2 * r, -1, e) != -1) owners[2 * r + 1] = e;
    }
}

__global__ void mirror_set_kernel(int nmol, int M, const int32_t *nergpairm, const int32_t *ergpairref,
                                  const int32_t *owners, int32_t *mirror) {
    const int m = blockIdx.x;
    const int n = nergpairm[m];
    for (int s = threadIdx.x; s < M; s += blockDim.x) {
        const int e = m * M + s;
        int v = -1;
        if (s < n) {
            const int r = ergpairref[e] - 1;
            const int a = owners[2 * r], b = owners[2 * r + 1];
            v = a == e ? b : a;
        }
        mirror[e] = v;
    }
}

__global__ void mol_radius_kernel(const int32_t *naf, const int32_t *nato, const float *xa, const float *ya,
                                  const float *za, int nmol, float *rad) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmol) return;
    float r = 0.0f;
    for (int a = naf[m]; a < naf[m] + nato[m]; ++a) r = fmaxf(r, sqrtf(xa[a] * xa[a] + ya[a] * ya[a] + za[a] * za[a]));
    rad[m] = r * 1.0001f + 1.0e-6f;
}

// ftest / ftestb: strict = the reference's sequential float sums
__global__ void fm_sums_kernel(const float *ergpair, int nintra, int ntot, const float *eintra, int nmol,
                               int strict, float *out2) {
    if (strict) {
        if (threadIdx.x == 0) {
            float ft = 0.0f, fb = 0.0f;
            for (int m = 0; m < nmol; ++m) fb = __fadd_rn(fb, eintra[m]);
            for (int g = nintra; g < ntot; ++g) ft = __fadd_rn(ft, ergpair[g]);
            out2[0] = __fdiv_rn(ft, (float)nmol);
            out2[1] = __fdiv_rn(fb, (float)nmol);
        }
        return;
    }
    double a = 0.0, b = 0.0;
    for (int g = nintra + threadIdx.x; g < ntot; g += blockDim.x) a += ergpair[g];
    for (int m = threadIdx.x; m < nmol; m += blockDim.x) b += eintra[m];
    __shared__ double sa[32], sb[32];
    a = warp_sum_d(a);
    b = warp_sum_d(b);
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = a;
        sb[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            ta += sa[w];
            tb += sb[w];
        }
        out2[0] = (float)(ta / nmol);
        out2[1] = (float)(tb / nmol);
    }
}

BoxDev make_boxdev(const epsr_box_t *b) {
    BoxDev B;
    B.L.cubic = b->cubic;
    B.L.alatx = b->lat[0];
    B.L.blatx = b->lat[1];
    B.L.clatx = b->lat[2];
    B.L.blaty = b->lat[3];
    B.L.claty = b->lat[4];
    B.L.clatz = b->lat[5];
    B.T.tab = (const float4 *)b->tab;
    B.T.xstar = b->xstar;
    B.T.ld = b->ld;
    B.T.npt2 = b->npt2;
    B.T.izcut = b->izcut < b->npt2 ? b->izcut : b->npt2;
    B.T.stepcl = b->stepcl;
    B.naf = b->naf;
    B.nato = b->nato;
    B.itype = b->itype;
    B.npairref = b->npairref;
    B.pos = (const float4 *)b->pos;
    B.ntype = b->ntype;
    return B;
}

__global__ void positions_kernel(const int32_t *naf, const int32_t *nato, const int32_t *itype, const float *xa,
                                 const float *ya, const float *za, const float *xadd, const float *yadd,
                                 const float *zadd, int nmol, float4 *pos) {
    int m = blockIdx.x;
    for (int a = naf[m] + threadIdx.x; a < naf[m] + nato[m]; a += blockDim.x)
        pos[a] = make_float4(__fadd_rn(xa[a], xadd[m]), __fadd_rn(ya[a], yadd[m]), __fadd_rn(za[a], zadd[m]),
                             __int_as_float(itype[a]));
}

}  // namespace epsr

using namespace epsr;

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int epsr_box_positions(const epsr_box_t *box, void *stream) {
    if (!box || !box->pos) {
        epsr_set_error("epsr_box_positions: null pointer");
        return EPSR_ERR_ARG;
    }
    positions_kernel<<<box->nmol, 32, 0, (cudaStream_t)stream>>>(box->naf, box->nato, box->itype, box->xa, box->ya,
                                                                 box->za, box->xadd, box->yadd, box->zadd,
                                                                 box->nmol, (float4 *)box->pos);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int64_t epsr_fmolec1_scratch_bytes(int32_t nmol, int32_t ncell, int32_t M) {
    size_t b = 0;
    b += align256(sizeof(int32_t) * (size_t)ncell * M);  // reg
    b += align256(sizeof(int32_t) * (size_t)ncell);      // nn
    b += 3 * align256(sizeof(int32_t) * ((size_t)nmol + 1));  // cnt, off, iidx
    b += align256(sizeof(int32_t) * (size_t)nmol);      // rowcnt
    b += align256(sizeof(float) * (size_t)nmol);        // rad
    b += align256(sizeof(int32_t) * 8);                 // err + misc
    b += align256(sizeof(float) * 2);
    b += align256(sizeof(int32_t) * 2 * ((size_t)nmol + (size_t)nmol * M / 2 + 16));  // mirror owners
    b += align256(sizeof(float) * (size_t)nmol * M);    // pair energies of the region entries
    return (int64_t)b;
}

extern "C" int epsr_fmolec1(const epsr_box_t *box, const epsr_cells_t *cells, const float *eintra,
                            epsr_store_t *store, void *scratch, int64_t scratch_bytes, int32_t strict,
                            float *out2_host, void *stream) {
    if (!box || !cells || !eintra || !store || !scratch || !out2_host) {
        epsr_set_error("epsr_fmolec1: null pointer");
        return EPSR_ERR_ARG;
    }
    const int nmol = box->nmol, ncell = cells->ncell, M = store->nnbrefmax;
    if (scratch_bytes < epsr_fmolec1_scratch_bytes(nmol, ncell, M)) {
        epsr_set_error("epsr_fmolec1: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += align256(bytes);
        return (void *)r;
    };
    int32_t *reg = (int32_t *)take(sizeof(int32_t) * (size_t)ncell * M);
    int32_t *nn = (int32_t *)take(sizeof(int32_t) * (size_t)ncell);
    int32_t *cnt = (int32_t *)take(sizeof(int32_t) * ((size_t)nmol + 1));
    int32_t *off = (int32_t *)take(sizeof(int32_t) * ((size_t)nmol + 1));
    int32_t *iidx = (int32_t *)take(sizeof(int32_t) * ((size_t)nmol + 1));
    int32_t *rowcnt = (int32_t *)take(sizeof(int32_t) * (size_t)nmol);
    float *rad = (float *)take(sizeof(float) * (size_t)nmol);
    int32_t *err = (int32_t *)take(sizeof(int32_t) * 8);
    float *sums = (float *)take(sizeof(float) * 2);
    const size_t own_n = 2 * ((size_t)nmol + (size_t)nmol * M / 2 + 16);
    int32_t *owners = (int32_t *)take(sizeof(int32_t) * own_n);
    float *ebuf = (float *)take(sizeof(float) * (size_t)nmol * M);
    EPSR_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t) * 8, s));

    BoxDev B = make_boxdev(box);
    Prefilter P;
    P.on = box->cubic ? 1 : 0;
    P.cut = (float)((double)(B.T.izcut - 1) * (double)box->stepcl * 1.00001 + 1.0e-6);
    P.rad = rad;
    P.xadd = box->xadd;
    P.yadd = box->yadd;
    P.zadd = box->zadd;
    const int noff = cells->ncellneighb;
    positions_kernel<<<nmol, 32, 0, s>>>(box->naf, box->nato, box->itype, box->xa, box->ya, box->za, box->xadd,
                                         box->yadd, box->zadd, nmol, (float4 *)box->pos);
    mol_radius_kernel<<<(nmol + 127) / 128, 128, 0, s>>>(box->naf, box->nato, box->xa, box->ya, box->za, nmol, rad);
    region_build_kernel<<<ncell, 256, sizeof(int32_t) * 2 * (size_t)noff, s>>>(
        cells->cell_start, cells->cell_mols, cells->offsets, noff, cells->ncelldiva, cells->ncelldivb,
        cells->ncelldivc, M, reg, nn, err);
    const size_t list_bytes = sizeof(int) * (size_t)M;
    if (list_bytes > 48 * 1024) EPSR_SMEM_OPTIN(fm_count_kernel);
    EPSR_TIMED("fm_count_kernel", s, fm_count_kernel<<<nmol, FM_THREADS, list_bytes, s>>>(B, P, cells->cell_mols, cells->molcellno, reg, nn, M, ebuf,
                                                         cnt));
    scan1_kernel<<<1, 1024, 0, s>>>(cnt, nmol, off, 0, nullptr);
    scan1_kernel<<<1, 1024, 0, s>>>(nullptr, nmol, iidx, 1, eintra);
    EPSR_CUDA(cudaGetLastError());
    int32_t totals[2];
    EPSR_D2H(&totals[0], iidx + nmol, sizeof(int32_t), s);
    EPSR_D2H(&totals[1], off + nmol, sizeof(int32_t), s);
    const int nintra = totals[0], npair = totals[1];
    const int64_t ntot = (int64_t)nintra + npair;
    if (ntot > store->capacity) {
        epsr_set_error("epsr_fmolec1: store capacity %d < %lld entries", store->capacity, (long long)ntot);
        return EPSR_ERR_CAPACITY;
    }
    fm_intra_kernel<<<(nmol + 127) / 128, 128, 0, s>>>(eintra, iidx, nmol, M, store->ergpair, rowcnt,
                                                      store->molergpair, store->ergpairref);
    fm_write_kernel<<<nmol, FM_THREADS, 0, s>>>(cells->cell_mols, cells->molcellno, reg, nn, M, ebuf, off, nintra,
                                                store->ergpair, rowcnt, store->molergpair, store->ergpairref, err);
    int maxrow = M;
    int cap = 1;
    while (cap < maxrow) cap <<= 1;
    size_t shm = sizeof(int32_t) * 2 * (size_t)cap;
    if (shm > 200 * 1024) {
        epsr_set_error("epsr_fmolec1: nnbrefmax %d too large for the row sort", M);
        return EPSR_ERR_CAPACITY;
    }
    if (shm > 48 * 1024) EPSR_SMEM_OPTIN(fm_sort_kernel);
    fm_sort_kernel<<<nmol, 256, shm, s>>>(M, rowcnt, store->nergpairm, store->molergpair, store->ergpairref, cap);
    fm_sums_kernel<<<1, strict ? 32 : 1024, 0, s>>>(store->ergpair, nintra, (int)ntot, eintra, nmol, strict, sums);
    if (store->mirror) {
        if ((size_t)2 * ntot > own_n) {
            epsr_set_error("epsr_fmolec1: mirror scratch too small");
            return EPSR_ERR_CAPACITY;
        }
        EPSR_CUDA(cudaMemsetAsync(owners, 0xff, sizeof(int32_t) * 2 * (size_t)ntot, s));
        mirror_claim_kernel<<<nmol, 128, 0, s>>>(nmol, M, store->nergpairm, store->ergpairref, owners);
        mirror_set_kernel<<<nmol, 128, 0, s>>>(nmol, M, store->nergpairm, store->ergpairref, owners, store->mirror);
    }
    EPSR_CUDA(cudaGetLastError());
    int32_t herr[1];
    int32_t hn = (int32_t)ntot;
    EPSR_H2D(store->nergpair, &hn, sizeof(int32_t), s);
    EPSR_D2H(herr, err, sizeof(int32_t), s);
    EPSR_D2H(out2_host, sums, sizeof(float) * 2, s);
    if (herr[0]) {
        epsr_set_error("epsr_fmolec1: neighbour region or row exceeds nnbrefmax=%d (code %d)", M, herr[0]);
        return EPSR_ERR_CAPACITY;
    }
    return EPSR_OK;
}
