// press.cu -- press (ato_manipulation_rev4.py:3903-4062): intermolecular energy and virial of
// the stored pairs, without three-body terms or coordination constraints.
//
// One CTA per molecule im (all but the last), one thread per stored partner slot: for a
// partner jm > im the thread sums, over im's atoms (outer) and jm's atoms (inner), the
// energy enwt + enpot into a float32 ergold and the virial terms into ergnew -- a float32
// add of the EP term prwt, then a double add of the reference-potential term prpot, stored
// back as float32 -- exactly as the reference (:3960-4040).  Pairs count only while the
// bin iz <= npt1.  The reduction then sums ergold in float32 and ergnew in double over
// (im, slot) in store order (:4041-4044): one thread, sequentially, for the reference's
// bits (strict), or in parallel in double (fast).
#include <string.h>

#include "common.cuh"

namespace epsr {

constexpr int PR_THREADS = 256;
constexpr int PR_MAXAT = 64;   // atoms of a molecule held in shared memory

struct PressDev {
    Lattice L;
    const float4 *tab;         // [npairs*ld] {xavs, xavs1, ecoul, ecoul1}
    const float *xstar;        // [ld]
    float stepcl;
    int npt1, ld, ntype, M;
    const int32_t *naf, *nato, *npairref, *nergpairm, *molergpair;
    const float *xadd, *yadd, *zadd;
    const float4 *pos;         // absolute atom positions, type bits in .w
    float *ergold, *ergnew;    // [nmol*M]
    double *sums;              // [2] {sumc, presst}
};

__global__ void __launch_bounds__(PR_THREADS) press_pairs_kernel(PressDev P) {
    extern __shared__ int list[];   // [M] slots with a partner jm > im, by partner atom count
    __shared__ float4 sa[PR_MAXAT];
    __shared__ int bk[PR_MAXAT + 2];
    const int im = blockIdx.x;
    const int a0 = P.naf[im], na = P.nato[im];
    const bool in_smem = na <= PR_MAXAT;   // larger molecules are read from global memory
    if (in_smem)
        for (int i = threadIdx.x; i < na; i += blockDim.x) sa[i] = P.pos[a0 + i];
    for (int i = threadIdx.x; i < PR_MAXAT + 2; i += blockDim.x) bk[i] = 0;
    __syncthreads();
    const float xc1 = P.xadd[im], yc1 = P.yadd[im], zc1 = P.zadd[im];
    const int nn = P.nergpairm[im];
    const size_t row = (size_t)im * P.M;
    // slots whose partner comes later are evaluated, listed by the partner's atom count so the
    // lanes of a warp run loops of the same length; the others hold 0
    auto nb_of = [&](int s) -> int {
        const int jm = P.molergpair[row + s];
        return jm > im ? min(P.nato[jm], PR_MAXAT) : 0;
    };
    for (int s = threadIdx.x; s < nn; s += blockDim.x) {
        const int nb = nb_of(s);
        if (nb > 0) {
            atomicAdd(&bk[nb], 1);
        } else {
            P.ergold[row + s] = 0.0f;
            P.ergnew[row + s] = 0.0f;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // bk[b] -> first list position of atom count b; bk[PR_MAXAT+1] = total
        int a = 0;
        for (int b = 0; b <= PR_MAXAT; ++b) {
            const int t = bk[b];
            bk[b] = a;
            a += t;
        }
        bk[PR_MAXAT + 1] = a;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < nn; s += blockDim.x) {
        const int nb = nb_of(s);
        if (nb > 0) list[atomicAdd(&bk[nb], 1)] = s;
    }
    __syncthreads();
    const int total = bk[PR_MAXAT + 1];
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int s = list[q];
        const int jm = P.molergpair[row + s];
        float eo = 0.0f, en = 0.0f;
        {
            // separation of the centres (the same for every atom pair of im, jm)
            float xcdif = __fsub_rn(P.xadd[jm], xc1), ycdif = __fsub_rn(P.yadd[jm], yc1),
                  zcdif = __fsub_rn(P.zadd[jm], zc1);
            minimagec(P.L, xcdif, ycdif, zcdif);
            const int b0 = P.naf[jm], nb = P.nato[jm];
            for (int ia = 0; ia < na; ++ia) {
                const float4 p1 = in_smem ? sa[ia] : __ldg(P.pos + a0 + ia);
                const int32_t *prow = P.npairref + __float_as_int(p1.w) * P.ntype;
                for (int ja = 0; ja < nb; ++ja) {
                    const float4 p2 = __ldg(P.pos + b0 + ja);
                    float xdif = __fsub_rn(p2.x, p1.x), ydif = __fsub_rn(p2.y, p1.y), zdif = __fsub_rn(p2.z, p1.z);
                    minimagec(P.L, xdif, ydif, zdif);
                    const float dsq =
                        __fadd_rn(__fadd_rn(__fmul_rn(xdif, xdif), __fmul_rn(ydif, ydif)), __fmul_rn(zdif, zdif));
                    const float dtest = __fsqrt_rn(dsq);
                    const int iz = ifix(__fdiv_rn(dtest, P.stepcl)) + 2;
                    // branch-free: tables read at iz clamped into 2..npt1, the sums kept unchanged
                    // outside that range, so consecutive pairs' loads can be in flight together
                    const bool in = iz >= 2 && iz <= P.npt1;
                    const int izc = min(max(iz, 2), P.npt1);
                    const int icref = __ldg(prow + __float_as_int(p2.w));
                    const float4 t = __ldg(P.tab + (size_t)icref * P.ld + izc);       // bin iz
                    const float4 tm = __ldg(P.tab + (size_t)icref * P.ld + izc - 1);  // bin iz-1
                    const float dtdif = __fsub_rn(dtest, __ldg(P.xstar + izc));
                    const float prfac =
                        dtest > 0.0f ? __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(xcdif, xdif), __fmul_rn(ycdif, ydif)),
                                                           __fmul_rn(zcdif, zdif)),
                                                 dtest)
                                     : 0.0f;
                    const float enpot = __fadd_rn(t.z, __fmul_rn(t.w, dtdif));
                    const double prpot = (double)__fmul_rn(__fmul_rn(0.5f, __fadd_rn(t.w, tm.w)), prfac);
                    const float enwt = __fadd_rn(t.x, __fmul_rn(t.y, dtdif));
                    const float prwt = __fmul_rn(__fmul_rn(0.5f, __fadd_rn(t.y, tm.y)), prfac);
                    const float eo2 = __fadd_rn(__fadd_rn(eo, enwt), enpot);
                    const float en2 = __double2float_rn(__dadd_rn((double)__fadd_rn(en, prwt), prpot));
                    eo = in ? eo2 : eo;
                    en = in ? en2 : en;
                }
            }
        }
        P.ergold[row + s] = eo;
        P.ergnew[row + s] = en;
    }
}

// sumc in float32 and presst in double over (im, slot) in store order, one thread
__global__ void press_sum_strict_kernel(PressDev P, int nmol) {
    float sumc = 0.0f;
    double presst = 0.0;
    for (int im = 0; im < nmol - 1; ++im) {
        const size_t row = (size_t)im * P.M;
        const int nn = P.nergpairm[im];
        for (int s = 0; s < nn; ++s) {
            sumc = __fadd_rn(sumc, P.ergold[row + s]);
            presst = __dadd_rn(presst, (double)P.ergnew[row + s]);
        }
    }
    P.sums[0] = (double)sumc;
    P.sums[1] = presst;
}

// both sums in double, in parallel (one CTA; a fixed order, so the result is reproducible):
// warp w takes molecules w, w+32, ..., its lanes the slots of each
__global__ void __launch_bounds__(1024) press_sum_fast_kernel(PressDev P, int nmol) {
    __shared__ double r0[32], r1[32];
    double a = 0.0, b = 0.0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int im = wid; im < nmol - 1; im += nwarp) {
        const size_t row = (size_t)im * P.M;
        const int nn = P.nergpairm[im];
        for (int s = lane; s < nn; s += 32) {
            a += (double)P.ergold[row + s];
            b += (double)P.ergnew[row + s];
        }
    }
    a = warp_sum_d(a);
    b = warp_sum_d(b);
    if (lane == 0) {
        r0[wid] = a;
        r1[wid] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < nwarp; ++w) {
            ta += r0[w];
            tb += r1[w];
        }
        P.sums[0] = (double)(float)ta;
        P.sums[1] = tb;
    }
}

}  // namespace epsr

using namespace epsr;

static inline size_t pr_al256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int64_t epsr_press_scratch_bytes(int32_t nmol, int32_t nnbrefmax) {
    return (int64_t)(2 * pr_al256(sizeof(float) * (size_t)nmol * (size_t)nnbrefmax) + pr_al256(sizeof(double) * 2));
}

extern "C" int epsr_press(const epsr_box_t *box, const epsr_store_t *store, int32_t npt1, void *scratch,
                          int64_t scratch_bytes, int32_t strict, double *sums_host, void *stream) {
    if (!box || !store || !scratch || !sums_host || !box->pos) {
        epsr_set_error("epsr_press: null pointer");
        return EPSR_ERR_ARG;
    }
    if (npt1 < 2 || npt1 >= box->ld) {
        epsr_set_error("epsr_press: npt1 %d outside 2..ld-1 (ld %d)", npt1, box->ld);
        return EPSR_ERR_ARG;
    }
    const int nmol = box->nmol, M = store->nnbrefmax;
    if (scratch_bytes < epsr_press_scratch_bytes(nmol, M)) {
        epsr_set_error("epsr_press: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    PressDev P;
    memset(&P, 0, sizeof(P));
    P.L.cubic = box->cubic;
    P.L.alatx = box->lat[0];
    P.L.blatx = box->lat[1];
    P.L.clatx = box->lat[2];
    P.L.blaty = box->lat[3];
    P.L.claty = box->lat[4];
    P.L.clatz = box->lat[5];
    P.tab = (const float4 *)box->tab;
    P.xstar = box->xstar;
    P.stepcl = box->stepcl;
    P.npt1 = npt1;
    P.ld = box->ld;
    P.ntype = box->ntype;
    P.M = M;
    P.naf = box->naf;
    P.nato = box->nato;
    P.npairref = box->npairref;
    P.nergpairm = store->nergpairm;
    P.molergpair = store->molergpair;
    P.xadd = box->xadd;
    P.yadd = box->yadd;
    P.zadd = box->zadd;
    P.pos = (const float4 *)box->pos;
    char *p = (char *)scratch;
    P.ergold = (float *)p;
    p += pr_al256(sizeof(float) * (size_t)nmol * M);
    P.ergnew = (float *)p;
    p += pr_al256(sizeof(float) * (size_t)nmol * M);
    P.sums = (double *)p;
    int rc = epsr_box_positions(box, stream);
    if (rc) return rc;
    if (nmol > 1) {
        const size_t list_bytes = sizeof(int) * (size_t)M;
        if (list_bytes > 48 * 1024) EPSR_SMEM_OPTIN(press_pairs_kernel);
        press_pairs_kernel<<<nmol - 1, PR_THREADS, list_bytes, s>>>(P);
        EPSR_CUDA(cudaGetLastError());
        if (strict) press_sum_strict_kernel<<<1, 1, 0, s>>>(P, nmol);
        else press_sum_fast_kernel<<<1, 1024, 0, s>>>(P, nmol);
        EPSR_CUDA(cudaGetLastError());
        EPSR_D2H(sums_host, P.sums, sizeof(double) * 2, s);
    } else {
        sums_host[0] = 0.0;
        sums_host[1] = 0.0;
    }
    return EPSR_OK;
}
