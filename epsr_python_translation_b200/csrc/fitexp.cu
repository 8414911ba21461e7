// fitexp.cu -- fit_expansion (epsr_standalone_rev3.py:4806-4921) on one thread-block cluster.
//
// The Monte Carlo fit is a chain of trials: perturb every coefficient (one ran1 draw each),
// evaluate chi^2 over all Q rows, Metropolis-accept (one more draw when 0 < exponent <= 20),
// smooth the coefficients every nfreq acceptances (smoop auxiliary_routines.py:744).
//
// The basis rows are split over the CTAs of a cluster so that each CTA keeps its rows in
// shared memory for the whole fit.  Per trial a CTA evaluates its rows (expand :4924, the
// sequential clamped sum of a row) and every CTA then forms the same chi^2 -- in the
// reference's row order through distributed shared memory (strict), or as a double sum
// (fast) -- so all CTAs take the same decisions without a second exchange.  A row is first
// summed without the clamp while tracking the largest partial sum; only a row whose partial
// sums could reach the clamp (|sum| > e^25) is summed again with it, so the result is the
// reference's either way.
//
// ran1: every CTA runs the same stream.  One warp generates the values of the next trial
// while thread 0 forms chi^2, keeping generation off the critical path; the state the
// reference leaves after the fit is rebuilt from the generator's batch checkpoints.
#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace epsr {

constexpr int FX_THREADS = 512;
constexpr int FX_GEN_WARP = 1;    // the warp that generates ran1 values
constexpr int FX_RING = 1024;     // ran1 values held (power of two)
constexpr int FX_CK = 64;         // batch checkpoints (power of two)
constexpr int FX_CKW = 36;        // ints per checkpoint: idum, iy, iv[32], pad[2]

struct FxDev {
    const float *yin, *expr;  // expr[(i-1)*nterms + m] (1-based flat, row-major by Q)
    float *yout, *wt_g, *wtold_g;
    int nmin, npt, ncfirst, nterms, nits, nfreq, strict, rpc;  // rpc: rows per CTA
    int32_t *ran1;
    float *scal;              // {stepr, acceptr, rejrat, chisq}
    long long *trials;
};

size_t fx_smem_bytes(int nt, int rpc, int ncta) {
    size_t f = (size_t)nt * rpc + 3 * (size_t)rpc + 2 * (size_t)(nt + 1) + FX_RING;
    size_t b = f * 4;
    b = (b + 15) & ~(size_t)15;
    b += 2 * sizeof(double);
    b += (size_t)FX_CK * FX_CKW * sizeof(int32_t);
    b += (size_t)FX_CK * sizeof(long long);
    b += sizeof(float) * ((size_t)ncta * rpc + 4);
    return b;
}

__global__ void __launch_bounds__(FX_THREADS) fitexp_cluster_kernel(FxDev F) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int ncta = (int)cl.num_blocks();
    extern __shared__ __align__(16) unsigned char fx_raw[];
    const int nt = F.nterms, rpc = F.rpc;
    float *ex = (float *)fx_raw;                    // [nt*rpc] term-major: ex[(m-1)*rpc + r]
    float *sq = ex + (size_t)nt * rpc;              // [2*rpc] double-buffered squared residuals
    float *yr = sq + 2 * rpc;                       // [rpc]
    float *wt = yr + rpc;                           // [nt+1]
    float *wtold = wt + (nt + 1);                   // [nt+1]
    float *ring = wtold + (nt + 1);                 // [FX_RING]
    size_t off = ((size_t)((unsigned char *)(ring + FX_RING) - fx_raw) + 15) & ~(size_t)15;
    double *part = (double *)(fx_raw + off);        // [2] fast-mode partial sums
    int32_t *ck = (int32_t *)(part + 2);            // [FX_CK][FX_CKW]
    long long *ckpos = (long long *)(ck + FX_CK * FX_CKW);  // [FX_CK]
    float *gat = (float *)(ckpos + FX_CK);          // [ncta*rpc] gathered residuals (16-byte aligned)
    __shared__ float s_val;
    __shared__ double s_red[FX_THREADS / 32];
    __shared__ int32_t g_tab[34];

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int row0 = 1 + rank * rpc;  // first (1-based) row of this CTA
    const int nrow = max(0, min(rpc, F.npt - row0 + 1));
    const float summax = exp_r(25.0f);
    const int K = nt - F.ncfirst + 1;  // draws per trial

    for (int idx = tid; idx < nt * rpc; idx += blockDim.x) {
        const int m = idx / rpc, r = idx - m * rpc;
        ex[idx] = r < nrow ? F.expr[1 + (size_t)(row0 - 1 + r) * nt + m] : 0.0f;
    }
    for (int r = tid; r < rpc; r += blockDim.x) yr[r] = r < nrow ? F.yin[row0 + r] : 0.0f;
    for (int i = tid; i <= nt; i += blockDim.x) {
        wtold[i] = F.wtold_g[i];
        wt[i] = wtold[i];
    }
    for (int i = tid; i < FX_CK; i += blockDim.x) ckpos[i] = -1;
    // generator warp state (the shuffle table lives one entry per lane)
    int32_t g_iv = 0, g_idum = 0, g_iy = 0;
    long long g_pos = 0, g_nb = 0;
    uint32_t g_mul = 16807u;
    if (wid == FX_GEN_WARP) {
        g_idum = F.ran1[0];
        g_iy = F.ran1[1];
        g_iv = F.ran1[3 + lane];
        for (int k = 0; k < lane; ++k) g_mul = r1_mulmod(g_mul, 16807u);
    }
    const int32_t mcall0 = F.ran1[2];
    cl.sync();

    // generate values up to stream index `until` (exclusive); warp FX_GEN_WARP only
    auto generate = [&](long long until) {
        if (wid != FX_GEN_WARP) return;
        while (g_pos < until) {
            const int slot = (int)(g_nb & (FX_CK - 1));
            ck[slot * FX_CKW + 2 + lane] = g_iv;
            if (lane == 0) {
                ck[slot * FX_CKW + 0] = g_idum;
                ck[slot * FX_CKW + 1] = g_iy;
                ckpos[slot] = g_pos;
            }
            ++g_nb;
            int32_t mine;
            const int cnt = ran1_warp_batch(g_idum, g_iy, g_iv, g_mul, 32, mine, g_tab);
            if (lane < cnt) ring[(g_pos + lane) & (FX_RING - 1)] = ran1_out(mine);
            g_pos += cnt;
        }
    };

    // chi^2 of the current wt over rows nmin..npt (all CTAs); while thread 0 sums, the
    // generator warp produces values up to `gen_until`.  Optionally writes yout (all rows).
    int buf = 0;
    auto chisq = [&](long long gen_until, bool write_yout, bool strict_sum) -> float {
        float *sqb = sq + buf * rpc;
        double mypart = 0.0;
        // the generator warp works while the others evaluate rows (two batches) and while
        // thread 0 forms chi^2 (the rest)
        generate(gen_until < g_pos + 64 ? gen_until : g_pos + 64);
        if (wid != FX_GEN_WARP) {
            const int w = wid > FX_GEN_WARP ? tid - 32 : tid;  // worker index
            const int nw = blockDim.x - 32;
            for (int r = w; r < nrow; r += nw) {
                const int i = row0 + r;
                float sum = 0.0f, mx = 0.0f;
                for (int m = 1; m <= nt; ++m) {
                    sum = __fadd_rn(sum, __fmul_rn(ex[(m - 1) * rpc + r], wt[m]));
                    mx = fmaxf(mx, fabsf(sum));
                }
                if (mx > summax) {  // the clamp may act: the reference's clamped sum
                    sum = 0.0f;
                    for (int m = 1; m <= nt; ++m) {
                        sum = __fadd_rn(sum, __fmul_rn(ex[(m - 1) * rpc + r], wt[m]));
                        if (fabsf(sum) > summax) sum = fsign(summax, sum);
                    }
                }
                const float term = __fsub_rn(yr[r], sum);
                const float q = __fmul_rn(term, term);
                sqb[r] = q;
                if (i >= F.nmin) mypart += (double)q;
                if (write_yout) F.yout[i] = sum;
            }
        }
        if (!strict_sum) {
            mypart = warp_sum_d(mypart);
            if (lane == 0) s_red[wid] = mypart;
        }
        __syncthreads();
        if (!strict_sum && tid == 0) {
            double t = 0.0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s_red[k];
            part[buf] = t;
        }
        cl.sync();  // every CTA's rows of this buffer are complete
        if (strict_sum) {
            // gather all rows' residuals into this CTA's gather buffer (remote rows through
            // distributed shared memory, in parallel), then sum them in the reference's order
            for (int q = 0; q < ncta; ++q) {
                const float *rs = q == rank ? sqb : cl.map_shared_rank(sq + buf * rpc, q);
                for (int r = tid; r < rpc; r += blockDim.x) gat[q * rpc + r] = rs[r];
            }
            __syncthreads();
            if (tid == 0) {
                const int a = F.nmin - 1, b = F.npt;  // 0-based rows a..b-1
                float c = 0.0f;
                int i = a;
                for (; i < b && (i & 3); ++i) c = __fadd_rn(c, gat[i]);
                const float4 *g4 = (const float4 *)gat;
                for (; i + 3 < b; i += 4) {
                    const float4 v = g4[i >> 2];
                    c = __fadd_rn(c, v.x);
                    c = __fadd_rn(c, v.y);
                    c = __fadd_rn(c, v.z);
                    c = __fadd_rn(c, v.w);
                }
                for (; i < b; ++i) c = __fadd_rn(c, gat[i]);
                s_val = c;
            }
            generate(gen_until);  // the generator warp, while thread 0 sums
        } else {
            generate(gen_until);
        }
        if (!strict_sum && tid == 0) {
            {
                double t = 0.0;
                for (int q = 0; q < ncta; ++q) t += *cl.map_shared_rank(part + buf, q);
                s_val = (float)t;
            }
        }
        __syncthreads();
        buf ^= 1;
        return s_val;
    };

    float stepr = F.scal[0];
    float rejrat = F.scal[2];
    float chisqnew = F.scal[3];
    const float acceptr = 0.05f;
    const int npoints = F.npt - F.nmin + 1;
    long long trials = 0, cursor = 0;
    float wtmax = 0.0f;
    for (int it = 1; it <= nt; ++it) {
        const float a = fabsf(wt[it]);
        wtmax = (a >= wtmax) ? a : wtmax;
    }
    if (stepr < __fmul_rn(1.0e-6f, wtmax)) stepr = __fmul_rn(2.0e-6f, wtmax);
    if (F.nits > 0) {
        int icount = 0;
        chisqnew = chisq(cursor + K, false, F.strict);
        float chisqold = chisqnew;
        float chisqtest = -1.0f;
        int itry = 0;
        while (itry < 10 || (itry < 150 && chisqtest < 1.0e-4f)) {
            ++itry;
            const float accept = __fdiv_rn(__fmul_rn(acceptr, chisqold), (float)npoints);
            rejrat = 0.0f;
            const float chisqstart = __fdiv_rn(chisqold, (float)npoints);
            for (int st = 1; st <= 100; ++st) {
                ++trials;
                // perturb coefficients ncfirst..nterms with the next K values (:4856-4861)
                for (int ic = F.ncfirst + tid; ic <= nt; ic += blockDim.x) {
                    const float u = ring[(cursor + ic - F.ncfirst) & (FX_RING - 1)];
                    const float du = __fsub_rn(__fmul_rn(2.0f, u), 1.0f);
                    if (fabsf(wtold[ic]) < 1.0f) wt[ic] = __fadd_rn(wtold[ic], __fmul_rn(stepr, du));
                    else wt[ic] = __fmul_rn(wtold[ic], __fadd_rn(1.0f, __fmul_rn(stepr, du)));
                }
                cursor += K;
                __syncthreads();
                // the conditional draw of this trial and the next trial's K draws
                chisqnew = chisq(cursor + 1 + K, false, F.strict);
                const float exponent = __fdiv_rn(__fsub_rn(chisqnew, chisqold), accept);
                float test;
                if (exponent > 0.0f && exponent <= 20.0f) {
                    test = __fsub_rn(exp_r(-exponent), ring[cursor & (FX_RING - 1)]);
                    cursor += 1;
                } else if (exponent > 20.0f) {
                    test = -1.0f;
                } else {
                    test = 1.0f;
                }
                if (test >= 0.0f) {
                    ++icount;
                    if (icount == F.nfreq) {
                        icount = 0;
                        if (tid == 0) {  // smoop(ncfirst, nterms, 1, wt)
                            const int n1 = F.ncfirst, n2 = nt;
                            if (!(n2 - 2 < n1)) {
                                float sm_ = 0.0f, sn = wt[n1];
                                float sum1 = __fmul_rn(0.25f, __fadd_rn(sm_, sn));
                                for (int i = n1; i <= n2; ++i) {
                                    sm_ = sn;
                                    sn = (i + 1) <= n2 ? wt[i + 1] : 0.0f;
                                    const float sum2 = __fmul_rn(0.25f, __fadd_rn(sm_, sn));
                                    wt[i] = __fadd_rn(sum1, sum2);
                                    sum1 = sum2;
                                }
                            }
                        }
                        __syncthreads();
                        chisqnew = chisq(cursor + K, false, F.strict);
                    }
                    chisqold = chisqnew;
                    for (int ic = 1 + tid; ic <= nt; ic += blockDim.x) wtold[ic] = wt[ic];
                } else {
                    rejrat = __fadd_rn(rejrat, 1.0f);
                }
                __syncthreads();
            }
            rejrat = __fdiv_rn(rejrat, 100.0f);
            const float chisqfinish = __fdiv_rn(chisqold, (float)npoints);
            if (chisqstart > 0.0f) chisqtest = __fdiv_rn(__fsub_rn(chisqfinish, chisqstart), chisqstart);
            else chisqtest = __fsub_rn(chisqfinish, chisqstart);
            const float rejfac = rejrat > 0.0f ? __fdiv_rn(0.75f, rejrat) : 2.0f;
            stepr = __fmul_rn(stepr, rejfac);
        }
        for (int ic = 1 + tid; ic <= nt; ic += blockDim.x) wt[ic] = wtold[ic];
        __syncthreads();
    }
    // final fit over rows 1..npt, chi^2 from nmin (:4908-4914); the chi^2 is strict here
    chisqnew = chisq(cursor, true, true);
    if (rank == 0) {
        for (int ic = tid; ic <= nt; ic += blockDim.x) {
            F.wt_g[ic] = wt[ic];
            F.wtold_g[ic] = wtold[ic];
        }
        if (tid == 0) {
            F.scal[0] = stepr;
            F.scal[1] = acceptr;
            F.scal[2] = rejrat;
            F.scal[3] = chisqnew;
            *F.trials = trials;
            // the stream state after exactly `cursor` draws: the last batch checkpoint at or
            // before it, advanced one draw at a time
            int best = -1;
            for (int k = 0; k < FX_CK; ++k)
                if (ckpos[k] >= 0 && ckpos[k] <= cursor && (best < 0 || ckpos[k] > ckpos[best])) best = k;
            Ran1 R;
            if (best >= 0) {
                R.idum = ck[best * FX_CKW + 0];
                R.iy = ck[best * FX_CKW + 1];
                for (int i = 0; i < 32; ++i) R.iv[i] = ck[best * FX_CKW + 2 + i];
                for (long long k = ckpos[best]; k < cursor; ++k) ran1_next(R);
            } else {
                ran1_load(R, F.ran1);
            }
            R.mcall = (int32_t)((uint32_t)mcall0 + (uint32_t)cursor);
            ran1_store(R, F.ran1);
        }
    }
    cl.sync();  // no CTA leaves while others may still read its shared memory
}

}  // namespace epsr

using namespace epsr;

static inline size_t al256f(size_t x) { return (x + 255) & ~(size_t)255; }

static int fx_cluster_size(int npt, int nterms, int *rpc_out) {
    const size_t budget = 200 * 1024;
    for (int c = 1; c <= 8; ++c) {
        const int rpc = (npt + c - 1) / c;
        if (fx_smem_bytes(nterms, rpc, c) <= budget) {
            *rpc_out = rpc;
            return c;
        }
    }
    return 0;
}

extern "C" int64_t epsr_fit_expansion_scratch_bytes(int32_t npt, int32_t nterms) {
    (void)npt;
    (void)nterms;
    return (int64_t)(al256f(sizeof(float) * 4) + al256f(sizeof(long long)));
}

extern "C" int epsr_fit_expansion(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                                  float *scal_host, int32_t nmin, int32_t npt, int32_t ncfirst, int32_t nterms,
                                  int32_t nits, int32_t nfreq, int32_t *ran1, void *scratch, int64_t scratch_bytes,
                                  int32_t strict, int64_t *trials_host, void *stream) {
    if (!yin || !expr || !yout || !wt || !wtold || !scal_host || !ran1 || !scratch || !trials_host || npt <= 0 ||
        nterms <= 0 || nmin < 1 || ncfirst < 1 || ncfirst > nterms) {
        epsr_set_error("epsr_fit_expansion: bad arguments");
        return EPSR_ERR_ARG;
    }
    if (scratch_bytes < epsr_fit_expansion_scratch_bytes(npt, nterms)) {
        epsr_set_error("epsr_fit_expansion: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    if (nterms + 64 > FX_RING) {
        epsr_set_error("epsr_fit_expansion: at most %d terms", FX_RING - 64);
        return EPSR_ERR_UNSUPPORTED;
    }
    int rpc = 0;
    const int csize = fx_cluster_size(npt, nterms, &rpc);
    if (!csize) {
        epsr_set_error("epsr_fit_expansion: %d rows x %d terms exceed 8 CTAs of shared memory", npt, nterms);
        return EPSR_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *p = (char *)scratch;
    float *scal = (float *)p;
    p += al256f(sizeof(float) * 4);
    long long *trials = (long long *)p;
    EPSR_CUDA(cudaMemcpyAsync(scal, scal_host, sizeof(float) * 4, cudaMemcpyHostToDevice, s));
    FxDev F;
    F.yin = yin;
    F.expr = expr;
    F.yout = yout;
    F.wt_g = wt;
    F.wtold_g = wtold;
    F.nmin = nmin;
    F.npt = npt;
    F.ncfirst = ncfirst;
    F.nterms = nterms;
    F.nits = nits;
    F.nfreq = nfreq;
    F.strict = strict ? 1 : 0;
    F.rpc = rpc;
    F.ran1 = ran1;
    F.scal = scal;
    F.trials = trials;
    const size_t shm = fx_smem_bytes(nterms, rpc, csize);
    EPSR_CUDA(cudaFuncSetAttribute(fitexp_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize, 1, 1);
    cfg.blockDim = dim3(FX_THREADS, 1, 1);
    cfg.dynamicSmemBytes = shm;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    EPSR_CUDA(cudaLaunchKernelEx(&cfg, fitexp_cluster_kernel, F));
    long long th = 0;
    EPSR_CUDA(cudaMemcpyAsync(scal_host, scal, sizeof(float) * 4, cudaMemcpyDeviceToHost, s));
    EPSR_CUDA(cudaMemcpyAsync(&th, trials, sizeof(long long), cudaMemcpyDeviceToHost, s));
    EPSR_CUDA(cudaStreamSynchronize(s));
    *trials_host = th;
    return EPSR_OK;
}
