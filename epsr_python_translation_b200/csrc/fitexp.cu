// fitexp.cu -- fit_expansion (epsr_standalone_rev3.py:4806-4921) as one persistent CTA.
//
// The Monte Carlo fit is a chain of trials: perturb every coefficient (one ran1 draw
// each), evaluate chi^2 over all Q rows, Metropolis-accept.  Per trial the rows are
// independent (one thread per row, expand :4924 is a sequential clamped sum over the terms)
// and chi^2 is the reference's sequential float32 sum over rows, so the chain is
// bit-identical up to the double-evaluated exp of the acceptance test.  The basis is read
// term-major (a transposed copy made once per call) so each term's row values are one
// coalesced load; it stays L2-resident across trials.
#include "common.cuh"

namespace epsr {

constexpr int FX_THREADS = 1024;

struct FxDev {
    const float *yin, *exprT;  // exprT[(m-1)*npt + (i-1)]
    float *yout, *wt_g, *wtold_g;
    int nmin, npt, ncfirst, nterms, nits, nfreq;
    int32_t *ran1;
    float *scal;         // device copy of {stepr, acceptr, rejrat, chisq}
    long long *trials;
};

__global__ void transpose_expr_kernel(const float *expr, int npt, int nterms, float *exprT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // row 0..npt-1
    const int m = blockIdx.y;                              // term 0..nterms-1
    if (i >= npt) return;
    exprT[(size_t)m * npt + i] = expr[1 + (size_t)i * nterms + m];
}

__device__ float chisq_rows(const FxDev &F, const float *wt, float *sq, float summax, bool write_yout) {
    for (int i = F.nmin + threadIdx.x; i <= F.npt; i += blockDim.x) {
        float sum = 0.0f;
        const float *e = F.exprT + (i - 1);
        for (int m = 1; m <= F.nterms; ++m) {
            sum = __fadd_rn(sum, __fmul_rn(__ldg(e + (size_t)(m - 1) * F.npt), wt[m]));
            if (fabsf(sum) > summax) sum = fsign(summax, sum);
        }
        const float term = __fsub_rn(F.yin[i], sum);
        sq[i] = __fmul_rn(term, term);
        if (write_yout) F.yout[i] = sum;
    }
    __syncthreads();
    __shared__ float result;
    if (threadIdx.x == 0) {
        float c = 0.0f;
        for (int i = F.nmin; i <= F.npt; ++i) c = __fadd_rn(c, sq[i]);
        result = c;
    }
    __syncthreads();
    return result;
}

__global__ void __launch_bounds__(FX_THREADS) fitexp_kernel(FxDev F) {
    extern __shared__ float sm[];
    float *wt = sm;                       // [nterms+1]
    float *wtold = wt + (F.nterms + 1);   // [nterms+1]
    float *sq = wtold + (F.nterms + 1);   // [npt+1]
    __shared__ Ran1 R;
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    const float summax = exp_r(25.0f);
    for (int i = tid; i <= F.nterms; i += blockDim.x) {
        wtold[i] = F.wtold_g[i];
        wt[i] = wtold[i];
    }
    if (tid == 0) ran1_load(R, F.ran1);
    __syncthreads();
    float stepr = F.scal[0];
    float rejrat = F.scal[2];
    float chisqnew = F.scal[3];
    const float acceptr = 0.05f;
    const int npoints = F.npt - F.nmin + 1;
    long long trials = 0;
    float wtmax = 0.0f;
    for (int it = 1; it <= F.nterms; ++it) {
        float a = fabsf(wt[it]);
        wtmax = (a >= wtmax) ? a : wtmax;
    }
    if (stepr < __fmul_rn(1.0e-6f, wtmax)) stepr = __fmul_rn(2.0e-6f, wtmax);
    if (F.nits > 0) {
        int icount = 0;
        chisqnew = chisq_rows(F, wt, sq, summax, false);
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
                if (tid == 0) {
                    for (int ic = F.ncfirst; ic <= F.nterms; ++ic) {
                        const float u = ran1_next(R);
                        const float du = __fsub_rn(__fmul_rn(2.0f, u), 1.0f);
                        if (fabsf(wtold[ic]) < 1.0f) wt[ic] = __fadd_rn(wtold[ic], __fmul_rn(stepr, du));
                        else wt[ic] = __fmul_rn(wtold[ic], __fadd_rn(1.0f, __fmul_rn(stepr, du)));
                    }
                }
                __syncthreads();
                chisqnew = chisq_rows(F, wt, sq, summax, false);
                if (tid == 0) {
                    const float exponent = __fdiv_rn(__fsub_rn(chisqnew, chisqold), accept);
                    float test;
                    if (exponent > 0.0f && exponent <= 20.0f) test = __fsub_rn(exp_r(-exponent), ran1_next(R));
                    else if (exponent > 20.0f) test = -1.0f;
                    else test = 1.0f;
                    int flag = 0;
                    if (test >= 0.0f) {
                        flag = 1;
                        ++icount;
                        if (icount == F.nfreq) {
                            icount = 0;
                            flag = 2;
                            // smoop(ncfirst, nterms, 1, wt) auxiliary_routines.py:744-763
                            const int n1 = F.ncfirst, n2 = F.nterms;
                            if (!(n2 - 2 < n1)) {
                                float sm_ = 0.0f, sn = wt[n1];
                                float sum1 = __fmul_rn(0.25f, __fadd_rn(sm_, sn));
                                for (int i = n1; i <= n2; ++i) {
                                    sm_ = sn;
                                    const int j = i + 1;
                                    sn = j <= n2 ? wt[j] : 0.0f;
                                    const float sum2 = __fmul_rn(0.25f, __fadd_rn(sm_, sn));
                                    wt[i] = __fadd_rn(sum1, sum2);
                                    sum1 = sum2;
                                }
                            }
                        }
                    }
                    s_flag = flag;
                }
                __syncthreads();
                const int flag = s_flag;
                if (flag == 2) chisqnew = chisq_rows(F, wt, sq, summax, false);
                if (flag) {
                    chisqold = chisqnew;
                    for (int ic = 1 + tid; ic <= F.nterms; ic += blockDim.x) wtold[ic] = wt[ic];
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
        for (int ic = 1 + tid; ic <= F.nterms; ic += blockDim.x) wt[ic] = wtold[ic];
        __syncthreads();
    }
    // final fit and chi^2 over rows 1..npt (chi^2 from nmin)
    {
        for (int i = 1 + tid; i <= F.npt; i += blockDim.x) {
            float sum = 0.0f;
            const float *e = F.exprT + (i - 1);
            for (int m = 1; m <= F.nterms; ++m) {
                sum = __fadd_rn(sum, __fmul_rn(__ldg(e + (size_t)(m - 1) * F.npt), wt[m]));
                if (fabsf(sum) > summax) sum = fsign(summax, sum);
            }
            F.yout[i] = sum;
            const float d = __fsub_rn(F.yin[i], sum);
            sq[i] = __fmul_rn(d, d);
        }
        __syncthreads();
        if (tid == 0) {
            float c = 0.0f;
            for (int i = F.nmin; i <= F.npt; ++i) c = __fadd_rn(c, sq[i]);
            chisqnew = c;
        }
    }
    for (int ic = tid; ic <= F.nterms; ic += blockDim.x) {
        F.wt_g[ic] = wt[ic];
        F.wtold_g[ic] = wtold[ic];
    }
    if (tid == 0) {
        F.scal[0] = stepr;
        F.scal[1] = acceptr;
        F.scal[2] = rejrat;
        F.scal[3] = chisqnew;
        *F.trials = trials;
        ran1_store(R, F.ran1);
    }
}

}  // namespace epsr

using namespace epsr;

static inline size_t al256f(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int64_t epsr_fit_expansion_scratch_bytes(int32_t npt, int32_t nterms) {
    return (int64_t)(al256f(sizeof(float) * (size_t)npt * nterms) + al256f(sizeof(float) * 4) +
                     al256f(sizeof(long long)));
}

extern "C" int epsr_fit_expansion(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                                  float *scal_host, int32_t nmin, int32_t npt, int32_t ncfirst, int32_t nterms,
                                  int32_t nits, int32_t nfreq, int32_t *ran1, void *scratch, int64_t scratch_bytes,
                                  int64_t *trials_host, void *stream) {
    if (!yin || !expr || !yout || !wt || !wtold || !scal_host || !ran1 || !scratch || !trials_host || npt <= 0 ||
        nterms <= 0 || nmin < 1 || ncfirst < 1) {
        epsr_set_error("epsr_fit_expansion: bad arguments");
        return EPSR_ERR_ARG;
    }
    if (scratch_bytes < epsr_fit_expansion_scratch_bytes(npt, nterms)) {
        epsr_set_error("epsr_fit_expansion: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    const size_t shm = sizeof(float) * (2 * (size_t)(nterms + 1) + (size_t)(npt + 1));
    if (shm > 200 * 1024) {
        epsr_set_error("epsr_fit_expansion: npt %d + nterms %d exceed shared memory", npt, nterms);
        return EPSR_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *p = (char *)scratch;
    float *exprT = (float *)p;
    p += al256f(sizeof(float) * (size_t)npt * nterms);
    float *scal = (float *)p;
    p += al256f(sizeof(float) * 4);
    long long *trials = (long long *)p;
    transpose_expr_kernel<<<dim3((npt + 127) / 128, nterms), 128, 0, s>>>(expr, npt, nterms, exprT);
    EPSR_CUDA(cudaMemcpyAsync(scal, scal_host, sizeof(float) * 4, cudaMemcpyHostToDevice, s));
    FxDev F;
    F.yin = yin;
    F.exprT = exprT;
    F.yout = yout;
    F.wt_g = wt;
    F.wtold_g = wtold;
    F.nmin = nmin;
    F.npt = npt;
    F.ncfirst = ncfirst;
    F.nterms = nterms;
    F.nits = nits;
    F.nfreq = nfreq;
    F.ran1 = ran1;
    F.scal = scal;
    F.trials = trials;
    if (shm > 48 * 1024) EPSR_CUDA(cudaFuncSetAttribute(fitexp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)shm));
    fitexp_kernel<<<1, FX_THREADS, shm, s>>>(F);
    EPSR_CUDA(cudaGetLastError());
    long long th = 0;
    EPSR_CUDA(cudaMemcpyAsync(scal_host, scal, sizeof(float) * 4, cudaMemcpyDeviceToHost, s));
    EPSR_CUDA(cudaMemcpyAsync(&th, trials, sizeof(long long), cudaMemcpyDeviceToHost, s));
    EPSR_CUDA(cudaStreamSynchronize(s));
    *trials_host = th;
    return EPSR_OK;
}
