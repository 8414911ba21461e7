// sums.cu -- running averages of the partial g(r) and S(Q) with their error bars: sumgr
// (epsr_standalone_rev3.py:3578-3637) and sumsq (:3642-3677), bit-identical.
//
// Every (pair, point) element is independent: the stored error bar and mean give back the
// mean square, both are folded with the new sample by fc2 (old) and fc1 (new) in double, as
// the reference's real*8 work space, and the mean and error bar are stored in float32.  One
// CTA per atom pair updates its points in parallel; sumgr's "zero limit" (a running double
// sum over r of ycoh*(g_inter - 1)) is then summed in r order by one thread of the CTA.
#include "common.cuh"

namespace epsr {

constexpr int SUM_THREADS = 256;

__device__ __forceinline__ void sum_update(double add1, double fc1, double fc2, float *mean, float *err) {
    double sumtot1 = (double)*mean, sumtot2 = (double)*err;
    const double add2 = __dmul_rn(add1, add1);
    sumtot2 = __dadd_rn(__dmul_rn(sumtot2, sumtot2), __dmul_rn(sumtot1, sumtot1));
    sumtot1 = __dadd_rn(__dmul_rn(fc2, sumtot1), __dmul_rn(fc1, add1));
    sumtot2 = __dadd_rn(__dmul_rn(fc2, sumtot2), __dmul_rn(fc1, add2));
    double errort = __dsub_rn(sumtot2, __dmul_rn(sumtot1, sumtot1));
    errort = errort > 0.0 ? __dsqrt_rn(errort) : 0.0;
    *mean = __double2float_rn(sumtot1);
    *err = __double2float_rn(errort);
}

__global__ void __launch_bounds__(SUM_THREADS) sumgr_kernel(int nz, int npairs, const float *wav, int ldw,
                                                            const float *ycoh, double fc1, double fc2,
                                                            float *gorintra, float *gorinter, float *gr2intra,
                                                            float *gr2inter, float *entsig) {
    const int id = blockIdx.x;
    const size_t row = (size_t)id * ldw, half = (size_t)npairs * ldw;
    for (int j = 2 + threadIdx.x; j <= nz; j += blockDim.x) {
        double a1 = 0.0, a2 = 0.0;
        const float yc = ycoh[j];
        if (yc > 0.0f) {
            a1 = (double)__fdiv_rn(wav[row + j], yc);
            a2 = (double)__fdiv_rn(wav[half + row + j], yc);
        }
        sum_update(a1, fc1, fc2, gorintra + row + j, gr2intra + row + j);
        sum_update(a2, fc1, fc2, gorinter + row + j, gr2inter + row + j);
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // the zero limit, in r order
        entsig[row + 1] = 0.0f;
        double zerolimit = 0.0;
        for (int j = 2; j <= nz; ++j) {
            zerolimit = __dadd_rn(zerolimit, (double)__fmul_rn(ycoh[j], __fsub_rn(gorinter[row + j], 1.0f)));
            entsig[row + j] = __double2float_rn(zerolimit);
        }
    }
}

__global__ void __launch_bounds__(SUM_THREADS) sumsq_kernel(int nq, int npairs, const float *qwind, int ldq,
                                                            double fc1, double fc2, float *soqintra,
                                                            float *soqinter, float *sq2intra, float *sq2inter) {
    const int id = blockIdx.x;
    const size_t row = (size_t)id * ldq, half = (size_t)npairs * ldq;
    for (int j = 1 + threadIdx.x; j <= nq; j += blockDim.x) {
        sum_update((double)qwind[row + j], fc1, fc2, soqintra + row + j, sq2intra + row + j);
        sum_update((double)qwind[half + row + j], fc1, fc2, soqinter + row + j, sq2inter + row + j);
    }
}

}  // namespace epsr

using namespace epsr;

extern "C" int epsr_sumgr(int32_t nz, int32_t npairs, const float *wav, int32_t ldw, const float *ycoh, double fc1,
                          double fc2, float *gorintra, float *gorinter, float *gr2intra, float *gr2inter,
                          float *entsig, void *stream) {
    if (nz < 1 || npairs <= 0 || nz + 1 > ldw || !wav || !ycoh || !gorintra || !gorinter || !gr2intra || !gr2inter ||
        !entsig) {
        epsr_set_error("epsr_sumgr: bad arguments");
        return EPSR_ERR_ARG;
    }
    sumgr_kernel<<<npairs, SUM_THREADS, 0, (cudaStream_t)stream>>>(nz, npairs, wav, ldw, ycoh, fc1, fc2, gorintra,
                                                                  gorinter, gr2intra, gr2inter, entsig);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_sumsq(int32_t nq, int32_t npairs, const float *qwind, int32_t ldq, double fc1, double fc2,
                          float *soqintra, float *soqinter, float *sq2intra, float *sq2inter, void *stream) {
    if (nq < 1 || npairs <= 0 || nq + 1 > ldq || !qwind || !soqintra || !soqinter || !sq2intra || !sq2inter) {
        epsr_set_error("epsr_sumsq: bad arguments");
        return EPSR_ERR_ARG;
    }
    sumsq_kernel<<<npairs, SUM_THREADS, 0, (cudaStream_t)stream>>>(nq, npairs, qwind, ldq, fc1, fc2, soqintra,
                                                                  soqinter, sq2intra, sq2inter);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
