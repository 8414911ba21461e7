// transforms.cu -- gensq (epsr_standalone_rev3.py:4731-4802) and stog
// (ato_manipulation_rev4.py:4067-4121) on the CUDA cores.
//
// Both are sums over one index with the other two free; the reference adds sequentially,
// so each output is one thread's sequential float32 sum (bit-identical for gensq; stog
// uses the double-evaluated sine, see common.cuh).  Consecutive threads take consecutive
// Q (gensq) or r (stog) points so every table read is coalesced.
#include "common.cuh"

namespace epsr {

__global__ void gensq_kernel(int nq, int npairs, int npt1, const float *wav, int ldw, const float *fq, long long sj,
                             long long si, const float *ycoh, const int32_t *n2extr, const float *natomsphere,
                             float *sofq) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int ic = blockIdx.y;
    if (i > nq) return;
    const float *w1 = wav + (size_t)ic * ldw;
    const float *w2 = wav + (size_t)(npairs + ic) * ldw;
    const float nsph = natomsphere[n2extr[ic]];
    float sum1 = 0.0f, sum2 = 0.0f, sum3 = 0.0f;
#pragma unroll 4
    for (int j = 2; j <= npt1; ++j) {   // branch-free, so the loads of several j are in flight
        const float f = __ldg(fq + (long long)j * sj + (long long)i * si);
        const float a1 = __ldg(w1 + j);
        const float t1 = __fadd_rn(sum1, __fmul_rn(a1, f));
        sum1 = fabsf(a1) > 0.0f ? t1 : sum1;
        const float b = __ldg(w2 + j);
        const float a2 = __fmul_rn(__fsub_rn(b, __ldg(ycoh + j)), nsph);
        sum2 = __fadd_rn(sum2, __fmul_rn(a2, f));
        sum3 = __fadd_rn(sum3, b);
    }
    if (sum3 <= 0.0f) sum2 = 0.0f;
    sofq[(size_t)ic * (nq + 1) + i] = sum1;
    sofq[(size_t)(npairs + ic) * (nq + 1) + i] = sum2;
}

// lorch(x) for every (pair, Q) (ato_manipulation_rev4.py:4113-4121): it depends on the pair
// only through qmax, so it is tabulated once instead of once per r point.
__global__ void lorch_kernel(const float *q, int ldq, int npairs, const int32_t *nqmax, float *lw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int in = blockIdx.y;
    if (i >= ldq) return;
    const float pi = 3.14159265358979323846f;
    const float qmax = __fdiv_rn(pi, q[min(ldq - 1, max(1, nqmax[in]))]);
    const float x = __fmul_rn(qmax, q[i]);
    float r;
    if (x == 0.0f) r = 1.0f;
    else if (x < pi) r = __fdiv_rn(sin_r(x), x);
    else r = 0.0f;
    lw[(size_t)in * ldq + i] = r;
}

__global__ void stog_kernel(float rho, const float *q, int ldq, const float *sofq, const float *r, int nr, int npairs,
                            const int32_t *nqmin, const int32_t *nqmax, const float *xwt, const float *lw,
                            float *gofr) {
    const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int in = blockIdx.y;
    if (j > nr) return;
    // sfac = 0.5*qstep/pi/pi/rho with qstep = q(4)-q(3) (ato_manipulation_rev4.py:4075-4076)
    const float pi = 3.14159265358979323846f;
    const float qstep = __fsub_rn(q[4], q[3]);
    const float sfac = __fdiv_rn(__fdiv_rn(__fdiv_rn(__fmul_rn(0.5f, qstep), pi), pi), rho);
    const float rr = r[j];
    const float *s = sofq + (size_t)in * ldq;
    const float *l = lw + (size_t)in * ldq;
    float sumi = 0.0f;
    const int i0 = max(1, nqmin[in]), i1 = min(ldq - 1, nqmax[in]);
    if (rr > 0.0f) {
        for (int i = i0; i <= i1; ++i) {
            const float qq = __ldg(q + i);
            const float prod = __fmul_rn(__fmul_rn(qq, sin_r(__fmul_rn(qq, rr))), __ldg(l + i));
            sumi = __fadd_rn(sumi, __fmul_rn(__ldg(s + i), prod));
        }
        gofr[(size_t)in * (nr + 1) + j] = __fadd_rn(xwt[in], __fdiv_rn(__fmul_rn(sfac, sumi), rr));
    } else {
        for (int i = i0; i <= i1; ++i) {
            const float qq = __ldg(q + i);
            const float prod = __fmul_rn(__fmul_rn(qq, qq), __ldg(l + i));
            sumi = __fadd_rn(sumi, __fmul_rn(__ldg(s + i), prod));
        }
        gofr[(size_t)in * (nr + 1) + j] = __fadd_rn(xwt[in], __fmul_rn(sfac, sumi));
    }
}

// The simulated fit of each data set (ptgnsq epsr_standalone_rev3.py:3844-3867): the sum
// over atom pairs of weight x intermolecular S(Q), sequential over pairs as the reference --
// the weights are real*8, so each step is sum = real(dble(sum) + cwt * dble(qwind)), one
// rounding to float32 per pair -- and its difference from the data, negated:
// out = -qtemp with the reference's Q window (:3856-3867): below max(qmin, q(nqmin)) the data
// are replaced by 0 or, when szeros is set, by the straight line from szeros at Q = q(1) to the
// data at nqmin; between nqmin and nqmax qtemp = data - sum; above nqmax 0.  Without window
// arrays (NULL) nqmin = 1, nqmax = nq, szeros = 0 and qmin = 0.  Thread per (set, Q).
// An X-ray data set (xray[d] != 0) weights each pair by its Q-dependent real*8 weight
// wq[d][ic][i] (x_rayf0.weightx) instead of cwt[d][ic] (:3850-3852).
__global__ void ptgnsq_diff_kernel(int ndata, int npairs, int nq, const float *data, const double *cwt,
                                   const float *qwind, const float *q, const int32_t *nqmin, const int32_t *nqmax,
                                   const float *szeros, float qmin, const double *wq, const int32_t *xray,
                                   float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int d = blockIdx.y;
    if (i > nq) return;
    const bool xr = wq && xray && xray[d] != 0;
    const double *w = xr ? wq + (size_t)d * npairs * (nq + 1) + i : cwt + (size_t)d * npairs;
    const size_t ws = xr ? (size_t)(nq + 1) : 1;
    const float *dd = data + (size_t)d * (nq + 1);
    float sum = 0.0f;
    for (int ic = 0; ic < npairs; ++ic)
        sum = __double2float_rn(__dadd_rn((double)sum, __dmul_rn(__ldg(w + ic * ws),
                                                                 (double)__ldg(qwind + (size_t)ic * (nq + 1) + i))));
    float qtemp;
    if (!q) {
        qtemp = __fsub_rn(dd[i], sum);
    } else {
        // the window as given, kept inside the row [1, nq] (the reference's window always is)
        int nqmn = nqmin ? nqmin[d] : 1, nqmx = nqmax ? nqmax[d] : nq;
        nqmn = nqmn < 1 ? 1 : (nqmn > nq ? nq : nqmn);
        nqmx = nqmx > nq ? nq : nqmx;
        const float sz = szeros ? szeros[d] : 0.0f;
        const float qn = q[nqmn];
        const float qthr = qn > qmin ? qn : qmin;          // max(qminptemp, q(nqmn))
        if (q[i] < qthr) {
            if (sz != 0.0f) {
                float grads0 = 0.0f, conss0 = 0.0f;
                if (nqmn > 1) {
                    grads0 = __fdiv_rn(__fsub_rn(dd[nqmn], sz), __fsub_rn(qn, q[1]));
                    conss0 = sz;
                }
                qtemp = __fsub_rn(__fadd_rn(conss0, __fmul_rn(grads0, __fsub_rn(q[i], q[1]))), sum);
            } else {
                qtemp = 0.0f;
            }
        } else if (i >= nqmn && i <= nqmx) {
            qtemp = __fsub_rn(dd[i], sum);
        } else {
            qtemp = 0.0f;
        }
    }
    out[(size_t)d * (nq + 1) + i] = -qtemp;
}

}  // namespace epsr

using namespace epsr;

extern "C" int epsr_ptgnsq_difference(int32_t ndata, int32_t npairs, int32_t nq, const float *data, const double *cwt,
                                      const float *qwind, const float *q, const int32_t *nqmin, const int32_t *nqmax,
                                      const float *szeros, float qmin, const double *wq, const int32_t *xray,
                                      float *out, void *stream) {
    if (ndata <= 0 || npairs <= 0 || nq <= 0 || !data || !cwt || !qwind || !out) {
        epsr_set_error("epsr_ptgnsq_difference: bad arguments");
        return EPSR_ERR_ARG;
    }
    ptgnsq_diff_kernel<<<dim3((nq + 1 + 127) / 128, ndata), 128, 0, (cudaStream_t)stream>>>(
        ndata, npairs, nq, data, cwt, qwind, q, nqmin, nqmax, szeros, qmin, wq, xray, out);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_gensq(int32_t nq, int32_t npairs, int32_t npt1, const float *wav, int32_t ldw, const float *foqols,
                          int64_t sj, int64_t si, const float *ycoh, const int32_t *n2extr, const float *natomsphere,
                          float *sofq, void *stream) {
    if (!wav || !foqols || !ycoh || !n2extr || !natomsphere || !sofq || nq <= 0 || npairs <= 0 || npt1 + 1 > ldw) {
        epsr_set_error("epsr_gensq: bad arguments");
        return EPSR_ERR_ARG;
    }
    dim3 grid((nq + 127) / 128, npairs);
    gensq_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(nq, npairs, npt1, wav, ldw, foqols, sj, si, ycoh, n2extr,
                                                         natomsphere, sofq);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int64_t epsr_stog_scratch_bytes(int32_t npairs, int32_t ldq) {
    return (int64_t)sizeof(float) * npairs * (int64_t)ldq + 256;
}

extern "C" int epsr_stog(float rho, const float *q, int32_t ldq, const float *sofq, const float *r, int32_t nr,
                         int32_t npairs, const int32_t *nqmin, const int32_t *nqmax, const float *xwt, float *gofr,
                         void *scratch, int64_t scratch_bytes, void *stream) {
    if (!q || !sofq || !r || !nqmin || !nqmax || !xwt || !gofr || !scratch || ldq < 5 || nr <= 0 || npairs <= 0) {
        epsr_set_error("epsr_stog: bad arguments");
        return EPSR_ERR_ARG;
    }
    if (scratch_bytes < epsr_stog_scratch_bytes(npairs, ldq)) {
        epsr_set_error("epsr_stog: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    float *lw = (float *)scratch;
    lorch_kernel<<<dim3((ldq + 127) / 128, npairs), 128, 0, s>>>(q, ldq, npairs, nqmax, lw);
    stog_kernel<<<dim3((nr + 127) / 128, npairs), 128, 0, s>>>(rho, q, ldq, sofq, r, nr, npairs, nqmin, nqmax, xwt,
                                                               lw, gofr);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
