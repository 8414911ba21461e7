// ep.cu -- the empirical potential rebuilt from its coefficients: generate_ep
// (epsr_standalone_rev3.py:5876-6022) on the device, and the basis matrices it reads,
// calc_pwrexpr_grad (:5230-5309) and calc_gaussr_grad (:5046-5096), on the host.
//
// The basis (the r-space gradient of every power-exponential or Gaussian basis function at
// every r point) depends only on the grid and the basis parameters, so it is built once on
// the host with the C library's logf/expf -- the functions the reference calls -- and kept
// on the device; the reference rebuilds the same matrix on every call.
//
// Device work of one call, bit-identical to the reference's float32 arithmetic:
//   kernel 1, one CTA per atom pair (rows of the pair in shared memory):
//     expand    every r point j <= npt2 is an independent sum over the basis terms, clamped at
//               +-exp(25) after every term (expand :4924): one thread per point.
//     integrate the potential from its gradient by the trapezoidal rule from the last point
//               inwards: the panel areas in parallel, their running difference sequentially in
//               r order by one thread (the reference's rounding order).
//     finish    x truncation wfac, x pressfac, + Coulomb term, forward-difference gradients.
//     Every CTA also forms abs_energy_ep (the largest max - min range of any coefficient set;
//     max and min are exact, so any order gives the reference's value) and pressfac, from the
//     coefficients as they are before the call.
//   kernel 2, one CTA: pwtold (the last pair's coefficients), multiply_pot_coeffs (each set
//     multiplied by pressfac once per pair that refers to it, in the same sequence of float32
//     products) and the step of the potential factor.
#include <math.h>

#include "common.cuh"

namespace epsr {

constexpr int EP_THREADS = 512;
constexpr int EP_COEF_THREADS = 256;
constexpr int EP_MAX_PAIRS = 960;   // pair -> coefficient set map travels in the launch parameters

struct EpArgs {
    int npairs, npt, npt2, nterms, nsets, ldc, ld;
    float dmax, summax, absolute_energy, erequnit, ereqstep, potfacamp;
    int changepotfac;
    const float *expgr, *xstar, *wfac, *ecoul;
    float *pcoefp, *xavs, *xavs1, *xavtot, *xavtot1, *pwtold, *potfac, *result;
    int32_t iref[EP_MAX_PAIRS];
};

// abs_energy_ep ato_manipulation_rev4.py:4128-4157 and the pressfac rules of generate_ep
// (:5966-5977).  min/max keep the first of equal values as Python's do; signed zeros cannot
// change the range (the running min starts at +0 and only moves to negatives, the max
// likewise), so the parallel order gives the reference's value.
__device__ void ep_pressfac(const EpArgs &a, float *red, float &energabs, float &pressfac) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float best = 0.0f;
    for (int k = warp; k < a.nsets; k += nw) {
        const float *p = a.pcoefp + (size_t)k * a.ldc;
        float lo = 0.0f, hi = 0.0f;
        for (int i = 2 + lane; i <= a.nterms; i += 32) {
            const float t = p[i];
            lo = t < lo ? t : lo;
            hi = t > hi ? t : hi;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
            lo = l2 < lo ? l2 : lo;
            hi = h2 > hi ? h2 : hi;
        }
        const float d = __fsub_rn(hi, lo);
        best = d > best ? d : best;
    }
    if (lane == 0) red[warp] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        float e = 0.0f;
        for (int w = 0; w < nw; ++w) e = red[w] > e ? red[w] : e;
        float pf = 1.0f;
        if (fabsf(a.absolute_energy) == 0.0f) {
            pf = 0.0f;
            e = 0.0f;
        } else if (fabsf(e) > 0.0f) {
            if (fabsf(e) < fabsf(a.erequnit)) {
                pf = __fdiv_rn(fabsf(a.erequnit), fabsf(e));
            } else {
                pf = __fdiv_rn(fabsf(a.absolute_energy), fabsf(e));
                if (pf > 1.0f && a.ereqstep == 0.0f) pf = 1.0f;
            }
        }
        red[0] = e;
        red[1] = pf;
    }
    __syncthreads();
    energabs = red[0];
    pressfac = red[1];
}

// Shared memory: s1[npt+1] (gradient), s[npt+1] (potential), t[npt+1] (panel areas, then the
// total potential), pw[nterms+1] (coefficients), red[32].
__global__ void __launch_bounds__(EP_THREADS) ep_pair_kernel(const __grid_constant__ EpArgs a) {
    extern __shared__ float sm[];
    const int n1 = a.npt + 1;
    float *__restrict__ s1 = sm;
    float *__restrict__ s = sm + n1;
    float *__restrict__ t = sm + 2 * n1;
    float *__restrict__ pw = sm + 3 * n1;
    float *red = pw + a.nterms + 1;
    const int ip = blockIdx.x, tid = threadIdx.x, npt = a.npt, npt2 = a.npt2;
    const size_t row = (size_t)ip * a.ld;
    const float *pc = a.pcoefp + (size_t)a.iref[ip] * a.ldc;
    // the coefficients without the first (:5921-5923)
    for (int i = 1 + tid; i <= a.nterms; i += blockDim.x) pw[i] = i >= 2 ? pc[i] : 0.0f;
    const float pc1 = pc[1];
    float energabs, pressfac;
    ep_pressfac(a, red, energabs, pressfac);   // its barriers also publish pw
    if (ip == 0 && tid == 0) {
        a.result[0] = energabs;
        a.result[1] = pressfac;
    }
    // expand (:5930-5932) and the dimensionless gradient (:5938-5942)
    for (int j = 1 + tid; j <= npt2; j += blockDim.x) {
        const float *e = a.expgr + (size_t)(j - 1) * a.nterms;
        float sum = 0.0f;
#pragma unroll 4
        for (int i = 1; i <= a.nterms; ++i) {
            sum = __fadd_rn(sum, __fmul_rn(__ldg(e + i - 1), pw[i]));
            if (fabsf(sum) > a.summax) sum = copysignf(a.summax, sum);
        }
        s1[j] = __fmul_rn(__fmul_rn(sum, pc1), a.dmax);
    }
    // the points the call does not rewrite keep the values they had (read by the reference too)
    for (int j = npt2 + 1 + tid; j < npt; j += blockDim.x) s1[j] = a.xavs1[row + j];
    const int jlo = npt - npt2;   // lowest point the integration reaches
    for (int j = 1 + tid; j < jlo; j += blockDim.x) s[j] = a.xavs[row + j];
    if (tid == 0) {
        s1[npt] = 0.0f;
        s[npt] = 0.0f;
    }
    __syncthreads();
    // panel areas of the trapezoidal rule (:5949-5957)
    for (int jr = jlo + tid; jr < npt; jr += blockDim.x)
        t[jr] = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(a.xstar[jr + 1], a.xstar[jr])), __fadd_rn(s1[jr + 1], s1[jr]));
    __syncthreads();
    if (tid == 0) {   // the potential from the last point inwards, in the reference's order
        float v = 0.0f;
#pragma unroll 8
        for (int jr = npt - 1; jr >= jlo; --jr) {
            v = __fsub_rn(v, t[jr]);
            s[jr] = v;
        }
    }
    __syncthreads();
    // truncation, pressfac and the total potential (:5961-5963, :5986-5988); points past npt2
    // keep their total potential
    for (int j = 1 + tid; j <= npt; j += blockDim.x) {
        if (j <= npt2) {
            const float v = __fmul_rn(__fmul_rn(s[j], a.wfac[j]), pressfac);
            s[j] = v;
            t[j] = __fadd_rn(a.ecoul[row + j], v);
        } else {
            t[j] = a.xavtot[row + j];
        }
    }
    __syncthreads();
    // forward-difference gradients (:5993-6009) and the tables out
    for (int j = 1 + tid; j <= npt; j += blockDim.x) {
        a.xavs[row + j] = s[j];
        if (j <= npt2) a.xavtot[row + j] = t[j];
        if (j >= 2) {
            const float xdif = __fsub_rn(a.xstar[j], a.xstar[j - 1]);
            a.xavs1[row + j - 1] = __fdiv_rn(__fsub_rn(s[j], s[j - 1]), xdif);
            a.xavtot1[row + j - 1] = __fdiv_rn(__fsub_rn(t[j], t[j - 1]), xdif);
        }
    }
    if (tid == 0) {
        a.xavs1[row + npt] = 0.0f;
        a.xavtot1[row + npt] = 0.0f;
    }
}

// pwtold (:5921-5923 of the last pair), multiply_pot_coeffs (:6493-6510) and the step of the
// potential factor (:6015-6022).  mult[k]: how many pairs refer to set k.
__global__ void __launch_bounds__(EP_COEF_THREADS) ep_coeff_kernel(const __grid_constant__ EpArgs a) {
    extern __shared__ int32_t mult[];
    const int tid = threadIdx.x;
    for (int k = tid; k < a.nsets; k += blockDim.x) mult[k] = 0;
    __syncthreads();
    for (int ip = tid; ip < a.npairs; ip += blockDim.x) atomicAdd(&mult[a.iref[ip]], 1);
    const float *last = a.pcoefp + (size_t)a.iref[a.npairs - 1] * a.ldc;
    for (int i = 1 + tid; i <= a.nterms; i += blockDim.x) a.pwtold[i] = i >= 2 ? last[i] : 0.0f;
    __syncthreads();
    const float energabs = a.result[0], pressfac = a.result[1];
    const int w = a.nterms - 1;
    for (int q = tid; q < a.nsets * w; q += blockDim.x) {
        const int k = q / w, ic = 2 + q % w;
        float *p = a.pcoefp + (size_t)k * a.ldc + ic;
        float v = *p;
        for (int r = mult[k]; r > 0; --r) v = __fmul_rn(v, pressfac);
        *p = v;
    }
    if (tid == 0 && a.changepotfac && a.absolute_energy > 0.0f) {
        float pf = *a.potfac;
        if (pf > 0.000001f && a.potfacamp > 0.0f) {
            float d = __fdiv_rn(__fsub_rn(a.absolute_energy, energabs), fabsf(__fmul_rn(a.potfacamp, a.absolute_energy)));
            if (fabsf(d) > 0.1f) d = copysignf(0.1f, d);
            pf = __fmul_rn(pf, __fadd_rn(1.0f, d));
            pf = pf < 0.000001f ? 0.000001f : pf;   // max(potfac, 1e-6): Python keeps the first of equals
            pf = 1.0f < pf ? 1.0f : pf;             // min(potfac, 1)
            *a.potfac = pf;
        }
    }
}

// The coefficient increment of ptgnsq epsr_standalone_rev3.py:3948-3962 for every data set in
// turn: pcoefp(ic, k) = real(dble(pcoefp(ic, k)) + (dble(pfact * efacp(k)) * cwtpot(ip, id)) *
// dble(pwtold_id(ic))) for each pair ip of set k, in pair order -- cwtpot is real*8, so the
// increment is formed in double and rounded once per step.  One thread per (set, coefficient).
struct EpUpdate {
    int ndata, npairs, nterms, nsets, ldc, ldw;
    float pfact;
    float *pcoefp;
    const float *efacp, *pwtold;
    const double *cwtpot;
    int32_t iref[EP_MAX_PAIRS];
};

__global__ void ep_update_kernel(const __grid_constant__ EpUpdate u) {
    const int w = u.nterms - 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= u.nsets * w) return;
    const int k = q / w, ic = 2 + q % w;
    float *p = u.pcoefp + (size_t)k * u.ldc + ic;
    float v = *p;
    const double fk = (double)__fmul_rn(u.pfact, u.efacp[k]);
    for (int id = 0; id < u.ndata; ++id) {
        const double pw = (double)u.pwtold[(size_t)id * u.ldw + ic];
        for (int ip = 0; ip < u.npairs; ++ip)
            if (u.iref[ip] == k)
                v = __double2float_rn(
                    __dadd_rn((double)v, __dmul_rn(__dmul_rn(fk, u.cwtpot[(size_t)id * u.npairs + ip]), pw)));
    }
    *p = v;
}

// The packed pair tables the energy kernels read: tab[(pair*ld + j)*4 + {0,1,2,3}] =
// {xavs, xavs1, ecoul, ecoul1}(j).
__global__ void ep_pack_kernel(int n, const float *xavs, const float *xavs1, const float *ecoul, const float *ecoul1,
                               float4 *tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) tab[i] = make_float4(xavs[i], xavs1[i], ecoul[i], ecoul1[i]);
}

}  // namespace epsr

using namespace epsr;

extern "C" int epsr_ep_update(int32_t ndata, int32_t npairs, int32_t nterms, float *pcoefp, int32_t nsets,
                              int32_t ldc, const int32_t *irefpcof_host, const float *efacp, const double *cwtpot,
                              const float *pwtold, int32_t ldw, float pfact, void *stream) {
    if (ndata < 1 || npairs < 1 || npairs > EP_MAX_PAIRS || nterms < 2 || nsets < 1 || ldc < nterms + 1 ||
        ldw < nterms + 1 || !pcoefp || !irefpcof_host || !efacp || !cwtpot || !pwtold) {
        epsr_set_error("epsr_ep_update: bad arguments");
        return EPSR_ERR_ARG;
    }
    EpUpdate u;
    u.ndata = ndata;
    u.npairs = npairs;
    u.nterms = nterms;
    u.nsets = nsets;
    u.ldc = ldc;
    u.ldw = ldw;
    u.pfact = pfact;
    u.pcoefp = pcoefp;
    u.efacp = efacp;
    u.cwtpot = cwtpot;
    u.pwtold = pwtold;
    for (int ip = 0; ip < npairs; ++ip) {
        if (irefpcof_host[ip] < 0 || irefpcof_host[ip] >= nsets) {
            epsr_set_error("epsr_ep_update: pair %d refers to coefficient set %d of %d", ip, irefpcof_host[ip], nsets);
            return EPSR_ERR_ARG;
        }
        u.iref[ip] = irefpcof_host[ip];
    }
    const int n = nsets * (nterms - 1);
    ep_update_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(u);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_pack_tables(int32_t npairs, int32_t ld, const float *xavs, const float *xavs1,
                                const float *ecoul, const float *ecoul1, float *tab, void *stream) {
    if (npairs < 1 || ld < 2 || !xavs || !xavs1 || !ecoul || !ecoul1 || !tab || ((uintptr_t)tab & 15)) {
        epsr_set_error("epsr_pack_tables: bad arguments (tab must be 16-byte aligned)");
        return EPSR_ERR_ARG;
    }
    const int n = npairs * ld;
    ep_pack_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, xavs, xavs1, ecoul, ecoul1, (float4 *)tab);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_generate_ep(int32_t npairs, int32_t npt, int32_t npt2, int32_t nterms, const float *expgr,
                                float *pcoefp, int32_t nsets, int32_t ldc, const int32_t *irefpcof_host, float dmax,
                                const float *xstar, const float *wfac, const float *ecoul, float *xavs, float *xavs1,
                                float *xavtot, float *xavtot1, int32_t ld, float *pwtold, float absolute_energy,
                                float erequnit, float ereqstep, float potfacamp, float *potfac, int32_t changepotfac,
                                float *result, void *stream) {
    if (npairs < 1 || npairs > EP_MAX_PAIRS || npt < 2 || npt2 < 1 || npt2 > npt - 1 || npt + 1 > ld ||
        nterms < 2 || nsets < 1 || ldc < nterms + 1 || !expgr || !pcoefp || !irefpcof_host || !xstar || !wfac ||
        !ecoul || !xavs || !xavs1 || !xavtot || !xavtot1 || !pwtold || !potfac || !result) {
        epsr_set_error("epsr_generate_ep: bad arguments (npairs %d of at most %d, npt %d, npt2 %d, ld %d, nterms %d, "
                       "nsets %d, ldc %d)", npairs, EP_MAX_PAIRS, npt, npt2, ld, nterms, nsets, ldc);
        return EPSR_ERR_ARG;
    }
    EpArgs a;
    a.npairs = npairs;
    a.npt = npt;
    a.npt2 = npt2;
    a.nterms = nterms;
    a.nsets = nsets;
    a.ldc = ldc;
    a.ld = ld;
    a.dmax = dmax;
    volatile float e25 = 25.0f;   // exp(25) from the C library at run time, as the reference
    a.summax = expf(e25);
    a.absolute_energy = absolute_energy;
    a.erequnit = erequnit;
    a.ereqstep = ereqstep;
    a.potfacamp = potfacamp;
    a.changepotfac = changepotfac != 0;
    a.expgr = expgr;
    a.xstar = xstar;
    a.wfac = wfac;
    a.ecoul = ecoul;
    a.pcoefp = pcoefp;
    a.xavs = xavs;
    a.xavs1 = xavs1;
    a.xavtot = xavtot;
    a.xavtot1 = xavtot1;
    a.pwtold = pwtold;
    a.potfac = potfac;
    a.result = result;
    for (int ip = 0; ip < npairs; ++ip) {
        if (irefpcof_host[ip] < 0 || irefpcof_host[ip] >= nsets) {
            epsr_set_error("epsr_generate_ep: pair %d refers to coefficient set %d of %d", ip, irefpcof_host[ip], nsets);
            return EPSR_ERR_ARG;
        }
        a.iref[ip] = irefpcof_host[ip];
    }
    const size_t smem = (size_t)(3 * (npt + 1) + nterms + 1 + 32) * sizeof(float);
    int dev = 0, mx = 0;
    EPSR_CUDA(cudaGetDevice(&dev));
    EPSR_CUDA(cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (smem > (size_t)mx || (size_t)nsets * sizeof(int32_t) > 48 * 1024) {
        epsr_set_error("epsr_generate_ep: npt %d / nterms %d / nsets %d need more shared memory than a CTA has", npt,
                       nterms, nsets);
        return EPSR_ERR_CAPACITY;
    }
    if (smem > 48 * 1024) EPSR_SMEM_OPTIN(ep_pair_kernel);
    cudaStream_t s = (cudaStream_t)stream;
    ep_pair_kernel<<<npairs, EP_THREADS, smem, s>>>(a);
    EPSR_CUDA(cudaGetLastError());
    ep_coeff_kernel<<<1, EP_COEF_THREADS, (size_t)nsets * sizeof(int32_t), s>>>(a);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

// ------------------------------------------------------------------ host: the basis matrices

// fctrln lngamma_mod.py:16-32: gamln[i] = log((i-1)!) in double, i = 1..n+1.
static void ep_gamln(int n, double *g) {
    double acc = 0.0, a = 0.0;
    for (int i = 1; i <= n + 1; ++i) {
        g[i] = acc;
        a = a + 1.0;
        acc = acc + log(a);
    }
}

// calc_pwrexpr_grad epsr_standalone_rev3.py:5230-5309 with dnext :5312-5326.
extern "C" int epsr_calc_pwrexpr_grad(int32_t lpt, int32_t nterms, float dmin, float dstep, float dmax, float sigmab,
                                      float rho, const float *xin, float *expr, float rmin, int32_t *ncfirst,
                                      float fbroad, float rbroad) {
    if (lpt < 1 || nterms < 1 || !xin || !expr || !ncfirst || !(sigmab > 0.0f)) {
        epsr_set_error("epsr_calc_pwrexpr_grad: bad arguments");
        return EPSR_ERR_ARG;
    }
    const float pi = 3.141592653f, expmax = 25.0f;
    const float ntf = dmax / sigmab + 3.0f;
    if (!(ntf < 1.0e7f)) {
        epsr_set_error("epsr_calc_pwrexpr_grad: dmax/sigmab %g is too large", (double)(dmax / sigmab));
        return EPSR_ERR_ARG;
    }
    const int ntmax = (int)ntf;   // ifix
    double *gamln = (double *)malloc(sizeof(double) * (size_t)(ntmax + 2));
    if (!gamln) {
        epsr_set_error("epsr_calc_pwrexpr_grad: out of host memory");
        return EPSR_ERR_CAPACITY;
    }
    ep_gamln(ntmax, gamln);
    float d = dstep, rootd = 1.0f;
    int nc = *ncfirst, rc = EPSR_OK;
    for (int m = 1; m <= nterms; ++m) {
        if (d < rmin) nc = m + 1;
        const float sigma = rootd * fbroad * sigmab;
        int n = 0;
        if (sigma <= d && sigma > 0.0f && m > 1) n = (int)(d / sigma - 1.0f);
        const int nref = n + 3;
        if (nref < 1 || nref > ntmax + 1) {
            epsr_set_error("epsr_calc_pwrexpr_grad: term %d needs log-factorial %d beyond the table (%d)", m, nref,
                           ntmax + 1);
            rc = EPSR_ERR_ARG;
            break;
        }
        const float gfac = 4.0f * pi * rho * sigma * sigma * sigma;
        const float gfacln = logf(gfac);
        float sigln = (float)(gamln[nref] + (double)gfacln);
        if (m == 1) sigln = sigln - rmin / sigma;
        for (int i = 1; i <= lpt; ++i) {
            const float r = xin[i];
            float fact = rbroad * r;
            const float rsigma = r / sigma;
            float expon;
            if (r > 0.0f) {
                const float rsigmaln = logf(rsigma);
                expon = (float)n * rsigmaln - rsigma - sigln - fact;
                fact = (float)n / r - 1.0f / sigma - rbroad;
            } else if (n == 0) {
                expon = -rsigma - sigln - fact;
                fact = -(1.0f / sigma + rbroad);
            } else if (n == 1) {
                expon = -rsigma - sigln - fact;
                fact = 1.0f / sigma;
            } else {
                expon = -2.0f * expmax;
                fact = 0.0f;
            }
            expr[(size_t)(i - 1) * nterms + (m - 1)] = expon > -expmax ? fact * expf(expon) : 0.0f;
        }
        // dnext
        float dn = d + dstep;
        const float dtest = d * dmin;
        if (dtest > dn) {
            dn = dtest;
            rootd = rootd * sqrtf(dmin);
        }
        d = dn;
    }
    free(gamln);
    *ncfirst = nc;
    return rc;
}

// calc_gaussr_grad epsr_standalone_rev3.py:5046-5096.
extern "C" int epsr_calc_gaussr_grad(int32_t lpt, int32_t nterms, float dstep, float dmax, float sigmab, float rho,
                                     const float *xin, float *expr, float rmin, int32_t *ncfirst, float fbroad,
                                     float rbroad) {
    (void)dmax;
    (void)rbroad;
    if (lpt < 1 || nterms < 1 || !xin || !expr || !ncfirst) {
        epsr_set_error("epsr_calc_gaussr_grad: bad arguments");
        return EPSR_ERR_ARG;
    }
    const float pi = (float)M_PI, expmax = 25.0f;
    const float piroot = sqrtf(0.5f * pi);
    const float gfac = piroot / (4.0f * pi * pi * rho);
    int nc = *ncfirst;
    for (int m = 1; m <= nterms; ++m) {
        const float d = (float)m * dstep;
        if (d < rmin) nc = m + 1;
        const float sigd = fbroad * sigmab;
        const float gfacs = gfac / sigd;
        const float sigd2 = sigd * sigd;
        for (int i = 1; i <= lpt; ++i) {
            const float r = xin[i];
            const float rmd = (r - d) / sigd, rpd = (r + d) / sigd;
            const float rmd2 = 0.5f * rmd * rmd, rpd2 = 0.5f * rpd * rpd;
            float sum = 0.0f, gfact = 0.0f;
            if (fabsf(r) > 0.0f && fabsf(d) > 0.0f) {
                gfact = gfacs / (r * d);
                if (rmd2 < expmax) sum = sum - (1.0f / r + (r - d) / sigd2) * expf(-rmd2);
                if (rpd2 < expmax) sum = sum + (1.0f / r + (r + d) / sigd2) * expf(-rpd2);
            }
            expr[(size_t)(i - 1) * nterms + (m - 1)] = gfact * sum;
        }
    }
    *ncfirst = nc;
    return EPSR_OK;
}
