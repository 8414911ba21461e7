// common.cuh -- device helpers shared by the EPSR pair-path kernels (sm_100a).
//
// Bit-exactness: the reference evaluates float32 scalars with no fused multiply-add, IEEE
// division and sqrt.  Every arithmetic step below that feeds a compared result uses the
// explicit round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, __fsqrt_rn), which
// the compiler never contracts, and the library is also built with -fmad=false.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/epsr_gpu.h"

namespace epsr {

// ----------------------------------------------------------------- Fortran intrinsics
// nint: round half away from zero (fortran/fmath.py:222).  x - trunc(x) is exact in float.
__device__ __forceinline__ float nint_f(float x) {
    float t = truncf(x);
    float fr = __fsub_rn(x, t);
    if (fr >= 0.5f) t = __fadd_rn(t, 1.0f);
    else if (fr <= -0.5f) t = __fsub_rn(t, 1.0f);
    return t;
}
__device__ __forceinline__ int nint_i(float x) { return (int)nint_f(x); }

// ifix: truncation toward zero (fortran/fmath.py:245)
__device__ __forceinline__ int ifix(float x) { return __float2int_rz(x); }

__device__ __forceinline__ float fsign(float a, float b) { return copysignf(fabsf(a), b); }

// Transcendentals: evaluated in double and rounded once to float, i.e. the correctly
// rounded value in all but a vanishing fraction of arguments.  glibc's float functions
// used by the reference are not correctly rounded (about 1.3% of sinf/cosf arguments and
// 0.07% of expf arguments differ by one ulp), so these are tolerance-checked, and the
// Monte Carlo kernel accepts injected cosine values to prove the rest bit-identical.
__device__ __forceinline__ float cos_r(float x) { return (float)cos((double)x); }
__device__ __forceinline__ float sin_r(float x) { return (float)sin((double)x); }
__device__ __forceinline__ float exp_r(float x) { return (float)exp((double)x); }

// ----------------------------------------------------------------- minimum image
struct Lattice {
    int cubic;
    float alatx, blatx, clatx, blaty, claty, clatz;
};

// minimagec.py:13-45
__device__ __forceinline__ void minimagec(const Lattice &L, float &x, float &y, float &z) {
    if (L.cubic) {
        z = __fsub_rn(z, nint_f(z));
        y = __fsub_rn(y, nint_f(y));
        x = __fsub_rn(x, nint_f(x));
        return;
    }
    float fc = __fdiv_rn(z, L.clatz);
    float fb = __fdiv_rn(__fsub_rn(y, __fmul_rn(fc, L.claty)), L.blaty);
    float fa = __fdiv_rn(__fsub_rn(__fsub_rn(x, __fmul_rn(fb, L.blatx)), __fmul_rn(fc, L.clatx)), L.alatx);
    fc = __fsub_rn(fc, nint_f(fc));
    fb = __fsub_rn(fb, nint_f(fb));
    fa = __fsub_rn(fa, nint_f(fa));
    z = __fmul_rn(fc, L.clatz);
    y = __fadd_rn(__fmul_rn(fb, L.blaty), __fmul_rn(fc, L.claty));
    x = __fadd_rn(__fadd_rn(__fmul_rn(fa, L.alatx), __fmul_rn(fb, L.blatx)), __fmul_rn(fc, L.clatx));
}

__device__ __forceinline__ float dist_f(const Lattice &L, float xd, float yd, float zd) {
    minimagec(L, xd, yd, zd);
    float dsq = __fadd_rn(__fadd_rn(__fmul_rn(xd, xd), __fmul_rn(yd, yd)), __fmul_rn(zd, zd));
    return __fsqrt_rn(dsq);
}

// ----------------------------------------------------------------- pair energy
struct Tables {
    const float4 *tab;   // [npairs*ld] {xavs, xavs1, ecoul, ecoul1}
    const float *xstar;  // [ld]
    int ld, npt2, izcut;
    float stepcl;
};

// en_atom_inter_scale molfit.py:1251-1279 (scalefac = 1).  d is the minimum-image distance.
// Beyond izcut every table entry is +0, so the reference's value there is exactly +0.
// Branch-free: the table is read at iz clamped into 2..izcut and the result replaced by +0
// outside that range, so the loads of consecutive pairs can be in flight together.
__device__ __forceinline__ float pair_energy_d(const Tables &T, float d, int icref) {
    float rat = __fdiv_rn(d, T.stepcl);
    int iz = ifix(rat) + 2;
    const bool in = iz >= 2 && iz <= T.izcut;  // iz < 2 only for a non-finite distance
    const int izc = min(max(iz, 2), T.izcut);
    const float4 t = __ldg(T.tab + (size_t)icref * T.ld + izc);
    const float dt = __fsub_rn(d, __ldg(T.xstar + izc));
    float sume = __fadd_rn(t.x, __fmul_rn(t.y, dt));
    sume = __fadd_rn(__fadd_rn(sume, t.z), __fmul_rn(t.w, dt));
    return in ? sume : 0.0f;
}

// A squared distance beyond which a pair is certainly past izcut (its value +0): the last
// table point's distance stepcl*(izcut-1), widened by 1e-5 twice to cover the roundings of
// the division and the square root, rounded up to float.
__host__ __device__ inline float skip_dsq(float stepcl, int izcut) {
    const double dc = (double)stepcl * (double)(izcut - 1) * (1.0 + 1e-5);
    return (float)(dc * dc * (1.0 + 1e-5)) * (1.0f + 1e-6f);
}

// pair_energy for a caller that expects most pairs out of range: a pair whose squared
// minimum-image distance exceeds dsq_skip (skip_dsq) contributes +0 without the square root,
// the division or the table reads; every other pair is evaluated exactly as pair_energy.
// Adding +0 to a sum started at +0 never changes it, so skipping is exact.
__device__ __forceinline__ float pair_energy_far(const Lattice &L, const Tables &T, float dsq_skip, float4 p1,
                                                 float4 p2, int icref) {
    float xd = __fsub_rn(p2.x, p1.x), yd = __fsub_rn(p2.y, p1.y), zd = __fsub_rn(p2.z, p1.z);
    minimagec(L, xd, yd, zd);
    const float dsq = __fadd_rn(__fadd_rn(__fmul_rn(xd, xd), __fmul_rn(yd, yd)), __fmul_rn(zd, zd));
    if (dsq > dsq_skip) return 0.0f;
    return pair_energy_d(T, __fsqrt_rn(dsq), icref);
}

__device__ __forceinline__ float pair_energy(const Lattice &L, const Tables &T, float4 p1, float4 p2,
                                             int icref) {
    // xdif = x2 - x1 (molfit.py:1257)
    float d = dist_f(L, __fsub_rn(p2.x, p1.x), __fsub_rn(p2.y, p1.y), __fsub_rn(p2.z, p1.z));
    return pair_energy_d(T, d, icref);
}

// ----------------------------------------------------------------- pair energy by bin edges
// The table index of en_atom_inter_scale is iz = ifix(d / stepcl) + 2 with the quotient
// rounded to float.  The rounded quotient is a non-decreasing function of d, so
// ifix(d / stepcl) >= n exactly when d >= D[n], D[n] being the smallest float whose rounded
// quotient is at least n (bin_edge, found by bisection over the float bit patterns with the
// same IEEE division).  An estimate n0 = ifix(d * cinv), with cinv chosen below 1/stepcl by
// about 2^-20 relative (bins_cinv), never exceeds the true index and falls short of it by at
// most one while n0 + 1 < 2^18, so the index is n0 + (d >= D[n0 + 1]): one multiplication, one
// conversion and one comparison against a tabulated edge instead of the division.  Beyond
// the last nonzero table point (n0 > izcut - 2) the pair is out of range whatever the
// correction, since the estimate never exceeds the index.  A NaN distance gives n0 = 0 and
// no correction, as ifix(NaN) = 0 in the division form, so the NaN propagates the same way.
struct Bins {
    const float4 *tab;    // [npairs*ld] {xavs, xavs1, ecoul, ecoul1}
    const float4 *edge;   // [max(izcut - 1, 1)] {D[n+1], xstar[n+2], xstar[n+3], 0} at n
    int ld, izcut;
    float cinv;
};

__device__ __forceinline__ float bin_edge(float stepcl, int n) {
    unsigned lo = 0u, hi = 0x7f800000u;   // +0 .. +inf
    const float fn = (float)n;
    while (lo < hi) {
        const unsigned mid = lo + ((hi - lo) >> 1);
        if (__fdiv_rn(__uint_as_float(mid), stepcl) >= fn) hi = mid;
        else lo = mid + 1u;
    }
    return __uint_as_float(lo);
}

// one entry of Bins::edge (n = 0 .. max(izcut - 2, 0)); xstar has ld entries
__device__ __forceinline__ float4 bin_edge_entry(float stepcl, const float *xstar, int ld, int n) {
    return make_float4(bin_edge(stepcl, n + 1), xstar[min(n + 2, ld - 1)], xstar[min(n + 3, ld - 1)], 0.0f);
}

// the estimate's multiplier: below 1/stepcl by 2^-20 relative, rounded down (host, double)
inline float bins_cinv(float stepcl) {
    const double c = (1.0 / (double)stepcl) * (1.0 - 1.0 / 1048576.0);
    float f = (float)c;
    if ((double)f > c) f = nextafterf(f, 0.0f);
    return f;
}

// The square of minimagec's cubic branch, (x - nint(x))^2.  nint rounds halves away from zero,
// rint to even; the two differ only when x is an odd multiple of one half, where x - nint(x)
// and x - rint(x) are +0.5 and -0.5 in some order -- the same square.  Away from those points
// they are the same integer, and x - rint(x) is exact (|x| < 2^23; beyond, both are x - x).
// rint is one instruction where the truncation form of nint takes six.
__device__ __forceinline__ float wrap_sq(float x) {
    const float r = __fsub_rn(x, rintf(x));
    return __fmul_rn(r, r);
}

// pair_energy for a cubic box, bit for bit: the same distance, index, table entry and sum
__device__ __forceinline__ float pair_energy_cubic_bins(const Bins &B, float4 p1, float4 p2, int icref) {
    const float d = __fsqrt_rn(__fadd_rn(__fadd_rn(wrap_sq(__fsub_rn(p2.x, p1.x)), wrap_sq(__fsub_rn(p2.y, p1.y))),
                                         wrap_sq(__fsub_rn(p2.z, p1.z))));
    const int n0 = __float2int_rz(__fmul_rn(d, B.cinv));
    const int izm2 = B.izcut - 2;
    const int nc = max(min(n0, izm2), 0);
    const float4 e = __ldg(B.edge + nc);
    const bool up = d >= e.x;
    const int iz = nc + 2 + (up ? 1 : 0);
    const bool in = n0 <= izm2 && iz <= B.izcut;
    const int izc = min(iz, B.izcut);
    const float4 t = __ldg(B.tab + (size_t)icref * B.ld + izc);
    const float dt = __fsub_rn(d, up ? e.z : e.y);
    float sume = __fadd_rn(t.x, __fmul_rn(t.y, dt));
    sume = __fadd_rn(__fadd_rn(sume, t.z), __fmul_rn(t.w, dt));
    return in ? sume : 0.0f;
}

// ----------------------------------------------------------------- ran1 (device, one lane)
// auxiliary_routines.py:324-391 with state {idum, iy, mcall, iv[32]}.
struct Ran1 {
    int32_t idum, iy, mcall;
    int32_t iv[32];
};

__device__ __forceinline__ int32_t ran1_lcg(int32_t idum) {
    int32_t k = idum / 127773;
    idum = 16807 * (idum - k * 127773) - 2836 * k;
    if (idum < 0) idum += 2147483647;
    return idum;
}

__device__ __forceinline__ float ran1_out(int32_t iy) {
    float r = __fmul_rn(4.656612873077393e-10f, (float)iy);
    return r > 0.9999998807907104f ? 0.9999998807907104f : r;
}

// Single-thread generator on a state held in shared or local memory.
__device__ __forceinline__ float ran1_next(Ran1 &s) {
    int32_t idum = s.idum, iy = s.iy;
    if (idum <= 0 || iy == 0) {
        int64_t neg = -(int64_t)idum;
        int32_t w = (int32_t)(uint32_t)(uint64_t)neg;
        idum = w > 1 ? w : 1;
        for (int j = 40; j >= 1; --j) {
            idum = ran1_lcg(idum);
            if (j <= 32) s.iv[j - 1] = idum;
        }
        iy = s.iv[0];
    }
    idum = ran1_lcg(idum);
    int j = iy >> 26;  // iy / NDIV, NDIV = 2^26, iy >= 0
    iy = s.iv[j];
    s.iv[j] = idum;
    s.idum = idum;
    s.iy = iy;
    s.mcall = (int32_t)((uint32_t)s.mcall + 1u);
    return ran1_out(iy);
}

__device__ __forceinline__ void ran1_load(Ran1 &s, const int32_t *g) {
    s.idum = g[0];
    s.iy = g[1];
    s.mcall = g[2];
    for (int i = 0; i < 32; ++i) s.iv[i] = g[3 + i];
}
__device__ __forceinline__ void ran1_store(const Ran1 &s, int32_t *g) {
    g[0] = s.idum;
    g[1] = s.iy;
    g[2] = s.mcall;
    for (int i = 0; i < 32; ++i) g[3 + i] = s.iv[i];
}

// ----------------------------------------------------------------- ran1 (device, one warp)
// a*b mod (2^31 - 1) for a, b < 2^31 - 1: the product is below 2^62 and 2^31 = 1 modulo the
// Mersenne prime, so the high and low 31-bit halves are added and at most two moduli
// subtracted -- the exact residue, as Schrage's method computes it.
__device__ __forceinline__ uint32_t r1_mulmod(uint32_t a, uint32_t b) {
    const uint64_t x = (uint64_t)a * (uint64_t)b;
    uint32_t r = (uint32_t)(x & 0x7fffffffull) + (uint32_t)(x >> 31);
    r = r >= 2147483647u ? r - 2147483647u : r;
    r = r >= 2147483647u ? r - 2147483647u : r;
    return r;
}

// 32 steps of the shuffle when no value of the batch can be zero: idl is this lane's Park-
// Miller value of the batch (step lane+1), iv this lane's table entry, iy warp-uniform.  The
// only dependence from step to step is the next slot, the top 5 bits of the value in slot
// j; each lane keeps those bits of its entry beside it, so a step's critical path is one
// shuffle of the 5-bit slot numbers.  The value itself and the step's Park-Miller value
// (which the lane owning slot j keeps) are shuffled beside it.  Returns the value of step
// `lane`; updates iv, iy.
__device__ __forceinline__ int32_t ran1_chain32(int32_t idl, int32_t &iv, int32_t &iy) {
    const int lane = threadIdx.x & 31;
    int32_t y = iy, mine = 0;
    int j = y >> 26;            // iy / NDIV, NDIV = 2^26
    int t5 = iv >> 26;          // the next slot after this lane's entry
#pragma unroll
    for (int s = 0; s < 32; ++s) {
        const int jn = __shfl_sync(0xffffffffu, t5, j);
        const int32_t id = __shfl_sync(0xffffffffu, idl, s);
        y = __shfl_sync(0xffffffffu, iv, j);
        const bool own = lane == j;
        iv = own ? id : iv;
        t5 = own ? (id >> 26) : t5;
        mine = (lane == s) ? y : mine;
        j = jn;
    }
    iy = y;
    return mine;
}

// Warp-cooperative batch of the ran1 stream: lane l holds table entry iv[l]; idum/iy are
// warp-uniform.  The Park-Miller values of the batch are jumped ahead (lane l: IA^(l+1) *
// idum mod IM, the value Schrage's method computes) and the Bays-Durham shuffle is walked
// with one shuffle per step.  When no value of the batch can be zero (no zero idum in the
// batch, no zero table entry, iy != 0) the 32 steps run unrolled without checks; otherwise
// the batch stops after a step that leaves idum or iy at zero, where the reference
// re-initialises (auxiliary_routines.py:346).  Returns the number of values produced; lane
// t < count receives its value in *mine.
__device__ __forceinline__ int ran1_warp_batch(int32_t &idum, int32_t &iy, int32_t &iv, uint32_t lane_mul, int want,
                                               int32_t &mine, int32_t *tab_tmp /* smem [34] */) {
    const int lane = threadIdx.x & 31;
    if (idum <= 0 || iy == 0) {  // (re)initialisation
        if (lane == 0) {
            int64_t neg = -(int64_t)idum;
            int32_t w = (int32_t)(uint32_t)(uint64_t)neg;
            int32_t d = w > 1 ? w : 1;
            for (int j = 40; j >= 1; --j) {
                d = ran1_lcg(d);
                if (j <= 32) tab_tmp[j - 1] = d;
            }
            tab_tmp[32] = d;
        }
        __syncwarp();
        idum = tab_tmp[32];
        iy = tab_tmp[0];
        iv = tab_tmp[lane];
        __syncwarp();
    }
    const int32_t idl = (int32_t)r1_mulmod(lane_mul, (uint32_t)idum);
    int cnt = want < 32 ? want : 32;
    const unsigned zero = __ballot_sync(0xffffffffu, idl == 0) | __ballot_sync(0xffffffffu, iv == 0);
    mine = 0;
    if (cnt == 32 && zero == 0u && iy != 0) {
        mine = ran1_chain32(idl, iv, iy);
        idum = __shfl_sync(0xffffffffu, idl, 31);
        return 32;
    }
    const unsigned z2 = __ballot_sync(0xffffffffu, lane < cnt && idl == 0);
    if (z2) cnt = __ffs(z2);
    int s = 0;
    while (s < cnt) {
        const int32_t id = __shfl_sync(0xffffffffu, idl, s);
        const int j = iy >> 26;
        const int32_t nxt = __shfl_sync(0xffffffffu, iv, j);
        if (lane == j) iv = id;
        iy = nxt;
        if (lane == s) mine = iy;
        ++s;
        if (iy == 0) break;
    }
    idum = __shfl_sync(0xffffffffu, idl, s - 1);
    return s;
}

// A warp's ran1 stream in batches of 32, the Park-Miller values of the next batch computed
// while the current batch's shuffle chain runs (they depend only on the batch's last value).
// Bit-identical to ran1_warp_batch, which it falls back to for batches that can meet a zero
// or a re-initialisation.  Once a batch has started from idum in 1..IM-1 with no zero table
// entry, every later value is a Park-Miller value of such an idum and so nonzero (IM is
// prime): the stream is `clean` and the checks are skipped from then on.
struct Ran1Warp {
    int32_t idum, iy, iv;   // idum, iy warp-uniform; iv this lane's table entry
    uint32_t mul;           // IA^(lane+1) mod IM
    int32_t idl;            // this lane's Park-Miller value of the next batch, when idl_ok
    bool idl_ok, clean;

    __device__ __forceinline__ void load(const int32_t *state) {
        const int lane = threadIdx.x & 31;
        idum = state[0];
        iy = state[1];
        iv = state[3 + lane];
        mul = 16807u;
        for (int k = 0; k < lane; ++k) mul = r1_mulmod(mul, 16807u);
        idl_ok = false;
        clean = false;
    }
    // Up to `want` (<= 32) values; lane t < return value receives value t in `mine`.
    __device__ __forceinline__ int next(int want, int32_t &mine, int32_t *tab_tmp) {
        if (want == 32 && (clean || (idum > 0 && idum < 2147483647 && iy != 0 &&
                                     __ballot_sync(0xffffffffu, iv == 0) == 0u))) {
            clean = true;
            if (!idl_ok) idl = (int32_t)r1_mulmod(mul, (uint32_t)idum);
            const int32_t last = __shfl_sync(0xffffffffu, idl, 31);
            const int32_t nidl = (int32_t)r1_mulmod(mul, (uint32_t)last);
            mine = ran1_chain32(idl, iv, iy);
            idum = last;
            idl = nidl;
            idl_ok = true;
            return 32;
        }
        idl_ok = false;
        return ran1_warp_batch(idum, iy, iv, mul, want, mine, tab_tmp);
    }
};

// ----------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace epsr

// Error plumbing shared by the ABI translation units.
// Kernel timing for measurement (epsr_timing_enable / epsr_timing_read): while enabled, the
// launches of the main kernels are bracketed by CUDA events on their launch stream.
// epsr_timing_mark(name, s, 0) before the launch, epsr_timing_mark(name, s, 1) after it.
extern int g_epsr_timing_on;
void epsr_timing_mark(const char *name, cudaStream_t s, int end);
#define EPSR_TIMED(name, s, ...)                           \
    do {                                                   \
        if (g_epsr_timing_on) epsr_timing_mark(name, s, 0); \
        __VA_ARGS__;                                       \
        if (g_epsr_timing_on) epsr_timing_mark(name, s, 1); \
    } while (0)
void epsr_set_error(const char *fmt, ...);
int epsr_cuda_check(cudaError_t e, const char *what);
int epsr_d2h(void *dst, const void *src, size_t bytes, cudaStream_t s);
int epsr_h2d(void *dst, const void *src, size_t bytes, cudaStream_t s);
// device -> pageable host copy after the stream drained (epsr_d2h); returns on error
#define EPSR_D2H(dst, src, bytes, s)                             \
    do {                                                         \
        const int _r = epsr_d2h((dst), (src), (bytes), (s));     \
        if (_r) return _r;                                       \
    } while (0)
#define EPSR_H2D(dst, src, bytes, s)                             \
    do {                                                         \
        const int _r = epsr_h2d((dst), (src), (bytes), (s));     \
        if (_r) return _r;                                       \
    } while (0)
#define EPSR_CUDA(call)                                              \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return epsr_cuda_check(_e, #call);    \
    } while (0)

// Raise a kernel's dynamic shared-memory limit to the device's opt-in maximum (less the
// kernel's static shared memory), once per
// kernel and device (ordinal < 64).  Changing a kernel's attribute waits for its running
// instances, so a call on every launch would serialise the same kernel across streams;
// after the first call no launch touches the attribute again.
#define EPSR_SMEM_OPTIN(kernel)                                                                      \
    do {                                                                                             \
        static std::atomic<unsigned long long> _optin_done{0};                                       \
        int _dev = 0;                                                                                \
        EPSR_CUDA(cudaGetDevice(&_dev));                                                             \
        if (_dev < 0 || _dev >= 64 || !((_optin_done.load() >> _dev) & 1ull)) {                      \
            int _mx = 0;                                                                             \
            cudaFuncAttributes _fa;                                                                  \
            EPSR_CUDA(cudaDeviceGetAttribute(&_mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, _dev));  \
            EPSR_CUDA(cudaFuncGetAttributes(&_fa, kernel));                                          \
            EPSR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                           _mx - (int)_fa.sharedSizeBytes));                         \
            if (_dev >= 0 && _dev < 64) _optin_done.fetch_or(1ull << _dev);                          \
        }                                                                                            \
    } while (0)
