// fitexp.cu -- fit_expansion (epsr_standalone_rev3.py:4806-4921) on one thread-block cluster.
//
// The Monte Carlo fit is a chain of trials: perturb every coefficient (one ran1 draw each),
// evaluate chi^2 over all Q rows, Metropolis-accept (one more draw when 0 < exponent <= 20),
// smooth the coefficients every nfreq acceptances (smoop auxiliary_routines.py:744).  One
// launch fits any number of data sets in turn on the same basis, continuing one ran1
// stream, as the reference's successive calls do.
//
// Layout.  The basis rows are split over the CTAs of a cluster; each keeps its rows in
// shared memory for the whole launch, four terms to a 16-byte word, except the first 64
// terms of each row, which its thread holds in registers; a thread evaluates its row per
// trial (expand :4924, the sequential clamped sum of a row).  Every partial
// sum of a row is bounded by the row's L1 norm times the largest |coefficient|; when that
// bound stays below the clamp level (e^25) the clamp cannot act and the plain sequential
// sum is the reference's value, otherwise the row is summed with the clamp.  The CTAs
// exchange their chi^2 contributions through distributed shared memory: each pushes its
// part (a double partial, or every residual for the reference's sequential float sum) into
// every CTA and arrives on that CTA's mbarrier; each then forms the same chi^2, so all take
// the same decisions without a second exchange.  Thread 0 of each CTA takes every decision
// (Metropolis test, smoothing, stopping) and broadcasts it through shared memory, so all
// threads pass the same barriers.
//
// ran1.  The chain is sequential; warp 15 of every CTA generates the same stream into a
// ring in its CTA's shared memory, running ahead of the trials (bounded by the ring) and
// publishing how many values exist.  Rows and coefficients are handled by the warps of the
// other three schedulers of the SM (warps 0-2, 4-6, 8-10, 12-14), so the generator's
// scheduler is left to it; warps 3, 7 and 11 only take part in the barriers.  The workers
// synchronise among themselves with a named barrier that the generator warp is not part of.
// At the end the state the reference leaves after exactly the values the fit consumed is
// rebuilt from the generator's per-batch checkpoints.
//
// Every wait (ring, exchange, ring space) is bounded in time: on timeout the kernel records
// status 1, stops the fit and returns.
#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace epsr {

constexpr int FX_THREADS = 512;
constexpr int FX_WARPS = FX_THREADS / 32;
constexpr int FX_GEN_WARP = 15;                 // the stream warp
constexpr int FX_NBAR = 480;                    // threads of the worker barrier (warps 0-14)
constexpr int FX_SLOTS = 384;                   // row / coefficient slots (12 warps, schedulers 0-2)
constexpr int FX_RQ = 16;                       // leading quads of a row held in its thread's registers
constexpr int FX_RING = 2048;                   // ran1 values held per worker CTA (power of two)
constexpr int FX_CK = 128;                      // generator checkpoints (power of two)
constexpr int FX_CKE = 8;                       // batches between checkpoints (power of two)
constexpr int FX_GB = 4;                        // generator batches between reads of the control words
constexpr int FX_CKW = 36;                      // ints per checkpoint: idum, iy, iv[32], pad[2]
constexpr unsigned long long FX_WAIT_NS = 2000000000ull;  // a wait gives up after 2 s

struct FxDev {
    const float *expr;        // expr[(i-1)*nterms + m] (1-based flat, row-major by Q)
    const float *yin;         // [nprob][npt+1]
    float *yout;              // [nprob][npt+1]
    float *wt_g, *wtold_g;    // [nprob][nterms+1]
    float *scal;              // [nprob][4] {stepr, acceptr, rejrat, chisq}
    long long *trials;        // [nprob]
    int *status;              // [1]: 0 ok, 1 a bounded wait gave up
    int nprob, nmin, npt, ncfirst, nterms, nits, nfreq, strict, rpc;
    int32_t *ran1;
};

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t map_rank(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cl_f32(uint32_t a, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cl_f64(uint32_t a, double v) {
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void st_cl_s64(uint32_t a, long long v) {
    asm volatile("st.shared::cluster.b64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release_cl_s64(uint32_t a, long long v) {
    asm volatile("st.release.cluster.shared::cluster.b64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release_cl_s32(uint32_t a, int v) {
    asm volatile("st.release.cluster.shared::cluster.b32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ long long ld_relaxed_cl_s64(uint32_t a) {
    long long v;
    asm volatile("ld.relaxed.cluster.shared::cluster.b64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ long long ld_acquire_s64(const long long *p) {
    long long v;
    asm volatile("ld.acquire.cluster.shared::cta.b64 %0, [%1];" : "=l"(v) : "r"(smem_addr(p)) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_s32(const int *p) {
    int v;
    asm volatile("ld.acquire.cluster.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(smem_addr(p)) : "memory");
    return v;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t a) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
// Barrier of the worker warps (0-14) after code in which a warp may have diverged (a
// bounded spin, a branch on the thread index): the warp is reconverged first, because the
// barrier requires every thread of a warp to arrive together.
__device__ __forceinline__ void block_sync() {
    __syncwarp();
    asm volatile("bar.sync 1, %0;" ::"n"(FX_NBAR) : "memory");
}
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct FxShared {                 // statically sized control block (one per CTA)
    long long cons;               // lowest stream index the workers may still read
    int done;                     // set by the workers when the fit is over
    int abort, stop;
    int accept, smooth, draw;     // thread 0's decision of the current trial
    float val;                    // chi^2 broadcast
    float wfix;                   // largest |wt| of the unperturbed terms 1..ncfirst-1
    float wmx[FX_WARPS];          // largest |wt| of the terms each warp perturbed
    double red[FX_WARPS];
};

__host__ __device__ inline int fx_ntq(int nt) { return (nt + 3) / 4; }
// quads of a row kept in shared memory (those after the first FX_RQ)
__host__ __device__ inline int fx_nsq(int nt) { return fx_ntq(nt) > FX_RQ ? fx_ntq(nt) - FX_RQ : 0; }
// floats per exchange buffer: every row of the cluster, padded to whole 16-byte words so the
// second buffer starts 16-byte aligned (it is read four rows at a time)
__host__ __device__ inline int fx_gstride(int nw, int rpc) { return (nw * rpc + 3) & ~3; }

size_t fx_smem_bytes(int nt, int rpc, int nw) {
    const int ntq = fx_ntq(nt);
    size_t b = 0;
    b += 16 * (size_t)fx_nsq(nt) * rpc;                 // ex4
    b += sizeof(float) * (size_t)rpc;                   // yr
    b += sizeof(float) * (size_t)rpc;                   // e1 (row L1 norms)
    b = (b + 15) & ~(size_t)15;
    b += sizeof(float) * (4 + 4 * (size_t)ntq);         // wt (wt + 1 16-byte aligned)
    b += sizeof(float) * (size_t)(nt + 1);              // wtold
    b = (b + 15) & ~(size_t)15;
    b += sizeof(unsigned long long) * FX_RING;          // ring
    b = (b + 15) & ~(size_t)15;
    b += sizeof(float) * 2 * (size_t)fx_gstride(nw, rpc);   // gat[2][gstride]
    b = (b + 15) & ~(size_t)15;
    b += sizeof(double) * 2 * (size_t)nw;               // parts[2][nw]
    b += sizeof(uint64_t) * 2;                          // exchange mbarriers
    b += sizeof(long long) * FX_CK;                     // ckpos
    b += sizeof(int32_t) * FX_CK * FX_CKW;              // checkpoints
    return b;
}

__global__ void __launch_bounds__(FX_THREADS, 1) fitexp_cluster_kernel(FxDev F) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int nw = (int)cl.num_blocks();
    extern __shared__ __align__(16) unsigned char fx_raw[];
    __shared__ FxShared S;
    __shared__ int32_t g_tab[34];
    const int nt = F.nterms, rpc = F.rpc, ntq = fx_ntq(nt);
    const int nsq = fx_nsq(nt);
    // [nsq*rpc]: ex4[q*rpc + r] = terms 4(FX_RQ+q)..4(FX_RQ+q)+3 of row r
    float4 *ex4 = (float4 *)fx_raw;
    float *yr = (float *)(ex4 + (size_t)nsq * rpc);     // [rpc]
    float *e1 = yr + rpc;                               // [rpc] sum over terms of |basis value|
    size_t off = ((size_t)((unsigned char *)(e1 + rpc) - fx_raw) + 15) & ~(size_t)15;
    float *wt = (float *)(fx_raw + off) + 3;            // wt[0..4*ntq]; wt + 1 is 16-byte aligned
    float *wtold = wt + 1 + 4 * ntq;                    // [nt+1]
    off = ((size_t)((unsigned char *)(wtold + nt + 1) - fx_raw) + 15) & ~(size_t)15;
    // [FX_RING] stream values, each with its position + 1 in the high word, so a reader knows
    // from the one 8-byte load whether the value it wants is there yet
    unsigned long long *ring = (unsigned long long *)(fx_raw + off);
    off = ((size_t)((unsigned char *)(ring + FX_RING) - fx_raw) + 15) & ~(size_t)15;
    float *gat = (float *)(fx_raw + off);               // [2][gstride] residuals by global row
    off = ((off + sizeof(float) * 2 * (size_t)fx_gstride(nw, rpc)) + 15) & ~(size_t)15;
    double *parts = (double *)(fx_raw + off);           // [2][nw]
    uint64_t *xbar = (uint64_t *)(parts + 2 * nw);      // [2]
    long long *ckpos = (long long *)(xbar + 2);         // [FX_CK]
    int32_t *ck = (int32_t *)(ckpos + FX_CK);           // [FX_CK][FX_CKW]

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    volatile FxShared *vs = &S;
    const int row0 = 1 + rank * rpc;                    // first (1-based) row of this CTA
    const int nrow = max(0, min(rpc, F.npt - row0 + 1));
    for (int idx = tid; idx < nsq * rpc; idx += blockDim.x) {
        const int q = idx / rpc, r = idx - q * rpc;
        float e[4];
        for (int j = 0; j < 4; ++j) {
            const int m = 4 * (FX_RQ + q) + j;          // 0-based term
            e[j] = (r < nrow && m < nt) ? F.expr[1 + (size_t)(row0 - 1 + r) * nt + m] : 0.0f;
        }
        ex4[idx] = make_float4(e[0], e[1], e[2], e[3]);
    }
    for (int i = tid; i <= 4 * ntq; i += blockDim.x) wt[i] = 0.0f;   // terms past nterms stay zero
    for (int r = tid; r < rpc; r += blockDim.x) {
        float a = 0.0f;
        for (int m = 0; m < nt && r < nrow; ++m) a = __fadd_ru(a, fabsf(F.expr[1 + (size_t)(row0 - 1 + r) * nt + m]));
        e1[r] = a;
    }
    for (int i = tid; i < FX_CK; i += blockDim.x) ckpos[i] = -1;
    for (int i = tid; i < FX_RING; i += blockDim.x) ring[i] = 0ull;   // no position yet
    if (tid < FX_WARPS) S.wmx[tid] = 0.0f;
    if (tid == 0) {
        S.cons = 0;
        S.done = 0;
        S.abort = 0;
        S.stop = 0;
        mbar_init(&xbar[0], (uint32_t)nw);
        mbar_init(&xbar[1], (uint32_t)nw);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const int32_t mcall0 = F.ran1[2];
    cl.sync();

    // ================================================================ stream warp
    if (wid == FX_GEN_WARP) {
        Ran1Warp g;
        g.load(F.ran1);
        long long pos = 0, nb = 0;
        unsigned long long t0 = 0;
        // the warp is converged at the top of every pass, so each control word is read by one
        // warp-wide load and every lane takes the same branch
        while (true) {
            __syncwarp();
            if (vs->done) break;
            const long long room = vs->cons + FX_RING - pos;
            if (room < 32) {   // ring full: wait for the workers (bounded)
                int give_up = 0;
                if (lane == 0) {
                    const unsigned long long t = now_ns();
                    if (t0 == 0) t0 = t;
                    else if (t - t0 > FX_WAIT_NS || vs->abort) {
                        atomicExch(F.status, 1);
                        vs->abort = 1;
                        give_up = 1;
                    }
                }
                if (__shfl_sync(0xffffffffu, give_up, 0)) break;
                __nanosleep(64);
                continue;
            }
            t0 = 0;
            // up to FX_GB batches before the control words are read again
            const int nbat = room >= 32 * FX_GB ? FX_GB : (int)(room >> 5);
            for (int bi = 0; bi < nbat; ++bi) {
                if ((nb & (FX_CKE - 1)) == 0) {   // the state before this batch, every FX_CKE batches
                    const int slot = (int)((nb / FX_CKE) & (FX_CK - 1));
                    ck[slot * FX_CKW + 2 + lane] = g.iv;
                    if (lane == 0) {
                        ck[slot * FX_CKW + 0] = g.idum;
                        ck[slot * FX_CKW + 1] = g.iy;
                        ckpos[slot] = pos;
                    }
                }
                ++nb;
                int32_t mine;
                const int cnt = g.next(32, mine, g_tab);
                if (lane < cnt) {
                    const long long q = pos + lane;
                    ring[q & (FX_RING - 1)] = ((unsigned long long)(uint32_t)(q + 1) << 32) |
                                              (unsigned long long)__float_as_uint(ran1_out(mine));
                }
                pos += cnt;
            }
        }
        __syncwarp();
        __syncthreads();   // meets the workers after they set done (barrier 0, all 512 threads)
        cl.sync();
        return;
    }

    // ================================================================ workers (warps 0-14)
    const float summax = exp_r(25.0f);
    const int K = nt - F.ncfirst + 1;                   // draws per trial
    // row / coefficient slot of this thread: the warps of schedulers 0-2, -1 otherwise
    const int slot = (wid & 3) != 3 ? (wid - (wid >> 2)) * 32 + lane : -1;
    const int swarp = (wid & 3) != 3 ? wid - (wid >> 2) : -1;   // slot warp 0..11
    const int ic = (slot >= 0 && slot < K) ? F.ncfirst + slot : -1;   // coefficient this thread perturbs
    // the first FX_RQ quads of this thread's row (row `slot`), in registers for the launch
    float4 rq[FX_RQ];
#pragma unroll
    for (int k = 0; k < FX_RQ; ++k) {
        float e[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (slot >= 0 && slot < nrow) {
            for (int j = 0; j < 4; ++j) {
                const int m = 4 * k + j;
                if (m < nt) e[j] = F.expr[1 + (size_t)(row0 - 1 + slot) * nt + m];
            }
        }
        rq[k] = make_float4(e[0], e[1], e[2], e[3]);
    }

    // stream value idx, once the generator has written it (a bounded wait, given up at once
    // after an abort)
    auto get = [&](long long idx) -> float {
        const volatile unsigned long long *e = ring + (idx & (FX_RING - 1));
        const uint32_t want = (uint32_t)(idx + 1);
        unsigned long long v = *e;
        if ((uint32_t)(v >> 32) != want) {
            const unsigned long long t0 = now_ns();
            while (true) {
                __nanosleep(32);
                v = *e;
                if ((uint32_t)(v >> 32) == want || vs->abort) break;
                if (now_ns() - t0 > FX_WAIT_NS) {
                    atomicExch(F.status, 1);
                    vs->abort = 1;
                    break;
                }
            }
        }
        return __uint_as_float((uint32_t)v);
    };

    // state of the trial loop that thread 0's Metropolis decision reads (the same in every
    // worker thread)
    long long cursor = 0;
    float chisqold = 0.0f, accept = 0.0f;
    int icount = 0;

    // the largest |wt| over the perturbed terms, for the clamp bound (thread 0; a barrier
    // follows before any row reads it)
    auto wmax_all = [&]() {
        float b = 0.0f;
        for (int m = F.ncfirst; m <= nt; ++m) b = fmaxf(b, fabsf(wt[m]));
        vs->wmx[0] = b;
        for (int k = 1; k < FX_WARPS; ++k) vs->wmx[k] = 0.0f;
    };
    // the Metropolis test (:4871-4880) and the smoothing (:4882-4893) of trial chi^2 cn,
    // taken by thread 0 and published in the control block
    auto decide = [&](float cn) {
        const float exponent = __fdiv_rn(__fsub_rn(cn, chisqold), accept);
        float test;
        int draw = 0;
        if (exponent > 0.0f && exponent <= 20.0f) {
            test = __fsub_rn(exp_r(-exponent), get(cursor));
            draw = 1;
        } else if (exponent > 20.0f) {
            test = -1.0f;
        } else {
            test = 1.0f;
        }
        const int acc = test >= 0.0f;
        int sm = 0;
        if (acc && icount + 1 == F.nfreq) {
            sm = 1;        // smoop(ncfirst, nterms, 1, wt)
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
            wmax_all();
        }
        vs->accept = acc;
        vs->smooth = sm;
        vs->draw = draw;
        vs->stop = vs->abort;
        vs->cons = cursor + draw;
    };

    int xb = 0;                                         // exchange buffer
    uint32_t xph = 0u;                                  // mbarrier phase parity, bit b for buffer b
    // chi^2 of the current wt over rows nmin..npt, the same value in every CTA, returned to
    // all workers; with `trial`, thread 0 also takes the Metropolis decision on it before the
    // result is published.  Rows, a worker barrier, then warp 0 alone: it forms this CTA's
    // part, lane d pushes it into CTA d and arrives on CTA d's mbarrier (the nw pushes in
    // parallel), lane 0 waits for every CTA's part and thread 0 forms the total in a fixed
    // order; a second barrier publishes it.  strict_sum: the reference's sequential float sum
    // over rows of the residuals that every row thread pushed to every CTA; else a double sum.
    // yout, if given, receives this CTA's row sums.
    auto chisq = [&](bool strict_sum, float *yout, bool trial) -> float {
        float *gb = gat + (size_t)xb * fx_gstride(nw, rpc);
        double mypart = 0.0;
        if (slot >= 0) {
            float wmax = vs->wfix;
            const float *wm = (const float *)S.wmx;   // complete since the last barrier
#pragma unroll
            for (int k = 0; k < FX_WARPS; ++k) wmax = fmaxf(wmax, wm[k]);
            if (slot < nrow) {
                const int r = slot;
                float sum = 0.0f;
                const float4 *w4 = (const float4 *)(wt + 1);
                const float4 *e4 = ex4 + r;
                // every partial sum is at most e1[r] * max|wt| (times 1 + 2^-20 for rounding)
                if (__fmul_ru(__fmul_ru(e1[r], wmax), 1.001f) < summax) {
#pragma unroll
                    for (int k = 0; k < FX_RQ; ++k) {
                        if (k < ntq) {
                            const float4 c = w4[k];
                            sum = __fadd_rn(sum, __fmul_rn(rq[k].x, c.x));
                            sum = __fadd_rn(sum, __fmul_rn(rq[k].y, c.y));
                            sum = __fadd_rn(sum, __fmul_rn(rq[k].z, c.z));
                            sum = __fadd_rn(sum, __fmul_rn(rq[k].w, c.w));
                        }
                    }
#pragma unroll 2
                    for (int q = 0; q < nsq; ++q) {
                        const float4 c = w4[FX_RQ + q];
                        const float4 e = e4[q * rpc];
                        sum = __fadd_rn(sum, __fmul_rn(e.x, c.x));
                        sum = __fadd_rn(sum, __fmul_rn(e.y, c.y));
                        sum = __fadd_rn(sum, __fmul_rn(e.z, c.z));
                        sum = __fadd_rn(sum, __fmul_rn(e.w, c.w));
                    }
                } else {  // the reference's clamped sum (expand :4924)
#pragma unroll
                    for (int k = 0; k < FX_RQ; ++k) {
                        const float ev[4] = {rq[k].x, rq[k].y, rq[k].z, rq[k].w};
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int m = 4 * k + j;
                            if (m < nt) {
                                sum = __fadd_rn(sum, __fmul_rn(ev[j], wt[1 + m]));
                                if (fabsf(sum) > summax) sum = fsign(summax, sum);
                            }
                        }
                    }
                    for (int m = 4 * FX_RQ; m < nt; ++m) {
                        const float *ee = (const float *)(e4 + ((m >> 2) - FX_RQ) * rpc);
                        sum = __fadd_rn(sum, __fmul_rn(ee[m & 3], wt[1 + m]));
                        if (fabsf(sum) > summax) sum = fsign(summax, sum);
                    }
                }
                const int i = row0 + r;
                const float term = __fsub_rn(yr[r], sum);
                const float q2 = __fmul_rn(term, term);
                if (yout) yout[i] = sum;
                if (strict_sum) {
                    const uint32_t la = smem_addr(gb + (rank * rpc + r));
                    for (int d = 0; d < nw; ++d) st_cl_f32(map_rank(la, (uint32_t)d), q2);
                } else if (i >= F.nmin) {
                    mypart += (double)q2;
                }
            }
        }
        __syncwarp();
        if (strict_sum) {
            fence_cluster();
        } else {
            mypart = warp_sum_d(mypart);
            if (lane == 0) vs->red[wid] = mypart;
        }
        block_sync();
        if (wid == 0) {
            const uint32_t ba = smem_addr(&xbar[xb]);
            double t = 0.0;
            if (!strict_sum) t = warp_sum_d(lane < FX_GEN_WARP ? vs->red[lane] : 0.0);
            if (lane < nw) {
                if (!strict_sum) st_cl_f64(map_rank(smem_addr(parts + xb * nw + rank), (uint32_t)lane), t);
                mbar_arrive_cluster(map_rank(ba, (uint32_t)lane));
            }
            if (lane == 0) {
                const uint32_t par = (xph >> xb) & 1u;
                if (!mbar_test(ba, par)) {
                    const unsigned long long t0 = now_ns();
                    while (!mbar_test(ba, par)) {
                        if (vs->abort || now_ns() - t0 > FX_WAIT_NS) {
                            atomicExch(F.status, 1);
                            vs->abort = 1;
                            break;
                        }
                    }
                }
                float v;
                if (strict_sum) {
                    const int a = F.nmin - 1, b = F.npt;    // 0-based rows a..b-1
                    float c = 0.0f;
                    int i = a;
                    for (; i < b && (i & 3); ++i) c = __fadd_rn(c, gb[i]);
                    const float4 *g4 = (const float4 *)gb;
                    for (; i + 3 < b; i += 4) {
                        const float4 u = g4[i >> 2];
                        c = __fadd_rn(c, u.x);
                        c = __fadd_rn(c, u.y);
                        c = __fadd_rn(c, u.z);
                        c = __fadd_rn(c, u.w);
                    }
                    for (; i < b; ++i) c = __fadd_rn(c, gb[i]);
                    v = c;
                } else {
                    double u = 0.0;
                    for (int q = 0; q < nw; ++q) u += parts[xb * nw + q];
                    v = (float)u;
                }
                vs->val = v;
                if (trial) decide(v);
            }
        }
        xph ^= 1u << xb;
        xb ^= 1;
        block_sync();
        return vs->val;
    };

    const float acceptr = 0.05f;
    const int npoints = F.npt - F.nmin + 1;
    for (int pi = 0; pi < F.nprob; ++pi) {
        const float *yin = F.yin + (size_t)pi * (F.npt + 1);
        float *yout = F.yout + (size_t)pi * (F.npt + 1);
        const float *wto_g = F.wtold_g + (size_t)pi * (nt + 1);
        float *scal = F.scal + (size_t)pi * 4;
        for (int r = tid; r < rpc; r += FX_NBAR) yr[r] = r < nrow ? yin[row0 + r] : 0.0f;
        for (int i = tid; i <= nt; i += FX_NBAR) {
            wtold[i] = wto_g[i];
            wt[i] = wtold[i];
        }
        block_sync();
        if (tid == 0) {
            float a = 0.0f;
            for (int m = 1; m < F.ncfirst; ++m) a = fmaxf(a, fabsf(wt[m]));
            vs->wfix = a;
            wmax_all();
        }
        block_sync();
        float stepr = scal[0];
        float rejrat = scal[2];
        float chisqnew = scal[3];
        long long trials = 0;
        float wtmax = 0.0f;
        for (int it = 1; it <= nt; ++it) {
            const float a = fabsf(wt[it]);
            wtmax = (a >= wtmax) ? a : wtmax;
        }
        if (stepr < __fmul_rn(1.0e-6f, wtmax)) stepr = __fmul_rn(2.0e-6f, wtmax);
        if (F.nits > 0 && !vs->stop) {
            icount = 0;
            chisqnew = chisq(F.strict != 0, nullptr, false);
            chisqold = chisqnew;
            float chisqtest = -1.0f;
            int itry = 0;
            bool stop = false;
            while (!stop && (itry < 10 || (itry < 150 && chisqtest < 1.0e-4f))) {
                ++itry;
                accept = __fdiv_rn(__fmul_rn(acceptr, chisqold), (float)npoints);
                rejrat = 0.0f;
                const float chisqstart = __fdiv_rn(chisqold, (float)npoints);
                for (int st = 1; st <= 100; ++st) {
                    ++trials;
                    // perturb coefficients ncfirst..nterms with the next K values (:4856-4861),
                    // each thread waiting for its own value
                    if (swarp >= 0 && swarp * 32 < K) {
                        float a = 0.0f;
                        if (ic > 0) {
                            const float du = __fsub_rn(__fmul_rn(2.0f, get(cursor + slot)), 1.0f);
                            float v;
                            if (fabsf(wtold[ic]) < 1.0f) v = __fadd_rn(wtold[ic], __fmul_rn(stepr, du));
                            else v = __fmul_rn(wtold[ic], __fadd_rn(1.0f, __fmul_rn(stepr, du)));
                            wt[ic] = v;
                            a = fabsf(v);
                        }
                        a = __int_as_float((int)__reduce_max_sync(0xffffffffu, (unsigned)__float_as_int(a)));
                        if (lane == 0) vs->wmx[swarp] = a;
                    }
                    cursor += K;
                    block_sync();
                    // chi^2 of the trial and thread 0's decision on it (Metropolis, smoothing)
                    const float cn = chisq(F.strict != 0, nullptr, true);
                    const int acc = vs->accept, sm = vs->smooth;
                    stop = vs->stop != 0;
                    cursor += vs->draw;
                    chisqnew = cn;
                    if (acc) {
                        ++icount;
                        if (sm) {
                            icount = 0;
                            chisqnew = chisq(F.strict != 0, nullptr, false);
                        }
                        chisqold = chisqnew;
                        // each thread keeps the coefficient it perturbs (terms below ncfirst
                        // never change); the next trial's perturbation reads only its own
                        if (ic > 0) wtold[ic] = wt[ic];
                    } else {
                        rejrat = __fadd_rn(rejrat, 1.0f);
                    }
                    if (stop) break;
                }
                rejrat = __fdiv_rn(rejrat, 100.0f);
                const float chisqfinish = __fdiv_rn(chisqold, (float)npoints);
                if (chisqstart > 0.0f) chisqtest = __fdiv_rn(__fsub_rn(chisqfinish, chisqstart), chisqstart);
                else chisqtest = __fsub_rn(chisqfinish, chisqstart);
                const float rejfac = rejrat > 0.0f ? __fdiv_rn(0.75f, rejrat) : 2.0f;
                stepr = __fmul_rn(stepr, rejfac);
            }
            block_sync();   // every thread's own wtold update is in
            for (int k = 1 + tid; k <= nt; k += FX_NBAR) wt[k] = wtold[k];
            block_sync();
            if (tid == 0) wmax_all();
            block_sync();
        }
        // final fit over rows 1..npt, chi^2 from nmin (:4908-4914), in the reference's order
        chisqnew = chisq(true, yout, false);
        if (rank == 0) {
            float *wt_g = F.wt_g + (size_t)pi * (nt + 1);
            float *wtold_o = F.wtold_g + (size_t)pi * (nt + 1);
            for (int k = tid; k <= nt; k += FX_NBAR) {
                wt_g[k] = wt[k];
                wtold_o[k] = wtold[k];
            }
            if (tid == 0) {
                scal[0] = stepr;
                scal[1] = acceptr;
                scal[2] = rejrat;
                scal[3] = chisqnew;
                F.trials[pi] = trials;
            }
        }
        block_sync();
    }
    // stop the stream warp, then rebuild the state after exactly `cursor` draws from the
    // last checkpoint at or before it (or from the launch's state when none is left)
    if (tid == 0) vs->done = 1;
    __syncwarp();
    __syncthreads();
    if (rank == 0 && tid == 0 && !vs->abort) {
        int best = -1;
        for (int k = 0; k < FX_CK; ++k)
            if (ckpos[k] >= 0 && ckpos[k] <= cursor && (best < 0 || ckpos[k] > ckpos[best])) best = k;
        Ran1 R;
        long long from = 0;
        ran1_load(R, F.ran1);
        if (best >= 0) {
            R.idum = ck[best * FX_CKW + 0];
            R.iy = ck[best * FX_CKW + 1];
            for (int i = 0; i < 32; ++i) R.iv[i] = ck[best * FX_CKW + 2 + i];
            from = ckpos[best];
        }
        for (long long k = from; k < cursor; ++k) ran1_next(R);
        R.mcall = (int32_t)((uint32_t)mcall0 + (uint32_t)cursor);
        ran1_store(R, F.ran1);
    }
    cl.sync();  // no CTA leaves while others may still write into its shared memory
}

}  // namespace epsr

using namespace epsr;

static inline size_t al256f(size_t x) { return (x + 255) & ~(size_t)255; }

// Smallest cluster whose CTAs hold their rows with one row per slot thread (at most 8 CTAs).
static int fx_workers(int npt, int nterms, int *rpc_out) {
    const size_t budget = 220 * 1024;
    for (int c = 1; c <= 8; ++c) {
        const int rpc = (npt + c - 1) / c;
        if (rpc <= FX_SLOTS && fx_smem_bytes(nterms, rpc, c) <= budget) {
            *rpc_out = rpc;
            return c;
        }
    }
    return 0;
}

extern "C" int64_t epsr_fit_expansion_batch_scratch_bytes(int32_t nprob, int32_t npt, int32_t nterms) {
    (void)npt;
    (void)nterms;
    if (nprob < 1) nprob = 1;
    return (int64_t)(al256f(sizeof(float) * 4 * (size_t)nprob) + al256f(sizeof(long long) * (size_t)nprob) +
                     al256f(sizeof(int)));
}

extern "C" int64_t epsr_fit_expansion_scratch_bytes(int32_t npt, int32_t nterms) {
    return epsr_fit_expansion_batch_scratch_bytes(1, npt, nterms);
}

extern "C" int epsr_fit_expansion_batch(int32_t nprob, const float *yin, const float *expr, float *yout, float *wt,
                                        float *wtold, float *scal_host, int32_t nmin, int32_t npt, int32_t ncfirst,
                                        int32_t nterms, int32_t nits, int32_t nfreq, int32_t *ran1, void *scratch,
                                        int64_t scratch_bytes, int32_t strict, int64_t *trials_host, void *stream) {
    if (nprob <= 0 || !yin || !expr || !yout || !wt || !wtold || !scal_host || !ran1 || !scratch || !trials_host ||
        npt <= 0 || nterms <= 0 || nmin < 1 || nmin > npt || ncfirst < 1 || ncfirst > nterms) {
        epsr_set_error("epsr_fit_expansion_batch: bad arguments");
        return EPSR_ERR_ARG;
    }
    if (scratch_bytes < epsr_fit_expansion_batch_scratch_bytes(nprob, npt, nterms)) {
        epsr_set_error("epsr_fit_expansion_batch: scratch too small");
        return EPSR_ERR_CAPACITY;
    }
    if (nterms - ncfirst + 1 > FX_SLOTS) {
        epsr_set_error("epsr_fit_expansion_batch: at most %d perturbed terms", FX_SLOTS);
        return EPSR_ERR_UNSUPPORTED;
    }
    int rpc = 0;
    const int nw = fx_workers(npt, nterms, &rpc);
    if (!nw) {
        epsr_set_error("epsr_fit_expansion_batch: %d rows x %d terms exceed 8 CTAs of shared memory", npt, nterms);
        return EPSR_ERR_UNSUPPORTED;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *p = (char *)scratch;
    float *scal = (float *)p;
    p += al256f(sizeof(float) * 4 * (size_t)nprob);
    long long *trials = (long long *)p;
    p += al256f(sizeof(long long) * (size_t)nprob);
    int *status = (int *)p;
    EPSR_H2D(scal, scal_host, sizeof(float) * 4 * (size_t)nprob, s);
    EPSR_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
    FxDev F;
    F.expr = expr;
    F.yin = yin;
    F.yout = yout;
    F.wt_g = wt;
    F.wtold_g = wtold;
    F.scal = scal;
    F.trials = trials;
    F.status = status;
    F.nprob = nprob;
    F.nmin = nmin;
    F.npt = npt;
    F.ncfirst = ncfirst;
    F.nterms = nterms;
    F.nits = nits;
    F.nfreq = nfreq;
    F.strict = strict ? 1 : 0;
    F.rpc = rpc;
    F.ran1 = ran1;
    const size_t shm = fx_smem_bytes(nterms, rpc, nw);
    EPSR_SMEM_OPTIN(fitexp_cluster_kernel);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nw, 1, 1);
    cfg.blockDim = dim3(FX_THREADS, 1, 1);
    cfg.dynamicSmemBytes = shm;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = nw;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    EPSR_TIMED("fitexp_cluster_kernel", s, EPSR_CUDA(cudaLaunchKernelEx(&cfg, fitexp_cluster_kernel, F)));
    int hstatus = 0;
    EPSR_D2H(scal_host, scal, sizeof(float) * 4 * (size_t)nprob, s);
    EPSR_D2H(trials_host, trials, sizeof(long long) * (size_t)nprob, s);
    EPSR_D2H(&hstatus, status, sizeof(int), s);
    if (hstatus) {
        epsr_set_error("epsr_fit_expansion: a bounded device wait gave up (results invalid)");
        return EPSR_ERR_TIMEOUT;
    }
    return EPSR_OK;
}

extern "C" int epsr_fit_expansion(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                                  float *scal_host, int32_t nmin, int32_t npt, int32_t ncfirst, int32_t nterms,
                                  int32_t nits, int32_t nfreq, int32_t *ran1, void *scratch, int64_t scratch_bytes,
                                  int32_t strict, int64_t *trials_host, void *stream) {
    return epsr_fit_expansion_batch(1, yin, expr, yout, wt, wtold, scal_host, nmin, npt, ncfirst, nterms, nits, nfreq,
                                    ran1, scratch, scratch_bytes, strict, trials_host, stream);
}
