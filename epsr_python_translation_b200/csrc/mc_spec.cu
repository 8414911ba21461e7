// mc_spec.cu -- molfit whole-molecule cycle (molfit.py:268-448) resolved speculatively.
//
// Within one cycle every molecule moves once, from its cycle-start position, with ran1
// draws at offsets fixed by the visit order (3 rotation + 3 translation + 1 acceptance
// draw per move, molfit.py:382-401).  Only the accept decisions chain the moves together:
// move k sees partner p at p's new position (and p's stored energy written by p's move)
// exactly when p was visited earlier and accepted.  So:
//
//   plan     per-move draw offsets; per-type step sizes (the first-visit initialisation);
//   draws    the cycle's ran1 values in one stream pass;
//   propose  every proposal (rotatm + movem) and its Metropolis threshold, in parallel;
//   energy   for every stored entry (k, p): A = E(new k, old p) and, if p is earlier in
//            the visit order, B = E(new k, new p) -- each in the reference's (ia, ja) order;
//   corr     per move the energy change assuming no earlier partner accepted (base) and
//            the correction c = (B - old') - (A - S) that applies if partner p accepted;
//   resolve  one CTA walks the moves in order: helper warps sum the corrections of
//            partners resolved more than 32 moves ago, the resolver warp adds those of the
//            last 32 with one shuffle reduction and compares with the precomputed threshold;
//   commit   coordinates, the energy store (the later accepted writer of a shared slot
//            wins), counters, step adaptation, fadds and the ran1 state.
//
// Energies of individual molecule pairs are bit-identical to the reference; each move's
// total is summed in double (the reference's float32 order is the sequential kernel in
// mc.cu).  The rare translation retry of movem (a move that leaves the centre unchanged
// doubles the step and draws again, molfit.py:752-758) shifts every later draw; the cycle is
// then discarded and the sequential kernel runs it instead, from the unchanged state.
#include "common.cuh"

namespace epsr {

constexpr int SP_W = 32;        // near window of the resolver (moves)
constexpr int SP_RING = 64;     // far-sum ring (moves)
constexpr int SP_MAXAT = 64;    // atoms of a moved molecule
constexpr int SP_ET = 256;      // threads of a move's energy CTA (its stored partners)
constexpr int SP_RT = 1024;     // resolver CTA: the resolver warp and 31 far-sum helper warps
constexpr long long SP_SPIN_LIMIT = 1ll << 26;

struct SpecDev {
    Lattice L;
    Tables T;
    int N, M, ntype, nmoltype, natom;
    const int32_t *naf, *nato, *mtype, *npairref, *visit;
    const float *xa, *ya, *za, *xadd, *yadd, *zadd;
    float *xa_w, *ya_w, *za_w, *xadd_w, *yadd_w, *zadd_w;
    const float4 *pos;
    float4 *pos_w;
    const int32_t *nergpairm, *molergpair, *ergpairref, *mirror;
    float *ergpair;
    // parameters and persistent state
    float simt, rejrate, stepr, stepm, trstepmax, trstepmin;
    int ireset;
    float *wholerot, *wholetrans, *internrot, *interntrans;
    int32_t *nwhole, *nmovem, *nstepreject;
    float *fadds;
    int32_t *ran1;
    const float *cos_override;
    float *trace_den;
    int32_t *trace_acc;
    int32_t *status;
    // scratch
    int32_t *vpos, *off, *rotidx, *flags;  // flags[0] retry, flags[1] resolver timeout
    float *rotstep, *transstep;            // [nmoltype]
    int32_t *tries_rot, *tries_tr, *rej_rot, *rej_tr, *cnt_type;  // [nmoltype]
    int32_t *ran1_next;                    // [35]
    float *draws;
    float *nx, *ny, *nz;                   // [natom] proposed offsets
    float4 *nc;                            // [N] proposed centres (by molecule)
    float4 *npos;                          // [natom] proposed absolute positions
    float *thr;                            // [N] Metropolis thresholds (by visit position)
    float *A, *B;                          // [N*M]
    double *base, *nearc, *farc;           // [N], [N*W], [N*M]
    int32_t *fv;                           // [N*M]
    int32_t *acc;                          // [N] by visit position
    float *fdiff;                          // [N] by visit position
    double *fadd_acc;                      // [1]
};

// ----------------------------------------------------------------- plan
__global__ void spec_plan_kernel(SpecDev S) {
    __shared__ int carry_s, carry_r;
    const int tid = threadIdx.x;
    if (tid == 0) {
        carry_s = 0;
        carry_r = 0;
    }
    for (int t = tid; t < S.nmoltype; t += blockDim.x) {
        S.rotstep[t] = S.wholerot[t];
        S.transstep[t] = S.wholetrans[t];
        S.tries_rot[t] = S.tries_tr[t] = S.rej_rot[t] = S.rej_tr[t] = S.cnt_type[t] = 0;
    }
    if (tid == 0) {
        S.flags[0] = 0;
        S.flags[1] = 0;
        *S.fadd_acc = 0.0;
    }
    __syncthreads();
    for (int base = 0; base < S.N; base += blockDim.x) {
        const int k = base + tid;
        int nd = 0, nr = 0;
        if (k < S.N) {
            const int m = S.visit[k];
            S.vpos[m] = k;
            const int n = S.nato[m];
            const int t = S.mtype[m];
            atomicAdd(S.cnt_type + t, 1);
            if (S.stepr > 0.0f && n > 1) {
                nd += 3;
                nr = 1;
                atomicAdd(S.tries_rot + t, 1);
            }
            if (S.stepm > 0.0f) {
                nd += 3;
                atomicAdd(S.tries_tr + t, 1);
            }
            nd += 1;
        }
        // block exclusive scans of nd and nr
        __shared__ int wsd[32], wsr[32];
        const int lane = tid & 31, wid = tid >> 5;
        int id = nd, ir = nr;
        for (int o = 1; o < 32; o <<= 1) {
            int a = __shfl_up_sync(0xffffffffu, id, o), b = __shfl_up_sync(0xffffffffu, ir, o);
            if (lane >= o) {
                id += a;
                ir += b;
            }
        }
        if (lane == 31) {
            wsd[wid] = id;
            wsr[wid] = ir;
        }
        __syncthreads();
        if (tid == 0) {
            int a = 0, b = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                int x = wsd[w], y = wsr[w];
                wsd[w] = a;
                wsr[w] = b;
                a += x;
                b += y;
            }
        }
        __syncthreads();
        if (k < S.N) {
            S.off[k] = carry_s + wsd[wid] + id - nd;
            S.rotidx[k] = carry_r + wsr[wid] + ir - nr;
        }
        __syncthreads();
        if (tid == blockDim.x - 1) {
            carry_s += wsd[wid] + id;
            carry_r += wsr[wid] + ir;
        }
        __syncthreads();
    }
    if (tid == 0) S.off[S.N] = carry_s;
    // per-type first-visit initialisation (molfit.py:377-394): a type whose molecules rotate
    // starts at rotstepmin if its step is not positive; otherwise its step is set to 0
    for (int t = tid; t < S.nmoltype; t += blockDim.x) {
        // no molecule of this path has rotational groups: every visited type's internrot is
        // set to 0 (molfit.py:358-360)
        if (S.cnt_type[t] > 0) S.internrot[t] = 0.0f;
        if (S.tries_rot[t] > 0) {
            if (S.rotstep[t] <= 0.0f) S.rotstep[t] = 1.0e-5f;
        }
        if (S.tries_tr[t] > 0) {
            if (S.transstep[t] <= 0.0f) S.transstep[t] = S.trstepmin;
        }
    }
}

// ----------------------------------------------------------------- propose
__device__ __forceinline__ float metropolis_threshold(float u) {
    // smallest e > 0 with exp(-e) <= u (double-evaluated exp rounded to float is monotone),
    // capped at 20: accept  <=>  ediff < threshold   (molfit.py:401-408)
    unsigned lo = 1u, hi = __float_as_uint(20.0f);
    if (!(exp_r(-20.0f) <= u)) return 20.0f;
    while (lo < hi) {
        const unsigned mid = lo + ((hi - lo) >> 1);
        if (exp_r(-__uint_as_float(mid)) <= u) hi = mid;
        else lo = mid + 1;
    }
    return __uint_as_float(lo);
}

__global__ void spec_propose_kernel(SpecDev S) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S.N) return;
    const float pi = 3.14159265358979323846f;
    const int m = S.visit[k];
    const int n = S.nato[m];
    const int a0 = S.naf[m];
    const int t = S.mtype[m];
    const float *u = S.draws + S.off[k];
    int q = 0;
    float x[SP_MAXAT], y[SP_MAXAT], z[SP_MAXAT];
    for (int i = 0; i < n; ++i) {
        x[i] = S.xa[a0 + i];
        y[i] = S.ya[a0 + i];
        z[i] = S.za[a0 + i];
    }
    if (S.stepr > 0.0f && n > 1) {
        const float step = S.rotstep[t];
        for (int ax = 0; ax < 3; ++ax) {
            const float phi = __fmul_rn(__fmul_rn(pi, step), __fsub_rn(__fmul_rn(2.0f, u[q++]), 1.0f));
            const float c = S.cos_override ? S.cos_override[3 * S.rotidx[k] + ax] : cos_r(phi);
            const float sn = fsign(__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(c, c))), phi);
            for (int i = 0; i < n; ++i) {
                if (ax == 0) {
                    const float xs = __fsub_rn(__fmul_rn(x[i], c), __fmul_rn(y[i], sn));
                    y[i] = __fadd_rn(__fmul_rn(x[i], sn), __fmul_rn(y[i], c));
                    x[i] = xs;
                } else if (ax == 1) {
                    const float zs = __fsub_rn(__fmul_rn(z[i], c), __fmul_rn(x[i], sn));
                    x[i] = __fadd_rn(__fmul_rn(z[i], sn), __fmul_rn(x[i], c));
                    z[i] = zs;
                } else {
                    const float ys = __fsub_rn(__fmul_rn(y[i], c), __fmul_rn(z[i], sn));
                    z[i] = __fadd_rn(__fmul_rn(y[i], sn), __fmul_rn(z[i], c));
                    y[i] = ys;
                }
            }
        }
    }
    float cx = S.xadd[m], cy = S.yadd[m], cz = S.zadd[m];
    if (S.stepm > 0.0f) {
        const float st = S.transstep[t];
        const float xs = cx, ys = cy, zs = cz;
        cz = __fadd_rn(cz, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, u[q++]), 1.0f)));
        cy = __fadd_rn(cy, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, u[q++]), 1.0f)));
        cx = __fadd_rn(cx, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, u[q++]), 1.0f)));
        if (xs == cx && ys == cy && zs == cz) atomicExch(S.flags, 1);  // retry: the cycle goes sequential
    }
    const float uacc = u[q];
    S.thr[k] = metropolis_threshold(uacc);
    for (int i = 0; i < n; ++i) {
        S.nx[a0 + i] = x[i];
        S.ny[a0 + i] = y[i];
        S.nz[a0 + i] = z[i];
        S.npos[a0 + i] = make_float4(__fadd_rn(x[i], cx), __fadd_rn(y[i], cy), __fadd_rn(z[i], cz), S.pos[a0 + i].w);
    }
    S.nc[m] = make_float4(cx, cy, cz, 0.0f);
}

// ----------------------------------------------------------------- energies
// E(a, b): a's atoms in shared memory (sa), b's absolute positions in global memory (read
// through the L1 cache for every atom of a, which keeps registers -- and so resident warps --
// free for latency hiding).  The sum runs ia outer, ja inner as en_change (molfit.py:851-882).
__device__ __forceinline__ float mol_energy(const Lattice &L, const Tables &T, const float4 *sa, int na,
                                            const float4 *__restrict__ pb, int nb, const int *spr, int ntype) {
    float sume = 0.0f;
    for (int ia = 0; ia < na; ++ia) {
        const float4 p1 = sa[ia];
        const int *row = spr + __float_as_int(p1.w) * ntype;
#pragma unroll 4
        for (int j = 0; j < nb; ++j) {
            const float4 p2 = __ldg(pb + j);
            sume = __fadd_rn(sume, pair_energy(L, T, p1, p2, row[__float_as_int(p2.w)]));
        }
    }
    return sume;
}

__global__ void __launch_bounds__(SP_ET) spec_energy_kernel(SpecDev S) {
    extern __shared__ int sdyn[];   // npairref [ntype*ntype], then the work list [2*M]
    __shared__ float4 sa[SP_MAXAT];
    __shared__ int cnt[SP_MAXAT + 2];
    if (S.flags[0]) return;
    int *spr = sdyn;
    int *list = sdyn + ((S.ntype * S.ntype + 3) & ~3);
    const int k = blockIdx.x;
    const int m = S.visit[k];
    const int na = S.nato[m], a0 = S.naf[m];
    for (int i = threadIdx.x; i < S.ntype * S.ntype; i += blockDim.x) spr[i] = S.npairref[i];
    for (int i = threadIdx.x; i < na; i += blockDim.x) sa[i] = S.npos[a0 + i];
    for (int i = threadIdx.x; i < SP_MAXAT + 2; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const int nn = S.nergpairm[m];
    const size_t row = (size_t)m * S.M;
    // work items: A for partners 1..nn-1 (item s-1), then B for the same partners (item
    // np+s-1) when the partner is earlier in the visit order.  The items are listed by the
    // partner's atom count, so the lanes of a warp run loops of the same length.
    const int np = nn - 1;
    auto item_nb = [&](int it) -> int {   // atom count (1..SP_MAXAT) of the item's partner, 0 if no item
        const bool second = it >= np;
        const int p = S.molergpair[row + 1 + (second ? it - np : it)];
        if (second && S.vpos[p] >= k) return 0;
        return S.nato[p];
    };
    for (int it = threadIdx.x; it < 2 * np; it += blockDim.x) {
        const int nb = item_nb(it);
        if (nb > 0) atomicAdd(&cnt[nb], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // cnt[b] -> first list position of atom count b; cnt[SP_MAXAT+1] = total
        int a = 0;
        for (int b = 0; b <= SP_MAXAT; ++b) {
            const int c = cnt[b];
            cnt[b] = a;
            a += c;
        }
        cnt[SP_MAXAT + 1] = a;
    }
    __syncthreads();
    for (int it = threadIdx.x; it < 2 * np; it += blockDim.x) {
        const int nb = item_nb(it);
        if (nb > 0) list[atomicAdd(&cnt[nb], 1)] = it;
    }
    __syncthreads();
    const int total = cnt[SP_MAXAT + 1];
    for (int q = threadIdx.x; q < total; q += blockDim.x) {
        const int it = list[q];
        const bool second = it >= np;
        const int s = 1 + (second ? it - np : it);
        const int p = S.molergpair[row + s];
        const int b0 = S.naf[p], nb = S.nato[p];
        const float e = __fadd_rn(0.0f, mol_energy(S.L, S.T, sa, na, (second ? S.npos : S.pos) + b0, nb, spr, S.ntype));
        if (second) S.B[row + s] = e;
        else S.A[row + s] = e;
    }
}

// ----------------------------------------------------------------- corrections
__global__ void __launch_bounds__(128) spec_corr_kernel(SpecDev S) {
    if (S.flags[0]) return;
    const int k = blockIdx.x;
    const int m = S.visit[k];
    const int nn = S.nergpairm[m];
    const size_t row = (size_t)m * S.M;
    double d0s = 0.0;
    for (int s = 1 + threadIdx.x; s < nn; s += blockDim.x) {
        const size_t e = row + s;
        const int p = S.molergpair[e];
        const int kp = S.vpos[p];
        const double sv = (double)S.ergpair[S.ergpairref[e] - 1];
        const double d0 = (double)S.A[e] - sv;
        d0s += d0;
        int fvv = -1;
        if (kp < k) {
            const int e2 = S.mirror[e];
            const int s2 = e2 % S.M;
            const double oldp = s2 >= 1 ? (double)S.A[e2] : sv;
            const double c = ((double)S.B[e] - oldp) - d0;
            const int dist = k - kp;
            if (dist <= SP_W) {
                S.nearc[(size_t)k * SP_W + dist - 1] = c;
            } else {
                S.farc[e] = c;
                fvv = kp;
            }
        }
        S.fv[e] = fvv;
    }
    d0s = warp_sum_d(d0s);
    __shared__ double ws[4];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = d0s;
    __syncthreads();
    if (threadIdx.x == 0) S.base[k] = ws[0] + ws[1] + ws[2] + ws[3];
}

// ----------------------------------------------------------------- resolve
__global__ void __launch_bounds__(SP_RT) spec_resolve_kernel(SpecDev S) {
    extern __shared__ unsigned accbits_raw[];
    volatile unsigned *accbits = accbits_raw;
    __shared__ volatile int progress;
    __shared__ volatile int abort_flag;
    __shared__ volatile int far_ready[SP_RING];
    __shared__ volatile double far_ring[SP_RING];
    if (S.flags[0]) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nwords = (S.N + 31) >> 5;
    for (int i = tid; i < nwords; i += blockDim.x) accbits[i] = 0u;
    for (int i = tid; i < SP_RING; i += blockDim.x) far_ready[i] = 0;
    if (tid == 0) {
        progress = 0;
        abort_flag = 0;
    }
    __syncthreads();
    const float temp = __fdiv_rn(1.0f, S.simt);
    if (wid == 0) {
        unsigned accmask = 0u;
        double fadd = 0.0;
        double cnext = S.N > 0 ? S.nearc[lane] : 0.0;
        float tnext = S.N > 0 ? S.thr[0] : 0.0f;
        for (int k = 0; k < S.N; ++k) {
            const double c = cnext;
            const float thr = tnext;
            if (k + 1 < S.N) {
                cnext = S.nearc[(size_t)(k + 1) * SP_W + lane];
                tnext = S.thr[k + 1];
            }
            const int slot = k % SP_RING;
            long long it = 0;
            while (far_ready[slot] != k + 1) {
                if (++it > SP_SPIN_LIMIT || abort_flag) break;
            }
            if (it > SP_SPIN_LIMIT || abort_flag) {
                if (lane == 0) {
                    abort_flag = 1;
                    S.flags[1] = 1;
                }
                break;
            }
            __threadfence_block();
            const double f = far_ring[slot];
            double v = ((accmask >> lane) & 1u) ? c : 0.0;
            v = warp_sum_d(v);
            const float fd = (float)(f + v);
            const float ediff = __fmul_rn(__fadd_rn(fd, 0.0f), temp);
            const unsigned a = ediff < thr ? 1u : 0u;
            accmask = (accmask << 1) | a;
            if (a) fadd += (double)fd;
            if (lane == 0) {
                S.acc[k] = (int)a;
                S.fdiff[k] = fd;
                if (a) accbits[k >> 5] |= 1u << (k & 31);
                __threadfence_block();
                progress = k + 1;
            }
            __syncwarp();
        }
        if (lane == 0) *S.fadd_acc = fadd;
    } else {
        const int nh = (blockDim.x >> 5) - 1;
        for (int k = wid - 1; k < S.N; k += nh) {
            const int need = max(k - SP_W, k - SP_RING + 1);
            long long it = 0;
            while (progress < need) {
                if (++it > SP_SPIN_LIMIT || abort_flag) break;
            }
            if (it > SP_SPIN_LIMIT || abort_flag) {
                if (lane == 0) {
                    abort_flag = 1;
                    S.flags[1] = 1;
                }
                break;
            }
            __threadfence_block();
            const int m = S.visit[k];
            const int nn = S.nergpairm[m];
            const size_t row = (size_t)m * S.M;
            // two partners per lane in flight; the correction is read whether or not it applies
            // (a stale value is masked), so its load does not wait for the partner's index
            double sum = 0.0;
            for (int s = 1 + lane; s < nn; s += 64) {
                const bool h2 = s + 32 < nn;
                const int kp0 = S.fv[row + s];
                const int kp1 = h2 ? S.fv[row + s + 32] : -1;
                const double f0 = S.farc[row + s];
                const double f1 = h2 ? S.farc[row + s + 32] : 0.0;
                const bool u0 = kp0 >= 0 && ((accbits[kp0 >> 5] >> (kp0 & 31)) & 1u);
                const bool u1 = kp1 >= 0 && ((accbits[kp1 >> 5] >> (kp1 & 31)) & 1u);
                sum += u0 ? f0 : 0.0;
                sum += u1 ? f1 : 0.0;
            }
            sum = warp_sum_d(sum);
            if (lane == 0) {
                far_ring[k % SP_RING] = S.base[k] + sum;
                __threadfence_block();
                far_ready[k % SP_RING] = k + 1;
            }
            __syncwarp();
        }
    }
}

// ----------------------------------------------------------------- commit
__global__ void spec_commit_moves_kernel(SpecDev S) {
    if (S.flags[0] || S.flags[1]) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S.N) return;
    const int m = S.visit[k];
    const int t = S.mtype[m];
    const int a0 = S.naf[m], n = S.nato[m];
    if (S.acc[k]) {
        for (int i = 0; i < n; ++i) {
            S.xa_w[a0 + i] = S.nx[a0 + i];
            S.ya_w[a0 + i] = S.ny[a0 + i];
            S.za_w[a0 + i] = S.nz[a0 + i];
            S.pos_w[a0 + i] = S.npos[a0 + i];
        }
        const float4 c = S.nc[m];
        S.xadd_w[m] = c.x;
        S.yadd_w[m] = c.y;
        S.zadd_w[m] = c.z;
        S.nstepreject[m] = 0;
    } else {
        S.nstepreject[m]++;
        if (S.stepr > 0.0f) atomicAdd(S.rej_rot + t, 1);
        if (S.stepm > 0.0f) atomicAdd(S.rej_tr + t, 1);
    }
    if (S.trace_den) S.trace_den[k] = S.fdiff[k];
    if (S.trace_acc) S.trace_acc[k] = S.acc[k];
}

__global__ void spec_commit_store_kernel(SpecDev S) {
    if (S.flags[0] || S.flags[1]) return;
    const int m = blockIdx.x;
    const int km = S.vpos[m];
    const int nn = S.nergpairm[m];
    const size_t row = (size_t)m * S.M;
    const int am = S.acc[km];
    if (!am) return;
    for (int s = 1 + threadIdx.x; s < nn; s += blockDim.x) {
        const size_t e = row + s;
        const int p = S.molergpair[e];
        const int kp = S.vpos[p];
        const int e2 = S.mirror[e];
        const int p_writes = S.acc[kp] && (e2 % S.M) >= 1;
        if (p_writes && kp > km) continue;  // the later accepted writer wins
        const float v = (kp < km && S.acc[kp]) ? S.B[e] : S.A[e];
        S.ergpair[S.ergpairref[e] - 1] = v;
    }
}

__global__ void spec_epilogue_kernel(SpecDev S) {
    if (threadIdx.x != 0) return;
    if (S.flags[1]) {
        if (S.status) S.status[0] = 2;
        return;
    }
    if (S.flags[0]) return;  // the sequential kernel runs this cycle
    const int nmt = S.nmoltype;
    const float rotstepmin = 1.0e-5f, rotstepmax = 1.0f;
    for (int t = 0; t < nmt; ++t) {
        // step values as the cycle leaves them: first-visit initialisation, or zero for a
        // visited type that does not rotate / translate (molfit.py:377-396)
        if (S.cnt_type[t] > 0) {
            S.wholerot[t] = S.tries_rot[t] > 0 ? S.rotstep[t] : 0.0f;
            S.wholetrans[t] = S.tries_tr[t] > 0 ? S.transstep[t] : 0.0f;
        }
        S.nwhole[t] = S.tries_rot[t];
        S.nwhole[nmt + t] = S.rej_rot[t];
        S.nmovem[t] = S.tries_tr[t];
        S.nmovem[nmt + t] = S.rej_tr[t];
    }
    if (S.ireset != 1) {
        for (int t = 0; t < nmt; ++t) {
            float it = __fmul_rn(S.interntrans[t], 1.0f);
            if (it > S.trstepmax) it = S.trstepmax;
            if (it < S.trstepmin && it != 0.0f) it = S.trstepmin;
            S.interntrans[t] = it;
            float ir = __fmul_rn(S.internrot[t], 1.0f);
            if (ir > rotstepmax) ir = rotstepmax;
            if (ir < rotstepmin && ir != 0.0f) ir = rotstepmin;
            S.internrot[t] = ir;
            float rat;
            if (S.nwhole[nmt + t] > 0) {
                rat = __fdiv_rn(__fmul_rn(S.rejrate, (float)S.nwhole[t]), (float)S.nwhole[nmt + t]);
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = S.nwhole[t] > 0 ? 1.1f : 1.0f;
            }
            float wr = __fmul_rn(S.wholerot[t], rat);
            if (wr > rotstepmax) wr = rotstepmax;
            if (wr < rotstepmin && wr != 0.0f) wr = rotstepmin;
            S.wholerot[t] = wr;
            if (S.nmovem[nmt + t] > 0) {
                rat = __fdiv_rn(__fmul_rn(S.rejrate, (float)S.nmovem[t]), (float)S.nmovem[nmt + t]);
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = S.nmovem[t] > 0 ? 1.1f : 1.0f;
            }
            float wt = __fmul_rn(S.wholetrans[t], rat);
            if (wt > S.trstepmax) wt = S.trstepmax;
            if (wt < S.trstepmin && wt != 0.0f) wt = S.trstepmin;
            S.wholetrans[t] = wt;
        }
    }
    S.fadds[0] = __fadd_rn(S.fadds[0], __fdiv_rn((float)(*S.fadd_acc), (float)S.N));
    for (int i = 0; i < 35; ++i) S.ran1[i] = S.ran1_next[i];
}

}  // namespace epsr

namespace epsr {
// ran1 draws for the cycle: n comes from the plan (device), the state is a copy so that a
// discarded cycle leaves the real state untouched
__global__ void ran1_copy_kernel(const int32_t *src, int32_t *dst) {
    if (threadIdx.x < 35) dst[threadIdx.x] = src[threadIdx.x];
}
int ran1_fill_device_count(int32_t *state, float *out, const int32_t *n_dev, int64_t n_max, cudaStream_t s);
int molfit_seq_launch(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                      void *scratch, int64_t scratch_bytes, cudaStream_t s, const int32_t *run_if);
}  // namespace epsr

using namespace epsr;

static inline size_t spal(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t spec_bytes(int N, int natom, int M, int nmt) {
    size_t b = 0;
    b += 3 * spal(sizeof(int32_t) * ((size_t)N + 1));             // vpos, off, rotidx
    b += spal(sizeof(int32_t) * 8);                                // flags
    b += 2 * spal(sizeof(float) * nmt) + 5 * spal(sizeof(int32_t) * nmt);
    b += spal(sizeof(int32_t) * 35);
    b += spal(sizeof(float) * ((size_t)N * 10 + 64));              // draws
    b += 3 * spal(sizeof(float) * natom) + spal(sizeof(float4) * N) + spal(sizeof(float4) * natom);
    b += spal(sizeof(float) * N);                                  // thr
    b += 2 * spal(sizeof(float) * (size_t)N * M);                  // A, B
    b += spal(sizeof(double) * N) + spal(sizeof(double) * (size_t)N * SP_W) + spal(sizeof(double) * (size_t)N * M);
    b += spal(sizeof(int32_t) * (size_t)N * M);                    // fv
    b += spal(sizeof(int32_t) * N) + spal(sizeof(float) * N) + spal(sizeof(double));
    return b;
}

extern "C" int64_t epsr_molfit_spec_scratch_bytes(int32_t nmol, int32_t natom, int32_t M, int32_t nmoltype) {
    return (int64_t)spec_bytes(nmol, natom, M, nmoltype);
}

int epsr_molfit_spec(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                     void *scratch, int64_t scratch_bytes, void *stream) {
    const int N = box->nmol, M = store->nnbrefmax, nmt = box->nmoltype, natom = box->natom;
    if (!store->mirror) {
        epsr_set_error("epsr_molfit: the fast path needs the store's mirror index (built by epsr_fmolec1)");
        return EPSR_ERR_ARG;
    }
    if ((int64_t)spec_bytes(N, natom, M, nmt) > scratch_bytes || !scratch) {
        epsr_set_error("epsr_molfit: scratch needs %lld bytes", (long long)spec_bytes(N, natom, M, nmt));
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    SpecDev S;
    memset(&S, 0, sizeof(S));
    S.L.cubic = box->cubic;
    S.L.alatx = box->lat[0];
    S.L.blatx = box->lat[1];
    S.L.clatx = box->lat[2];
    S.L.blaty = box->lat[3];
    S.L.claty = box->lat[4];
    S.L.clatz = box->lat[5];
    S.T.tab = (const float4 *)box->tab;
    S.T.xstar = box->xstar;
    S.T.ld = box->ld;
    S.T.npt2 = box->npt2;
    S.T.izcut = box->izcut < box->npt2 ? box->izcut : box->npt2;
    S.T.stepcl = box->stepcl;
    S.N = N;
    S.M = M;
    S.ntype = box->ntype;
    S.nmoltype = nmt;
    S.natom = natom;
    S.naf = box->naf;
    S.nato = box->nato;
    S.mtype = box->mtype;
    S.npairref = box->npairref;
    S.visit = cells->cell_mols;
    S.xa = S.xa_w = box->xa;
    S.ya = S.ya_w = box->ya;
    S.za = S.za_w = box->za;
    S.xadd = S.xadd_w = box->xadd;
    S.yadd = S.yadd_w = box->yadd;
    S.zadd = S.zadd_w = box->zadd;
    S.pos = S.pos_w = (float4 *)box->pos;
    S.nergpairm = store->nergpairm;
    S.molergpair = store->molergpair;
    S.ergpairref = store->ergpairref;
    S.mirror = store->mirror;
    S.ergpair = store->ergpair;
    S.simt = mc->simt;
    S.rejrate = mc->rejrate;
    S.stepr = mc->stepr;
    S.stepm = mc->stepm;
    S.trstepmax = mc->trstepmax;
    S.trstepmin = mc->trstepmin;
    S.ireset = mc->ireset;
    S.wholerot = mc->wholerot;
    S.wholetrans = mc->wholetrans;
    S.internrot = mc->internrot;
    S.interntrans = mc->interntrans;
    S.nwhole = mc->nwhole;
    S.nmovem = mc->nmovem;
    S.nstepreject = mc->nstepreject;
    S.fadds = mc->fadds;
    S.ran1 = mc->ran1;
    S.cos_override = mc->cos_override;
    S.trace_den = mc->trace_den;
    S.trace_acc = mc->trace_acc;
    S.status = mc->status;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += spal(bytes);
        return (void *)r;
    };
    S.vpos = (int32_t *)take(sizeof(int32_t) * ((size_t)N + 1));
    S.off = (int32_t *)take(sizeof(int32_t) * ((size_t)N + 1));
    S.rotidx = (int32_t *)take(sizeof(int32_t) * ((size_t)N + 1));
    S.flags = (int32_t *)take(sizeof(int32_t) * 8);
    S.rotstep = (float *)take(sizeof(float) * nmt);
    S.transstep = (float *)take(sizeof(float) * nmt);
    S.tries_rot = (int32_t *)take(sizeof(int32_t) * nmt);
    S.tries_tr = (int32_t *)take(sizeof(int32_t) * nmt);
    S.rej_rot = (int32_t *)take(sizeof(int32_t) * nmt);
    S.rej_tr = (int32_t *)take(sizeof(int32_t) * nmt);
    S.cnt_type = (int32_t *)take(sizeof(int32_t) * nmt);
    S.ran1_next = (int32_t *)take(sizeof(int32_t) * 35);
    S.draws = (float *)take(sizeof(float) * ((size_t)N * 10 + 64));
    S.nx = (float *)take(sizeof(float) * natom);
    S.ny = (float *)take(sizeof(float) * natom);
    S.nz = (float *)take(sizeof(float) * natom);
    S.nc = (float4 *)take(sizeof(float4) * N);
    S.npos = (float4 *)take(sizeof(float4) * natom);
    S.thr = (float *)take(sizeof(float) * N);
    S.A = (float *)take(sizeof(float) * (size_t)N * M);
    S.B = (float *)take(sizeof(float) * (size_t)N * M);
    S.base = (double *)take(sizeof(double) * N);
    S.nearc = (double *)take(sizeof(double) * (size_t)N * SP_W);
    S.farc = (double *)take(sizeof(double) * (size_t)N * M);
    S.fv = (int32_t *)take(sizeof(int32_t) * (size_t)N * M);
    S.acc = (int32_t *)take(sizeof(int32_t) * N);
    S.fdiff = (float *)take(sizeof(float) * N);
    S.fadd_acc = (double *)take(sizeof(double));

    spec_plan_kernel<<<1, 1024, 0, s>>>(S);
    ran1_copy_kernel<<<1, 64, 0, s>>>(mc->ran1, S.ran1_next);
    int rc = ran1_fill_device_count(S.ran1_next, S.draws, S.off + N, (int64_t)N * 7 + 1, s);
    if (rc) return rc;
    spec_propose_kernel<<<(N + 127) / 128, 128, 0, s>>>(S);
    const size_t en_bytes = sizeof(int) * ((((size_t)box->ntype * box->ntype + 3) & ~(size_t)3) + 2 * (size_t)M);
    if (en_bytes > 48 * 1024) EPSR_SMEM_OPTIN(spec_energy_kernel);
    EPSR_TIMED("spec_energy_kernel", s, spec_energy_kernel<<<N, SP_ET, en_bytes, s>>>(S));
    EPSR_CUDA(cudaMemsetAsync(S.nearc, 0, sizeof(double) * (size_t)N * SP_W, s));
    EPSR_TIMED("spec_corr_kernel", s, spec_corr_kernel<<<N, 128, 0, s>>>(S));
    const size_t bits = sizeof(unsigned) * (((size_t)N + 31) / 32);
    if (bits > 48 * 1024) EPSR_SMEM_OPTIN(spec_resolve_kernel);
    EPSR_TIMED("spec_resolve_kernel", s, spec_resolve_kernel<<<1, SP_RT, bits, s>>>(S));
    spec_commit_moves_kernel<<<(N + 127) / 128, 128, 0, s>>>(S);
    spec_commit_store_kernel<<<N, 128, 0, s>>>(S);
    spec_epilogue_kernel<<<1, 32, 0, s>>>(S);
    EPSR_CUDA(cudaGetLastError());
    // a cycle with a translation retry runs on the sequential kernel (no-op otherwise)
    return molfit_seq_launch(box, cells, store, mc, nullptr, 0, s, S.flags);
}
