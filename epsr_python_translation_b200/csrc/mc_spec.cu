// mc_spec.cu -- molfit whole-molecule cycle (molfit.py:268-448) resolved speculatively.
//
// Within one cycle every molecule moves once, from its cycle-start position, with ran1
// draws at offsets fixed by the visit order (3 rotation + 3 translation + 1 acceptance
// draw per move, molfit.py:382-401).  Only the accept decisions chain the moves together:
// move k sees partner p at p's new position (and p's stored energy written by p's move)
// exactly when p was visited earlier and accepted.  So:
//
//   plan     per-move draw offsets; per-type step sizes (the first-visit initialisation);
//   draws    the cycle's ran1 values in one stream pass -- or, when the caller gave a
//            draws-ahead buffer and the previous cycle left the stream where the values in it
//            start, those values, generated on a second stream while the previous cycle ran;
//   propose  every proposal (rotatm + movem) and its Metropolis threshold, in parallel;
//   energy   for every stored entry (k, p): A = E(new k, old p) and, if p is earlier in
//            the visit order, B = E(new k, new p) -- each in the reference's (ia, ja) order;
//   corr     per move the energy change assuming no earlier partner accepted (base) and
//            the correction c = (B - old') - (A - S) that applies if partner p accepted;
//            the corrections of partners visited at most 64 moves earlier are kept by the
//            earlier move (its row: the effect of its acceptance on each of the next 64 moves)
//   resolve  one CTA walks the moves in order.  The resolver warp holds a running sum for
//            each of the next 64 moves (two per lane); deciding a move is one comparison in
//            the lane that holds its sum and a ballot, after which every lane adds the
//            decided move's row entry for its two moves -- no reduction on the decision
//            chain.  The rows and thresholds arrive by bulk copies into a four-block ring of
//            shared memory.  Helper warps sum, per move, the corrections of accepted partners
//            visited more than 64 moves earlier, reading the decisions the resolver publishes
//            once per 32 moves; each handoff is a 64-bit word carrying its own tag, so no
//            fence sits on the decision chain;
//   commit   coordinates, the energy store (the later accepted writer of a shared slot
//            wins), counters, step adaptation, fadds and the ran1 state.
//
// Energies of individual molecule pairs are bit-identical to the reference; each move's
// total is summed in double (the reference's float32 order is the sequential kernel in
// mc.cu).  The rare translation retry of movem (a move that leaves the centre unchanged
// doubles the step and draws again, molfit.py:752-758) shifts every later draw; the cycle is
// then discarded and the sequential kernel runs it instead, from the unchanged state.
#include "common.cuh"
#include "umma.cuh"

namespace epsr {

constexpr int SP_W = 64;        // near window of the resolver (moves): two running sums per lane
constexpr int SP_FR = 128;      // far-sum ring (moves)
constexpr int SP_BLK = 32;      // moves per staged block (and per published decision word)
constexpr int SP_NSLOT = 4;     // staged blocks held in shared memory
constexpr int SP_NH = 24;       // helper warps: warps 1..31 outside scheduler 0
constexpr int SP_MAXAT = 64;    // atoms of a moved molecule
constexpr int SP_ET = 320;      // threads of a move's energy CTA (its stored partners: about 300 at 0.1 atoms/A^3)
constexpr int SP_RT = 1024;     // resolver CTA: warp 0 resolves, the warps of schedulers 1-3 help
constexpr long long SP_SPIN_LIMIT = 1ll << 26;
// words of the draws-ahead buffer (described with the draws-ahead kernels below)
constexpr int AH_VALID = 0, AH_COUNT = 1, AH_USES = 2, AH_START = 4, AH_END = 40, AH_VALS = 80;
constexpr int SP_MAXEDGE = 16384;  // table points indexed by bin edges (beyond: the energy pass divides)

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
    int32_t *vpos, *off, *rotidx, *flags;  // flags[0] retry, [1] resolver timeout, [2] values to walk, [3] draws ahead
                                           // taken, [4] CTAs of the commit pass done
    float *rotstep, *transstep;            // [nmoltype]
    int32_t *tries_rot, *tries_tr, *rej_rot, *rej_tr, *cnt_type;  // [nmoltype]
    int32_t *ran1_next;                    // [35]
    float *draws;
    int32_t *ahead;                        // the draws-ahead buffer (AH_* words), or NULL
    const float *ahead_vals;               // the draws-ahead values, or NULL
    const int32_t *use_ahead;              // [1] 1: this cycle reads ahead_vals (NULL: never)
    float *nx, *ny, *nz;                   // [natom] proposed offsets
    float4 *nc;                            // [N] proposed centres (by molecule)
    float4 *npos;                          // [natom] proposed absolute positions
    float *thr;                            // [N] Metropolis thresholds (by visit position)
    float *A, *B;                          // [N*M]
    double *base;                          // [N] each move's change if no earlier partner accepted
    float2 *nearT;                         // [Npad*W] near terms {rejected, accepted}, by the earlier move
    int32_t *farkp;                        // [N*M] far partners by visit position: the partner's visit position
    float2 *fart;                          // [N*M] and its two terms {rejected, accepted}
    int32_t *nnk;                          // [N] far partners listed for each move
    int32_t *acc;                          // [N] by visit position
    float *fdiff;                          // [N] by visit position
    double *fadd_acc;                      // [1]
    Bins bins;                             // the energy pass's table index by bin edges (cubic boxes)
    float4 *edge_w;                        // [nedge] written by the propose pass
    int nedge;                             // 0: the energy pass divides (triclinic box, or too many bins)
    int ev;                                // the energy pass's staged values per chunk (>= 2 maxat^2)
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
        S.flags[4] = 0;
        *S.fadd_acc = 0.0;
    }
    __syncthreads();
    for (int base = 0; base < S.N; base += blockDim.x) {
        const int k = base + tid;
        int nd = 0, nr = 0, t = -1;
        bool istr = false;
        if (k < S.N) {
            const int m = S.visit[k];
            S.vpos[m] = k;
            const int n = S.nato[m];
            t = S.mtype[m];
            if (S.stepr > 0.0f && n > 1) {
                nd += 3;
                nr = 1;
            }
            if (S.stepm > 0.0f) {
                nd += 3;
                istr = true;
            }
            nd += 1;
        }
        // per-type counts, one atomic per type present in the warp (integers: any order)
        {
            const unsigned same = __match_any_sync(0xffffffffu, t);
            const unsigned rotb = __ballot_sync(0xffffffffu, nr != 0), trb = __ballot_sync(0xffffffffu, istr);
            if (t >= 0 && (int)(threadIdx.x & 31) == __ffs(same) - 1) {
                atomicAdd(S.cnt_type + t, __popc(same));
                if (rotb & same) atomicAdd(S.tries_rot + t, __popc(rotb & same));
                if (trb & same) atomicAdd(S.tries_tr + t, __popc(trb & same));
            }
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
    __syncthreads();   // off[N], the cycle's draw count
    if (tid >= 32) return;
    // the cycle's ran1 values, from a copy of the state (a discarded cycle leaves the real state
    // untouched): the draws ahead when the previous cycle left them for exactly this state and
    // count, else walked here by this warp
    const int lane = tid;
    for (int i = lane; i < 35; i += 32) S.ran1_next[i] = S.ran1[i];
    const int32_t count = S.off[S.N];
    bool ok = false;
    if (S.ahead) {
        bool same = S.ahead[AH_START + lane] == S.ran1[lane];
        if (lane < 3) same = same && S.ahead[AH_START + 32 + lane] == S.ran1[32 + lane];
        ok = __all_sync(0xffffffffu, same) && S.ahead[AH_VALID] == 1 && S.ahead[AH_COUNT] == count;
    }
    __syncwarp();
    if (ok) {
        S.ran1_next[lane] = S.ahead[AH_END + lane];
        if (lane < 3) S.ran1_next[32 + lane] = S.ahead[AH_END + 32 + lane];
    }
    if (lane == 0) {
        S.flags[2] = ok ? 0 : count;
        S.flags[3] = ok ? 1 : 0;
        if (ok) S.ahead[AH_USES] += 1;
    }
    __syncwarp();
    if (ok || count == 0) return;
    __shared__ int32_t tab[34];
    Ran1Warp g;
    g.load(S.ran1_next);
    const int32_t mcall = S.ran1_next[2];
    __syncwarp();
    int64_t done = 0;
    while (done < count) {
        const int64_t left = count - done;
        int32_t mine;
        const int cnt = g.next(left > 32 ? 32 : (int)left, mine, tab);
        if (lane < cnt) S.draws[done + lane] = ran1_out(mine);
        done += cnt;
    }
    __syncwarp();
    S.ran1_next[3 + lane] = g.iv;
    if (lane == 0) {
        S.ran1_next[0] = g.idum;
        S.ran1_next[1] = g.iy;
        S.ran1_next[2] = (int32_t)((uint32_t)mcall + (uint32_t)count);
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
    if (k < S.nedge) S.edge_w[k] = bin_edge_entry(S.T.stepcl, S.T.xstar, S.T.ld, k);
    if (k >= S.N) return;
    const float pi = 3.14159265358979323846f;
    const int m = S.visit[k];
    const int n = S.nato[m];
    if (n > SP_MAXAT) {   // beyond this path's per-molecule arrays: the sequential kernel refuses the cycle
        atomicExch(S.flags, 1);
        return;
    }
    const int a0 = S.naf[m];
    const int t = S.mtype[m];
    const float *u = (S.use_ahead && *S.use_ahead ? S.ahead_vals : S.draws) + S.off[k];
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
// free for latency hiding).
// Both energies of one partner in one pass over its atoms: A against its cycle-start
// position (pa), B against its proposed position (pn) when has_b; each summed ia outer, ja
// inner as en_change, so each is the reference's value.
__device__ __forceinline__ void mol_energy_ab(const Lattice &L, const Tables &T, const float4 *sa, int na,
                                              const float4 *__restrict__ pa, const float4 *__restrict__ pn, int nb,
                                              bool has_b, const int *spr, int ntype, float &ea, float &eb) {
    float xa = 0.0f, xb = 0.0f;
    for (int ia = 0; ia < na; ++ia) {
        const float4 p1 = sa[ia];
        const int *row = spr + __float_as_int(p1.w) * ntype;
#pragma unroll 2
        for (int j = 0; j < nb; ++j) {
            const float4 p2 = __ldg(pa + j);
            const int ic = row[__float_as_int(p2.w)];
            xa = __fadd_rn(xa, pair_energy(L, T, p1, p2, ic));
            if (has_b) xb = __fadd_rn(xb, pair_energy(L, T, p1, __ldg(pn + j), ic));
        }
    }
    ea = xa;
    eb = xb;
}

// One CTA per move.  The stored partners are taken in chunks of at most one per thread whose
// pair values fit the staging area; a chunk is spread over the CTA as items (partner, partner
// atom ja, which position: cycle start or proposed), each item evaluating its atom against
// every atom ia of the moved molecule into the staging area at [ia][ja], and then one thread
// per partner sums its values in the reference's order (ia outer, ja inner, from +0).  Every
// pair value is pair_energy of the same operands as en_change, so A and B are the values of
// mol_energy_ab bit for bit; the items keep a partner's nine (water) or more pair evaluations
// independent of each other instead of one thread's dependent chain of table loads.

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

// four CTAs of the energy pass per SM (40 warps): its shared memory allows four, and the
// register budget that gives (51 a thread) holds the three pair evaluations in flight unspilled
constexpr int SP_EN_MINB = 4;
template <bool BINS>
__global__ void __launch_bounds__(SP_ET, SP_EN_MINB) spec_energy_kernel(SpecDev S) {
    extern __shared__ __align__(16) unsigned char en_smem[];
    const int ev = S.ev;                                                 // staged values per chunk
    float *vals = reinterpret_cast<float *>(en_smem);                  // [ev]
    uint16_t *items = reinterpret_cast<uint16_t *>(vals + ev);           // [ev] (chunk thread << 7) | item
    int *spr = reinterpret_cast<int *>(items + ((ev + 1) & ~1));          // npairref [ntype*ntype]
    __shared__ float4 sa[SP_MAXAT];
    __shared__ int c_b0[SP_ET], c_nb[SP_ET], c_voff[SP_ET];
    __shared__ int ws_v[SP_ET / 32], ws_i[SP_ET / 32];
    __shared__ int s_nitems;
    if (S.flags[0]) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int k = blockIdx.x;
    const int m = S.visit[k];
    const int na = S.nato[m], a0 = S.naf[m];
    const int ntype = S.ntype;
    const Lattice L = S.L;
    const Tables T = S.T;
    const float4 *__restrict__ pos = S.pos;
    const float4 *__restrict__ npos = S.npos;
    for (int i = tid; i < ntype * ntype; i += blockDim.x) spr[i] = S.npairref[i];
    for (int i = tid; i < na; i += blockDim.x) sa[i] = S.npos[a0 + i];
    const int nn = S.nergpairm[m];
    const size_t row = (size_t)m * S.M;
    __syncthreads();
    for (int s0 = 1; s0 < nn;) {
        // 1. this thread's partner (slot s0 + tid) and the value / item offsets of the chunk
        const int s = s0 + tid;
        int b0 = 0, nb = 0, nv = 0, ni = 0;
        bool hb = false;
        if (s < nn) {
            const int p = S.molergpair[row + s];
            b0 = S.naf[p];
            nb = S.nato[p];
            hb = S.vpos[p] < k;
            ni = hb ? 2 * nb : nb;
            nv = na * ni;
        }
        int iv = warp_incl_scan(nv, lane), ii = warp_incl_scan(ni, lane);
        if (lane == 31) {
            ws_v[wid] = iv;
            ws_i[wid] = ii;
        }
        __syncthreads();
        for (int w = 0; w < wid; ++w) {
            iv += ws_v[w];
            ii += ws_i[w];
        }
        // the chunk is the prefix of partners whose values fit (at least the first: nv <= ev)
        const bool take = s < nn && iv <= ev;
        if (take) {
            c_b0[tid] = b0;
            c_nb[tid] = nb;
            c_voff[tid] = iv - nv;
            for (int j = 0; j < ni; ++j) items[ii - ni + j] = (uint16_t)((tid << 7) | j);
        }
        const int ntake = __syncthreads_count(take);
        if (take && tid == ntake - 1) s_nitems = ii;
        __syncthreads();
        // 2. items: (partner, ja, position) against every atom of the moved molecule
        const int nit = s_nitems;
        for (int it = tid; it < nit; it += blockDim.x) {
            const int code = items[it];
            const int t = code >> 7, j = code & 127;
            const int pb = c_b0[t], pn = c_nb[t];
            const bool nw_pos = j >= pn;
            const int ja = nw_pos ? j - pn : j;
            const float4 p2 = nw_pos ? npos[pb + ja] : __ldg(pos + pb + ja);
            float *v = vals + c_voff[t] + (nw_pos ? na * pn : 0) + ja;
            const int *col = spr + __float_as_int(p2.w);
            // three atoms of the moved molecule at a time (independent evaluations in flight; a
            // short last group repeats the molecule's last atom and stores nothing for it)
            for (int ia = 0; ia < na; ia += 3) {
                const int i1 = min(ia + 1, na - 1), i2 = min(ia + 2, na - 1);
                const float4 q0 = sa[ia], q1 = sa[i1], q2 = sa[i2];
                const int c0 = col[__float_as_int(q0.w) * ntype], c1 = col[__float_as_int(q1.w) * ntype],
                          c2 = col[__float_as_int(q2.w) * ntype];
                float e0, e1, e2;
                if (BINS) {
                    e0 = pair_energy_cubic_bins(S.bins, q0, p2, c0);
                    e1 = pair_energy_cubic_bins(S.bins, q1, p2, c1);
                    e2 = pair_energy_cubic_bins(S.bins, q2, p2, c2);
                } else {
                    e0 = pair_energy(L, T, q0, p2, c0);
                    e1 = pair_energy(L, T, q1, p2, c1);
                    e2 = pair_energy(L, T, q2, p2, c2);
                }
                v[ia * pn] = e0;
                if (ia + 1 < na) v[i1 * pn] = e1;
                if (ia + 2 < na) v[i2 * pn] = e2;
            }
        }
        __syncthreads();
        // 3. each taken partner's A (and B) summed in the reference's order
        if (take) {
            const float *v = vals + c_voff[tid];
            const int n2 = na * nb;
            float xa = 0.0f;
            for (int q = 0; q < n2; ++q) xa = __fadd_rn(xa, v[q]);
            S.A[row + s] = xa;
            if (hb) {
                float xb = 0.0f;
                for (int q = 0; q < n2; ++q) xb = __fadd_rn(xb, v[n2 + q]);
                S.B[row + s] = xb;
            }
        }
        s0 += ntake;
        __syncthreads();   // the staging area and chunk tables are rewritten by the next chunk
    }
}

// ----------------------------------------------------------------- corrections
// Per move k (one CTA): base[k] = sum over its partners visited later of A - S, and for each
// partner p visited earlier both terms it can bring: A - S if p was rejected, B - (p's stored
// energy after its move) if it was accepted.  Partners at most SP_W moves earlier go into p's
// row of nearT (the resolver adds the term that applies as decisions are taken); the others
// are listed for the helpers in store order, compacted to the front of k's rows of farkp/fart as
// (partner's visit position, both terms) words (nnk[k] of them).  Carrying both terms, never
// their difference, keeps an energy that the final configuration does not contain (A against
// a partner that has moved away) out of every sum.
__global__ void __launch_bounds__(128) spec_corr_kernel(SpecDev S) {
    __shared__ double ws[4];
    __shared__ int wcount[4];
    if (S.flags[0]) return;
    const int k = blockIdx.x;
    const int m = S.visit[k];
    const int nn = S.nergpairm[m];
    const size_t row = (size_t)m * S.M, krow = (size_t)k * S.M;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double d0s = 0.0;
    int nfar = 0;   // far partners listed so far (block-uniform)
    for (int s0 = 1; s0 < nn; s0 += blockDim.x) {
        const int s = s0 + threadIdx.x;
        bool far = false;
        int kp = -1;
        float ca = 0.0f, cb = 0.0f;
        if (s < nn) {
            const size_t e = row + s;
            const int p = S.molergpair[e];
            kp = S.vpos[p];
            const double sv = (double)S.ergpair[S.ergpairref[e] - 1];
            const double d0 = (double)S.A[e] - sv;
            if (kp < k) {
                // the term if p was rejected (A - S) and if it was accepted (B against p's stored
                // energy after its move); the resolver or a helper adds the one that applies
                const int e2 = S.mirror[e];
                const int s2 = e2 % S.M;
                const double oldp = s2 >= 1 ? (double)S.A[e2] : sv;
                ca = (float)d0;
                cb = (float)((double)S.B[e] - oldp);
                const int dist = k - kp;
                if (dist <= SP_W) S.nearT[(size_t)kp * SP_W + dist - 1] = make_float2(ca, cb);
                else far = true;
            } else {
                d0s += d0;   // a later partner: its term is A - S
            }
        }
        // ordered compaction of this chunk's far partners
        const unsigned bal = __ballot_sync(0xffffffffu, far);
        if (lane == 0) wcount[wid] = __popc(bal);
        __syncthreads();
        int off = nfar, tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            if (w < wid) off += wcount[w];
            tot += wcount[w];
        }
        if (far) {
            const int i = off + __popc(bal & ((1u << lane) - 1u));
            S.farkp[krow + i] = kp;
            S.fart[krow + i] = make_float2(ca, cb);
        }
        nfar += tot;
        __syncthreads();
    }
    d0s = warp_sum_d(d0s);
    if (lane == 0) ws[wid] = d0s;
    __syncthreads();
    if (threadIdx.x == 0) {
        S.base[k] = ws[0] + ws[1] + ws[2] + ws[3];
        S.nnk[k] = nfar;
    }
}

// ----------------------------------------------------------------- resolve
// Loads of data the previous kernels wrote and this one only reads, issued at their place in
// the program (the compiler neither sinks them to their first use nor merges them away).
__device__ __forceinline__ int ldg_pinned(const int32_t *p) {
    int r;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(r) : "l"(p));
    return r;
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(umma::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(umma::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ double ldg_pinned(const double *p) {
    double r;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(r) : "l"(p));
    return r;
}

// Shared memory of the resolver CTA (dynamic): the staged rows ({rejected, accepted} terms),
// the staged thresholds, the blocks' mbarriers, the far-sum ring (one tagged word a move: the
// tag in the high half, the float far part in the low), each helper's two staged far lists,
// and the published decision words (tag in the high half, one bit a move in the low).
constexpr int SP_SROWS = SP_NSLOT * SP_BLK * SP_W * 8;
constexpr int SP_STHR = SP_NSLOT * SP_BLK * 4;
constexpr int SP_HCAP = 256;                                  // far partners a helper stages per move
constexpr int SP_HSTAGE = SP_HCAP * 12;                       // one staged list: terms, then positions
constexpr int SP_HOFF = SP_SROWS + SP_STHR + SP_NSLOT * 8 + SP_FR * 8;
constexpr int SP_SHDR = SP_HOFF + SP_NH * 2 * SP_HSTAGE;

__host__ __device__ constexpr size_t spec_resolve_smem(int N) {
    return (size_t)SP_SHDR + 8 * (size_t)((N + SP_BLK - 1) / SP_BLK);
}

__global__ void __launch_bounds__(SP_RT, 1) spec_resolve_kernel(SpecDev S) {
    extern __shared__ __align__(128) unsigned char rsm[];
    float2 *srows = reinterpret_cast<float2 *>(rsm);
    float *sthr = reinterpret_cast<float *>(rsm + SP_SROWS);
    uint64_t *bars = reinterpret_cast<uint64_t *>(rsm + SP_SROWS + SP_STHR);
    volatile uint64_t *vfar = reinterpret_cast<volatile uint64_t *>(rsm + SP_SROWS + SP_STHR + SP_NSLOT * 8);
    volatile uint64_t *vpub = reinterpret_cast<volatile uint64_t *>(rsm + SP_SHDR);
    __shared__ volatile int abort_flag;
    if (S.flags[0]) return;
    const int N = S.N;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nblk = (N + SP_BLK - 1) / SP_BLK;
    for (int i = tid; i < SP_FR; i += blockDim.x) vfar[i] = 0ull;
    for (int i = tid; i < nblk; i += blockDim.x) vpub[i] = 0ull;
    if (tid == 0) {
        abort_flag = 0;
        for (int i = 0; i < SP_NSLOT; ++i) umma::mbar_init(&bars[i], 1);
        umma::fence_mbar_init();
    }
    __syncthreads();
    const float temp = __fdiv_rn(1.0f, S.simt);
    auto fail = [&]() {
        abort_flag = 1;
        S.flags[1] = 1;
    };

    if (wid == 0) {
        // ---- the resolver warp
        auto stage = [&](int b) {   // lane 0: rows and thresholds of block b into its slot
            const int slot = b % SP_NSLOT;
            const int nr = min(SP_BLK, N - SP_BLK * b);
            const uint32_t rb = (uint32_t)nr * SP_W * 8, tb = ((uint32_t)nr * 4 + 15u) & ~15u;
            umma::mbar_expect_tx(&bars[slot], rb + tb);
            umma::bulk_load(srows + (size_t)slot * SP_BLK * SP_W, S.nearT + (size_t)b * SP_BLK * SP_W, rb, &bars[slot]);
            umma::bulk_load(sthr + slot * SP_BLK, S.thr + (size_t)b * SP_BLK, tb, &bars[slot]);
        };
        int issued = 0, waited = 0;
        if (lane == 0)
            for (; issued < min(nblk, SP_NSLOT - 1); ++issued) stage(issued);
        float A0 = 0.0f, A1 = 0.0f;   // running sums of the pending moves = lane, lane + 32 (mod 64)
        double fadd = 0.0;
        int err = 0;
        for (int b = 0; b < nblk && !err; ++b) {
            const int slot = b % SP_NSLOT;
            if (lane == 0 && issued < nblk) {   // the slot block b-1 used: this warp has read it
                umma::fence_proxy_async();
                stage(issued++);
            }
            // every lane waits on the block's mbarrier (its completion makes the copied bytes visible)
            const bool got = umma::mbar_wait(&bars[slot], (uint32_t)((b / SP_NSLOT) & 1), nullptr);
            if (__any_sync(0xffffffffu, !got)) {
                err = 1;
                break;
            }
            ++waited;
            const float2 *rows = srows + (size_t)slot * SP_BLK * SP_W;
            const float *th = sthr + slot * SP_BLK;
            const int nr = min(SP_BLK, N - SP_BLK * b);
            // lane i owns move 32 b + i of the block: its threshold and its far part (which the
            // helpers completed while the block before was walked) are read once, by that lane
            const int ko = SP_BLK * b + lane;
            const bool mine = lane < nr;
            const float thr_own = mine ? th[lane] : 0.0f;
            const int fs = ko % SP_FR;
            const uint32_t tag = (uint32_t)(ko + 1);
            uint64_t w = 0ull;
            bool ready = true;
            if (mine) {
                w = vfar[fs];
                ready = (uint32_t)(w >> 32) == tag;
            }
            for (long long it = 0; !__all_sync(0xffffffffu, ready);) {
                if (__any_sync(0xffffffffu, ++it > SP_SPIN_LIMIT || abort_flag)) {
                    err = 1;
                    break;
                }
                if (!ready) {
                    w = vfar[fs];
                    ready = (uint32_t)(w >> 32) == tag;
                }
            }
            if (err) break;
            const float f_own = __uint_as_float((uint32_t)w);
            float fd_own = 0.0f;
            unsigned wbits = 0u;
            // this lane's two entries of row i (the terms move 32 b + i brings to the two pending
            // moves this lane holds, {rejected, accepted})
            auto row_c = [&](int i, float2 &c0, float2 &c1) {
                const int j0 = (lane + SP_W - 1 - ((SP_BLK * b + i) & (SP_W - 1))) & (SP_W - 1);
                c0 = rows[i * SP_W + j0];
                c1 = rows[i * SP_W + ((j0 + 32) & (SP_W - 1))];
            };
            const bool r1 = (b & 1) != 0;   // the register of the block's moves: (32 b + i) & 32
            float2 c0n, c1n;
            row_c(0, c0n, c1n);
            int i = 0;
            // two moves a step: the second move's test is formed for both outcomes of the first
            // (its sum with the first's rejected or accepted term), and two ballots decide both --
            // bit i and i+1 of the first the first move's test and the second's if the first
            // rejects, the second the second's if the first accepts
            auto pair = [&](int i) {
                const float2 ca0 = c0n, ca1 = c1n;
                float2 cb0, cb1;
                row_c(i + 1, cb0, cb1);
                const float asel = r1 ? A1 : A0;
                const float2 cs = r1 ? ca1 : ca0;
                const bool own0 = lane == i, own1 = lane == i + 1;
                // lane i: move i's own sum; lane i+1: its sum with move i rejected / accepted
                const float fdA = __fadd_rn(f_own, own1 ? __fadd_rn(asel, cs.x) : asel);
                const float fdB = __fadd_rn(f_own, __fadd_rn(asel, cs.y));
                const float eA = __fmul_rn(__fadd_rn(fdA, 0.0f), temp);
                const float eB = __fmul_rn(__fadd_rn(fdB, 0.0f), temp);
                const unsigned bA = __ballot_sync(0xffffffffu, (own0 || own1) && eA < thr_own);
                const unsigned bB = __ballot_sync(0xffffffffu, own1 && eB < thr_own);
                if (i + 2 < nr) row_c(i + 2, c0n, c1n);
                const bool ak = (bA >> i) & 1u;
                const bool ak1 = ak ? bB != 0u : ((bA >> (i + 1)) & 1u) != 0u;
                const float dk0 = ak ? ca0.y : ca0.x, dk1 = ak ? ca1.y : ca1.x;
                A0 = (own0 && !r1) ? dk0 : __fadd_rn(A0, dk0);
                A1 = (own0 && r1) ? dk1 : __fadd_rn(A1, dk1);
                const float dl0 = ak1 ? cb0.y : cb0.x, dl1 = ak1 ? cb1.y : cb1.x;
                A0 = (own1 && !r1) ? dl0 : __fadd_rn(A0, dl0);
                A1 = (own1 && r1) ? dl1 : __fadd_rn(A1, dl1);
                fd_own = own0 ? fdA : (own1 ? (ak ? fdB : fdA) : fd_own);
                wbits |= ((ak ? 1u : 0u) | (ak1 ? 2u : 0u)) << i;
            };
            if (nr == SP_BLK) {   // a full block: the walk written out, its registers renamed by the compiler
#pragma unroll
                for (int i2 = 0; i2 < SP_BLK; i2 += 2) pair(i2);
                i = SP_BLK;
            } else {
                for (; i + 1 < nr; i += 2) pair(i);
            }
            if (i < nr) {   // an odd last move
                const float2 ca0 = c0n, ca1 = c1n;
                const float fdA = __fadd_rn(f_own, r1 ? A1 : A0);
                const float eA = __fmul_rn(__fadd_rn(fdA, 0.0f), temp);
                const bool own0 = lane == i;
                const bool ak = __ballot_sync(0xffffffffu, own0 && eA < thr_own) != 0u;
                const float dk0 = ak ? ca0.y : ca0.x, dk1 = ak ? ca1.y : ca1.x;
                A0 = (own0 && !r1) ? dk0 : __fadd_rn(A0, dk0);
                A1 = (own0 && r1) ? dk1 : __fadd_rn(A1, dk1);
                fd_own = own0 ? fdA : fd_own;
                wbits |= (ak ? 1u : 0u) << i;
            }
            if (mine) {
                const bool acc = (wbits >> lane) & 1u;
                S.acc[ko] = acc ? 1 : 0;
                S.fdiff[ko] = fd_own;
                if (acc) fadd += (double)fd_own;
            }
            if (lane == 0) vpub[b] = ((uint64_t)(uint32_t)(b + 1) << 32) | wbits;
        }
        if (lane == 0) {
            if (err) {
                fail();
                // the copies still in flight land before the CTA's shared memory goes away
                for (int b = waited; b < issued; ++b) umma::mbar_wait(&bars[b % SP_NSLOT], (uint32_t)((b / SP_NSLOT) & 1), nullptr);
            }
        }
        fadd = warp_sum_d(fadd);   // each lane's accepted moves, then the lanes in a fixed order
        if (lane == 0) *S.fadd_acc = fadd;
    } else if ((wid & 3) != 0) {
        // ---- helper warps: the far part of each move's change, one move a step.  A move's
        // listed far partners (up to SP_HCAP; a longer list reads the rest from global memory)
        // are copied into one of the helper's two shared-memory stages by cp.async one step
        // before they are summed, with its list length and base loaded two steps before; those
        // two scalars live in three register sets that take turns (the loop body is written
        // out three times), so nothing waits on a load in flight.
        const int h = wid - 1 - (wid >> 2);
        const int M = S.M;
        const int st = SP_NH;
        unsigned char *hb = rsm + SP_HOFF + (size_t)h * 2 * SP_HSTAGE;
        struct Scal {
            int nf;
            double bk;
        };
        auto load = [&](int kk, Scal &g) {
            g.nf = kk < N ? ldg_pinned(S.nnk + kk) : 0;
            g.bk = kk < N ? ldg_pinned(S.base + kk) : 0.0;
        };
        auto issue = [&](int kk, int nfk, int sg) {   // move kk's list into stage sg
            if (kk < N) {
                const size_t r = (size_t)kk * M;
                float2 *t = reinterpret_cast<float2 *>(hb + sg * SP_HSTAGE);
                int *q = reinterpret_cast<int *>(hb + sg * SP_HSTAGE + SP_HCAP * 8);
                const int n = min(nfk, SP_HCAP);
                for (int i = lane; i < n; i += 32) {
                    cp_async8(t + i, S.fart + r + i);
                    cp_async4(q + i, S.farkp + r + i);
                }
            }
            cp_async_commit();
        };
        // the far part of move kk from stage sg; false when a wait gave up (uniform over the warp)
        auto process = [&](int kk, const Scal &g, int sg) -> bool {
            const float2 *t = reinterpret_cast<const float2 *>(hb + sg * SP_HSTAGE);
            const int *q = reinterpret_cast<const int *>(hb + sg * SP_HSTAGE + SP_HCAP * 8);
            double sum = 0.0;
            bool bad = false;
            // the decision of partner kq (published in word kq / 32), waiting for the word
            auto accepted = [&](int kq) -> bool {
                const int w = kq / SP_BLK;
                uint64_t v = vpub[w];
                long long it = 0;
                while ((uint32_t)(v >> 32) != (uint32_t)(w + 1)) {
                    if (++it > SP_SPIN_LIMIT || abort_flag) {
                        bad = true;
                        return false;
                    }
                    __nanosleep(32);
                    v = vpub[w];
                }
                return (v >> (kq % SP_BLK)) & 1ull;
            };
            // the ring slot of move kk was last read by the resolver in move kk - SP_FR's block
            const uint64_t vring = (kk >= SP_FR && lane == 0) ? vpub[(kk - SP_FR) / SP_BLK] : 0ull;
            // the listed order, lane by lane (entry lane + 32 j), four entries at a time: their
            // positions, then their decision words, are read together
            const int n = min(g.nf, SP_HCAP);
            for (int c0 = 0; c0 < n; c0 += 128) {
                int kq[4];
                uint64_t v[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) kq[j] = c0 + lane + 32 * j < n ? q[c0 + lane + 32 * j] : -1;
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = kq[j] >= 0 ? vpub[kq[j] / SP_BLK] : 0ull;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (kq[j] >= 0) {
                        const bool got = (uint32_t)(v[j] >> 32) == (uint32_t)(kq[j] / SP_BLK + 1);
                        const bool acc = got ? ((v[j] >> (kq[j] % SP_BLK)) & 1ull) != 0ull : accepted(kq[j]);
                        const float2 tt = t[c0 + lane + 32 * j];
                        sum += (double)(acc ? tt.y : tt.x);
                    }
                }
            }
            for (int i = SP_HCAP + lane; i < g.nf; i += 32) {   // lists longer than SP_HCAP
                const float2 tt = S.fart[(size_t)kk * M + i];
                sum += (double)(accepted(S.farkp[(size_t)kk * M + i]) ? tt.y : tt.x);
            }
            if (kk >= SP_FR && lane == 0 && (uint32_t)(vring >> 32) != (uint32_t)((kk - SP_FR) / SP_BLK + 1))
                accepted(kk - SP_FR);
            if (__any_sync(0xffffffffu, bad)) {
                if (lane == 0) fail();
                return false;
            }
            sum = warp_sum_d(sum);
            if (lane == 0) {
                const float fk = (float)(g.bk + sum);
                vfar[kk % SP_FR] = ((uint64_t)(uint32_t)(kk + 1) << 32) | __float_as_uint(fk);
            }
            return true;
        };
        // one step: stage the next move's list, load the scalars of the move after it, wait
        // for this move's list and sum it
        int sg = 0;
        auto body = [&](int kk, const Scal &cur, const Scal &nxt, Scal &fill) -> bool {
            issue(kk + st, nxt.nf, sg ^ 1);
            load(kk + 2 * st, fill);
            cp_async_wait1();   // this lane's copies of move kk
            __syncwarp();       // and every lane's
            const bool ok = process(kk, cur, sg);
            __syncwarp();       // stage sg is read; the next step but one refills it
            sg ^= 1;
            return ok;
        };
        Scal g0, g1, g2;
        load(h, g0);
        load(h + st, g1);
        issue(h, g0.nf, 0);
        for (int k = h; k < N; k += 3 * st) {
            if (!body(k, g0, g1, g2) || k + st >= N) break;
            if (!body(k + st, g1, g2, g0) || k + 2 * st >= N) break;
            if (!body(k + 2 * st, g2, g0, g1)) break;
        }
        cp_async_wait_all();   // no copy lands after the CTA's shared memory goes away
    }
}

// ----------------------------------------------------------------- commit
// The cycle's commits in one pass, one warp per molecule m (visited at position km), four
// molecules a CTA: if its move was accepted, its stored energies (the later accepted writer of a
// shared slot wins) and its coordinates; its counters either way.  The CTA that finishes last
// then runs the epilogue (counts, step adaptation, fadds, the ran1 state), every other CTA's
// counts being complete.
constexpr int SP_CW = 4;   // molecules (warps) per CTA of the commit pass

__device__ void spec_epilogue(const SpecDev &S);

__global__ void __launch_bounds__(32 * SP_CW) spec_commit_kernel(SpecDev S) {
    __shared__ int s_last;
    const int lane = threadIdx.x & 31;
    const int m = blockIdx.x * SP_CW + (threadIdx.x >> 5);
    if (m < S.N && !(S.flags[0] || S.flags[1])) {
        const int km = S.vpos[m];
        const int am = S.acc[km];
        if (am) {
            const int nn = S.nergpairm[m];
            const size_t row = (size_t)m * S.M;
            for (int s = 1 + lane; s < nn; s += 32) {
                const size_t e = row + s;
                const int p = S.molergpair[e];
                const int kp = S.vpos[p];
                const int e2 = S.mirror[e];
                const int p_writes = S.acc[kp] && (e2 % S.M) >= 1;
                if (p_writes && kp > km) continue;  // the later accepted writer wins
                const float v = (kp < km && S.acc[kp]) ? S.B[e] : S.A[e];
                S.ergpair[S.ergpairref[e] - 1] = v;
            }
            const int a0 = S.naf[m], n = S.nato[m];
            for (int i = lane; i < n; i += 32) {
                S.xa_w[a0 + i] = S.nx[a0 + i];
                S.ya_w[a0 + i] = S.ny[a0 + i];
                S.za_w[a0 + i] = S.nz[a0 + i];
                S.pos_w[a0 + i] = S.npos[a0 + i];
            }
            if (lane == 0) {
                const float4 c = S.nc[m];
                S.xadd_w[m] = c.x;
                S.yadd_w[m] = c.y;
                S.zadd_w[m] = c.z;
                S.nstepreject[m] = 0;
            }
        } else if (lane == 0) {
            const int t = S.mtype[m];
            S.nstepreject[m]++;
            if (S.stepr > 0.0f) atomicAdd(S.rej_rot + t, 1);
            if (S.stepm > 0.0f) atomicAdd(S.rej_tr + t, 1);
        }
        if (lane == 0) {
            if (S.trace_den) S.trace_den[km] = S.fdiff[km];
            if (S.trace_acc) S.trace_acc[km] = am;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(S.flags + 4, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        spec_epilogue(S);
    }
}

__device__ void spec_epilogue(const SpecDev &S) {
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
        S.nwhole[nmt + t] = *(volatile const int32_t *)(S.rej_rot + t);   // counted by other CTAs' atomics
        S.nmovem[t] = S.tries_tr[t];
        S.nmovem[nmt + t] = *(volatile const int32_t *)(S.rej_tr + t);
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

// Draws ahead.  The values a cycle draws are the next off[N] values of the one ran1 stream, a
// function of the state the cycle starts from and of that count only.  While a cycle runs, a
// second stream walks the stream on from where this cycle's draws end, into the caller's
// buffer (int32 words):
//   [AH_VALID] 1 once the values are complete   [AH_COUNT] how many   [AH_USES] cycles that took them
//   [AH_START..+35) the state they start from   [AH_END..+35) the state after them
//   [AH_VALS..) the values (float bits)
// The next cycle takes them only when its starting state equals AH_START word for word and
// it needs exactly AH_COUNT values; otherwise (another stage drew from the stream in
// between, the cycle was redone by the sequential kernel, the caller set a new state) it
// walks the stream itself.  Either way it draws the same values.

__global__ void ahead_fill_kernel(const int32_t *state, int32_t *ahead, const int32_t *count) {
    const int lane = threadIdx.x;
    __shared__ int32_t tab[34];
    const int64_t n = *count;
    if (lane == 0) ahead[AH_VALID] = 0;
    ahead[AH_START + lane] = state[lane];
    if (lane < 3) ahead[AH_START + 32 + lane] = state[32 + lane];
    Ran1Warp g;
    g.load(state);
    const int32_t mcall = state[2];
    float *out = reinterpret_cast<float *>(ahead + AH_VALS);
    __syncwarp();
    int64_t done = 0;
    while (done < n) {
        const int64_t left = n - done;
        int32_t mine;
        const int cnt = g.next(left > 32 ? 32 : (int)left, mine, tab);
        if (lane < cnt) out[done + lane] = ran1_out(mine);
        done += cnt;
    }
    ahead[AH_END + 3 + lane] = g.iv;
    if (lane == 0) {
        ahead[AH_END + 0] = g.idum;
        ahead[AH_END + 1] = g.iy;
        ahead[AH_END + 2] = (int32_t)((uint32_t)mcall + (uint32_t)n);
        ahead[AH_COUNT] = (int32_t)n;
        __threadfence();
        ahead[AH_VALID] = 1;
    }
}

// The second stream and its two events, one set per host thread and device: boxes driven
// from different threads never share them, and one thread's cycles run one after another.
struct AheadStream {
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
static thread_local AheadStream g_ahead_streams[16];

static size_t g_ahead_smem = 0;   // dynamic shared memory of the draws-ahead walk

static int ahead_stream(AheadStream **out) {
    int dev = 0;
    EPSR_CUDA(cudaGetDevice(&dev));
    if (!g_ahead_smem) {
        int optin = 0;
        EPSR_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        g_ahead_smem = (size_t)optin - 256;   // room for the kernel's own static table
    }
    if (dev < 0 || dev >= 16) {
        epsr_set_error("epsr_molfit: device ordinal %d beyond the draws-ahead table", dev);
        return EPSR_ERR_ARG;
    }
    AheadStream &a = g_ahead_streams[dev];
    if (!a.st) {
        EPSR_CUDA(cudaStreamCreateWithFlags(&a.st, cudaStreamNonBlocking));
        EPSR_CUDA(cudaEventCreateWithFlags(&a.fork, cudaEventDisableTiming));
        EPSR_CUDA(cudaEventCreateWithFlags(&a.join, cudaEventDisableTiming));
    }
    *out = &a;
    return EPSR_OK;
}
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
    b += spal(sizeof(float) * ((size_t)N + SP_BLK));                 // thr (+ the last staged block's tail)
    b += 2 * spal(sizeof(float) * (size_t)N * M);                  // A, B
    const size_t npad = ((size_t)N + SP_BLK - 1) / SP_BLK * SP_BLK;
    b += spal(sizeof(double) * N) + spal(sizeof(float2) * npad * SP_W) + spal(sizeof(int32_t) * (size_t)N * M) +
         spal(sizeof(float2) * (size_t)N * M);
    b += spal(sizeof(int32_t) * N);   // nnk
    b += spal(sizeof(int32_t) * N) + spal(sizeof(float) * N) + spal(sizeof(double));
    b += spal(sizeof(float4) * SP_MAXEDGE);   // bin edges of the energy pass
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
    {
        int dev = 0, optin = 0;
        EPSR_CUDA(cudaGetDevice(&dev));
        EPSR_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        if (spec_resolve_smem(N) > (size_t)optin) {
            epsr_set_error("epsr_molfit: %d molecules need %zu bytes of shared memory in the resolver (at most %d)", N,
                           spec_resolve_smem(N), optin);
            return EPSR_ERR_CAPACITY;
        }
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
    S.thr = (float *)take(sizeof(float) * ((size_t)N + SP_BLK));
    S.A = (float *)take(sizeof(float) * (size_t)N * M);
    S.B = (float *)take(sizeof(float) * (size_t)N * M);
    S.base = (double *)take(sizeof(double) * N);
    const size_t npad = ((size_t)N + SP_BLK - 1) / SP_BLK * SP_BLK;
    S.nearT = (float2 *)take(sizeof(float2) * npad * SP_W);
    S.farkp = (int32_t *)take(sizeof(int32_t) * (size_t)N * M);
    S.fart = (float2 *)take(sizeof(float2) * (size_t)N * M);
    S.nnk = (int32_t *)take(sizeof(int32_t) * N);
    S.acc = (int32_t *)take(sizeof(int32_t) * N);
    S.fdiff = (float *)take(sizeof(float) * N);
    S.fadd_acc = (double *)take(sizeof(double));
    {
        float4 *edge = (float4 *)take(sizeof(float4) * SP_MAXEDGE);
        const int nedge = max(S.T.izcut - 1, 1);
        if (box->cubic && nedge <= SP_MAXEDGE && S.T.stepcl > 0.0f) {
            S.nedge = nedge;
            S.edge_w = edge;
            S.bins.tab = S.T.tab;
            S.bins.edge = edge;
            S.bins.ld = S.T.ld;
            S.bins.izcut = S.T.izcut;
            S.bins.cinv = bins_cinv(S.T.stepcl);
        }
    }

    // draws ahead: only with a buffer that holds a whole cycle's values (at most 7 a move)
    const bool ahead = mc->ahead && mc->ahead_cap >= (int64_t)N * 7;
    int32_t *use = S.flags + 3;
    if (ahead) {
        S.ahead_vals = reinterpret_cast<const float *>(mc->ahead + AH_VALS);
        S.use_ahead = use;
    }
    if (ahead) S.ahead = mc->ahead;
    int rc = EPSR_OK;
    EPSR_TIMED("spec_plan_kernel", s, spec_plan_kernel<<<1, 1024, 0, s>>>(S));
    EPSR_CUDA(cudaGetLastError());
    EPSR_TIMED("spec_propose_kernel", s, spec_propose_kernel<<<(max(N, S.nedge) + 127) / 128, 128, 0, s>>>(S));
    // the next cycle's values, from the state after this cycle's draws, on the second stream
    // once nothing of this cycle reads the buffer any more; joined before this call returns
    AheadStream *as = nullptr;
    if (ahead) {
        rc = ahead_stream(&as);
        if (rc) return rc;
        EPSR_CUDA(cudaEventRecord(as->fork, s));
        EPSR_CUDA(cudaStreamWaitEvent(as->st, as->fork, 0));
        // the walk is one warp's chain of dependent shuffles: other CTAs on its SM would take
        // issue slots from it, so it asks for all the shared memory a CTA may have, which keeps
        // the SM to itself for the 2-3 ms it runs
        EPSR_SMEM_OPTIN(ahead_fill_kernel);
        EPSR_TIMED("ahead_fill_kernel", as->st,
                   ahead_fill_kernel<<<1, 32, g_ahead_smem, as->st>>>(S.ran1_next, mc->ahead, S.off + N));
        EPSR_CUDA(cudaGetLastError());
        EPSR_CUDA(cudaEventRecord(as->join, as->st));
    }
    {
        const int ma = box->maxat > 0 && box->maxat <= SP_MAXAT ? box->maxat : SP_MAXAT;
        S.ev = max(2 * ma * ma, 4096);
    }
    const size_t en_bytes = sizeof(float) * (size_t)S.ev + sizeof(uint16_t) * (size_t)((S.ev + 1) & ~1) +
                            sizeof(int) * (size_t)box->ntype * box->ntype;
    if (S.nedge) {
        EPSR_SMEM_OPTIN(spec_energy_kernel<true>);
        EPSR_TIMED("spec_energy_kernel", s, spec_energy_kernel<true><<<N, SP_ET, en_bytes, s>>>(S));
    } else {
        EPSR_SMEM_OPTIN(spec_energy_kernel<false>);
        EPSR_TIMED("spec_energy_kernel", s, spec_energy_kernel<false><<<N, SP_ET, en_bytes, s>>>(S));
    }
    EPSR_CUDA(cudaMemsetAsync(S.nearT, 0, sizeof(float2) * npad * SP_W, s));
    EPSR_TIMED("spec_corr_kernel", s, spec_corr_kernel<<<N, 128, 0, s>>>(S));
    // the walk is latency-bound on its scheduler: the CTA asks for all the shared memory a CTA
    // may have (its own need, spec_resolve_smem(N), is checked above), so no other kernel's CTA
    // shares the SM and takes issue slots from it
    size_t rsmem = spec_resolve_smem(N);
    {
        int dev = 0, optin = 0;
        EPSR_CUDA(cudaGetDevice(&dev));
        EPSR_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        rsmem = max(rsmem, (size_t)optin - 1024);
    }
    EPSR_SMEM_OPTIN(spec_resolve_kernel);
    EPSR_TIMED("spec_resolve_kernel", s, spec_resolve_kernel<<<1, SP_RT, rsmem, s>>>(S));
    EPSR_TIMED("spec_commit_kernel", s, spec_commit_kernel<<<(N + SP_CW - 1) / SP_CW, 32 * SP_CW, 0, s>>>(S));
    EPSR_CUDA(cudaGetLastError());
    if (ahead) EPSR_CUDA(cudaStreamWaitEvent(s, as->join, 0));
    // a cycle with a translation retry runs on the sequential kernel (no-op otherwise)
    return molfit_seq_launch(box, cells, store, mc, nullptr, 0, s, S.flags);
}
