// shake.cu -- the intramolecular branch of molfit (molfit.py:124-174, the cycle taken when
// nisum >= intra): every molecule's atoms moved at random (movei :545, movea :556), the change of
// its intramolecular energy (en_change_intra :763 -> en_mole_intra :1327 -> en_atom_intra :923),
// the Metropolis test and, on acceptance, the centre of mass put back at the molecule centre
// (centreofmassi ato_manipulation_rev4.py:442); then the step adaptation (:465-536).  A box
// with rotational groups also rotates each molecule's groups after its atom moves (:175-245),
// tested with the intermolecular change; that cycle runs on the sequential kernel of mc.cu.
//
// Every moved molecule draws three values per atom and one for its test, so its place in the
// ran1 stream is known before the cycle starts.  The stream is generated once; every
// molecule's trial coordinates and new intramolecular energy are computed in parallel (one
// thread per molecule, the atom pairs in the reference's order); one thread then walks the
// molecules in order for the little that chains them: the first stored energy the test
// compares against (the reference's ergold(1), which a molecule with an empty list inherits
// from the molecule before it, and which an earlier accepted molecule rewrites when the two
// share that slot), the running float32 sum faddb and the per-type counts.  Accepted moves are
// applied in parallel.
#include <string.h>

#include "common.cuh"
#include "intra.cuh"

namespace epsr {

constexpr int SH_THREADS = 1024;
constexpr int SH_TILE = 1024;       // molecules per tile of the ordered pass

// en_mole_intra with the molecule's atom pairs spread over the lanes of one warp: every lane
// evaluates pairs (flattened in the reference's (ia, ja) order) into the warp's slice of
// shared memory, then lane 0 sums them in that order.  Molecules of more than SH_WAT atoms fall
// back to one thread.  The value is returned on lane 0.
constexpr int SH_WAT = 64;
constexpr int SH_WPAIRS = SH_WAT * (SH_WAT - 1) / 2;
constexpr int SH_WARPS = 4;   // warps (molecules) per CTA of the warp kernels

__device__ float warp_en_mole_intra(const IntraDev &I, int im, const float *x, const float *y, const float *z,
                                    float *pe, int lane) {
    const int a0 = I.naf[im], n = I.nato[im];
    if (n > SH_WAT) return lane == 0 ? en_mole_intra_d(I, im, x, y, z) : 0.0f;
    const int np = n * (n - 1) / 2;
    for (int p = lane; p < np; p += 32) {
        int i = 0, q = p;
        while (q >= n - 1 - i) {   // row i holds the pairs (i, i+1..n-1)
            q -= n - 1 - i;
            ++i;
        }
        const int ia = a0 + i, ja = a0 + i + 1 + q;
        pe[p] = en_atom_intra_d(I, im, ia, ja, x[ia], y[ia], z[ia], x[ja], y[ja], z[ja]);
    }
    __syncwarp();
    float e = 0.0f;
    if (lane == 0) {
        for (int p = 0; p < np; ++p) e = __fadd_rn(e, pe[p]);
        if (has_dihedral_term(I, im)) e = __fadd_rn(e, dihedral_term_d(I, im, x, y, z));
    }
    return e;
}

__global__ void __launch_bounds__(32 * SH_WARPS) en_mole_intra_kernel(IntraDev I, int nmol, const float *xa,
                                                                       const float *ya, const float *za, float *out) {
    __shared__ float pe[SH_WARPS][SH_WPAIRS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int im = blockIdx.x * SH_WARPS + w;
    if (im >= nmol) return;
    const float e = warp_en_mole_intra(I, im, xa, ya, za, pe[w], lane);
    if (lane == 0) out[im] = e;
}

// ---------------------------------------------------------------- the cycle

struct ShakeDev {
    IntraDev I;
    int nmol, nmoltype, M, ireset;
    float stepmi, simt, rejrate, trstepmax, trstepmin;
    float *xa, *ya, *za;
    const int32_t *nergpairm, *molergpair, *ergpairref;
    float *ergpair;
    float *wholerot, *wholetrans, *internrot, *interntrans, *fadds, *faddbs;
    int32_t *nwhole, *nmovem, *nmovei;
    // scratch
    long long *off;      // [nmol] first ran1 value of each molecule, -1: not moved
    long long *total;    // [2]: the draw count, then the status (1: a molecule with rotational groups)
    int32_t *status;     // = (int32_t *)(total + 1)
    const float *vals;   // [total] the cycle's ran1 values
    float *xt, *yt, *zt; // [natom] trial coordinates
    float *enew;         // [nmol]
    int32_t *acc;        // [nmol]
};

// The draws of every molecule (3 per atom + 1 when it is moved), their offsets in the stream,
// and the per-type settings the reference makes while it walks the molecules: interntrans(mt)
// set to trstepmin where it was 0 for types with a moved molecule (:135-138), internrot(mt) = 0
// for types with a molecule without rotational groups (:246-247).
__global__ void __launch_bounds__(SH_THREADS) shake_plan_kernel(ShakeDev D) {
    __shared__ long long wsum[SH_THREADS / 32];
    __shared__ long long carry;
    __shared__ int moved_t[64], plain_t[64], bad;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) {
        carry = 0;
        bad = 0;
    }
    for (int t = tid; t < 64; t += blockDim.x) moved_t[t] = plain_t[t] = 0;
    __syncthreads();
    for (int base = 0; base < D.nmol; base += SH_THREADS) {
        const int m = base + tid;
        long long d = 0;
        if (m < D.nmol) {
            const int n = D.I.nato[m];
            if (D.I.ngrot[m] > 0) atomicOr(&bad, 1);
            const int mt = D.I.mtype[m];
            if (n > 1 && D.stepmi > 0.0f) {
                d = 3LL * n + 1;
                if (mt < 64) moved_t[mt] = 1;
            }
            if (mt < 64) plain_t[mt] = 1;
        }
        long long v = d;   // inclusive warp scan
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        if (lane == 31) wsum[w] = v;
        __syncthreads();
        if (w == 0) {
            long long s = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const long long u = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += u;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const long long excl = carry + (w > 0 ? wsum[w - 1] : 0) + v - d;
        if (m < D.nmol) D.off[m] = d > 0 ? excl : -1;
        __syncthreads();
        if (tid == 0) carry += wsum[31];
        __syncthreads();
    }
    if (tid == 0) {
        D.total[0] = carry;
        D.status[0] = bad;
    }
    if (bad) return;
    for (int t = tid; t < D.nmoltype && t < 64; t += blockDim.x) {
        if (moved_t[t] && D.interntrans[t] == 0.0f) D.interntrans[t] = D.trstepmin;
        if (plain_t[t]) D.internrot[t] = 0.0f;
    }
}

// movei/movea (:545-567): atom by atom, z then y then x, x += step * (2 r - 1); then the new
// intramolecular energy of the trial coordinates.  One warp per molecule.
__global__ void __launch_bounds__(32 * SH_WARPS) shake_trial_kernel(ShakeDev D) {
    __shared__ float pe[SH_WARPS][SH_WPAIRS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int im = blockIdx.x * SH_WARPS + w;
    if (im >= D.nmol) return;
    const long long o = D.off[im];
    if (o < 0) return;
    const int a0 = D.I.naf[im], n = D.I.nato[im];
    const float step = D.interntrans[D.I.mtype[im]];
    const float *r = D.vals + o;
    for (int k = lane; k < n; k += 32) {
        const int a = a0 + k;
        D.zt[a] = __fadd_rn(D.za[a], __fmul_rn(step, __fsub_rn(__fmul_rn(2.0f, r[3 * k]), 1.0f)));
        D.yt[a] = __fadd_rn(D.ya[a], __fmul_rn(step, __fsub_rn(__fmul_rn(2.0f, r[3 * k + 1]), 1.0f)));
        D.xt[a] = __fadd_rn(D.xa[a], __fmul_rn(step, __fsub_rn(__fmul_rn(2.0f, r[3 * k + 2]), 1.0f)));
    }
    __syncwarp();
    const float e = warp_en_mole_intra(D.I, im, D.xt, D.yt, D.zt, pe[w], lane);
    if (lane == 0) D.enew[im] = e;
}

// The Metropolis test value of en_change_intra's difference (molfit.py:147-154).
__device__ __forceinline__ float metropolis_etest(float enew, float eold, float temp) {
    const float ediff = __fmul_rn(__fsub_rn(enew, eold), temp);
    if (ediff <= 0.0f) return 10.0f;
    if (ediff < 20.0f) return exp_r(-ediff);
    return 0.0f;
}

// The same, out of line: the ordered pass calls it only when a chained energy changed the
// comparison, so the exponential stays off its path.
__device__ __noinline__ float metropolis_etest_call(float enew, float eold, float temp) {
    return metropolis_etest(enew, eold, temp);
}

// The ordered pass (:119-170 per molecule) and the step adaptation (:465-536).  Per tile of
// molecules: every thread loads one molecule's inputs and forms its Metropolis decisions against
// its own first stored energy and, where an earlier molecule shares that stored slot, against
// that molecule's trial energy (what the slot holds once that molecule is accepted); one thread
// walks the tile in order carrying ergold(1) and faddb in registers, reading eight molecules'
// inputs ahead of the chain and picking the decision by the earlier molecule's acceptance (only a
// molecule with an empty list, compared against the carried energy, forms its own); the threads
// then count tries and rejections per type.
#define SHF_MV 1      // the molecule was moved (a trial)
#define SHF_NN 2      // its stored list is not empty
#define SHF_PREV 4    // an earlier molecule shares its first stored slot
#define SHF_ACC 8     // the decision against its own first stored energy
#define SHF_ACCP 16   // the decision against the trial energy of the earlier molecule sharing it
#define SH_AHEAD 8
__global__ void __launch_bounds__(SH_THREADS) shake_resolve_kernel(ShakeDev D) {
    __shared__ float s_enew[SH_TILE], s_r[SH_TILE], s_v1[SH_TILE], s_enp[SH_TILE];
    __shared__ int s_prev[SH_TILE], s_mt[SH_TILE];
    __shared__ int s_slot[SH_TILE];
    __shared__ unsigned char s_fl[SH_TILE], s_acc[SH_TILE];
    __shared__ int cnt[2 * 64];
    __shared__ float s_faddb, s_ergold1;
    const int tid = threadIdx.x;
    const float temp = __fdiv_rn(1.0f, D.simt);
    for (int t = tid; t < 2 * 64; t += blockDim.x) cnt[t] = 0;
    if (tid == 0) {
        s_faddb = 0.0f;
        s_ergold1 = 0.0f;   // a molecule with an empty list before any loaded one compares against 0
    }
    __syncthreads();
    for (int base = 0; base < D.nmol; base += SH_TILE) {
        const int nt = min(SH_TILE, D.nmol - base);
        const int ntp = (nt + SH_AHEAD - 1) / SH_AHEAD * SH_AHEAD;   // <= SH_TILE (a multiple of SH_AHEAD)
        for (int k = tid; k < ntp; k += blockDim.x) {
            if (k >= nt) {              // padding: no trial, no list -- the walk leaves the chain alone
                s_fl[k] = 0;
                s_enew[k] = s_r[k] = s_v1[k] = s_enp[k] = 0.0f;
                s_prev[k] = -1;
                s_slot[k] = 0;
                continue;
            }
            const int m = base + k;
            const long long o = D.off[m];
            const int nn = D.nergpairm[m];
            s_mt[k] = D.I.mtype[m];
            float en = 0.0f, r = 0.0f;
            if (o >= 0) {
                en = D.enew[m];
                r = D.vals[o + 3LL * D.I.nato[m]];
            }
            s_enew[k] = en;
            s_r[k] = r;
            int prev = -1, slot = 0;
            float v1 = 0.0f;
            if (nn >= 1) {
                const size_t row = (size_t)m * D.M;
                slot = D.ergpairref[row];
                v1 = D.ergpair[slot - 1];
                // an earlier molecule whose first slot is the same stored energy (a shared pair
                // that is the first entry of both lists) rewrites it when its move is accepted
                const int p = D.molergpair[row];
                if (p >= 0 && p < m && D.nergpairm[p] >= 1 && D.ergpairref[(size_t)p * D.M] == slot) prev = p;
            }
            const float enp = prev >= 0 ? D.enew[prev] : 0.0f;
            s_slot[k] = slot;
            s_v1[k] = v1;
            s_prev[k] = prev;
            s_enp[k] = enp;
            int fl = (o >= 0 ? SHF_MV : 0) | (nn >= 1 ? SHF_NN : 0) | (prev >= 0 ? SHF_PREV : 0);
            if (o >= 0 && nn >= 1 && r < metropolis_etest(en, v1, temp)) fl |= SHF_ACC;
            if (o >= 0 && prev >= 0 && r < metropolis_etest(en, enp, temp)) fl |= SHF_ACCP;
            s_fl[k] = (unsigned char)fl;
        }
        __syncthreads();
        if (tid == 0) {
            float faddb = s_faddb, ergold1 = s_ergold1;
            for (int k0 = 0; k0 < ntp; k0 += SH_AHEAD) {
                int fl[SH_AHEAD], pv[SH_AHEAD];
                float en[SH_AHEAD], v1[SH_AHEAD], enp[SH_AHEAD];
#pragma unroll
                for (int j = 0; j < SH_AHEAD; ++j) {
                    fl[j] = s_fl[k0 + j];
                    en[j] = s_enew[k0 + j];
                    v1[j] = s_v1[k0 + j];
                    enp[j] = s_enp[k0 + j];
                    pv[j] = s_prev[k0 + j];
                }
#pragma unroll
                for (int j = 0; j < SH_AHEAD; ++j) {
                    const int k = k0 + j, f = fl[j];
                    const bool nn = (f & SHF_NN) != 0, mv = (f & SHF_MV) != 0;
                    int pa = 0;
                    if (f & SHF_PREV) {
                        const int p = pv[j];
                        pa = p >= base ? s_acc[p - base] : D.acc[p];
                    }
                    // make_neighbour_list_from_mols: ergold(1) is the first stored energy (as the
                    // sharing molecule left it); a molecule with an empty list keeps the carried one
                    const float e1 = nn ? (pa ? enp[j] : v1[j]) : ergold1;
                    // the decisions were formed in parallel against both energies the slot can
                    // hold here; only a molecule with an empty list compares against the carried one
                    int a;
                    if (mv && !nn) a = s_r[k] < metropolis_etest_call(en[j], e1, temp);
                    else a = mv && (f & (pa ? SHF_ACCP : SHF_ACC)) != 0;
                    const float fsum = __fadd_rn(faddb, __fsub_rn(en[j], e1));
                    faddb = a ? fsum : faddb;
                    const bool save = a && nn;                          // save_energies + save_erg_pairs
                    ergold1 = save ? en[j] : e1;
                    if (save) D.ergpair[s_slot[k] - 1] = en[j];
                    s_acc[k] = (unsigned char)a;
                }
            }
            s_faddb = faddb;
            s_ergold1 = ergold1;
        }
        __syncthreads();
        for (int k = tid; k < nt; k += blockDim.x) {
            const int a = s_acc[k];
            D.acc[base + k] = a;
            if ((s_fl[k] & SHF_MV) && s_mt[k] < 64) {
                atomicAdd(&cnt[s_mt[k]], 1);
                if (!a) atomicAdd(&cnt[64 + s_mt[k]], 1);
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int nmt = D.nmoltype;
        const float rotstepmin = 1.0e-5f, rotstepmax = 1.0f;
        for (int t = 0; t < nmt; ++t) {
            const int tries = t < 64 ? cnt[t] : 0, rej = t < 64 ? cnt[64 + t] : 0;
            D.nmovei[t] = tries;
            D.nmovei[nmt + t] = rej;
            D.nwhole[t] = D.nwhole[nmt + t] = 0;
            D.nmovem[t] = D.nmovem[nmt + t] = 0;
            if (D.ireset != 1) {
                float rat;
                if (rej > 0) {
                    rat = __fdiv_rn(__fmul_rn(D.rejrate, (float)tries), (float)rej);
                    if (rat > 1.1f) rat = 1.1f;
                    if (rat < 0.9f) rat = 0.9f;
                } else {
                    rat = tries > 0 ? 1.1f : 1.0f;
                }
                float it = __fmul_rn(D.interntrans[t], rat);
                if (it > D.trstepmax) it = D.trstepmax;
                if (it < D.trstepmin && it != 0.0f) it = D.trstepmin;
                D.interntrans[t] = it;
                float ir = __fmul_rn(D.internrot[t], 1.0f);      // no internal rotations: ninter 0
                if (ir > rotstepmax) ir = rotstepmax;
                if (ir < rotstepmin && ir != 0.0f) ir = rotstepmin;
                D.internrot[t] = ir;
                float wr = __fmul_rn(D.wholerot[t], 1.0f);       // no whole-molecule moves this cycle
                if (wr > rotstepmax) wr = rotstepmax;
                if (wr < rotstepmin && wr != 0.0f) wr = rotstepmin;
                D.wholerot[t] = wr;
                float wt = __fmul_rn(D.wholetrans[t], 1.0f);
                if (wt > D.trstepmax) wt = D.trstepmax;
                if (wt < D.trstepmin && wt != 0.0f) wt = D.trstepmin;
                D.wholetrans[t] = wt;
            }
        }
        D.fadds[0] = __fadd_rn(D.fadds[0], __fdiv_rn(0.0f, (float)D.nmol));
        D.faddbs[0] = __fadd_rn(D.faddbs[0], __fdiv_rn(s_faddb, (float)D.nmol));
    }
}

// Accepted moves: the trial coordinates, then centreofmassi (mass-weighted centre of the
// non-q atoms, summed in atom order, subtracted from every atom).
__global__ void shake_apply_kernel(ShakeDev D) {
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= D.nmol || D.off[im] < 0 || !D.acc[im]) return;
    const int a0 = D.I.naf[im], n = D.I.nato[im];
    float x1 = 0.0f, y1 = 0.0f, z1 = 0.0f, summass = 0.0f;
    for (int k = 0; k < n; ++k) {
        const int a = a0 + k;
        if (D.I.qtype[a] == 0) {
            const float am = D.I.amassa[D.I.itype[a]];
            x1 = __fadd_rn(x1, __fmul_rn(D.xt[a], am));
            y1 = __fadd_rn(y1, __fmul_rn(D.yt[a], am));
            z1 = __fadd_rn(z1, __fmul_rn(D.zt[a], am));
            summass = __fadd_rn(summass, am);
        }
    }
    if (summass > 0.0f) {
        x1 = __fdiv_rn(x1, summass);
        y1 = __fdiv_rn(y1, summass);
        z1 = __fdiv_rn(z1, summass);
    }
    for (int k = 0; k < n; ++k) {
        const int a = a0 + k;
        D.xa[a] = __fsub_rn(D.xt[a], x1);
        D.ya[a] = __fsub_rn(D.yt[a], y1);
        D.za[a] = __fsub_rn(D.zt[a], z1);
    }
}

__global__ void minimage_centres_kernel(Lattice L, int nmol, float *xadd, float *yadd, float *zadd) {
    const int im = blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= nmol) return;
    float x = xadd[im], y = yadd[im], z = zadd[im];
    minimagec(L, x, y, z);
    xadd[im] = x;
    yadd[im] = y;
    zadd[im] = z;
}

size_t al256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace epsr

namespace epsr {
int molfit_shake_rot_launch(const epsr_box_t *box, epsr_store_t *store, epsr_mc_t *mc, const epsr_intra_t *in,
                            float stepmi, int32_t *nmovei, float *faddbs, void *scratch, int64_t scratch_bytes,
                            cudaStream_t s);
}

using namespace epsr;

static int intra_check(const epsr_box_t *box, const epsr_intra_t *in, const char *who) {
    if (!box || !in || !in->nbond || !in->iabond || !in->tbond || in->maxbond < 1 || !in->imageatom || !in->qtype ||
        !in->amassa || !in->amassr || !in->xav || !in->xav1 || !in->ngrot || !(in->stepcl > 0.0f)) {
        epsr_set_error("%s: bad arguments", who);
        return EPSR_ERR_ARG;
    }
    return EPSR_OK;
}

extern "C" int epsr_en_mole_intra(const epsr_box_t *box, const epsr_intra_t *in, float *out, void *stream) {
    int rc = intra_check(box, in, "epsr_en_mole_intra");
    if (rc) return rc;
    if (!out || box->nmol < 1) {
        epsr_set_error("epsr_en_mole_intra: bad arguments");
        return EPSR_ERR_ARG;
    }
    const IntraDev I = make_intradev(box, in);
    en_mole_intra_kernel<<<(box->nmol + SH_WARPS - 1) / SH_WARPS, 32 * SH_WARPS, 0, (cudaStream_t)stream>>>(
        I, box->nmol, box->xa, box->ya,
                                                                                  box->za, out);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}

extern "C" int epsr_minimage_centres(const epsr_box_t *box, void *stream) {
    if (!box || box->nmol < 1 || !box->xadd || !box->yadd || !box->zadd) {
        epsr_set_error("epsr_minimage_centres: bad arguments");
        return EPSR_ERR_ARG;
    }
    Lattice L;
    L.cubic = box->cubic;
    L.alatx = box->lat[0];
    L.blatx = box->lat[1];
    L.clatx = box->lat[2];
    L.blaty = box->lat[3];
    L.claty = box->lat[4];
    L.clatz = box->lat[5];
    minimage_centres_kernel<<<(box->nmol + 127) / 128, 128, 0, (cudaStream_t)stream>>>(L, box->nmol, box->xadd,
                                                                                       box->yadd, box->zadd);
    EPSR_CUDA(cudaGetLastError());
    return epsr_box_positions(box, stream);
}

extern "C" int64_t epsr_molfit_shake_scratch_bytes(int32_t nmol, int32_t natom) {
    if (nmol < 1 || natom < 1) return -1;
    return (int64_t)(al256(8 * (size_t)nmol) + 256 + 256 + al256(4 * (3 * (size_t)natom + nmol)) +
                     3 * al256(4 * (size_t)natom) + al256(4 * (size_t)nmol) + al256(4 * (size_t)nmol));
}

extern "C" int epsr_molfit_shake(const epsr_box_t *box, epsr_store_t *store, epsr_mc_t *mc, const epsr_intra_t *in,
                                 float stepmi, int32_t *nmovei, float *faddbs, void *scratch, int64_t scratch_bytes,
                                 void *stream) {
    int rc = intra_check(box, in, "epsr_molfit_shake");
    if (rc) return rc;
    if (!store || !mc || !nmovei || !faddbs || !scratch || !mc->ran1 || !mc->fadds || !mc->internrot ||
        !mc->interntrans || !mc->wholerot || !mc->wholetrans || !mc->nwhole || !mc->nmovem || box->nmoltype > 64) {
        epsr_set_error("epsr_molfit_shake: bad arguments (at most 64 molecule types)");
        return EPSR_ERR_ARG;
    }
    const int64_t need = epsr_molfit_shake_scratch_bytes(box->nmol, box->natom);
    if (scratch_bytes < need) {
        epsr_set_error("epsr_molfit_shake: scratch %lld < %lld bytes", (long long)scratch_bytes, (long long)need);
        return EPSR_ERR_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    ShakeDev D;
    memset(&D, 0, sizeof(D));
    D.I = make_intradev(box, in);
    D.nmol = box->nmol;
    D.nmoltype = box->nmoltype;
    D.M = store->nnbrefmax;
    D.ireset = mc->ireset;
    D.stepmi = stepmi;
    D.simt = mc->simt;
    D.rejrate = mc->rejrate;
    D.trstepmax = mc->trstepmax;
    D.trstepmin = mc->trstepmin;
    D.xa = box->xa;
    D.ya = box->ya;
    D.za = box->za;
    D.nergpairm = store->nergpairm;
    D.molergpair = store->molergpair;
    D.ergpairref = store->ergpairref;
    D.ergpair = store->ergpair;
    D.wholerot = mc->wholerot;
    D.wholetrans = mc->wholetrans;
    D.internrot = mc->internrot;
    D.interntrans = mc->interntrans;
    D.fadds = mc->fadds;
    D.faddbs = faddbs;
    D.nwhole = mc->nwhole;
    D.nmovem = mc->nmovem;
    D.nmovei = nmovei;
    unsigned char *p = (unsigned char *)scratch;
    D.off = (long long *)p;
    p += al256(8 * (size_t)D.nmol);
    D.total = (long long *)p;
    D.status = (int32_t *)(D.total + 1);
    p += 256;
    p += 256;
    float *vals = (float *)p;
    D.vals = vals;
    p += al256(4 * (3 * (size_t)box->natom + D.nmol));
    D.xt = (float *)p;
    p += al256(4 * (size_t)box->natom);
    D.yt = (float *)p;
    p += al256(4 * (size_t)box->natom);
    D.zt = (float *)p;
    p += al256(4 * (size_t)box->natom);
    D.enew = (float *)p;
    p += al256(4 * (size_t)D.nmol);
    D.acc = (int32_t *)p;

    shake_plan_kernel<<<1, SH_THREADS, 0, s>>>(D);
    EPSR_CUDA(cudaGetLastError());
    long long tot2[2] = {0, 0};
    EPSR_D2H(tot2, D.total, sizeof(tot2), s);
    const long long total = tot2[0];
    const int32_t status = (int32_t)(tot2[1] & 0xffffffff);
    if (status) {
        // molecules with rotational groups: after each molecule's atom moves its groups are
        // rotated and tested with the intermolecular change (molfit.py:175-245), which chains the
        // molecules in index order -- the sequential kernel runs the whole cycle
        if (!mc->rot_nrf || !mc->rot_nrl || !mc->rot_axis || !mc->rot_first || !mc->rot_last || !mc->rot_atoms ||
            !mc->ninter || !mc->nstepreject) {
            epsr_set_error("epsr_molfit_shake: molecules with rotational groups need the groups (rot_*), ninter and "
                           "nstepreject in the mc state");
            return EPSR_ERR_UNSUPPORTED;
        }
        rc = molfit_shake_rot_launch(box, store, mc, in, stepmi, nmovei, faddbs, scratch, scratch_bytes, s);
        if (rc) return rc;
        return epsr_box_positions(box, stream);
    }
    if (total > 3LL * box->natom + D.nmol) {
        epsr_set_error("epsr_molfit_shake: %lld draws exceed the stream buffer", total);
        return EPSR_ERR_CAPACITY;
    }
    if (total > 0) {
        rc = epsr_ran1_fill(mc->ran1, vals, total, stream);
        if (rc) return rc;
    }
    const int nb = (D.nmol + 127) / 128;
    shake_trial_kernel<<<(D.nmol + SH_WARPS - 1) / SH_WARPS, 32 * SH_WARPS, 0, s>>>(D);
    EPSR_CUDA(cudaGetLastError());
    shake_resolve_kernel<<<1, SH_THREADS, 0, s>>>(D);
    EPSR_CUDA(cudaGetLastError());
    shake_apply_kernel<<<nb, 128, 0, s>>>(D);
    EPSR_CUDA(cudaGetLastError());
    return epsr_box_positions(box, stream);
}
