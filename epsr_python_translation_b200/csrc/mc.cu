// mc.cu -- molfit whole-molecule cycle (molfit.py:52-541) on one box.
//
// Sequential kernel: one CTA walks the molecules in cell-visit order exactly as the
// reference (the ran1 stream and the accept decisions chain every move to the previous
// one).  Per move: one thread draws the rotation (rotatm :672) and translation (movem :733,
// including the step-doubling retry); all threads evaluate the moved molecule against its
// stored neighbours, one neighbour per thread in the reference's (ia, ja) order so each
// neighbour energy is bit-identical (en_change :806); then the Metropolis test (:401-408),
// the store update (save_energies/save_erg_pairs) and the coordinate commit or restore.
#include <string.h>

#include "common.cuh"
#include "intra.cuh"

namespace epsr {

constexpr int MC_THREADS = 512;
constexpr int MC_MAXAT = 64;  // atoms per molecule handled by the kernel

struct McDev {
    Lattice L;
    Tables T;
    int nmol, ntype, nmoltype, M;
    const int32_t *naf, *nato, *mtype, *npairref, *visit;
    float *xa, *ya, *za, *xadd, *yadd, *zadd;
    float4 *pos;
    const int32_t *nergpairm, *molergpair, *ergpairref;
    float *ergpair;
    // parameters
    float simt, rejrate, stepr, stepm, trstepmax, trstepmin;
    int ireset, strict;
    float *wholerot, *wholetrans, *internrot, *interntrans;
    int32_t *nwhole, *nmovem, *nstepreject;
    float *fadds;
    int32_t *ran1;
    const float *cos_override;
    float *trace_den;
    int32_t *trace_acc;
    float *ergnew_g;   // [M] global fallback when M is large
    int use_smem;
    int32_t *status;
    const int32_t *run_if;  // when set, the kernel runs only if *run_if != 0
    // internal rotations of rotational groups (molfit.py:295-360), when has_rot
    int has_rot, rotcycle;
    float stepri;
    IntraDev I;
    const int32_t *ngrot, *rot_nrf, *rot_nrl, *rot_axis, *rot_first, *rot_last, *rot_atoms;
    int32_t *ninter;
    float *faddbs;
    // the intramolecular cycle of a box with rotational groups (molfit.py:124-267), when shake:
    // molecules in index order, atom moves (stepmi) then internal rotations, no whole-molecule move
    int shake;
    float stepmi;
    int32_t *nmovei;   // [2*nmoltype] tries then rejections of the atom moves
};

// rotati molfit.py:589-660 after its angle: rotate the atoms of group ig about the axis from
// its first axis atom to its second by the angle whose cosine and sine are cphi and sphi, on
// the molecule's offsets x/y/z (local atom index = global - a0), in the reference's float
// operation order (scapro, vecpro auxiliary_routines.py:231-244).
__device__ __forceinline__ void rotati_d(const McDev &D, int a0, int ig, float cphi, float sphi, float *x, float *y,
                                        float *z) {
    const int k1 = D.rot_axis[2 * ig] - a0, k2 = D.rot_axis[2 * ig + 1] - a0;
    float p1 = __fsub_rn(x[k2], x[k1]), p2 = __fsub_rn(y[k2], y[k1]), p3 = __fsub_rn(z[k2], z[k1]);
    const float rab2 = __fadd_rn(__fadd_rn(__fmul_rn(p1, p1), __fmul_rn(p2, p2)), __fmul_rn(p3, p3));
    if (!(rab2 > 0.0f)) return;
    const float rab = __fsqrt_rn(rab2);
    p1 = __fdiv_rn(p1, rab);
    p2 = __fdiv_rn(p2, rab);
    p3 = __fdiv_rn(p3, rab);
    for (int ia = D.rot_first[ig]; ia <= D.rot_last[ig]; ++ia) {
        const int k = D.rot_atoms[ia] - a0;
        const float v1 = __fsub_rn(x[k], x[k1]), v2 = __fsub_rn(y[k], y[k1]), v3 = __fsub_rn(z[k], z[k1]);
        const float frac = __fadd_rn(__fadd_rn(__fmul_rn(p1, v1), __fmul_rn(p2, v2)), __fmul_rn(p3, v3));
        const float q1 = __fmul_rn(frac, p1), q2 = __fmul_rn(frac, p2), q3 = __fmul_rn(frac, p3);
        const float r1 = __fsub_rn(v1, q1), r2 = __fsub_rn(v2, q2), r3 = __fsub_rn(v3, q3);
        const float w1 = __fsub_rn(__fmul_rn(p2, r3), __fmul_rn(p3, r2));
        const float w2 = __fsub_rn(__fmul_rn(p3, r1), __fmul_rn(p1, r3));
        const float w3 = __fsub_rn(__fmul_rn(p1, r2), __fmul_rn(p2, r1));
        const float xs = __fadd_rn(x[k1], q1), ys = __fadd_rn(y[k1], q2), zs = __fadd_rn(z[k1], q3);
        x[k] = __fadd_rn(__fadd_rn(xs, __fmul_rn(r1, cphi)), __fmul_rn(w1, sphi));
        y[k] = __fadd_rn(__fadd_rn(ys, __fmul_rn(r2, cphi)), __fmul_rn(w2, sphi));
        z[k] = __fadd_rn(__fadd_rn(zs, __fmul_rn(r3, cphi)), __fmul_rn(w3, sphi));
    }
}

__device__ __forceinline__ float next_cos(const McDev &D, int &kcos, float phi) {
    if (D.cos_override) return D.cos_override[kcos++];
    ++kcos;
    return cos_r(phi);
}

__global__ void __launch_bounds__(MC_THREADS) molfit_seq_kernel(McDev D) {
    extern __shared__ float dyn[];  // ergnew[M], ergold[M] when use_smem
    __shared__ Ran1 R;
    __shared__ float4 mv[MC_MAXAT];
    __shared__ float nx[MC_MAXAT], ny[MC_MAXAT], nz[MC_MAXAT];
    __shared__ float sx[MC_MAXAT], sy[MC_MAXAT], sz[MC_MAXAT];
    __shared__ int sh_im, sh_n, sh_acc, sh_bad, sh_rot;
    __shared__ float sh_cx, sh_cy, sh_cz, sh_fdiff;
    __shared__ double red[MC_THREADS / 32];
    if (D.run_if && *D.run_if == 0) return;
    float *ergnew = D.use_smem ? dyn : D.ergnew_g;
    float *ergold = D.use_smem ? dyn + D.M : D.ergnew_g + D.M;
    const int tid = threadIdx.x;
    const int nmt = D.nmoltype;
    const float pi = 3.14159265358979323846f;
    const float rotstepmin = 1.0e-5f, rotstepmax = 1.0f;
    int kcos = 0;
    float fadd = 0.0f, faddb = 0.0f;
    // the reference's ergold(1) (molfit's work array): the first stored energy of the last
    // molecule whose list was loaded, as updated by that molecule's accepted moves
    float eold0 = 0.0f, p0 = 0.0f;
    if (tid == 0) {
        ran1_load(R, D.ran1);
        for (int k = 0; k < 2 * nmt; ++k) {
            D.nwhole[k] = 0;
            D.nmovem[k] = 0;
            if (D.ninter) D.ninter[k] = 0;
            if (D.nmovei) D.nmovei[k] = 0;
        }
    }
    const float temp = __fdiv_rn(1.0f, D.simt);
    __syncthreads();
    // en_change (molfit.py:806-919) of molecule sh_im at positions mv[] over its stored list:
    // ergnew/ergold filled for slots 1.., the change summed in list order (strict) or in double
    auto en_change_mv = [&](int im, int n) -> float {
        const size_t row = (size_t)im * D.M;
        const int nn = D.nergpairm[im];
        double part = 0.0;
        for (int inn = 1 + tid; inn < nn; inn += MC_THREADS) {
            const int jm = D.molergpair[row + inn];
            const int b0 = D.naf[jm], b1 = b0 + D.nato[jm];
            float sume = 0.0f;
            for (int ia = 0; ia < n; ++ia) {
                const float4 p1 = mv[ia];
                const int it = __float_as_int(p1.w);
                for (int ja = b0; ja < b1; ++ja) {
                    const float4 p2 = D.pos[ja];
                    const int icref = __ldg(D.npairref + it * D.ntype + __float_as_int(p2.w));
                    sume = __fadd_rn(sume, pair_energy(D.L, D.T, p1, p2, icref));
                }
            }
            const float en = __fadd_rn(0.0f, sume);
            const float eo = D.ergpair[D.ergpairref[row + inn] - 1];
            ergnew[inn] = en;
            ergold[inn] = eo;
            part += (double)en - (double)eo;
        }
        float fdiff;
        if (D.strict) {
            __syncthreads();
            if (tid == 0) {
                float f = 0.0f;
                for (int inn = 1; inn < nn; ++inn) f = __fsub_rn(__fadd_rn(f, ergnew[inn]), ergold[inn]);
                red[0] = (double)f;
            }
            __syncthreads();
            fdiff = (float)red[0];
        } else {
            part = warp_sum_d(part);
            if ((tid & 31) == 0) red[tid >> 5] = part;
            __syncthreads();
            double t = 0.0;
            for (int w = 0; w < MC_THREADS / 32; ++w) t += red[w];
            fdiff = (float)t;
        }
        __syncthreads();
        return fdiff;
    };
    for (int v = 0; v < D.nmol; ++v) {
        if (tid == 0) {
            const int im = D.shake ? v : D.visit[v];
            const int n = D.nato[im];
            sh_bad = n > MC_MAXAT;
        }
        __syncthreads();
        if (sh_bad) {
            if (tid == 0 && D.status) D.status[0] = 1;
            return;
        }
        // ---- internal rotations of the molecule's rotational groups (molfit.py:295-360), in
        // the intramolecular cycle after the molecule's atom moves (:141-267)
        if (tid == 0) {
            const int im = D.shake ? v : D.visit[v];
            const int n = D.nato[im];
            const int mt = D.mtype[im];
            const size_t row = (size_t)im * D.M;
            if (D.nergpairm[im] >= 1) eold0 = D.ergpair[D.ergpairref[row] - 1];   // make_neighbour_list_from_mols
            if (D.shake && n > 1 && D.stepmi > 0.0f) {
                // movei/movea (:545-567) on the offsets, en_change_intra against ergold(1), the
                // Metropolis test; on acceptance the store's first slot (save_energies,
                // save_erg_pairs) and the centre of mass put back (centreofmassi)
                float step = D.interntrans[mt];
                if (step == 0.0f) step = D.trstepmin;
                D.interntrans[mt] = step;
                const int a0 = D.naf[im];
                for (int k = 0; k < n; ++k) {
                    sx[k] = D.xa[a0 + k];
                    sy[k] = D.ya[a0 + k];
                    sz[k] = D.za[a0 + k];
                }
                D.nmovei[mt]++;
                for (int k = 0; k < n; ++k) {
                    const int a = a0 + k;
                    D.za[a] = __fadd_rn(D.za[a], __fmul_rn(step, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                    D.ya[a] = __fadd_rn(D.ya[a], __fmul_rn(step, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                    D.xa[a] = __fadd_rn(D.xa[a], __fmul_rn(step, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                }
                const float enew = en_mole_intra_d(D.I, im, D.xa, D.ya, D.za);
                const float fdiffb = __fsub_rn(enew, eold0);
                const float ediff = __fmul_rn(fdiffb, temp);
                float etest;
                if (ediff <= 0.0f) etest = 10.0f;
                else if (ediff < 20.0f) etest = exp_r(-ediff);
                else etest = 0.0f;
                if (ran1_next(R) < etest) {
                    faddb = __fadd_rn(faddb, fdiffb);
                    if (D.nergpairm[im] >= 1) {
                        eold0 = enew;
                        D.ergpair[D.ergpairref[row] - 1] = enew;
                    }
                    float x1 = 0.0f, y1 = 0.0f, z1 = 0.0f, summass = 0.0f;
                    for (int k = 0; k < n; ++k) {
                        const int a = a0 + k;
                        if (D.I.qtype[a] == 0) {
                            const float am = D.I.amassa[D.I.itype[a]];
                            x1 = __fadd_rn(x1, __fmul_rn(D.xa[a], am));
                            y1 = __fadd_rn(y1, __fmul_rn(D.ya[a], am));
                            z1 = __fadd_rn(z1, __fmul_rn(D.za[a], am));
                            summass = __fadd_rn(summass, am);
                        }
                    }
                    if (summass > 0.0f) {
                        x1 = __fdiv_rn(x1, summass);
                        y1 = __fdiv_rn(y1, summass);
                        z1 = __fdiv_rn(z1, summass);
                    }
                    const float cx = D.xadd[im], cy = D.yadd[im], cz = D.zadd[im];
                    for (int k = 0; k < n; ++k) {
                        const int a = a0 + k;
                        D.xa[a] = __fsub_rn(D.xa[a], x1);
                        D.ya[a] = __fsub_rn(D.ya[a], y1);
                        D.za[a] = __fsub_rn(D.za[a], z1);
                        D.pos[a] = make_float4(__fadd_rn(D.xa[a], cx), __fadd_rn(D.ya[a], cy), __fadd_rn(D.za[a], cz),
                                               D.pos[a].w);
                    }
                } else {
                    D.nmovei[nmt + mt]++;
                    for (int k = 0; k < n; ++k) {
                        D.xa[a0 + k] = sx[k];
                        D.ya[a0 + k] = sy[k];
                        D.za[a0 + k] = sz[k];
                    }
                }
            }
            const int ng = D.ngrot ? D.ngrot[im] : 0;
            sh_rot = D.has_rot && D.stepri > 0.0f && ng > 0 && (D.rotcycle || D.shake);
            sh_im = im;
            sh_n = n;
            if (sh_rot) {
                if (D.internrot[mt] == 0.0f) D.internrot[mt] = rotstepmin;
                D.ninter[mt]++;
                const int a0 = D.naf[im];
                for (int k = 0; k < n; ++k) {
                    sx[k] = D.xa[a0 + k];
                    sy[k] = D.ya[a0 + k];
                    sz[k] = D.za[a0 + k];
                    nx[k] = sx[k];
                    ny[k] = sy[k];
                    nz[k] = sz[k];
                }
                const float step = D.internrot[mt];
                for (int ig = D.rot_nrf[im]; ig <= D.rot_nrl[im]; ++ig) {
                    const float phi = __fmul_rn(__fmul_rn(pi, step), __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f));
                    const float c = next_cos(D, kcos, phi);
                    const float sp = fsign(__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(c, c))), phi);
                    rotati_d(D, a0, ig, c, sp, nx, ny, nz);
                }
                const float cx = D.xadd[im], cy = D.yadd[im], cz = D.zadd[im];
                for (int k = 0; k < n; ++k) {
                    D.xa[a0 + k] = nx[k];   // the trial lives in the offsets, as the reference's
                    D.ya[a0 + k] = ny[k];
                    D.za[a0 + k] = nz[k];
                    mv[k] = make_float4(__fadd_rn(nx[k], cx), __fadd_rn(ny[k], cy), __fadd_rn(nz[k], cz),
                                        D.pos[a0 + k].w);
                }
            } else if (!D.ngrot || D.ngrot[im] == 0) {
                D.internrot[mt] = 0.0f;
            }
        }
        __syncthreads();
        if (sh_rot) {
            const int im = sh_im, n = sh_n;
            const float fdiff = en_change_mv(im, n);
            if (tid == 0) {
                const int mt = D.mtype[im];
                const int a0 = D.naf[im];
                // en_change_intra: the new intramolecular energy against ergold(1)
                const float enew0 = en_mole_intra_d(D.I, im, D.xa, D.ya, D.za);
                const float fdiffb = __fsub_rn(enew0, eold0);
                p0 = enew0;
                const float ediff = __fmul_rn(__fadd_rn(fdiff, fdiffb), temp);
                float etest;
                if (ediff <= 0.0f) etest = 10.0f;
                else if (ediff < 20.0f) etest = exp_r(-ediff);
                else etest = 0.0f;
                const int acc = ran1_next(R) < etest;
                const size_t row = (size_t)im * D.M;
                const int nn = D.nergpairm[im];
                if (acc) {
                    D.nstepreject[im] = 0;
                    fadd = __fadd_rn(fadd, fdiff);
                    faddb = __fadd_rn(faddb, fdiffb);
                    eold0 = enew0;
                    if (nn >= 1) D.ergpair[D.ergpairref[row] - 1] = enew0;
                    for (int k = 0; k < n; ++k) D.pos[a0 + k] = mv[k];
                } else {
                    D.nstepreject[im]++;
                    for (int k = 0; k < n; ++k) {
                        D.xa[a0 + k] = sx[k];
                        D.ya[a0 + k] = sy[k];
                        D.za[a0 + k] = sz[k];
                    }
                    D.ninter[nmt + mt]++;
                }
                sh_acc = acc;
            }
            __syncthreads();
            if (sh_acc) {
                const size_t row = (size_t)im * D.M;
                const int nn = D.nergpairm[im];
                for (int inn = 1 + tid; inn < nn; inn += MC_THREADS) D.ergpair[D.ergpairref[row + inn] - 1] = ergnew[inn];
            }
            __syncthreads();
        }
        if (D.shake) continue;   // the intramolecular cycle moves no molecule whole (uniform branch)
        // ---- whole-molecule rotation and translation (molfit.py:362-448)
        if (tid == 0) {
            const int im = sh_im;
            const int n = sh_n;
            const int a0 = D.naf[im];
            const int mt = D.mtype[im];
            for (int k = 0; k < n; ++k) {
                nx[k] = D.xa[a0 + k];
                ny[k] = D.ya[a0 + k];
                nz[k] = D.za[a0 + k];
            }
            if (D.stepr > 0.0f && n > 1) {
                if (D.wholerot[mt] <= 0.0f) D.wholerot[mt] = rotstepmin;
                D.nwhole[mt]++;
                const float step = D.wholerot[mt];
                // rotatm: about z, then y, then x (molfit.py:683-710)
                for (int ax = 0; ax < 3; ++ax) {
                    float phi = __fmul_rn(__fmul_rn(pi, step), __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f));
                    float c = next_cos(D, kcos, phi);
                    float sgn = fsign(__fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(c, c))), phi);
                    for (int k = 0; k < n; ++k) {
                        if (ax == 0) {
                            float xs = __fsub_rn(__fmul_rn(nx[k], c), __fmul_rn(ny[k], sgn));
                            ny[k] = __fadd_rn(__fmul_rn(nx[k], sgn), __fmul_rn(ny[k], c));
                            nx[k] = xs;
                        } else if (ax == 1) {
                            float zs = __fsub_rn(__fmul_rn(nz[k], c), __fmul_rn(nx[k], sgn));
                            nx[k] = __fadd_rn(__fmul_rn(nz[k], sgn), __fmul_rn(nx[k], c));
                            nz[k] = zs;
                        } else {
                            float ys = __fsub_rn(__fmul_rn(ny[k], c), __fmul_rn(nz[k], sgn));
                            nz[k] = __fadd_rn(__fmul_rn(ny[k], sgn), __fmul_rn(nz[k], c));
                            ny[k] = ys;
                        }
                    }
                }
            } else {
                D.wholerot[mt] = 0.0f;
            }
            float cx = D.xadd[im], cy = D.yadd[im], cz = D.zadd[im];
            if (D.stepm > 0.0f) {
                if (D.wholetrans[mt] <= 0.0f) D.wholetrans[mt] = D.trstepmin;
                D.nmovem[mt]++;
                float st = D.wholetrans[mt];
                const float xs = cx, ys = cy, zs = cz;
                cz = __fadd_rn(cz, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                cy = __fadd_rn(cy, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                cx = __fadd_rn(cx, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                while (xs == cx && ys == cy && zs == cz) {
                    st = __fmul_rn(st, 2.0f);
                    cz = __fadd_rn(cz, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                    cy = __fadd_rn(cy, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                    cx = __fadd_rn(cx, __fmul_rn(st, __fsub_rn(__fmul_rn(2.0f, ran1_next(R)), 1.0f)));
                }
                D.wholetrans[mt] = st;
            } else {
                D.wholetrans[mt] = 0.0f;
            }
            for (int k = 0; k < n; ++k)
                mv[k] = make_float4(__fadd_rn(nx[k], cx), __fadd_rn(ny[k], cy), __fadd_rn(nz[k], cz),
                                    D.pos[a0 + k].w);
            sh_cx = cx;
            sh_cy = cy;
            sh_cz = cz;
        }
        __syncthreads();
        const int im = sh_im, n = sh_n;
        const size_t row = (size_t)im * D.M;
        const int nn = D.nergpairm[im];
        const float fdiff = en_change_mv(im, n);
        if (tid == 0) {
            const int mt = D.mtype[im];
            const float ediff = __fmul_rn(__fadd_rn(fdiff, 0.0f), temp);
            float etest;
            if (ediff <= 0.0f) etest = 10.0f;
            else if (ediff < 20.0f) etest = exp_r(-ediff);
            else etest = 0.0f;
            const int acc = ran1_next(R) < etest;
            if (acc) {
                D.nstepreject[im] = 0;
                fadd = __fadd_rn(fadd, fdiff);
                // save_energies copies every slot, the first one included: after an internal
                // rotation of this visit it holds the rotation's intramolecular energy even when
                // that rotation was rejected (molfit.py:215, :419; ergpairreference.py:192-210)
                if (sh_rot) {
                    eold0 = p0;
                    if (nn >= 1) D.ergpair[D.ergpairref[row] - 1] = p0;
                }
            } else {
                D.nstepreject[im]++;
                if (D.stepr > 0.0f) D.nwhole[nmt + mt]++;
                if (D.stepm > 0.0f) D.nmovem[nmt + mt]++;
            }
            if (D.trace_den) D.trace_den[v] = fdiff;
            if (D.trace_acc) D.trace_acc[v] = acc;
            sh_acc = acc;
        }
        __syncthreads();
        if (sh_acc) {
            for (int inn = 1 + tid; inn < nn; inn += MC_THREADS) D.ergpair[D.ergpairref[row + inn] - 1] = ergnew[inn];
            const int a0 = D.naf[im];
            for (int k = tid; k < n; k += MC_THREADS) {
                D.xa[a0 + k] = nx[k];
                D.ya[a0 + k] = ny[k];
                D.za[a0 + k] = nz[k];
                D.pos[a0 + k] = mv[k];
            }
            if (tid == 0) {
                D.xadd[im] = sh_cx;
                D.yadd[im] = sh_cy;
                D.zadd[im] = sh_cz;
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        // step adaptation (molfit.py:465-536); nmovei counts only in the intramolecular cycle
        if (D.ireset != 1) {
            for (int t = 0; t < nmt; ++t) {
                float rat0;
                const int nm1 = D.nmovei ? D.nmovei[t] : 0, nm2 = D.nmovei ? D.nmovei[nmt + t] : 0;
                if (nm2 > 0) {
                    rat0 = __fdiv_rn(__fmul_rn(D.rejrate, (float)nm1), (float)nm2);
                    if (rat0 > 1.1f) rat0 = 1.1f;
                    if (rat0 < 0.9f) rat0 = 0.9f;
                } else {
                    rat0 = nm1 > 0 ? 1.1f : 1.0f;
                }
                float it = __fmul_rn(D.interntrans[t], rat0);
                if (it > D.trstepmax) it = D.trstepmax;
                if (it < D.trstepmin && it != 0.0f) it = D.trstepmin;
                D.interntrans[t] = it;
                float rat;
                const int ni1 = D.ninter ? D.ninter[t] : 0, ni2 = D.ninter ? D.ninter[nmt + t] : 0;
                if (ni2 > 0) {
                    rat = __fdiv_rn(__fmul_rn(D.rejrate, (float)ni1), (float)ni2);
                    if (rat > 1.1f) rat = 1.1f;
                    if (rat < 0.9f) rat = 0.9f;
                } else {
                    rat = ni1 > 0 ? 1.1f : 1.0f;
                }
                float ir = __fmul_rn(D.internrot[t], rat);
                if (ir > rotstepmax) ir = rotstepmax;
                if (ir < rotstepmin && ir != 0.0f) ir = rotstepmin;
                D.internrot[t] = ir;
                if (D.nwhole[nmt + t] > 0) {
                    rat = __fdiv_rn(__fmul_rn(D.rejrate, (float)D.nwhole[t]), (float)D.nwhole[nmt + t]);
                    if (rat > 1.1f) rat = 1.1f;
                    if (rat < 0.9f) rat = 0.9f;
                } else {
                    rat = D.nwhole[t] > 0 ? 1.1f : 1.0f;
                }
                float wr = __fmul_rn(D.wholerot[t], rat);
                if (wr > rotstepmax) wr = rotstepmax;
                if (wr < rotstepmin && wr != 0.0f) wr = rotstepmin;
                D.wholerot[t] = wr;
                if (D.nmovem[nmt + t] > 0) {
                    rat = __fdiv_rn(__fmul_rn(D.rejrate, (float)D.nmovem[t]), (float)D.nmovem[nmt + t]);
                    if (rat > 1.1f) rat = 1.1f;
                    if (rat < 0.9f) rat = 0.9f;
                } else {
                    rat = D.nmovem[t] > 0 ? 1.1f : 1.0f;
                }
                float wt = __fmul_rn(D.wholetrans[t], rat);
                if (wt > D.trstepmax) wt = D.trstepmax;
                if (wt < D.trstepmin && wt != 0.0f) wt = D.trstepmin;
                D.wholetrans[t] = wt;
            }
        }
        D.fadds[0] = __fadd_rn(D.fadds[0], __fdiv_rn(fadd, (float)D.nmol));
        if (D.faddbs) D.faddbs[0] = __fadd_rn(D.faddbs[0], __fdiv_rn(faddb, (float)D.nmol));
        ran1_store(R, D.ran1);
    }
    (void)sh_fdiff;
}

// en_change for one molecule at its current coordinates (no move)
__global__ void en_change_kernel(McDev D, int im, float *ergnew_out, float *fdiff_out) {
    __shared__ double red[MC_THREADS / 32];
    const int tid = threadIdx.x;
    const size_t row = (size_t)im * D.M;
    const int nn = D.nergpairm[im];
    const int a0 = D.naf[im], n = D.nato[im];
    for (int inn = 1 + tid; inn < nn; inn += blockDim.x) {
        const int jm = D.molergpair[row + inn];
        const int b0 = D.naf[jm], b1 = b0 + D.nato[jm];
        float sume = 0.0f;
        for (int ia = a0; ia < a0 + n; ++ia) {
            const float4 p1 = D.pos[ia];
            const int it = __float_as_int(p1.w);
            for (int ja = b0; ja < b1; ++ja) {
                const float4 p2 = D.pos[ja];
                sume = __fadd_rn(sume, pair_energy(D.L, D.T, p1, p2,
                                                   __ldg(D.npairref + it * D.ntype + __float_as_int(p2.w))));
            }
        }
        ergnew_out[inn] = __fadd_rn(0.0f, sume);
    }
    __syncthreads();
    if (tid == 0) {
        float f = 0.0f;
        for (int inn = 1; inn < nn; ++inn)
            f = __fsub_rn(__fadd_rn(f, ergnew_out[inn]), D.ergpair[D.ergpairref[row + inn] - 1]);
        *fdiff_out = f;
    }
    (void)red;
}

__global__ void en_mole_pair_kernel(McDev D, const int32_t *im, const int32_t *jm, int n, float *out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = im[k], j = jm[k];
    float sume = 0.0f;
    for (int ia = D.naf[i]; ia < D.naf[i] + D.nato[i]; ++ia) {
        const float4 p1 = D.pos[ia];
        const int it = __float_as_int(p1.w);
        for (int ja = D.naf[j]; ja < D.naf[j] + D.nato[j]; ++ja) {
            const float4 p2 = D.pos[ja];
            sume = __fadd_rn(sume, pair_energy(D.L, D.T, p1, p2, __ldg(D.npairref + it * D.ntype + __float_as_int(p2.w))));
        }
    }
    out[k] = sume;
}

McDev make_mcdev(const epsr_box_t *b, const epsr_cells_t *c, const epsr_store_t *s) {
    McDev D;
    memset(&D, 0, sizeof(D));
    D.L.cubic = b->cubic;
    D.L.alatx = b->lat[0];
    D.L.blatx = b->lat[1];
    D.L.clatx = b->lat[2];
    D.L.blaty = b->lat[3];
    D.L.claty = b->lat[4];
    D.L.clatz = b->lat[5];
    D.T.tab = (const float4 *)b->tab;
    D.T.xstar = b->xstar;
    D.T.ld = b->ld;
    D.T.npt2 = b->npt2;
    D.T.izcut = b->izcut < b->npt2 ? b->izcut : b->npt2;
    D.T.stepcl = b->stepcl;
    D.nmol = b->nmol;
    D.ntype = b->ntype;
    D.nmoltype = b->nmoltype;
    D.naf = b->naf;
    D.nato = b->nato;
    D.mtype = b->mtype;
    D.npairref = b->npairref;
    D.visit = c ? c->cell_mols : nullptr;
    D.xa = b->xa;
    D.ya = b->ya;
    D.za = b->za;
    D.xadd = b->xadd;
    D.yadd = b->yadd;
    D.zadd = b->zadd;
    D.pos = (float4 *)b->pos;
    if (s) {
        D.M = s->nnbrefmax;
        D.nergpairm = s->nergpairm;
        D.molergpair = s->molergpair;
        D.ergpairref = s->ergpairref;
        D.ergpair = s->ergpair;
    }
    return D;
}

}  // namespace epsr

using namespace epsr;

extern "C" int64_t epsr_molfit_spec_scratch_bytes(int32_t nmol, int32_t natom, int32_t M, int32_t nmoltype);

extern "C" int64_t epsr_molfit_scratch_bytes(int32_t nmol, int32_t natom, int32_t M) {
    // the sequential kernel needs 2*M floats when M is too large for shared memory; the fast
    // path needs its per-cycle buffers (up to 64 molecule types)
    const int64_t seq = (int64_t)sizeof(float) * 2 * (int64_t)(M > 0 ? M : 1) + 256;
    const int64_t spec = epsr_molfit_spec_scratch_bytes(nmol, natom, M, 64);
    return seq > spec ? seq : spec;
}

static int check_box(const epsr_box_t *b, const char *who) {
    if (!b || !b->naf || !b->nato || !b->itype || !b->pos || !b->tab || !b->xstar || !b->npairref) {
        epsr_set_error("%s: box has null pointers", who);
        return EPSR_ERR_ARG;
    }
    return EPSR_OK;
}

namespace epsr {
// The intramolecular cycle's settings when the sequential kernel runs it (shake mode).
struct ShakeRot {
    const epsr_intra_t *intra;
    float stepmi;
    int32_t *nmovei;
    float *faddbs;
};

static int seq_launch(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                      void *scratch, int64_t scratch_bytes, cudaStream_t s, const int32_t *run_if, const ShakeRot *sr);

int molfit_seq_launch(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                      void *scratch, int64_t scratch_bytes, cudaStream_t s, const int32_t *run_if) {
    return seq_launch(box, cells, store, mc, scratch, scratch_bytes, s, run_if, nullptr);
}

// molfit's intramolecular cycle (nisum >= intra) for a box whose molecules have rotational
// groups, on the sequential kernel: the rotations test the intermolecular change, which chains
// every molecule to the ones before it.  mc must carry the groups (rot_*), ninter and stepri.
int molfit_shake_rot_launch(const epsr_box_t *box, epsr_store_t *store, epsr_mc_t *mc, const epsr_intra_t *in,
                            float stepmi, int32_t *nmovei, float *faddbs, void *scratch, int64_t scratch_bytes,
                            cudaStream_t s) {
    const ShakeRot sr{in, stepmi, nmovei, faddbs};
    return seq_launch(box, nullptr, store, mc, scratch, scratch_bytes, s, nullptr, &sr);
}

static int seq_launch(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                      void *scratch, int64_t scratch_bytes, cudaStream_t s, const int32_t *run_if, const ShakeRot *sr) {
    McDev D = make_mcdev(box, cells, store);
    D.simt = mc->simt;
    D.rejrate = mc->rejrate;
    D.stepr = mc->stepr;
    D.stepm = mc->stepm;
    D.trstepmax = mc->trstepmax;
    D.trstepmin = mc->trstepmin;
    D.ireset = mc->ireset;
    D.strict = run_if ? 0 : mc->strict;
    D.wholerot = mc->wholerot;
    D.wholetrans = mc->wholetrans;
    D.internrot = mc->internrot;
    D.interntrans = mc->interntrans;
    D.nwhole = mc->nwhole;
    D.nmovem = mc->nmovem;
    D.nstepreject = mc->nstepreject;
    D.fadds = mc->fadds;
    D.ran1 = mc->ran1;
    D.cos_override = mc->cos_override;
    D.trace_den = mc->trace_den;
    D.trace_acc = mc->trace_acc;
    D.status = mc->status;
    D.run_if = run_if;
    D.faddbs = mc->faddbs;
    if (sr || mc->intra) {
        const epsr_intra_t *in = sr ? sr->intra : (const epsr_intra_t *)mc->intra;
        D.I = make_intradev(box, in);
        D.ngrot = in->ngrot;
        D.has_rot = mc->rot_nrf && mc->rot_nrl && mc->rot_axis && mc->rot_first && mc->rot_last && mc->rot_atoms;
        D.rot_nrf = mc->rot_nrf;
        D.rot_nrl = mc->rot_nrl;
        D.rot_axis = mc->rot_axis;
        D.rot_first = mc->rot_first;
        D.rot_last = mc->rot_last;
        D.rot_atoms = mc->rot_atoms;
        D.stepri = mc->stepri;
        D.rotcycle = mc->rotcycle;
        D.ninter = mc->ninter;
        if (D.has_rot && !D.ninter) {
            epsr_set_error("epsr_molfit: internal rotations need the ninter counters");
            return EPSR_ERR_ARG;
        }
    }
    if (sr) {
        if (!D.has_rot || !sr->nmovei) {
            epsr_set_error("epsr_molfit_shake: a box with rotational groups needs the groups (rot_*), ninter and nmovei");
            return EPSR_ERR_ARG;
        }
        D.shake = 1;
        D.strict = 1;
        D.stepmi = sr->stepmi;
        D.nmovei = sr->nmovei;
        D.faddbs = sr->faddbs;
        D.visit = nullptr;
    }
    const size_t need = sizeof(float) * 2 * (size_t)(D.M > 0 ? D.M : 1);
    size_t shm = 0;
    if (need <= 160 * 1024) {
        D.use_smem = 1;
        shm = need;
    } else {
        if (!scratch || scratch_bytes < (int64_t)need) {
            epsr_set_error("epsr_molfit: scratch needs %zu bytes", need);
            return EPSR_ERR_CAPACITY;
        }
        D.use_smem = 0;
        D.ergnew_g = (float *)scratch;
    }
    if (shm > 48 * 1024)
        EPSR_SMEM_OPTIN(molfit_seq_kernel);
    EPSR_TIMED("molfit_seq_kernel", s, molfit_seq_kernel<<<1, MC_THREADS, shm, s>>>(D));
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
}  // namespace epsr

int epsr_molfit_spec(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                     void *scratch, int64_t scratch_bytes, void *stream);

extern "C" int epsr_molfit(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                           void *scratch, int64_t scratch_bytes, void *stream) {
    int rc = check_box(box, "epsr_molfit");
    if (rc) return rc;
    if (!cells || !store || !mc || !mc->wholerot || !mc->wholetrans || !mc->nwhole || !mc->nmovem ||
        !mc->nstepreject || !mc->fadds || !mc->ran1 || !mc->internrot || !mc->interntrans) {
        epsr_set_error("epsr_molfit: null pointer");
        return EPSR_ERR_ARG;
    }
    // internal rotations (and the internrot rule that needs every molecule's ngrot) run in the
    // sequential kernel
    if (mc->strict || mc->intra)
        return molfit_seq_launch(box, cells, store, mc, scratch, scratch_bytes, (cudaStream_t)stream, nullptr);
    return epsr_molfit_spec(box, cells, store, mc, scratch, scratch_bytes, stream);
}

extern "C" int epsr_en_change(const epsr_box_t *box, const epsr_store_t *store, int32_t im, float *ergnew,
                              float *out_host, void *stream) {
    int rc = check_box(box, "epsr_en_change");
    if (rc) return rc;
    if (!store || !ergnew || !out_host || im < 0 || im >= box->nmol) {
        epsr_set_error("epsr_en_change: bad arguments");
        return EPSR_ERR_ARG;
    }
    McDev D = make_mcdev(box, nullptr, store);
    cudaStream_t s = (cudaStream_t)stream;
    en_change_kernel<<<1, 256, 0, s>>>(D, im, ergnew, ergnew);  // the total goes to slot 0
    EPSR_CUDA(cudaGetLastError());
    EPSR_D2H(out_host, ergnew, sizeof(float), s);
    return EPSR_OK;
}

extern "C" int epsr_en_mole_pair(const epsr_box_t *box, const int32_t *im, const int32_t *jm, int32_t n, float *out,
                                 void *stream) {
    int rc = check_box(box, "epsr_en_mole_pair");
    if (rc) return rc;
    if (!im || !jm || !out || n < 0) {
        epsr_set_error("epsr_en_mole_pair: bad arguments");
        return EPSR_ERR_ARG;
    }
    if (n == 0) return EPSR_OK;
    McDev D = make_mcdev(box, nullptr, nullptr);
    en_mole_pair_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(D, im, jm, n, out);
    EPSR_CUDA(cudaGetLastError());
    return EPSR_OK;
}
