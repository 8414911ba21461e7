// intra.cuh -- the intramolecular energy of a molecule on the device (en_mole_intra
// molfit.py:1327-1350 -> en_atom_intra :923-1045): bonds and bond-angle pairs as harmonic
// terms, the intramolecular reference potential xav for the other pairs, image atoms, q-type
// atoms and refine_intra's EP term.  Shared by the intramolecular cycle (shake.cu) and the
// internal rotations of the whole-molecule cycle (mc.cu).
#pragma once

#include <string.h>

#include "common.cuh"

namespace epsr {

struct IntraDev {
    Lattice L;
    const int32_t *naf, *nato, *mtype, *itype, *npairref, *ngrot;
    const int32_t *nbond, *iabond, *imageatom, *qtype;
    const float *tbond, *amassa, *amassr, *xav, *xav1, *xstar;
    const float4 *tab;
    int32_t maxbond, ld, npt2, ntype, natom, refine_intra;
    float stepcl, sizefactor, tempb, tempang, simt, refine_intra_fac;
    // dihedral angles of the rotational groups (grp_nrf NULL: none)
    const int32_t *grp_nrf, *grp_nrl, *grp_axis, *grp_dih0, *grp_isdih, *dih_atoms;
    const float *dih_cos, *dih_sin;
    float tempdih;
};

static inline IntraDev make_intradev(const epsr_box_t *b, const epsr_intra_t *in) {
    IntraDev I;
    memset(&I, 0, sizeof(I));
    I.L.cubic = b->cubic;
    I.L.alatx = b->lat[0];
    I.L.blatx = b->lat[1];
    I.L.clatx = b->lat[2];
    I.L.blaty = b->lat[3];
    I.L.claty = b->lat[4];
    I.L.clatz = b->lat[5];
    I.naf = b->naf;
    I.nato = b->nato;
    I.mtype = b->mtype;
    I.itype = b->itype;
    I.npairref = b->npairref;
    I.ngrot = in->ngrot;
    I.nbond = in->nbond;
    I.iabond = in->iabond;
    I.imageatom = in->imageatom;
    I.qtype = in->qtype;
    I.tbond = in->tbond;
    I.amassa = in->amassa;
    I.amassr = in->amassr;
    I.xav = in->xav;
    I.xav1 = in->xav1;
    I.xstar = b->xstar;
    I.tab = (const float4 *)b->tab;
    I.maxbond = in->maxbond;
    I.ld = b->ld;
    I.npt2 = b->npt2;
    I.ntype = b->ntype;
    I.natom = b->natom;
    I.refine_intra = in->refine_intra;
    I.stepcl = in->stepcl;
    I.sizefactor = in->sizefactor;
    I.tempb = in->tempb;
    I.tempang = in->tempang;
    I.simt = in->simt;
    I.refine_intra_fac = in->refine_intra_fac;
    if (in->grp_nrf && in->grp_nrl && in->grp_axis && in->grp_dih0 && in->grp_isdih) {
        I.grp_nrf = in->grp_nrf;
        I.grp_nrl = in->grp_nrl;
        I.grp_axis = in->grp_axis;
        I.grp_dih0 = in->grp_dih0;
        I.grp_isdih = in->grp_isdih;
        I.dih_atoms = in->dih_atoms;
        I.dih_cos = in->dih_cos;
        I.dih_sin = in->dih_sin;
        I.tempdih = in->tempdih;
    }
    return I;
}

// The bond of atom `a` to atom `ja` (first in a's list), or -1.
__device__ __forceinline__ int find_bond(const IntraDev &I, int a, int ja) {
    const int nb = min(I.nbond[a], I.maxbond);
    for (int k = 0; k < nb; ++k)
        if (I.iabond[(size_t)a * I.maxbond + k] == ja) return k;
    return -1;
}

// The EP term refine_intra adds (molfit.py:993-996 / :1037-1040).
__device__ __forceinline__ float ep_term(const IntraDev &I, int iz, int icref, float dtdif) {
    const float4 t = I.tab[(size_t)icref * I.ld + iz];
    return __fmul_rn(I.refine_intra_fac, __fadd_rn(t.x, __fmul_rn(t.y, dtdif)));
}

// en_atom_intra :999-1016: is (ia, ja) one of the dihedral atom pairs of molecule im's groups?
__device__ __forceinline__ bool dihedral_pair_d(const IntraDev &I, int im, int ia, int ja) {
    if (!I.grp_nrf) return false;
    for (int ir = I.grp_nrf[im]; ir <= I.grp_nrl[im]; ++ir)
        for (int kd = I.grp_dih0[ir]; kd < I.grp_dih0[ir + 1]; ++kd) {
            const int io1 = I.dih_atoms[2 * kd], io2 = I.dih_atoms[2 * kd + 1];
            if ((io1 == ia && io2 == ja) || (io1 == ja && io2 == ia)) return true;
        }
    return false;
}

// vecpro, scapro auxiliary_routines.py:231-244 in the reference's order
__device__ __forceinline__ void vecpro_d(const float *a, const float *b, float *c) {
    c[0] = __fsub_rn(__fmul_rn(a[1], b[2]), __fmul_rn(a[2], b[1]));
    c[1] = __fsub_rn(__fmul_rn(a[2], b[0]), __fmul_rn(a[0], b[2]));
    c[2] = __fsub_rn(__fmul_rn(a[0], b[1]), __fmul_rn(a[1], b[0]));
}
__device__ __forceinline__ float scapro_d(const float *a, const float *b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
}

// en_dihedral molfit.py:1487-1524 with the angle's cosine and sine given
__device__ __forceinline__ float en_dihedral_d(const float *co1, const float *co2, const float *cd, float cosdih,
                                               float sindih) {
    float cv1[3], cv2[3], cpar[3];
    vecpro_d(co1, cd, cv1);
    vecpro_d(co2, cd, cv2);
    float dmag = __fsqrt_rn(scapro_d(cv1, cv1));
    for (int i = 0; i < 3; ++i) cv1[i] = __fdiv_rn(cv1[i], dmag);
    dmag = __fsqrt_rn(scapro_d(cv2, cv2));
    for (int i = 0; i < 3; ++i) cv2[i] = __fdiv_rn(cv2[i], dmag);
    float cosphi = scapro_d(cv1, cv2);
    if (cosphi > 1.0f) cosphi = 1.0f;
    if (cosphi < -1.0f) cosphi = -1.0f;
    vecpro_d(cv1, cv2, cpar);
    const float sinphi = scapro_d(cpar, cd);
    const float difc = __fsub_rn(cosdih, cosphi), difs = __fsub_rn(sindih, sinphi);
    return __fadd_rn(__fmul_rn(difc, difc), __fmul_rn(difs, difs));
}

// en_mole_dihedral molfit.py:1353-1410: the DIH groups of molecule im on the offsets x/y/z
static __device__ float en_mole_dihedral_d(const IntraDev &I, int im, const float *x, const float *y, const float *z) {
    float e = 0.0f;
    if (!I.grp_nrf) return e;
    for (int ir = I.grp_nrf[im]; ir <= I.grp_nrl[im]; ++ir) {
        if (!I.grp_isdih[ir]) continue;
        const int ia1 = I.grp_axis[2 * ir], ia2 = I.grp_axis[2 * ir + 1];
        const float x1 = x[ia1], y1 = y[ia1], z1 = z[ia1], x2 = x[ia2], y2 = y[ia2], z2 = z[ia2];
        float cd[3] = {__fsub_rn(x2, x1), __fsub_rn(y2, y1), __fsub_rn(z2, z1)};
        const float dmag = __fsqrt_rn(scapro_d(cd, cd));
        for (int i = 0; i < 3; ++i) cd[i] = __fdiv_rn(cd[i], dmag);
        for (int kd = I.grp_dih0[ir]; kd < I.grp_dih0[ir + 1]; ++kd) {
            const int io1 = I.dih_atoms[2 * kd], io2 = I.dih_atoms[2 * kd + 1];
            const float co1[3] = {__fsub_rn(x[io1], x1), __fsub_rn(y[io1], y1), __fsub_rn(z[io1], z1)};
            const float co2[3] = {__fsub_rn(x[io2], x2), __fsub_rn(y[io2], y2), __fsub_rn(z[io2], z2)};
            e = __fadd_rn(e, en_dihedral_d(co1, co2, cd, I.dih_cos[kd], I.dih_sin[kd]));
        }
    }
    return e;
}

// The dihedral part en_mole_intra adds after its atom pairs (:1345-1348), or +0 when none.
__device__ __forceinline__ bool has_dihedral_term(const IntraDev &I, int im) {
    return I.tempdih > 0.0f && I.ngrot && I.ngrot[im] > 0;
}
__device__ __forceinline__ float dihedral_term_d(const IntraDev &I, int im, const float *x, const float *y,
                                                 const float *z) {
    return __fmul_rn(__fmul_rn(I.tempdih, I.simt), en_mole_dihedral_d(I, im, x, y, z));
}

// en_atom_intra molfit.py:923-1045 for atoms ia, ja (0-based) of molecule im.
static __device__ float en_atom_intra_d(const IntraDev &I, int im, int ia, int ja, float x1, float y1, float z1,
                                        float x2, float y2, float z2) {
    if (ja == I.imageatom[ia]) return 0.0f;
    const int icref = I.npairref[I.itype[ia] * I.ntype + I.itype[ja]];
    const bool notq = I.qtype[ia] == 0 && I.qtype[ja] == 0;
    const float xdifs = __fsub_rn(x2, x1), ydifs = __fsub_rn(y2, y1), zdifs = __fsub_rn(z2, z1);
    int image = ia, jref = find_bond(I, ia, ja);
    if (jref < 0) {
        image = I.imageatom[ia];
        jref = (image >= 0 && image < I.natom) ? find_bond(I, image, ja) : -1;
    }
    if (jref >= 0) {
        float xd = xdifs, yd = ydifs, zd = zdifs;
        minimagec(I.L, xd, yd, zd);
        const float dsq = __fadd_rn(__fadd_rn(__fmul_rn(xd, xd), __fmul_rn(yd, yd)), __fmul_rn(zd, zd));
        const float dtest = __fsqrt_rn(dsq);
        const int iz = ifix(__fdiv_rn(dtest, I.stepcl)) + 2;
        const float tbv = I.tbond[(size_t)image * I.maxbond + jref];
        const float atb = fabsf(tbv);
        const float tb = atb > I.stepcl ? atb : I.stepcl;      // max(stepcl, |tbond|)
        float wtm = __fdiv_rn(I.amassr[icref], tb);
        if (tbv < 0.0f) wtm = __fmul_rn(wtm, I.tempang);
        const float ddif = __fsub_rn(tb, dtest);
        float sume = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(wtm, ddif), ddif), I.tempb), I.simt);
        if (I.refine_intra && iz <= I.npt2 && notq) sume = __fadd_rn(sume, ep_term(I, iz, icref, __fsub_rn(dtest, I.xstar[iz])));
        return sume;
    }
    if (dihedral_pair_d(I, im, ia, ja)) return 0.0f;   // a dihedral's pair: its energy is the dihedral term
    float xd = __fmul_rn(xdifs, I.sizefactor), yd = __fmul_rn(ydifs, I.sizefactor), zd = __fmul_rn(zdifs, I.sizefactor);
    minimagec(I.L, xd, yd, zd);
    const float dsq = __fadd_rn(__fadd_rn(__fmul_rn(xd, xd), __fmul_rn(yd, yd)), __fmul_rn(zd, zd));
    const float dtest = __fsqrt_rn(dsq);
    const int iz = ifix(__fdiv_rn(dtest, I.stepcl)) + 2;
    float sume = 0.0f;
    if (iz <= I.npt2) {
        const float dtdif = __fsub_rn(dtest, I.xstar[iz]);
        const size_t k = (size_t)icref * I.ld + iz;
        sume = __fadd_rn(I.xav[k], __fmul_rn(I.xav1[k], dtdif));
        if (I.refine_intra && notq) sume = __fadd_rn(sume, ep_term(I, iz, icref, dtdif));
    }
    return sume;
}

// en_mole_intra molfit.py:1327-1350 on the coordinates x/y/z (indexed by global atom).
static __device__ float en_mole_intra_d(const IntraDev &I, int im, const float *x, const float *y, const float *z) {
    const int a0 = I.naf[im], n = I.nato[im];
    float e = 0.0f;
    for (int i = 0; i < n - 1; ++i) {
        const int ia = a0 + i;
        const float x1 = x[ia], y1 = y[ia], z1 = z[ia];
        for (int j = i + 1; j < n; ++j) {
            const int ja = a0 + j;
            e = __fadd_rn(e, en_atom_intra_d(I, im, ia, ja, x1, y1, z1, x[ja], y[ja], z[ja]));
        }
    }
    if (has_dihedral_term(I, im)) e = __fadd_rn(e, dihedral_term_d(I, im, x, y, z));
    return e;
}

}  // namespace epsr
