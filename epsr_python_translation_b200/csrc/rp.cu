// rp.cu -- the reference potential tables: generate_mp (ato_manipulation_rev4.py:2816-2902, the
// WCA core of intramolecular pairs, xav/xav1) and generate_rp (epsr_standalone_rev3.py:5675-5873:
// n-6 Lennard-Jones + charged-sphere Coulomb (chsph ato_manipulation_rev4.py:589, sum1/sum2),
// Gaussians or the modified Morse of gauss6pot (:562), the repulsive core, and the forward-
// difference gradients), host functions.
//
// These tables are built once per run and again whenever the reference potential changes
// (a few hundred points per atom pair, a handful of single-precision transcendentals each);
// they are built on the host with the C library's logf/expf/sinhf/powf -- the functions the
// reference calls -- so the tables are bit-identical, and the caller uploads them with the
// other tables (epsr_pack_tables builds the energy kernels' packed form on the device).
#include <math.h>
#include <string.h>

#include "common.cuh"

namespace {

// sum1 / sum2 ato_manipulation_rev4.py: the overlapping-sphere integral in two parts.
float rp_sum1(float r, float a, float b, float aup, float alo) {
    float cof[7];
    const float a2 = a * a, b2 = b * b, r2 = r * r;
    cof[6] = 1.0f / 6.0f;
    cof[5] = 3.0f * r / 5.0f;
    cof[4] = -(3.0f * (a2 - r2) + b2) / 4.0f;
    cof[3] = -r * (3.0f * (a2 + b2) - r2) / 3.0f;
    cof[2] = 3.0f * b2 * (a2 - r2) / 2.0f;
    cof[1] = r * b2 * (3.0f * a2 - r2);
    const float fac = 3.0f / (8.0f * a2 * a * b2 * b * r);
    float sumu = 0.0f, suml = 0.0f;
    for (int i = 1; i <= 6; ++i) {
        const int ir = 7 - i;
        sumu = aup * (sumu + cof[ir]);
        suml = alo * (suml + cof[ir]);
    }
    return fac * (sumu - suml);
}

float rp_sum2(float r, float b, float aup, float alo) {
    float cof[4];
    const float b2 = b * b;
    cof[3] = -1.0f / 3.0f;
    cof[2] = 0.0f;
    cof[1] = b2;
    const float fac = 3.0f / (4.0f * r * b2 * b);
    float sumu = 0.0f, suml = 0.0f;
    for (int i = 1; i <= 3; ++i) {
        const int ir = 4 - i;
        sumu = aup * (sumu + cof[ir]);
        suml = alo * (suml + cof[ir]);
    }
    return fac * (sumu - suml);
}

// chsph: Coulomb interaction of two uniformly charged spheres of radii sig1, sig2 at r.
float rp_chsph(float sig1, float sig2, float r) {
    float ra = sig1, rb = sig2;
    if (sig2 > sig1) {
        ra = sig2;
        rb = sig1;
    }
    if (r >= ra + rb) return 1.0f / r;
    if (r <= ra - rb) return ra > 0.0f ? (3.0f * (ra * ra - 0.2f * rb * rb) - r * r) / (2.0f * ra * ra * ra) : 1.0e20f;
    return rp_sum1(r, ra, rb, ra - r, -rb) + rp_sum2(r, rb, +rb, ra - r);
}

// gauss6pot: a Gaussian core minus an r**-6 term from the overlapping-sphere Coulomb function
// (coul**6 as (c*c*c)*(c*c*c)); sigg clipped to 0.29.
float rp_gauss6pot(float r, float sig, float sigg) {
    const float x = r / sig;
    const float coul = rp_chsph(0.5f, 0.5f, x);
    const float c3 = coul * coul * coul;
    const float london = -(c3 * c3);
    if (sigg > 0.29f) sigg = 0.29f;
    const float ampgln = 0.5f / (sigg * sigg);
    float arg = x / sigg;
    arg = 0.5f * arg * arg - ampgln;
    const float term = arg < 30.0f ? expf(-arg) : 0.0f;
    return term + london;
}

// The n-6 Lennard-Jones of generate_mp/generate_rp: 2 fac sinh(pwr2) exp(pwr1).
float rp_lj(float power, float fac, float ddif) {
    const float xx = logf(ddif);
    float pwr1 = 0.5f * (power + 6.0f) * xx;
    if (fabsf(pwr1) > 20.0f) pwr1 = copysignf(20.0f, pwr1);
    float pwr2 = 0.5f * (power - 6.0f) * xx;
    if (fabsf(pwr2) > 40.0f) pwr2 = copysignf(40.0f, pwr2);
    return 2.0f * fac * sinhf(pwr2) * expf(pwr1);
}

// Forward differences on xstar (j = 2..npt into j-1), the last point 0.
void rp_slopes(const float *t, const float *xstar, int npt, float *t1) {
    float s1 = t[1], x1 = xstar[1];
    for (int j = 2; j <= npt; ++j) {
        const float x2 = xstar[j], s2 = t[j];
        t1[j - 1] = (s2 - s1) / (x2 - x1);
        x1 = x2;
        s1 = s2;
    }
}

}  // namespace

extern "C" int epsr_generate_rp(const epsr_rp_t *p) {
    if (!p || p->npairs < 1 || p->npt < 3 || p->npt2 < 1 || p->npt2 > p->npt || p->ld < p->npt + 1 || !p->x ||
        !p->xstar || !p->wfac || !p->wfacc || !p->n1extr || !p->n2extr || !p->irefpcof || !p->qradius || !p->ecor ||
        !p->qcor || !p->dcor || !p->coulfac || !p->pcoefex || !p->rminex || !p->npgauss || (p->maxgauss > 0 &&
        (!p->wpgauss || !p->rpgauss || !p->hpgauss)) || !p->epot || !p->epot1 || !p->ecoul || !p->ecoul1 ||
        !p->xav || !p->xav1 || !(p->power > 6.0f)) {
        epsr_set_error("epsr_generate_rp: bad arguments");
        return EPSR_ERR_ARG;
    }
    const int npt = p->npt, npt2 = p->npt2;
    const float *x = p->x, *xstar = p->xstar, power = p->power;
    // the prefactor of the well depth (generate_mp :2845-2851 = generate_rp :5721-5727)
    const float rat = 6.0f / power;
    const float rat1 = sqrtf(rat);
    const float rat2 = 1.0f / rat1;
    const float power1 = (power + 6.0f) / (power - 6.0f);
    const float rat3 = powf(rat1, power1);
    const float prefac = 1.0f / ((rat2 - rat1) * rat3);
    // generate_mp: the WCA core of every pair (the same for all pairs)
    const float rat4 = 1.0f / (power - 6.0f);
    const float dcm = p->dcore / p->sizefactor;
    const float rmaxwca = dcm * powf(power / 6.0f, rat4);
    // generate_rp's limit on the repulsive gradient
    float gradlimit = p->expecfpwr, loggradlimit = 0.0f;
    if (gradlimit > 0.0f) loggradlimit = logf(gradlimit);
    else gradlimit = 0.0f;
    for (int ic = 0; ic < p->npairs; ++ic) {
        const size_t row = (size_t)ic * p->ld;
        float *xav = p->xav + row, *xav1 = p->xav1 + row, *epot = p->epot + row, *epot1 = p->epot1 + row;
        float *ecoul = p->ecoul + row, *ecoul1 = p->ecoul1 + row;
        // ---- generate_mp (:2866-2896)
        for (int j = 2; j <= npt; ++j) {
            const float x2 = x[j];
            const float ddif = dcm / x2;
            float s = 0.0f;
            if (ddif > 0.0f && p->ecore > 0.0f && x2 < rmaxwca) s = rp_lj(power, prefac * p->ecore, ddif) + p->ecore;
            xav[j] = s * p->wfac[j];
        }
        xav[1] = xav[2];
        rp_slopes(xav, xstar, npt, xav1);
        xav1[npt] = 0.0f;
    }
    for (int ic = 0; ic < p->npairs; ++ic) {
        const size_t row = (size_t)ic * p->ld;
        float *xav = p->xav + row, *xav1 = p->xav1 + row, *epot = p->epot + row, *epot1 = p->epot1 + row;
        float *ecoul = p->ecoul + row, *ecoul1 = p->ecoul1 + row;
        const int k = p->irefpcof[ic];
        const float ra = p->qradius[p->n1extr[ic]], rb = p->qradius[p->n2extr[ic]];
        const float ect = p->ecor[ic], qct = p->qcor[ic] * p->coulfac[k], dc = p->dcor[ic];
        // ---- Lennard-Jones + Coulomb, Gaussians (:5741-5800)
        for (int j = 2; j <= npt; ++j) {
            const float x2 = x[j];
            const float ddif = dc / x2;
            float sumlj = (ddif > 0.0f && ect > 0.0f) ? rp_lj(power, prefac * ect, ddif) : 0.0f;
            float sumc = qct * rp_chsph(ra, rb, x2);
            sumlj = p->refpotfac * sumlj * p->wfac[j];
            sumc = p->refpotfac * sumc * p->wfacc[j];
            epot[j] = sumlj + sumc;
            ecoul[j] = sumlj + sumc;
            for (int ig = 0; ig < p->npgauss[k] && ig < p->maxgauss; ++ig) {
                const size_t g = (size_t)k * p->maxgauss + ig;
                const float wpg = fabsf(p->wpgauss[g]);
                if (wpg > 0.0f) {
                    const float rpg = fabsf(p->rpgauss[g]), hpg = p->hpgauss[g];
                    float add = 0.0f;
                    if (ig == 0 && p->modmorse) {
                        add = fabsf(hpg) * rp_gauss6pot(x[j], rpg, wpg);
                    } else {
                        const float rdiff = (x[j] - rpg) / wpg;
                        const float term = logf(fabsf(hpg)) - 0.5f * rdiff * rdiff;
                        if (fabsf(term) < 25.0f) add = copysignf(1.0f, hpg) * expf(term);
                    }
                    ecoul[j] = ecoul[j] + add * p->wfac[j];
                }
            }
            if (p->coul_intra) xav[j] = p->coul_intra_fac * ecoul[j];
        }
        // ---- the repulsive core (:5805-5833)
        if (fabsf(p->pcoefex[k]) > 0.0f && fabsf(p->rminex[k]) > 0.0f) {
            const float expecfuse = p->expecf * sqrtf(fabsf(p->rminex[k]));
            if (!p->harmonic) {
                const float rminextest = fabsf(p->rminex[k]);
                for (int j = 1; j <= npt2; ++j) {
                    const float dd = (rminextest - x[j]) / expecfuse;
                    const float add = (gradlimit > 0.0f && dd >= loggradlimit)
                                          ? p->pcoefex[k] * gradlimit * (1.0f + dd - loggradlimit)
                                          : p->pcoefex[k] * expf(dd);
                    ecoul[j] = ecoul[j] + add * p->wfac[j];
                }
            } else {
                const float rminextest = fabsf(p->rminex[k]) + expecfuse;
                for (int j = 1; j <= npt2; ++j) {
                    const float dd = (rminextest - x[j]) / expecfuse;
                    if (dd > 0.0f) {
                        const float add = (gradlimit > 0.0f && dd >= gradlimit)
                                              ? 0.5f * p->pcoefex[k] * gradlimit * (2.0f * dd - gradlimit)
                                              : 0.5f * p->pcoefex[k] * dd * dd;
                        ecoul[j] = ecoul[j] + add * p->wfac[j];
                    }
                }
            }
        }
        epot[1] = epot[2];
        ecoul[1] = ecoul[2];
        xav[1] = xav[2];
        // ---- gradients (:5837-5858)
        rp_slopes(epot, xstar, npt, epot1);
        rp_slopes(ecoul, xstar, npt, ecoul1);
        rp_slopes(xav, xstar, npt, xav1);
        epot1[npt] = 0.0f;
        ecoul1[npt] = 0.0f;
        xav[npt] = 0.0f;   // xav, not xav1, as the reference
    }
    return EPSR_OK;
}
