/*
 * epsr_oracle.c -- CPU restatement of the EPSR minimum-image pair path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the device path is compared with; it is
 * never linked into, called by or shipped with the product library.  Only the tests, the
 * smoke check and the CPU-baseline leg of the benchmark load it.
 *
 * Each routine restates the reference translation (IzzyRodger-edb/EPSR_python_translation,
 * package src/epsr26) statement by statement in float32, with the same operation order.
 * The reference evaluates every `real` as a NumPy float32 scalar with no fused
 * multiply-add and calls glibc libm (expf/sinf/cosf/powf) through ctypes; this file is
 * compiled with -ffp-contract=off and calls the same glibc functions, so on the same
 * machine its results are bit-identical to the reference's.  Parity is pinned by the
 * golden vectors under tests/golden, produced by running the reference itself.
 *
 * Indexing: molecules, atoms, types and pairs are 0-based; the r-grid index iz and the
 * Q index keep the reference's 1-based meaning (tables are stored [pair][ld] with iz in
 * 1..npt, element 0 unused), because the bin arithmetic `ifix(d/stepcl)+2` depends on it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ Fortran intrinsics */

/* nint: round half away from zero (fortran/fmath.py:222-236, gfortran lroundf). */
static inline int32_t f_nint(float x) {
    if (!(x >= -2147483648.0f && x < 2147483648.0f)) return 0;
    double t = trunc((double)x);
    double fr = (double)x - t;
    if (fr >= 0.5) t += 1.0;
    else if (fr <= -0.5) t -= 1.0;
    return (int32_t)(int64_t)t;
}

/* ifix: truncation toward zero; out of range -> INT_MIN (fortran/fmath.py:245-253). */
static inline int32_t f_ifix(float x) {
    if (!(x > -2147483649.0f && x < 2147483648.0f)) return INT32_MIN;
    return (int32_t)x;
}

/* sign(a,b) for reals: |a| with the sign of b (fortran/fmath.py:284). */
static inline float f_sign(float a, float b) { return copysignf(fabsf(a), b); }

/* ------------------------------------------------------------------ ran1 */
/* auxiliary_routines.py:324-391; constants common/ran1com.py:13-21. */
typedef struct {
    int32_t idum, iy, mcall;
    int32_t iv[32];
} oracle_ran1_state;

#define R_IA 16807
#define R_IM 2147483647
#define R_IQ 127773
#define R_IR 2836
#define R_NTAB 32
#define R_NDIV 67108864

float oracle_ran1(oracle_ran1_state *s) {
    const float am = 4.656612873077393e-10f;   /* f32(1/IM) */
    const float rnmx = 0.9999998807907104f;    /* f32(1 - 1.2e-7) */
    int32_t idum = s->idum, iy = s->iy;
    if (idum <= 0 || iy == 0) {
        int64_t neg = -(int64_t)idum;
        int32_t w = (int32_t)(uint32_t)(uint64_t)neg;   /* wrap32 */
        idum = w > 1 ? w : 1;
        for (int j = R_NTAB + 8; j >= 1; --j) {
            int32_t k = idum / R_IQ;
            idum = R_IA * (idum - k * R_IQ) - R_IR * k;
            if (idum < 0) idum += R_IM;
            if (j <= R_NTAB) s->iv[j - 1] = idum;
        }
        iy = s->iv[0];
    }
    int32_t k = idum / R_IQ;
    idum = R_IA * (idum - k * R_IQ) - R_IR * k;
    if (idum < 0) idum += R_IM;
    int32_t j = iy / R_NDIV;                /* 0-based slot (1 + iy/NDIV in 1-based) */
    iy = s->iv[j];
    s->iv[j] = idum;
    float r = am * (float)iy;
    if (rnmx < r) r = rnmx;
    s->idum = idum;
    s->iy = iy;
    s->mcall = (int32_t)((uint32_t)s->mcall + 1u);
    return r;
}

void oracle_ran1_fill(oracle_ran1_state *s, float *out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) out[i] = oracle_ran1(s);
}

/* ------------------------------------------------------------------ system description */
typedef struct {
    int32_t nmol, natom, ntype, npairs, nmoltype;
    const int32_t *naf, *nato, *mtype, *itype; /* 0-based */
    float *xa, *ya, *za;                       /* atom offsets (box units) */
    float *xadd, *yadd, *zadd;                 /* molecule centres (box units) */
    const int32_t *npairref;                   /* [ntype*ntype] 0-based pair index */
    const float *xstar;                        /* [ld], 1-based */
    const float *xavs, *xavs1, *ecoul, *ecoul1;/* [npairs*ld] */
    int32_t ld, npt2;
    float stepcl;
    int32_t cubic;
    float lat[6]; /* alatx, blatx, clatx, blaty, claty, clatz (box units) */
} oracle_sys;

/* minimagec.py:13-62 */
static inline void minimagec(const oracle_sys *S, float *x, float *y, float *z) {
    if (S->cubic) {
        *z = *z - (float)f_nint(*z);
        *y = *y - (float)f_nint(*y);
        *x = *x - (float)f_nint(*x);
        return;
    }
    const float alatx = S->lat[0], blatx = S->lat[1], clatx = S->lat[2];
    const float blaty = S->lat[3], claty = S->lat[4], clatz = S->lat[5];
    float fc = *z / clatz;
    float fb = (*y - fc * claty) / blaty;
    float fa = (*x - fb * blatx - fc * clatx) / alatx;
    fc = fc - (float)f_nint(fc);
    fb = fb - (float)f_nint(fb);
    fa = fa - (float)f_nint(fa);
    *z = fc * clatz;
    *y = fb * blaty + fc * claty;
    *x = fa * alatx + fb * blatx + fc * clatx;
}

/* en_atom_inter_scale molfit.py:1251-1279 with scalefac = 1 (no coarse graining). */
static inline float en_atom_inter(const oracle_sys *S, float x1, float y1, float z1, float x2, float y2,
                                  float z2, int icref) {
    float sume = 0.0f;
    float xd = x2 - x1, yd = y2 - y1, zd = z2 - z1;
    minimagec(S, &xd, &yd, &zd);
    float dsq = xd * xd + yd * yd + zd * zd;
    float dtest = sqrtf(dsq);
    float rat = dtest / S->stepcl;
    int32_t iz = f_ifix(rat) + 2;
    const size_t base = (size_t)icref * (size_t)S->ld;
    if (iz <= S->npt2) {
        float dtdif = dtest - S->xstar[iz];
        sume = S->xavs[base + iz] + S->xavs1[base + iz] * dtdif;
    }
    dtest = dtest * 1.0f;
    rat = dtest / S->stepcl;
    iz = f_ifix(rat) + 2;
    if (iz <= S->npt2) {
        float dtdif = dtest - S->xstar[iz];
        sume = sume + S->ecoul[base + iz] + S->ecoul1[base + iz] * dtdif;
    }
    return sume;
}

/* en_mole_pair molfit.py:1528-1578 (no tethering, no coordination constraints). */
float oracle_en_mole_pair(const oracle_sys *S, int im, int jm) {
    float sume = 0.0f;
    const int a0 = S->naf[im], a1 = a0 + S->nato[im];
    const int b0 = S->naf[jm], b1 = b0 + S->nato[jm];
    for (int ia = a0; ia < a1; ++ia) {
        const int it = S->itype[ia];
        const float x1 = S->xa[ia] + S->xadd[im];
        const float y1 = S->ya[ia] + S->yadd[im];
        const float z1 = S->za[ia] + S->zadd[im];
        for (int ja = b0; ja < b1; ++ja) {
            const int icref = S->npairref[it * S->ntype + S->itype[ja]];
            const float x2 = S->xa[ja] + S->xadd[jm];
            const float y2 = S->ya[ja] + S->yadd[jm];
            const float z2 = S->za[ja] + S->zadd[jm];
            sume = sume + en_atom_inter(S, x1, y1, z1, x2, y2, z2, icref);
        }
    }
    return sume;
}

/* ------------------------------------------------------------------ cell list */
/* cellneighbourlist.py:23-90 (initialise), :97-183 (makecellneighbourlist),
 * :266-305 (findperiodiccell, cellcoord, atomcellno). Lattice in box units. */
typedef struct {
    int32_t ncelldiva, ncelldivb, ncelldivc, ncell, ncellneighb, maxcellno;
    int32_t *molcellno;   /* [nmol] 1-based cell number */
    int32_t *cell_start;  /* [ncell+1] CSR offsets (0-based cell index) */
    int32_t *cell_mols;   /* [nmol] molecules (0-based) in reference order */
    int32_t *ia_off, *ib_off, *ic_off; /* [ncellneighb] */
} oracle_cells;

static int cellcoord(float x, int ncelldiv) {
    float x1 = x - (float)f_nint(x);
    int ix = f_ifix((x1 + 0.5f) * (float)ncelldiv);
    while (ix < 0) ix += ncelldiv;
    while (ix >= ncelldiv) ix -= ncelldiv;
    return ix;
}

static int atomcellno(const float *lat, int na, int nb, int nc, float x, float y, float z) {
    const float alatx = lat[0], blatx = lat[1], clatx = lat[2];
    const float blaty = lat[3], claty = lat[4], clatz = lat[5];
    float fc = z / clatz;
    float fb = (y - fc * claty) / blaty;
    float fa = (x - fb * blatx - fc * clatx) / alatx;
    int ia = cellcoord(fa, na), ib = cellcoord(fb, nb), ic = cellcoord(fc, nc);
    return 1 + ia + na * (ib + nb * ic);
}

/* First pass: sizes.  Writes ncelldiv*, ncell.  Returns 0. */
int oracle_cell_dims(int nmolcellin, int nmol, const float *lat, int32_t *dims /* [4] */) {
    int nmolcell = nmolcellin > nmol ? nmol : nmolcellin;
    /* ncelldiv = nint(powf(f32(nmol)/f32(nmolcell), 1/3)) */
    float ratio = (float)nmol / (float)nmolcell;
    int ncelldiv = f_nint(powf(ratio, 1.0f / 3.0f));
    if (ncelldiv < 1) ncelldiv = 1;
    float mn = lat[0];
    if (lat[3] < mn) mn = lat[3];
    if (lat[5] < mn) mn = lat[5];
    /* Python min(alatx, blaty, clatz) returns the first minimal value */
    float cellsize = 2.0f * mn / (float)ncelldiv;
    dims[0] = 2 * f_ifix(lat[0] / cellsize) + 1;
    dims[1] = 2 * f_ifix(lat[3] / cellsize) + 1;
    dims[2] = 2 * f_ifix(lat[5] / cellsize) + 1;
    dims[3] = dims[0] * dims[1] * dims[2];
    return 0;
}

/* Second pass.  lat9 = alatc[3], blatc[3], clatc[3]. Offsets arrays must hold ncell. */
int oracle_cell_list(int nmolcellin, const float *xadd, const float *yadd, const float *zadd, int nmol,
                     float rmax, const float *lat, const float *lat9, oracle_cells *C) {
    int32_t dims[4];
    oracle_cell_dims(nmolcellin, nmol, lat, dims);
    C->ncelldiva = dims[0];
    C->ncelldivb = dims[1];
    C->ncelldivc = dims[2];
    C->ncell = dims[3];
    const int ncell = C->ncell;
    int32_t *count = (int32_t *)calloc((size_t)ncell, sizeof(int32_t));
    int maxc = 0;
    for (int im = 0; im < nmol; ++im) {
        int c = atomcellno(lat, dims[0], dims[1], dims[2], xadd[im], yadd[im], zadd[im]);
        C->molcellno[im] = c;
        count[c - 1]++;
        if (count[c - 1] > maxc) maxc = count[c - 1];
    }
    C->maxcellno = maxc;
    C->cell_start[0] = 0;
    for (int c = 0; c < ncell; ++c) C->cell_start[c + 1] = C->cell_start[c] + count[c];
    memset(count, 0, sizeof(int32_t) * (size_t)ncell);
    for (int im = 0; im < nmol; ++im) {
        int c = C->molcellno[im] - 1;
        C->cell_mols[C->cell_start[c] + count[c]] = im;
        count[c]++;
    }
    free(count);
    /* makecellneighbourlist (cellneighbourlist.py:97-183) */
    const float *alatc = lat9, *blatc = lat9 + 3, *clatc = lat9 + 6;
    float cella = 1.0f / (float)C->ncelldiva, cellb = 1.0f / (float)C->ncelldivb,
          cellc = 1.0f / (float)C->ncelldivc;
    float cella2 = 0.5f * cella, cellb2 = 0.5f * cellb, cellc2 = 0.5f * cellc;
    float xc[8], yc[8], zc[8];
    int nf = 0;
    for (int ic = -1; ic <= 1; ic += 2) {
        float cx = (float)ic * cellc2 * clatc[0], cy = (float)ic * cellc2 * clatc[1],
              cz = (float)ic * cellc2 * clatc[2];
        for (int ib = -1; ib <= 1; ib += 2) {
            float bx = (float)ib * cellb2 * blatc[0], by = (float)ib * cellb2 * blatc[1],
                  bz = (float)ib * cellb2 * blatc[2];
            for (int ia = -1; ia <= 1; ia += 2) {
                float ax = (float)ia * cella2 * alatc[0], ay = (float)ia * cella2 * alatc[1],
                      az = (float)ia * cella2 * alatc[2];
                xc[nf] = ax + bx + cx;
                yc[nf] = ay + by + cy;
                zc[nf] = az + bz + cz;
                nf++;
            }
        }
    }
    int nra = (C->ncelldiva - 1) / 2, nrb = (C->ncelldivb - 1) / 2, nrc = (C->ncelldivc - 1) / 2;
    float rmaxsq = rmax * rmax;
    int found_n = 0;
    for (int ic = -nrc; ic <= nrc; ++ic) {
        float cx = (float)ic * cellc * clatc[0], cy = (float)ic * cellc * clatc[1], cz = (float)ic * cellc * clatc[2];
        for (int ib = -nrb; ib <= nrb; ++ib) {
            float bx = (float)ib * cellb * blatc[0], by = (float)ib * cellb * blatc[1],
                  bz = (float)ib * cellb * blatc[2];
            for (int ia = -nra; ia <= nra; ++ia) {
                float ax = (float)ia * cella * alatc[0], ay = (float)ia * cella * alatc[1],
                      az = (float)ia * cella * alatc[2];
                float xdc = ax + bx + cx, ydc = ay + by + cy, zdc = az + bz + cz;
                int found = 0;
                for (int f1 = 0; f1 < 8 && !found; ++f1)
                    for (int f2 = 0; f2 < 8 && !found; ++f2) {
                        float xd = xdc + xc[f1] - xc[f2];
                        float yd = ydc + yc[f1] - yc[f2];
                        float zd = zdc + zc[f1] - zc[f2];
                        float r2 = xd * xd + yd * yd + zd * zd;
                        found = (r2 < rmaxsq) || (ia == 0 && ib == 0 && ic == 0);
                    }
                if (found) {
                    C->ia_off[found_n] = ia;
                    C->ib_off[found_n] = ib;
                    C->ic_off[found_n] = ic;
                    found_n++;
                }
            }
        }
    }
    C->ncellneighb = found_n;
    return 0;
}

static inline int fold(int x, int n) {
    while (x < 0) x += n;
    while (x >= n) x -= n;
    return x;
}

/* make_neighbour_list_from_cells cellneighbourlist.py:187-207 (0-based cell ic). */
int oracle_region(const oracle_cells *C, int ic, int32_t *nbref) {
    int c0 = ic;
    int icc = c0 / (C->ncelldiva * C->ncelldivb);
    int ibb = (c0 - icc * C->ncelldiva * C->ncelldivb) / C->ncelldiva;
    int iaa = c0 - C->ncelldiva * (ibb + C->ncelldivb * icc);
    int n = 0;
    for (int k = 0; k < C->ncellneighb; ++k) {
        int a = fold(iaa + C->ia_off[k], C->ncelldiva);
        int b = fold(ibb + C->ib_off[k], C->ncelldivb);
        int c = fold(icc + C->ic_off[k], C->ncelldivc);
        int cell = a + C->ncelldiva * (b + C->ncelldivb * c);
        for (int p = C->cell_start[cell]; p < C->cell_start[cell + 1]; ++p) nbref[n++] = C->cell_mols[p];
    }
    return n;
}

/* get_nnbrefmax cellneighbourlist.py:211-233 */
int oracle_nnbrefmax(const oracle_cells *C) {
    int mx = 0;
    for (int ic = 0; ic < C->ncell; ++ic) {
        int c0 = ic;
        int icc = c0 / (C->ncelldiva * C->ncelldivb);
        int ibb = (c0 - icc * C->ncelldiva * C->ncelldivb) / C->ncelldiva;
        int iaa = c0 - C->ncelldiva * (ibb + C->ncelldivb * icc);
        int n = 0;
        for (int k = 0; k < C->ncellneighb; ++k) {
            int a = fold(iaa + C->ia_off[k], C->ncelldiva);
            int b = fold(ibb + C->ib_off[k], C->ncelldivb);
            int c = fold(icc + C->ic_off[k], C->ncelldivc);
            int cell = a + C->ncelldiva * (b + C->ncelldivb * c);
            n += C->cell_start[cell + 1] - C->cell_start[cell];
        }
        if (n > mx) mx = n;
    }
    return mx;
}

/* ------------------------------------------------------------------ pair-energy store */
/* ergpairreference.py:63-126 (initialise_ergpair, set_ergpair), fmolec1
 * ato_manipulation_rev4.py:2374-2528.  Store layout: molergpair/ergpairref [nmol][nnbrefmax]
 * (slot-major per molecule, 0-based slots), ergpair[] 0-based values, refs 1-based as in
 * the reference (ergpairref value k means ergpair[k-1]). */
typedef struct {
    int32_t nnbrefmax, nergpair, nergpairmax;
    int32_t *nergpairm;  /* [nmol] */
    int32_t *molergpair; /* [nmol*nnbrefmax], partner molecule (0-based) */
    int32_t *ergpairref; /* [nmol*nnbrefmax], 1-based index into ergpair */
    float *ergpair;      /* [nergpairmax] */
} oracle_store;

static void set_ergpair(oracle_store *E, int im, int jm, float energy) {
    const int M = E->nnbrefmax;
    if (E->nergpairm[im] < M && E->nergpairm[jm] < M && energy != 0.0f) {
        E->nergpair++;
        if (E->nergpair > E->nergpairmax) return; /* caller sizes the store; checked after */
        E->ergpair[E->nergpair - 1] = energy;
        if (jm == im) {
            E->nergpairm[im] = 1;
            E->molergpair[(size_t)im * M + 0] = im;
            E->ergpairref[(size_t)im * M + 0] = E->nergpair;
        } else {
            E->nergpairm[im]++;
            E->nergpairm[jm]++;
            E->molergpair[(size_t)im * M + E->nergpairm[im] - 1] = jm;
            E->molergpair[(size_t)jm * M + E->nergpairm[jm] - 1] = im;
            E->ergpairref[(size_t)im * M + E->nergpairm[im] - 1] = E->nergpair;
            E->ergpairref[(size_t)jm * M + E->nergpairm[jm] - 1] = E->nergpair;
        }
    }
}

/* fmolec1: eintra[] are the en_mole_intra values (an input).  out2 = {ftest, ftestb}
 * (per molecule, as returned).  Returns 0, or 1 when ergpair capacity was exceeded. */
int oracle_fmolec1(const oracle_sys *S, const oracle_cells *C, const float *eintra, oracle_store *E,
                   float *out2) {
    const int nmol = S->nmol;
    const int M = E->nnbrefmax;
    E->nergpair = 0;
    for (int im = 0; im < nmol; ++im) E->nergpairm[im] = 0;
    float ftest = 0.0f, ftestb = 0.0f;
    for (int im = 0; im < nmol; ++im) {
        float e = eintra[im];
        ftestb = ftestb + e;
        set_ergpair(E, im, im, e);
    }
    int32_t *nbref = (int32_t *)malloc(sizeof(int32_t) * (size_t)(M > 0 ? M : 1));
    float *ergold = (float *)malloc(sizeof(float) * (size_t)(M > 0 ? M : 1));
    for (int ic = 0; ic < C->ncell; ++ic) {
        if (C->cell_start[ic + 1] - C->cell_start[ic] <= 0) continue;
        int nn = oracle_region(C, ic, nbref);
        for (int p = C->cell_start[ic]; p < C->cell_start[ic + 1]; ++p) {
            int im = C->cell_mols[p];
            for (int inn = 0; inn < nn; ++inn) {
                int jm = nbref[inn];
                ergold[inn] = 0.0f;
                if (jm > im) ergold[inn] = oracle_en_mole_pair(S, im, jm);
            }
            /* the store loop starts at the second neighbour (ato_manipulation_rev4.py:2466-2474) */
            for (int inn = 1; inn < nn; ++inn) {
                int jm = nbref[inn];
                if (ergold[inn] != 0.0f && jm > im) {
                    set_ergpair(E, im, jm, ergold[inn]);
                    ftest = ftest + ergold[inn];
                }
            }
        }
    }
    free(nbref);
    free(ergold);
    out2[0] = ftest / (float)nmol;
    out2[1] = ftestb / (float)nmol;
    return E->nergpair > E->nergpairmax ? 1 : 0;
}

/* ------------------------------------------------------------------ molfit sweep */
/* ------------------------------------------------------------------ press */
/* press ato_manipulation_rev4.py:3903-4062 without three-body terms or coordination
 * constraints: for every molecule im but the last (0..nmol-2) and every stored partner
 * jm > im, in store order, the energy (ergold, float32, ia outer / ja inner) and the virial
 * term (ergnew: float32 add of prwt, then double add of prpot, stored back as float32) of
 * all atom pairs with iz <= npt1 (:3960-4040); then sumc += ergold in float32 and presst +=
 * ergnew in double over (im, jref) (:4041-4044).  Returns sumc; out2[0] = presst and, for
 * checking sums made in another order, out2[1] = the double sum of the same float32 ergold
 * values. */
float oracle_press(const oracle_sys *S, const oracle_store *E, int32_t npt1, double *out2) {
    const int M = E->nnbrefmax;
    float sumc = 0.0f;
    double presst = 0.0, sum64 = 0.0;
    for (int im = 0; im < S->nmol - 1; ++im) {
        const float xc1 = S->xadd[im], yc1 = S->yadd[im], zc1 = S->zadd[im];
        const int a0 = S->naf[im], a1 = a0 + S->nato[im];
        const int nn = E->nergpairm[im];
        for (int s = 0; s < nn; ++s) {
            const int jm = E->molergpair[(size_t)im * M + s];
            float ergold = 0.0f, ergnew = 0.0f;
            if (jm > im) {
                const int b0 = S->naf[jm], b1 = b0 + S->nato[jm];
                for (int ia = a0; ia < a1; ++ia) {
                    const int it = S->itype[ia];
                    const float x1 = S->xa[ia] + xc1, y1 = S->ya[ia] + yc1, z1 = S->za[ia] + zc1;
                    for (int ja = b0; ja < b1; ++ja) {
                        const float xc2 = S->xadd[jm], yc2 = S->yadd[jm], zc2 = S->zadd[jm];
                        const int icref = S->npairref[it * S->ntype + S->itype[ja]];
                        const float x2 = S->xa[ja] + xc2, y2 = S->ya[ja] + yc2, z2 = S->za[ja] + zc2;
                        float xdif = x2 - x1, ydif = y2 - y1, zdif = z2 - z1;
                        minimagec(S, &xdif, &ydif, &zdif);
                        float xcdif = xc2 - xc1, ycdif = yc2 - yc1, zcdif = zc2 - zc1;
                        minimagec(S, &xcdif, &ycdif, &zcdif);
                        const float dsq = xdif * xdif + ydif * ydif + zdif * zdif;
                        const float dtest = sqrtf(dsq);
                        const float rat = dtest / S->stepcl;
                        const int32_t iz = f_ifix(rat) + 2;
                        if (iz <= npt1) {
                            const size_t b = (size_t)icref * (size_t)S->ld;
                            const float dtdif = dtest - S->xstar[iz];
                            const int32_t ipz = iz;
                            float prfac;
                            if (dtest > 0.0f) prfac = (xcdif * xdif + ycdif * ydif + zcdif * zdif) / dtest;
                            else prfac = 0.0f;
                            const float enpot = S->ecoul[b + iz] + S->ecoul1[b + iz] * dtdif;
                            const double prpot = (double)(0.5f * (S->ecoul1[b + ipz] + S->ecoul1[b + ipz - 1]) * prfac);
                            const float enwt = S->xavs[b + iz] + S->xavs1[b + iz] * dtdif;
                            const float prwt = 0.5f * (S->xavs1[b + ipz] + S->xavs1[b + ipz - 1]) * prfac;
                            ergold = ergold + enwt + enpot;
                            ergnew = (float)((double)(ergnew + prwt) + prpot);
                        }
                    }
                }
            }
            sumc = sumc + ergold;
            presst = presst + (double)ergnew;
            sum64 += (double)ergold;
        }
    }
    out2[0] = presst;
    out2[1] = sum64;
    return sumc;
}

typedef struct {
    float simt, rejrate, stepr, stepm, trstepmax, trstepmin;
    int32_t ireset;
    float *wholerot, *wholetrans;      /* [nmoltype] */
    int32_t *nwhole, *nmovem;          /* [2*nmoltype]: [0..nmt) tries, [nmt..2nmt) rejections */
    int32_t *nstepreject;              /* [nmol] */
    float *internrot, *interntrans;    /* [nmoltype] */
    const int32_t *ngrot;              /* [nmol] (0 here) */
} oracle_mcpar;

typedef struct {
    int32_t nmoves;
    int32_t *im;     /* [nmol] */
    float *den;      /* [nmol] en_change value */
    int32_t *acc;    /* [nmol] */
    float *cosv;     /* [3*nmol] cos values used (glibc cosf), or NULL */
    int32_t ncos;
    double *den64;   /* [nmol] FP64 energy change of the proposed move, or NULL */
    double *scale64; /* [nmol] sum of |FP64 pair energies| before and after the move */
    float *u;        /* [nmol] the ran1 value of the Metropolis test, or NULL */
} oracle_trace;

/* FP64 restatement of en_atom_inter_scale (molfit.py:1251-1279): the same tables and bin
 * rule evaluated in double precision; the interpolation is continuous across bins, so it
 * is the reference value the float32 energies are checked against. */
static double en_atom_inter64(const oracle_sys *S, double x1, double y1, double z1, double x2, double y2,
                              double z2, int icref) {
    double xd = x2 - x1, yd = y2 - y1, zd = z2 - z1;
    xd -= round(xd);
    yd -= round(yd);
    zd -= round(zd);
    double d = sqrt(xd * xd + yd * yd + zd * zd);
    int iz = (int)(d / (double)S->stepcl) + 2;
    if (iz > S->npt2) return 0.0;
    const size_t base = (size_t)icref * (size_t)S->ld;
    double dt = d - (double)S->xstar[iz];
    return (double)S->xavs[base + iz] + (double)S->xavs1[base + iz] * dt + (double)S->ecoul[base + iz] +
           (double)S->ecoul1[base + iz] * dt;
}

/* FP64 energy of molecule im (atom offsets xo/yo/zo, centre cx/cy/cz) with molecule jm;
 * *absum accumulates the magnitudes of the atom-pair terms. */
static double en_mole_pair64(const oracle_sys *S, int im, const float *xo, const float *yo, const float *zo,
                             float cx, float cy, float cz, int jm, double *absum) {
    double e = 0.0;
    const int n = S->nato[im];
    const int b0 = S->naf[jm], b1 = b0 + S->nato[jm];
    for (int k = 0; k < n; ++k) {
        const int it = S->itype[S->naf[im] + k];
        const double x1 = (double)xo[k] + cx, y1 = (double)yo[k] + cy, z1 = (double)zo[k] + cz;
        for (int ja = b0; ja < b1; ++ja) {
            const int icref = S->npairref[it * S->ntype + S->itype[ja]];
            double v = en_atom_inter64(S, x1, y1, z1, (double)S->xa[ja] + S->xadd[jm], (double)S->ya[ja] + S->yadd[jm],
                                       (double)S->za[ja] + S->zadd[jm], icref);
            e += v;
            *absum += fabs(v);
        }
    }
    return e;
}

/* en_change molfit.py:806-919.  d64/sc64 (optional): the exact (double) sum of the same
 * float32 terms and the sum of their magnitudes -- the FP64 reference of the accumulation. */
static float en_change(const oracle_sys *S, int im, const oracle_store *E, float *ergnew, double *d64,
                       double *sc64) {
    const int M = E->nnbrefmax;
    const int nn = E->nergpairm[im];
    const int32_t *nb = E->molergpair + (size_t)im * M;
    const int32_t *rf = E->ergpairref + (size_t)im * M;
    for (int inn = 1; inn < nn; ++inn) ergnew[inn] = 0.0f;
    for (int inn = 1; inn < nn; ++inn) {
        int jm = nb[inn];
        float sume = oracle_en_mole_pair(S, im, jm);
        ergnew[inn] = ergnew[inn] + sume;
    }
    float fdiff = 0.0f;
    double d = 0.0, sc = 0.0;
    for (int inn = 1; inn < nn; ++inn) {
        const float old = E->ergpair[rf[inn] - 1];
        fdiff = fdiff + ergnew[inn] - old;
        d += (double)ergnew[inn] - (double)old;
        sc += fabs((double)ergnew[inn]) + fabs((double)old);
    }
    if (d64) *d64 = d;
    if (sc64) *sc64 = sc;
    return fdiff;
}

float oracle_en_change(const oracle_sys *S, int im, const oracle_store *E, float *ergnew, double *d64_sc64) {
    return en_change(S, im, E, ergnew, d64_sc64, d64_sc64 ? d64_sc64 + 1 : 0);
}

/* rotatm molfit.py:672-711 */
static void rotatm(oracle_sys *S, int im, float stepsz, oracle_ran1_state *R, oracle_trace *T) {
    const float pi = 3.14159265358979323846f; /* f32(math.pi) */
    const int a0 = S->naf[im], a1 = a0 + S->nato[im];
    if (a1 - 1 > a0) {
        float phi, cphi, sphi;
        phi = pi * stepsz * (2.0f * oracle_ran1(R) - 1.0f);
        cphi = cosf(phi);
        if (T && T->cosv) T->cosv[T->ncos++] = cphi;
        sphi = f_sign(sqrtf(1.0f - cphi * cphi), phi);
        for (int ia = a0; ia < a1; ++ia) {
            float xs = S->xa[ia] * cphi - S->ya[ia] * sphi;
            S->ya[ia] = S->xa[ia] * sphi + S->ya[ia] * cphi;
            S->xa[ia] = xs;
        }
        phi = pi * stepsz * (2.0f * oracle_ran1(R) - 1.0f);
        cphi = cosf(phi);
        if (T && T->cosv) T->cosv[T->ncos++] = cphi;
        sphi = f_sign(sqrtf(1.0f - cphi * cphi), phi);
        for (int ia = a0; ia < a1; ++ia) {
            float zs = S->za[ia] * cphi - S->xa[ia] * sphi;
            S->xa[ia] = S->za[ia] * sphi + S->xa[ia] * cphi;
            S->za[ia] = zs;
        }
        phi = pi * stepsz * (2.0f * oracle_ran1(R) - 1.0f);
        cphi = cosf(phi);
        if (T && T->cosv) T->cosv[T->ncos++] = cphi;
        sphi = f_sign(sqrtf(1.0f - cphi * cphi), phi);
        for (int ia = a0; ia < a1; ++ia) {
            float ys = S->ya[ia] * cphi - S->za[ia] * sphi;
            S->za[ia] = S->ya[ia] * sphi + S->za[ia] * cphi;
            S->ya[ia] = ys;
        }
    }
}

/* movem molfit.py:733-759 (the step is doubled until the position changes). */
static float movem(oracle_sys *S, int im, float stepsz, oracle_ran1_state *R) {
    float xs = S->xadd[im], ys = S->yadd[im], zs = S->zadd[im];
    S->zadd[im] = S->zadd[im] + stepsz * (2.0f * oracle_ran1(R) - 1.0f);
    S->yadd[im] = S->yadd[im] + stepsz * (2.0f * oracle_ran1(R) - 1.0f);
    S->xadd[im] = S->xadd[im] + stepsz * (2.0f * oracle_ran1(R) - 1.0f);
    int nochange = xs == S->xadd[im] && ys == S->yadd[im] && zs == S->zadd[im];
    while (nochange) {
        stepsz = stepsz * 2.0f;
        S->zadd[im] = S->zadd[im] + stepsz * (2.0f * oracle_ran1(R) - 1.0f);
        S->yadd[im] = S->yadd[im] + stepsz * (2.0f * oracle_ran1(R) - 1.0f);
        S->xadd[im] = S->xadd[im] + stepsz * (2.0f * oracle_ran1(R) - 1.0f);
        nochange = xs == S->xadd[im] && ys == S->yadd[im] && zs == S->zadd[im];
    }
    return stepsz;
}

/* trstepmax/trstepmin of molfit.py:96-101 */
void oracle_trsteps(int natomr, float *out2) {
    float t = 1.0f / (float)natomr;
    t = powf(t, 1.0f / 3.0f);
    out2[0] = t;
    float a = 0.0001f * t;
    out2[1] = a > 1.0e-6f ? a : 1.0e-6f;
    /* Python max(a, b) returns a when a >= b: same value */
    if (!(a > 1.0e-6f) && a == 1.0e-6f) out2[1] = a;
}

/* ------------------------------------------------------------------ atogen */
/* ato_manipulation_rev4.py:3640-3899, no coarse graining, no container forces.
 * wav: [2][npairs][ld] (ld >= npt1+1, iz 1-based). ycoh: [ld].  rminex: [npairs].
 * out_ngrsamples: returned value.  Returns ngrsamples. */
int oracle_atogen(const oracle_sys *S, float *wav, float *potex, int ngrsamples, int npt1, float sizefactor,
                  float dmax, const float *rminex, const float *cfrac, int natomr, const float *ycoh,
                  oracle_ran1_state *R) {
    const int nmol = S->nmol, npairs = S->npairs, ld = S->ld, ntype = S->ntype;
    const size_t half = (size_t)npairs * (size_t)ld;
    for (size_t i = 0; i < 2 * half; ++i) wav[i] = 0.0f;
    for (int ic = 0; ic < npairs; ++ic) potex[ic] = 0.0f;
    const float stepcl = S->stepcl;
    /* intramolecular (:3696-3725) */
    for (int im = 0; im < nmol; ++im) {
        if (S->nato[im] > 1) {
            const int a0 = S->naf[im], a1 = a0 + S->nato[im];
            for (int ia = a0; ia < a1 - 1; ++ia) {
                float x1 = S->xa[ia], y1 = S->ya[ia], z1 = S->za[ia];
                for (int ja = ia + 1; ja < a1; ++ja) {
                    int icref = S->npairref[S->itype[ia] * ntype + S->itype[ja]];
                    float xx = (x1 - S->xa[ja]) * sizefactor;
                    float yy = (y1 - S->ya[ja]) * sizefactor;
                    float zz = (z1 - S->za[ja]) * sizefactor;
                    minimagec(S, &xx, &yy, &zz);
                    float dtest = sqrtf(xx * xx + yy * yy + zz * zz);
                    int iz1 = f_nint(dtest / stepcl) + 2;
                    if (iz1 > 1 && iz1 <= npt1) wav[(size_t)icref * ld + iz1] = wav[(size_t)icref * ld + iz1] + 2.0f;
                }
            }
        }
    }
    /* intermolecular (:3739-3838) */
    float *csampled = (float *)calloc((size_t)ntype, sizeof(float));
    int *molsampled = (int *)calloc((size_t)S->nmoltype, sizeof(int));
    float *molfraction = (float *)calloc((size_t)S->nmoltype, sizeof(float));
    int32_t *izv = (int32_t *)calloc((size_t)S->natom, sizeof(int32_t));
    int32_t *icv = (int32_t *)calloc((size_t)S->natom, sizeof(int32_t));
    if (ngrsamples <= 0) ngrsamples = 1000;
    if (ngrsamples > nmol) ngrsamples = nmol;
    float probaccept = (float)ngrsamples / (float)nmol;
    for (int im = 0; im < nmol; ++im) molfraction[S->mtype[im]] = molfraction[S->mtype[im]] + 1.0f;
    for (int t = 0; t < S->nmoltype; ++t) molfraction[t] = molfraction[t] / (float)nmol;
    int im1 = 0, im2 = nmol - 1;
    float addwav = 1.0f;
    if (probaccept >= 1.0f) {
        im2 = nmol - 2;
        addwav = 2.0f;
        const int a0 = S->naf[nmol - 1];
        for (int ia = a0; ia < a0 + S->nato[nmol - 1]; ++ia) csampled[S->itype[ia]] = csampled[S->itype[ia]] + 1.0f;
    }
    for (int im = im1; im <= im2; ++im) {
        float u = oracle_ran1(R);
        int mt = S->mtype[im];
        if (u < probaccept || molsampled[mt] < 1 || molfraction[mt] < probaccept) {
            molsampled[mt]++;
            float xc1 = S->xadd[im], yc1 = S->yadd[im], zc1 = S->zadd[im];
            int jm1 = 0, jm2 = nmol - 1;
            if (probaccept >= 1.0f) jm1 = im + 1;
            const int a0 = S->naf[im], a1 = a0 + S->nato[im];
            for (int ia = a0; ia < a1; ++ia) csampled[S->itype[ia]] = csampled[S->itype[ia]] + 1.0f;
            for (int ia = a0; ia < a1; ++ia) {
                float x1 = S->xa[ia] + xc1, y1 = S->ya[ia] + yc1, z1 = S->za[ia] + zc1;
                int it = S->itype[ia];
                for (int jm = jm1; jm <= jm2; ++jm) {
                    const int b0 = S->naf[jm], b1 = b0 + S->nato[jm];
                    if (jm != im) {
                        float xc2 = S->xadd[jm], yc2 = S->yadd[jm], zc2 = S->zadd[jm];
                        for (int ja = b0; ja < b1; ++ja) {
                            int icref = S->npairref[it * ntype + S->itype[ja]];
                            float x2 = S->xa[ja] + xc2, y2 = S->ya[ja] + yc2, z2 = S->za[ja] + zc2;
                            float xx = x1 - x2, yy = y1 - y2, zz = z1 - z2;
                            minimagec(S, &xx, &yy, &zz);
                            float dtest = sqrtf(xx * xx + yy * yy + zz * zz);
                            int iz1 = f_nint(dtest / stepcl) + 2;
                            if (iz1 > 1 && iz1 <= npt1) {
                                izv[ja] = iz1;
                                icv[ja] = icref;
                            } else {
                                izv[ja] = 0;
                            }
                            float dtt = dtest * dmax;
                            if (dtt < 1.0f * fabsf(rminex[icref])) potex[icref] = potex[icref] + 1.0f;
                        }
                    } else {
                        for (int ja = b0; ja < b1; ++ja) izv[ja] = 0;
                    }
                }
                int ja0 = S->naf[jm1], ja1 = S->naf[jm2] + S->nato[jm2];
                for (int ja = ja0; ja < ja1; ++ja) {
                    if (izv[ja] > 0) {
                        size_t k = half + (size_t)icv[ja] * ld + izv[ja];
                        wav[k] = wav[k] + addwav;
                    }
                }
            }
        }
    }
    /* normalisation (:3857-3897) */
    for (int ic = 0; ic < npairs; ++ic) {
        int it = -1, jt = -1;
        for (int a = 0; a < ntype && it < 0; ++a)
            for (int b = a; b < ntype; ++b)
                if (S->npairref[a * ntype + b] == ic) { it = a; jt = b; break; }
        float cprod = cfrac[it] * cfrac[jt] * (float)natomr;
        float cprod2 = csampled[it] * cfrac[jt];
        if (it != jt) {
            cprod = cprod * 2.0f;
            cprod2 = cprod2 + csampled[jt] * cfrac[it];
        }
        float *w1 = wav + (size_t)ic * ld;
        float *w2 = wav + half + (size_t)ic * ld;
        if (cprod > 0.0f) {
            for (int iz = 1; iz <= npt1; ++iz) w1[iz] = w1[iz] / cprod;
        } else {
            for (int iz = 1; iz <= npt1; ++iz) w1[iz] = 0.0f;
        }
        if (cprod2 > 0.0f) {
            for (int iz = 1; iz <= npt1; ++iz) w2[iz] = w2[iz] / cprod2;
            potex[ic] = potex[ic] * cfrac[jt] / cprod2;
        } else {
            for (int iz = 1; iz <= npt1; ++iz) w2[iz] = ycoh[iz];
        }
    }
    free(csampled);
    free(molsampled);
    free(molfraction);
    free(izv);
    free(icv);
    return ngrsamples;
}

/* ------------------------------------------------------------------ gensq */
/* epsr_standalone_rev3.py:4731-4802.  wav [2][npairs][ldw]; foqols [nq+1][ldf] row i holds
 * F[j,i] for j in 1..npt1 (ldf >= npt1+1); sofq out [2][npairs][nq+1]. natomsphere [ntype]. */
void oracle_gensq(int nq, int npairs, int npt1, const float *wav, int ldw, const float *foqols, int ldf,
                  const float *ycoh, const int32_t *n2extr, const float *natomsphere, float *sofq) {
    const size_t half = (size_t)npairs * (size_t)ldw;
    const size_t shalf = (size_t)npairs * (size_t)(nq + 1);
    for (int ic = 0; ic < npairs; ++ic) {
        const float *w1 = wav + (size_t)ic * ldw;
        const float *w2 = wav + half + (size_t)ic * ldw;
        const float nsph = natomsphere[n2extr[ic]];
        for (int i = 1; i <= nq; ++i) {
            const float *fq = foqols + (size_t)i * ldf;
            float sum1 = 0.0f, sum2 = 0.0f, sum3 = 0.0f;
            for (int j = 2; j <= npt1; ++j) {
                float add1 = w1[j];
                if (fabsf(add1) > 0.0f) sum1 = sum1 + add1 * fq[j];
            }
            for (int j = 2; j <= npt1; ++j) {
                float add2 = (w2[j] - ycoh[j]) * nsph;
                sum2 = sum2 + add2 * fq[j];
                sum3 = sum3 + w2[j];
            }
            if (sum3 <= 0.0f) sum2 = 0.0f;
            sofq[(size_t)ic * (nq + 1) + i] = sum1;
            sofq[shalf + (size_t)ic * (nq + 1) + i] = sum2;
        }
    }
}

/* ------------------------------------------------------------------ running averages */
/* One element of the running average with its error bar (the k loop of sumgr
 * epsr_standalone_rev3.py:3619-3629 and sumsq :3667-3677), in double as the reference's
 * real*8 work space: the stored error bar and mean give back the mean square, both are
 * folded with the new sample by fc2 (old) and fc1 (new), and the error bar is the square
 * root of the variance (0 when it is not positive).  *mean and *err are the float32 arrays. */
static void sum_update(double add1, double fc1, double fc2, float *mean, float *err) {
    double sumtot1 = (double)*mean, sumtot2 = (double)*err;
    const double add2 = add1 * add1;
    sumtot2 = sumtot2 * sumtot2 + sumtot1 * sumtot1;
    sumtot1 = fc2 * sumtot1 + fc1 * add1;
    sumtot2 = fc2 * sumtot2 + fc1 * add2;
    double errort = sumtot2 - sumtot1 * sumtot1;
    errort = errort > 0.0 ? sqrt(errort) : 0.0;
    *mean = (float)sumtot1;
    *err = (float)errort;
}

/* sumgr epsr_standalone_rev3.py:3578-3637: wav [2][npairs][ldw] (r index 1-based, 2..nz
 * used), ycoh [ldw]; gorintra, gorinter, gr2intra, gr2inter, entsig [npairs][ldw].  The new
 * sample is wav/ycoh in float32 (0 where ycoh <= 0); entsig[j] is the running double sum
 * over j of ycoh*(gorinter-1) in float32 (the "zero limit"), entsig[1] = 0. */
void oracle_sumgr(int nz, int npairs, const float *wav, int ldw, const float *ycoh, double fc1, double fc2,
                  float *gorintra, float *gorinter, float *gr2intra, float *gr2inter, float *entsig) {
    const size_t half = (size_t)npairs * (size_t)ldw;
    for (int id = 0; id < npairs; ++id) {
        const size_t row = (size_t)id * ldw;
        entsig[row + 1] = 0.0f;
        double zerolimit = 0.0;
        for (int j = 2; j <= nz; ++j) {
            double a1 = 0.0, a2 = 0.0;
            if (ycoh[j] > 0.0f) {
                a1 = (double)(wav[row + j] / ycoh[j]);
                a2 = (double)(wav[half + row + j] / ycoh[j]);
            }
            sum_update(a1, fc1, fc2, &gorintra[row + j], &gr2intra[row + j]);
            sum_update(a2, fc1, fc2, &gorinter[row + j], &gr2inter[row + j]);
            zerolimit = zerolimit + (double)(ycoh[j] * (gorinter[row + j] - 1.0f));
            entsig[row + j] = (float)zerolimit;
        }
    }
}

/* sumsq epsr_standalone_rev3.py:3642-3677: qwind [2][npairs][ldq] (Q index 1-based, 1..nq);
 * soqintra, soqinter, sq2intra, sq2inter [npairs][ldq]. */
void oracle_sumsq(int nq, int npairs, const float *qwind, int ldq, double fc1, double fc2, float *soqintra,
                  float *soqinter, float *sq2intra, float *sq2inter) {
    const size_t half = (size_t)npairs * (size_t)ldq;
    for (int id = 0; id < npairs; ++id) {
        const size_t row = (size_t)id * ldq;
        for (int j = 1; j <= nq; ++j) {
            sum_update((double)qwind[row + j], fc1, fc2, &soqintra[row + j], &sq2intra[row + j]);
            sum_update((double)qwind[half + row + j], fc1, fc2, &soqinter[row + j], &sq2inter[row + j]);
        }
    }
}

/* ------------------------------------------------------------------ intramolecular moves */
typedef struct {
    const int32_t *nbond, *iabond; /* [natom], [natom*maxbond] 0-based partners */
    const float *tbond;            /* [natom*maxbond] */
    int32_t maxbond;
    const int32_t *imageatom;      /* [natom] 0-based, -1 none */
    const int32_t *qtype;          /* [natom] */
    const float *amassa, *amassr;  /* [ntype], [npairs] */
    const float *xav, *xav1;       /* [npairs*ld] */
    const int32_t *ngrot;          /* [nmol] */
    float stepcl, sizefactor, tempb, tempang, simt;
    int32_t refine_intra;
    float refine_intra_fac;
    /* dihedral angles of the rotational groups (molecom labrotdih / ndihedralang / dihedralang):
     * their energy for DIH groups (en_mole_dihedral molfit.py:1353), and their atom pairs left
     * out of the reference potential (en_atom_intra :999-1020).  grp_nrf NULL: no groups. */
    int32_t ndih;
    const int32_t *grp_nrf, *grp_nrl;   /* [nmol] 0-based group range (nrl < nrf: none) */
    const int32_t *grp_axis;            /* [ngroups*2] the two base atoms (labaxi) */
    const int32_t *grp_dih0;            /* [ngroups+1] each group's range in dih_* */
    const int32_t *grp_isdih;           /* [ngroups] 1 for a group of type DIH */
    const int32_t *dih_atoms;           /* [ndih*2] io1 (by base atom 1), io2 (by base atom 2) */
    const float *dih_cos, *dih_sin;     /* [ndih] cosf, sinf of the dihedral angle */
    float tempdih;                      /* molecom.tempdih */
} oracle_intra;

/* en_atom_intra :999-1016: is (ia, ja) one of the dihedral atom pairs of molecule im's groups? */
static int dihedral_pair(const oracle_intra *I, int im, int ia, int ja) {
    if (!I->grp_nrf) return 0;
    for (int ir = I->grp_nrf[im]; ir <= I->grp_nrl[im]; ++ir)
        for (int kd = I->grp_dih0[ir]; kd < I->grp_dih0[ir + 1]; ++kd) {
            const int io1 = I->dih_atoms[2 * kd], io2 = I->dih_atoms[2 * kd + 1];
            if ((io1 == ia && io2 == ja) || (io1 == ja && io2 == ia)) return 1;
        }
    return 0;
}

/* en_dihedral molfit.py:1487-1524 with vecpro / scapro auxiliary_routines.py:231-244: the
 * dihedral angle's cosine and sine already taken (cosf, sinf of dihedralang) */
static float en_dihedral(const float *co1, const float *co2, const float *cd, float cosdih, float sindih) {
    float cv1[3], cv2[3], cpar[3];
    cv1[0] = co1[1] * cd[2] - co1[2] * cd[1];
    cv1[1] = co1[2] * cd[0] - co1[0] * cd[2];
    cv1[2] = co1[0] * cd[1] - co1[1] * cd[0];
    cv2[0] = co2[1] * cd[2] - co2[2] * cd[1];
    cv2[1] = co2[2] * cd[0] - co2[0] * cd[2];
    cv2[2] = co2[0] * cd[1] - co2[1] * cd[0];
    float dmag = sqrtf(cv1[0] * cv1[0] + cv1[1] * cv1[1] + cv1[2] * cv1[2]);
    cv1[0] = cv1[0] / dmag;
    cv1[1] = cv1[1] / dmag;
    cv1[2] = cv1[2] / dmag;
    dmag = sqrtf(cv2[0] * cv2[0] + cv2[1] * cv2[1] + cv2[2] * cv2[2]);
    cv2[0] = cv2[0] / dmag;
    cv2[1] = cv2[1] / dmag;
    cv2[2] = cv2[2] / dmag;
    float cosphi = cv1[0] * cv2[0] + cv1[1] * cv2[1] + cv1[2] * cv2[2];
    if (cosphi > 1.0f) cosphi = 1.0f;
    if (cosphi < -1.0f) cosphi = -1.0f;
    cpar[0] = cv1[1] * cv2[2] - cv1[2] * cv2[1];
    cpar[1] = cv1[2] * cv2[0] - cv1[0] * cv2[2];
    cpar[2] = cv1[0] * cv2[1] - cv1[1] * cv2[0];
    const float sinphi = cpar[0] * cd[0] + cpar[1] * cd[1] + cpar[2] * cd[2];
    const float difc = cosdih - cosphi, difs = sindih - sinphi;
    return difc * difc + difs * difs;
}

/* en_mole_dihedral molfit.py:1353-1410: the DIH groups of molecule im at its offsets */
static float en_mole_dihedral(const oracle_sys *S, const oracle_intra *I, int im) {
    float e = 0.0f;
    if (!I->grp_nrf) return e;
    for (int ir = I->grp_nrf[im]; ir <= I->grp_nrl[im]; ++ir) {
        if (!I->grp_isdih[ir]) continue;
        const int ia1 = I->grp_axis[2 * ir], ia2 = I->grp_axis[2 * ir + 1];
        const float x1 = S->xa[ia1], y1 = S->ya[ia1], z1 = S->za[ia1];
        const float x2 = S->xa[ia2], y2 = S->ya[ia2], z2 = S->za[ia2];
        float cd[3] = {x2 - x1, y2 - y1, z2 - z1};
        const float dmag = sqrtf(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
        cd[0] = cd[0] / dmag;
        cd[1] = cd[1] / dmag;
        cd[2] = cd[2] / dmag;
        for (int kd = I->grp_dih0[ir]; kd < I->grp_dih0[ir + 1]; ++kd) {
            const int io1 = I->dih_atoms[2 * kd], io2 = I->dih_atoms[2 * kd + 1];
            const float co1[3] = {S->xa[io1] - x1, S->ya[io1] - y1, S->za[io1] - z1};
            const float co2[3] = {S->xa[io2] - x2, S->ya[io2] - y2, S->za[io2] - z2};
            e = e + en_dihedral(co1, co2, cd, I->dih_cos[kd], I->dih_sin[kd]);
        }
    }
    return e;
}

/* en_atom_intra molfit.py:923-1045 */
static float en_atom_intra(const oracle_sys *S, const oracle_intra *I, int im, int ia, int ja, float x1, float y1,
                           float z1, float x2, float y2, float z2) {
    if (ja == I->imageatom[ia]) return 0.0f;
    const int icref = S->npairref[S->itype[ia] * S->ntype + S->itype[ja]];
    const int notq = I->qtype[ia] == 0 && I->qtype[ja] == 0;
    float sume = 0.0f;
    const float xdifs = x2 - x1, ydifs = y2 - y1, zdifs = z2 - z1;
    int image = ia, iflag = -1;
    for (int k = 0; k < I->nbond[image] && iflag < 0; ++k)
        if (I->iabond[(size_t)image * I->maxbond + k] == ja) iflag = k;
    if (iflag < 0) {
        image = I->imageatom[ia];
        if (image >= 0)
            for (int k = 0; k < I->nbond[image] && iflag < 0; ++k)
                if (I->iabond[(size_t)image * I->maxbond + k] == ja) iflag = k;
    }
    if (iflag >= 0) {
        float xdif = xdifs, ydif = ydifs, zdif = zdifs;
        minimagec(S, &xdif, &ydif, &zdif);
        const float dtest = sqrtf(xdif * xdif + ydif * ydif + zdif * zdif);
        const int iz = f_ifix(dtest / I->stepcl) + 2;
        const float t = I->tbond[(size_t)image * I->maxbond + iflag];
        const float tb = fabsf(t) > I->stepcl ? fabsf(t) : I->stepcl;
        float wtm = I->amassr[icref] / tb;
        if (t < 0.0f) wtm = wtm * I->tempang;
        const float ddif = tb - dtest;
        sume = wtm * ddif * ddif * I->tempb * I->simt;
        if (I->refine_intra && iz <= S->npt2 && notq) {
            const float dtdif = dtest - S->xstar[iz];
            const size_t k = (size_t)icref * S->ld + iz;
            sume = sume + I->refine_intra_fac * (S->xavs[k] + S->xavs1[k] * dtdif);
        }
    } else if (!dihedral_pair(I, im, ia, ja)) {
        float xdif = xdifs * I->sizefactor, ydif = ydifs * I->sizefactor, zdif = zdifs * I->sizefactor;
        minimagec(S, &xdif, &ydif, &zdif);
        const float dtest = sqrtf(xdif * xdif + ydif * ydif + zdif * zdif);
        const int iz = f_ifix(dtest / I->stepcl) + 2;
        if (iz <= S->npt2) {
            const float dtdif = dtest - S->xstar[iz];
            const size_t k = (size_t)icref * S->ld + iz;
            sume = I->xav[k] + I->xav1[k] * dtdif;
            if (I->refine_intra && notq) sume = sume + I->refine_intra_fac * (S->xavs[k] + S->xavs1[k] * dtdif);
        }
    }
    return sume;
}

/* runepsr17 epsr_standalone_rev3.py:1332-1335: every molecule centre put back in the box */
void oracle_minimage_centres(oracle_sys *S) {
    for (int im = 0; im < S->nmol; ++im) minimagec(S, &S->xadd[im], &S->yadd[im], &S->zadd[im]);
}

/* en_mole_intra molfit.py:1327-1350 */
float oracle_en_mole_intra(const oracle_sys *S, const oracle_intra *I, int im) {
    const int a0 = S->naf[im], n = S->nato[im];
    float e = 0.0f;
    for (int ia = a0; ia < a0 + n - 1; ++ia)
        for (int ja = ia + 1; ja < a0 + n; ++ja)
            e = e + en_atom_intra(S, I, im, ia, ja, S->xa[ia], S->ya[ia], S->za[ia], S->xa[ja], S->ya[ja], S->za[ja]);
    if (I->tempdih > 0.0f && I->ngrot && I->ngrot[im] > 0) {   /* :1345-1348 */
        const float sume = I->tempdih * I->simt * en_mole_dihedral(S, I, im);
        e = e + sume;
    }
    return e;
}

void oracle_en_mole_intra_all(const oracle_sys *S, const oracle_intra *I, float *out) {
    for (int im = 0; im < S->nmol; ++im) out[im] = oracle_en_mole_intra(S, I, im);
}

/* ------------------------------------------------------------------ internal rotations */
/* Rotational groups (molfit.py:295-360): per molecule the group range nrf..nrl, per group the
 * two axis atoms and the range first..last of its rotated atoms in atoms[] (0-based, global). */
typedef struct {
    const oracle_intra *I;
    const int32_t *nrf, *nrl, *axis, *first, *last, *atoms;
    float stepri;
    int32_t rotcycle;
    int32_t *ninter;   /* [2*nmoltype] tries then rejections */
    float *faddbs;     /* in/out, or NULL */
} oracle_rot;

/* rotati molfit.py:589-660 with scapro / vecpro auxiliary_routines.py:231-244 */
static void rotati(oracle_sys *S, const oracle_rot *RT, int ig, float steprithis, oracle_ran1_state *R,
                   oracle_trace *T) {
    const float pi = 3.14159265358979323846f;
    float phi = pi * steprithis * (2.0f * oracle_ran1(R) - 1.0f);
    float cphi = cosf(phi);
    if (T && T->cosv) T->cosv[T->ncos++] = cphi;
    float sphi = f_sign(sqrtf(1.0f - cphi * cphi), phi);
    const int a1 = RT->axis[2 * ig], a2 = RT->axis[2 * ig + 1];
    float p1 = S->xa[a2] - S->xa[a1], p2 = S->ya[a2] - S->ya[a1], p3 = S->za[a2] - S->za[a1];
    float rab2 = p1 * p1 + p2 * p2 + p3 * p3;
    if (rab2 > 0.0f) {
        float rab = sqrtf(rab2);
        p1 = p1 / rab;
        p2 = p2 / rab;
        p3 = p3 / rab;
        for (int ia = RT->first[ig]; ia <= RT->last[ig]; ++ia) {
            const int nat = RT->atoms[ia];
            float v1 = S->xa[nat] - S->xa[a1], v2 = S->ya[nat] - S->ya[a1], v3 = S->za[nat] - S->za[a1];
            float frac = p1 * v1 + p2 * v2 + p3 * v3;
            float q1 = frac * p1, q2 = frac * p2, q3 = frac * p3;
            float r1 = v1 - q1, r2 = v2 - q2, r3 = v3 - q3;
            float w1 = p2 * r3 - p3 * r2, w2 = p3 * r1 - p1 * r3, w3 = p1 * r2 - p2 * r1;
            S->xa[nat] = S->xa[a1] + q1;
            S->ya[nat] = S->ya[a1] + q2;
            S->za[nat] = S->za[a1] + q3;
            S->xa[nat] = S->xa[nat] + r1 * cphi + w1 * sphi;
            S->ya[nat] = S->ya[nat] + r2 * cphi + w2 * sphi;
            S->za[nat] = S->za[nat] + r3 * cphi + w3 * sphi;
        }
    }
}

/* One molfit cycle, whole-molecule branch (molfit.py:268-448) with the internal rotations of
 * rotational groups of type ROT every rotfreq cycles (:295-360, rotati :589) when RT is given,
 * plus step adaptation (:465-536).  fadds (and RT->faddbs) are updated in place (:538-539). */
static int molfit_impl(oracle_sys *S, const oracle_cells *C, oracle_store *E, oracle_mcpar *P,
                       oracle_ran1_state *R, float *fadds, oracle_trace *T, const oracle_rot *RT) {
    const int nmt = S->nmoltype;
    const float temp = 1.0f / P->simt;
    const float rotstepmax = 1.0f, rotstepmin = 1.0e-5f;
    for (int k = 0; k < 2 * nmt; ++k) {
        P->nwhole[k] = 0;
        P->nmovem[k] = 0;
        if (RT && RT->ninter) RT->ninter[k] = 0;
    }
    float fadd = 0.0f, faddb = 0.0f;
    /* molfit's work array ergold(1): the first stored energy of the last loaded list */
    float eold0 = 0.0f, p0 = 0.0f;
    const int M = E->nnbrefmax;
    float *ergnew = (float *)malloc(sizeof(float) * (size_t)(M > 0 ? M : 1));
    float xr[4096], yr[4096], zr[4096];
    if (T) { T->nmoves = 0; T->ncos = 0; }
    for (int ic = 0; ic < C->ncell; ++ic) {
        for (int p = C->cell_start[ic]; p < C->cell_start[ic + 1]; ++p) {
            const int im = C->cell_mols[p];
            const int n = S->nato[im];
            const int mt = S->mtype[im];
            const int a0 = S->naf[im];
            const int32_t *rf0 = E->ergpairref + (size_t)im * M;
            const int nn = E->nergpairm[im];
            if (nn >= 1) eold0 = E->ergpair[rf0[0] - 1];
            const int rot = RT && RT->stepri > 0.0f && P->ngrot[im] > 0 && RT->rotcycle;
            if (rot) {
                if (P->internrot[mt] == 0.0f) P->internrot[mt] = rotstepmin;
                RT->ninter[mt]++;
                for (int k = 0; k < n; ++k) { xr[k] = S->xa[a0 + k]; yr[k] = S->ya[a0 + k]; zr[k] = S->za[a0 + k]; }
                for (int ig = RT->nrf[im]; ig <= RT->nrl[im]; ++ig) rotati(S, RT, ig, P->internrot[mt], R, T);
                const float enew0 = oracle_en_mole_intra(S, RT->I, im);
                const float fdiffb = enew0 - eold0;
                p0 = enew0;
                double r64 = 0.0, rs64 = 0.0;
                const float fdiff = en_change(S, im, E, ergnew, &r64, &rs64);
                const float ediff = (fdiff + fdiffb) * temp;
                float etest;
                if (ediff <= 0.0f) etest = 10.0f;
                else if (ediff < 20.0f) etest = expf(-ediff);
                else etest = 0.0f;
                if (oracle_ran1(R) < etest) {
                    P->nstepreject[im] = 0;
                    fadd = fadd + fdiff;
                    faddb = faddb + fdiffb;
                    eold0 = enew0;
                    if (nn >= 1) E->ergpair[rf0[0] - 1] = enew0;
                    for (int inn = 1; inn < nn; ++inn) E->ergpair[rf0[inn] - 1] = ergnew[inn];
                } else {
                    P->nstepreject[im]++;
                    for (int k = 0; k < n; ++k) { S->xa[a0 + k] = xr[k]; S->ya[a0 + k] = yr[k]; S->za[a0 + k] = zr[k]; }
                    RT->ninter[nmt + mt]++;
                }
            } else if (P->ngrot[im] == 0) {
                P->internrot[mt] = 0.0f;
            }
            for (int k = 0; k < n; ++k) { xr[k] = S->xa[a0 + k]; yr[k] = S->ya[a0 + k]; zr[k] = S->za[a0 + k]; }
            const float xs = S->xadd[im], ys = S->yadd[im], zs = S->zadd[im];
            if (P->stepr > 0.0f && n > 1) {
                if (P->wholerot[mt] <= 0.0f) P->wholerot[mt] = rotstepmin;
                P->nwhole[mt]++;
                rotatm(S, im, P->wholerot[mt], R, T);
            } else {
                P->wholerot[mt] = 0.0f;
            }
            if (P->stepm > 0.0f) {
                if (P->wholetrans[mt] <= 0.0f) P->wholetrans[mt] = P->trstepmin;
                P->nmovem[mt]++;
                P->wholetrans[mt] = movem(S, im, P->wholetrans[mt], R);
            } else {
                P->wholetrans[mt] = 0.0f;
            }
            double d64 = 0.0, sc64 = 0.0;
            float fdiff = en_change(S, im, E, ergnew, &d64, &sc64);
            if (T && T->den64) {
                T->den64[T->nmoves] = d64;
                T->scale64[T->nmoves] = sc64;
            }
            float ediff = (fdiff + 0.0f) * temp;
            float etest;
            if (ediff <= 0.0f) etest = 10.0f;
            else if (ediff < 20.0f) etest = expf(-ediff);
            else etest = 0.0f;
            const float udraw = oracle_ran1(R);
            int acc = udraw < etest;
            if (T && T->u) T->u[T->nmoves] = udraw;
            if (acc) {
                P->nstepreject[im] = 0;
                fadd = fadd + fdiff;
                const int32_t *rf = E->ergpairref + (size_t)im * M;
                for (int inn = 1; inn < E->nergpairm[im]; ++inn) E->ergpair[rf[inn] - 1] = ergnew[inn];
                /* save_energies copies ergnew(1) too: the rotation's intramolecular energy of this
                 * visit, accepted or not (ergpairreference.py:192-210) */
                if (rot) {
                    eold0 = p0;
                    if (nn >= 1) E->ergpair[rf[0] - 1] = p0;
                }
            } else {
                P->nstepreject[im]++;
                for (int k = 0; k < n; ++k) { S->xa[a0 + k] = xr[k]; S->ya[a0 + k] = yr[k]; S->za[a0 + k] = zr[k]; }
                S->xadd[im] = xs;
                S->yadd[im] = ys;
                S->zadd[im] = zs;
                if (P->stepr > 0.0f) P->nwhole[nmt + mt]++;
                if (P->stepm > 0.0f) P->nmovem[nmt + mt]++;
            }
            if (T) {
                T->im[T->nmoves] = im;
                T->den[T->nmoves] = fdiff;
                T->acc[T->nmoves] = acc;
                T->nmoves++;
            }
        }
    }
    free(ergnew);
    if (P->ireset != 1) {
        for (int t = 0; t < nmt; ++t) {
            float rat;
            /* nmovei stays 0 in this branch, so its ratio is 1.0 (molfit.py:469-483) */
            P->interntrans[t] = P->interntrans[t] * 1.0f;
            if (P->interntrans[t] > P->trstepmax) P->interntrans[t] = P->trstepmax;
            if (P->interntrans[t] < P->trstepmin && P->interntrans[t] != 0.0f) P->interntrans[t] = P->trstepmin;
            const int ni1 = RT && RT->ninter ? RT->ninter[t] : 0, ni2 = RT && RT->ninter ? RT->ninter[nmt + t] : 0;
            if (ni2 > 0) {
                rat = P->rejrate * (float)ni1 / (float)ni2;
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = ni1 > 0 ? 1.1f : 1.0f;
            }
            P->internrot[t] = P->internrot[t] * rat;
            if (P->internrot[t] > rotstepmax) P->internrot[t] = rotstepmax;
            if (P->internrot[t] < rotstepmin && P->internrot[t] != 0.0f) P->internrot[t] = rotstepmin;
            if (P->nwhole[nmt + t] > 0) {
                rat = P->rejrate * (float)P->nwhole[t] / (float)P->nwhole[nmt + t];
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = P->nwhole[t] > 0 ? 1.1f : 1.0f;
            }
            P->wholerot[t] = P->wholerot[t] * rat;
            if (P->wholerot[t] > rotstepmax) P->wholerot[t] = rotstepmax;
            if (P->wholerot[t] < rotstepmin && P->wholerot[t] != 0.0f) P->wholerot[t] = rotstepmin;
            if (P->nmovem[nmt + t] > 0) {
                rat = P->rejrate * (float)P->nmovem[t] / (float)P->nmovem[nmt + t];
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = P->nmovem[t] > 0 ? 1.1f : 1.0f;
            }
            P->wholetrans[t] = P->wholetrans[t] * rat;
            if (P->wholetrans[t] > P->trstepmax) P->wholetrans[t] = P->trstepmax;
            if (P->wholetrans[t] < P->trstepmin && P->wholetrans[t] != 0.0f) P->wholetrans[t] = P->trstepmin;
        }
    }
    *fadds = *fadds + fadd / (float)S->nmol;
    if (RT && RT->faddbs) *RT->faddbs = *RT->faddbs + faddb / (float)S->nmol;
    return 0;
}

int oracle_molfit(oracle_sys *S, const oracle_cells *C, oracle_store *E, oracle_mcpar *P,
                  oracle_ran1_state *R, float *fadds, oracle_trace *T) {
    return molfit_impl(S, C, E, P, R, fadds, T, NULL);
}

int oracle_molfit_rot(oracle_sys *S, const oracle_cells *C, oracle_store *E, oracle_mcpar *P,
                      oracle_ran1_state *R, float *fadds, oracle_trace *T, const oracle_rot *RT) {
    return molfit_impl(S, C, E, P, R, fadds, T, RT);
}


/* The intramolecular branch of molfit (molfit.py:119-174 with :246-247; no rotational groups),
 * then the step adaptation :465-536, in the reference's order.  *ergold1 is the reference's
 * work value ergold(1) (in/out).  Returns 1 for a molecule with rotational groups. */
int oracle_molfit_shake(oracle_sys *S, oracle_store *E, oracle_mcpar *P, const oracle_intra *I, float stepmi,
                        oracle_ran1_state *R, float *fadds, float *faddbs, int32_t *nmovei, float *ergold1) {
    const int nmt = S->nmoltype, M = E->nnbrefmax;
    for (int im = 0; im < S->nmol; ++im)
        if (I->ngrot[im] > 0) return 1;
    for (int t = 0; t < 2 * nmt; ++t) {
        nmovei[t] = 0;
        P->nwhole[t] = 0;
        P->nmovem[t] = 0;
    }
    const float temp = 1.0f / P->simt;
    float faddb = 0.0f, eo1 = *ergold1;
    float xr[4096], yr[4096], zr[4096];
    for (int im = 0; im < S->nmol; ++im) {
        const int nn = E->nergpairm[im];
        if (nn >= 1) eo1 = E->ergpair[E->ergpairref[(size_t)im * M] - 1];   /* make_neighbour_list_from_mols */
        const int n = S->nato[im], a0 = S->naf[im], mt = S->mtype[im];
        if (n > 1 && stepmi > 0.0f && n <= 4096) {
            float step = P->interntrans[mt];
            if (stepmi > 0.0f && step == 0.0f) step = P->trstepmin;
            P->interntrans[mt] = step;
            for (int k = 0; k < n; ++k) {
                xr[k] = S->xa[a0 + k];
                yr[k] = S->ya[a0 + k];
                zr[k] = S->za[a0 + k];
            }
            nmovei[mt] += 1;
            for (int k = 0; k < n; ++k) {                                    /* movei / movea */
                const int a = a0 + k;
                S->za[a] = S->za[a] + step * (2.0f * oracle_ran1(R) - 1.0f);
                S->ya[a] = S->ya[a] + step * (2.0f * oracle_ran1(R) - 1.0f);
                S->xa[a] = S->xa[a] + step * (2.0f * oracle_ran1(R) - 1.0f);
            }
            const float enew = oracle_en_mole_intra(S, I, im);
            const float fdiffb = enew - eo1;
            const float ediff = fdiffb * temp;
            const float etest = ediff <= 0.0f ? 10.0f : (ediff < 20.0f ? expf(-ediff) : 0.0f);
            if (oracle_ran1(R) < etest) {
                faddb = faddb + fdiffb;
                if (nn >= 1) {                                                 /* save_energies */
                    eo1 = enew;
                    E->ergpair[E->ergpairref[(size_t)im * M] - 1] = eo1;     /* save_erg_pairs */
                }
                float x1 = 0.0f, y1 = 0.0f, z1 = 0.0f, summass = 0.0f;        /* centreofmassi */
                for (int k = 0; k < n; ++k) {
                    const int a = a0 + k;
                    if (I->qtype[a] == 0) {
                        const float am = I->amassa[S->itype[a]];
                        x1 = x1 + S->xa[a] * am;
                        y1 = y1 + S->ya[a] * am;
                        z1 = z1 + S->za[a] * am;
                        summass = summass + am;
                    }
                }
                if (summass > 0.0f) {
                    x1 = x1 / summass;
                    y1 = y1 / summass;
                    z1 = z1 / summass;
                }
                for (int k = 0; k < n; ++k) {
                    S->xa[a0 + k] = S->xa[a0 + k] - x1;
                    S->ya[a0 + k] = S->ya[a0 + k] - y1;
                    S->za[a0 + k] = S->za[a0 + k] - z1;
                }
            } else {
                nmovei[nmt + mt] += 1;
                for (int k = 0; k < n; ++k) {
                    S->xa[a0 + k] = xr[k];
                    S->ya[a0 + k] = yr[k];
                    S->za[a0 + k] = zr[k];
                }
            }
        }
        P->internrot[mt] = 0.0f;   /* no rotational groups (:246-247) */
    }
    if (P->ireset != 1) {
        const float rotstepmin = 1.0e-5f, rotstepmax = 1.0f;
        for (int t = 0; t < nmt; ++t) {
            float rat;
            if (nmovei[nmt + t] > 0) {
                rat = P->rejrate * (float)nmovei[t] / (float)nmovei[nmt + t];
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = nmovei[t] > 0 ? 1.1f : 1.0f;
            }
            P->interntrans[t] = P->interntrans[t] * rat;
            if (P->interntrans[t] > P->trstepmax) P->interntrans[t] = P->trstepmax;
            if (P->interntrans[t] < P->trstepmin && P->interntrans[t] != 0.0f) P->interntrans[t] = P->trstepmin;
            P->internrot[t] = P->internrot[t] * 1.0f;
            if (P->internrot[t] > rotstepmax) P->internrot[t] = rotstepmax;
            if (P->internrot[t] < rotstepmin && P->internrot[t] != 0.0f) P->internrot[t] = rotstepmin;
            P->wholerot[t] = P->wholerot[t] * 1.0f;
            if (P->wholerot[t] > rotstepmax) P->wholerot[t] = rotstepmax;
            if (P->wholerot[t] < rotstepmin && P->wholerot[t] != 0.0f) P->wholerot[t] = rotstepmin;
            P->wholetrans[t] = P->wholetrans[t] * 1.0f;
            if (P->wholetrans[t] > P->trstepmax) P->wholetrans[t] = P->trstepmax;
            if (P->wholetrans[t] < P->trstepmin && P->wholetrans[t] != 0.0f) P->wholetrans[t] = P->trstepmin;
        }
    }
    *fadds = *fadds + 0.0f / (float)S->nmol;
    *faddbs = *faddbs + faddb / (float)S->nmol;
    *ergold1 = eo1;
    return 0;
}

/* centreofmassi ato_manipulation_rev4.py:442: the molecule's offsets moved so that their
 * centre of mass (atoms that are not q-type, weighted by amassa) is at the molecule centre */
static void centreofmassi(oracle_sys *S, const oracle_intra *I, int im) {
    const int a0 = S->naf[im], n = S->nato[im];
    float x1 = 0.0f, y1 = 0.0f, z1 = 0.0f, summass = 0.0f;
    for (int k = 0; k < n; ++k) {
        const int a = a0 + k;
        if (I->qtype[a] == 0) {
            const float am = I->amassa[S->itype[a]];
            x1 = x1 + S->xa[a] * am;
            y1 = y1 + S->ya[a] * am;
            z1 = z1 + S->za[a] * am;
            summass = summass + am;
        }
    }
    if (summass > 0.0f) {
        x1 = x1 / summass;
        y1 = y1 / summass;
        z1 = z1 / summass;
    }
    for (int k = 0; k < n; ++k) {
        S->xa[a0 + k] = S->xa[a0 + k] - x1;
        S->ya[a0 + k] = S->ya[a0 + k] - y1;
        S->za[a0 + k] = S->za[a0 + k] - z1;
    }
}

/* The intramolecular branch of molfit for a box with rotational groups of type ROT
 * (molfit.py:124-267): molecules in index order; each one's atoms moved at random (movei :545,
 * movea :556) and tested on its intramolecular change against ergold(1) (en_change_intra :763),
 * the centre of mass restored on acceptance; then, when stepri > 0 and the molecule has groups,
 * every group rotated (rotati :589) and the rotation tested on the intramolecular change plus
 * the intermolecular change over the stored list (en_change :806).  Then the step adaptation
 * :465-536 with nmovei and RT->ninter.  *ergold1 is molfit's work value ergold(1) (in/out);
 * T->cosv (optional) records rotati's cosines in order.  fadds gains the rotations' accepted
 * intermolecular changes, *faddbs the accepted intramolecular ones, over nmol. */
int oracle_molfit_shake_rot(oracle_sys *S, oracle_store *E, oracle_mcpar *P, const oracle_rot *RT, float stepmi,
                            oracle_ran1_state *R, float *fadds, float *faddbs, int32_t *nmovei, float *ergold1,
                            oracle_trace *T) {
    const int nmt = S->nmoltype, M = E->nnbrefmax;
    const float rotstepmin = 1.0e-5f, rotstepmax = 1.0f;
    for (int t = 0; t < 2 * nmt; ++t) {
        nmovei[t] = 0;
        RT->ninter[t] = 0;
        P->nwhole[t] = 0;
        P->nmovem[t] = 0;
    }
    if (T) T->ncos = 0;
    const float temp = 1.0f / P->simt;
    float fadd = 0.0f, faddb = 0.0f, eo1 = *ergold1;
    float *ergnew = (float *)malloc(sizeof(float) * (size_t)(M > 0 ? M : 1));
    float xr[4096], yr[4096], zr[4096];
    for (int im = 0; im < S->nmol; ++im) {
        const int nn = E->nergpairm[im];
        const int32_t *rf = E->ergpairref + (size_t)im * M;
        if (nn >= 1) eo1 = E->ergpair[rf[0] - 1];   /* make_neighbour_list_from_mols */
        const int n = S->nato[im], a0 = S->naf[im], mt = S->mtype[im];
        if (n > 4096) { free(ergnew); return 1; }
        if (n > 1 && stepmi > 0.0f) {
            float step = P->interntrans[mt];
            if (stepmi > 0.0f && step == 0.0f) step = P->trstepmin;
            P->interntrans[mt] = step;
            for (int k = 0; k < n; ++k) { xr[k] = S->xa[a0 + k]; yr[k] = S->ya[a0 + k]; zr[k] = S->za[a0 + k]; }
            nmovei[mt] += 1;
            for (int k = 0; k < n; ++k) {                                    /* movei / movea */
                const int a = a0 + k;
                S->za[a] = S->za[a] + step * (2.0f * oracle_ran1(R) - 1.0f);
                S->ya[a] = S->ya[a] + step * (2.0f * oracle_ran1(R) - 1.0f);
                S->xa[a] = S->xa[a] + step * (2.0f * oracle_ran1(R) - 1.0f);
            }
            const float enew = oracle_en_mole_intra(S, RT->I, im);
            const float fdiffb = enew - eo1;
            const float ediff = fdiffb * temp;
            const float etest = ediff <= 0.0f ? 10.0f : (ediff < 20.0f ? expf(-ediff) : 0.0f);
            if (oracle_ran1(R) < etest) {
                faddb = faddb + fdiffb;
                if (nn >= 1) {                                 /* save_energies, save_erg_pairs */
                    eo1 = enew;
                    E->ergpair[rf[0] - 1] = eo1;
                }
                centreofmassi(S, RT->I, im);
            } else {
                nmovei[nmt + mt] += 1;
                for (int k = 0; k < n; ++k) { S->xa[a0 + k] = xr[k]; S->ya[a0 + k] = yr[k]; S->za[a0 + k] = zr[k]; }
            }
        }
        if (RT->stepri > 0.0f && P->ngrot[im] > 0) {
            if (P->internrot[mt] == 0.0f) P->internrot[mt] = rotstepmin;
            RT->ninter[mt]++;
            for (int k = 0; k < n; ++k) { xr[k] = S->xa[a0 + k]; yr[k] = S->ya[a0 + k]; zr[k] = S->za[a0 + k]; }
            for (int ig = RT->nrf[im]; ig <= RT->nrl[im]; ++ig) rotati(S, RT, ig, P->internrot[mt], R, T);
            const float enew = oracle_en_mole_intra(S, RT->I, im);
            const float fdiffb = enew - eo1;
            const float fdiff = en_change(S, im, E, ergnew, NULL, NULL);
            const float ediff = (fdiff + fdiffb) * temp;
            const float etest = ediff <= 0.0f ? 10.0f : (ediff < 20.0f ? expf(-ediff) : 0.0f);
            if (oracle_ran1(R) < etest) {
                P->nstepreject[im] = 0;
                fadd = fadd + fdiff;
                faddb = faddb + fdiffb;
                if (nn >= 1) {                                 /* save_energies, save_erg_pairs */
                    eo1 = enew;
                    E->ergpair[rf[0] - 1] = enew;
                }
                for (int inn = 1; inn < nn; ++inn) E->ergpair[rf[inn] - 1] = ergnew[inn];
            } else {
                P->nstepreject[im]++;
                for (int k = 0; k < n; ++k) { S->xa[a0 + k] = xr[k]; S->ya[a0 + k] = yr[k]; S->za[a0 + k] = zr[k]; }
                RT->ninter[nmt + mt]++;
            }
        } else if (P->ngrot[im] == 0) {
            P->internrot[mt] = 0.0f;
        }
    }
    free(ergnew);
    if (P->ireset != 1) {
        for (int t = 0; t < nmt; ++t) {
            float rat;
            if (nmovei[nmt + t] > 0) {
                rat = P->rejrate * (float)nmovei[t] / (float)nmovei[nmt + t];
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = nmovei[t] > 0 ? 1.1f : 1.0f;
            }
            P->interntrans[t] = P->interntrans[t] * rat;
            if (P->interntrans[t] > P->trstepmax) P->interntrans[t] = P->trstepmax;
            if (P->interntrans[t] < P->trstepmin && P->interntrans[t] != 0.0f) P->interntrans[t] = P->trstepmin;
            if (RT->ninter[nmt + t] > 0) {
                rat = P->rejrate * (float)RT->ninter[t] / (float)RT->ninter[nmt + t];
                if (rat > 1.1f) rat = 1.1f;
                if (rat < 0.9f) rat = 0.9f;
            } else {
                rat = RT->ninter[t] > 0 ? 1.1f : 1.0f;
            }
            P->internrot[t] = P->internrot[t] * rat;
            if (P->internrot[t] > rotstepmax) P->internrot[t] = rotstepmax;
            if (P->internrot[t] < rotstepmin && P->internrot[t] != 0.0f) P->internrot[t] = rotstepmin;
            P->wholerot[t] = P->wholerot[t] * 1.0f;
            if (P->wholerot[t] > rotstepmax) P->wholerot[t] = rotstepmax;
            if (P->wholerot[t] < rotstepmin && P->wholerot[t] != 0.0f) P->wholerot[t] = rotstepmin;
            P->wholetrans[t] = P->wholetrans[t] * 1.0f;
            if (P->wholetrans[t] > P->trstepmax) P->wholetrans[t] = P->trstepmax;
            if (P->wholetrans[t] < P->trstepmin && P->wholetrans[t] != 0.0f) P->wholetrans[t] = P->trstepmin;
        }
    }
    *fadds = *fadds + fadd / (float)S->nmol;
    *faddbs = *faddbs + faddb / (float)S->nmol;
    *ergold1 = eo1;
    return 0;
}

/* ------------------------------------------------------------------ generate_ep */
/* generate_ep epsr_standalone_rev3.py:5876-5995 with the Poisson basis already built
 * (calc_pwrexpr_grad, host): expgr [npt2][nterms] (row j-1 of the reference's flat expgr).
 * pcoefp [nsets][ldc] (coefficient ic at [set][ic], 1-based ic), iref [npairs] the set of
 * each pair (irefpcof - 1); tables xavs, xavs1, xavtot, xavtot1, ecoul [npairs][ld] (r index
 * 1-based), xstar, wfac [ld].  par = {absolute_energy, erequnit, ereqstep, potfacamp}.
 * Updates the tables, pcoefp (multiply_pot_coeffs), pwtold (the last pair's coefficients)
 * and *potfac; returns energabs and pressfac in out2. */
void oracle_generate_ep(int npairs, int npt, int npt2, int nterms, const float *expgr, float *pcoefp, int nsets,
                        int ldc, const int32_t *iref, float dmax, const float *xstar, const float *wfac, const float *ecoul,
                        float *xavs, float *xavs1, float *xavtot, float *xavtot1, int ld, float *pwtold,
                        const float *par, float *potfac, int changepotfac, float *out2) {
    volatile float e25 = 25.0f;   /* exp(25) from the C library at run time, as the reference */
    const float summax = expf(e25);
    const int w = ldc;
    /* the EP gradient of every pair from its coefficients (:5905-5920) */
    for (int ip = 0; ip < npairs; ++ip) {
        const float *pc = pcoefp + (size_t)iref[ip] * w;
        for (int ic = 2; ic <= nterms; ++ic) pwtold[ic] = pc[ic];
        pwtold[1] = 0.0f;
        for (int j = 1; j <= npt2; ++j) {
            const float *e = expgr + (size_t)(j - 1) * nterms;
            float sum = 0.0f;
            for (int i = 1; i <= nterms; ++i) {     /* expand :4924 */
                sum = sum + e[i - 1] * pwtold[i];
                if (fabsf(sum) > summax) sum = copysignf(summax, sum);
            }
            xavs1[(size_t)ip * ld + j] = sum * pc[1];
        }
    }
    /* the potential integrated from the last point, then truncated (:5922-5948) */
    for (int ip = 0; ip < npairs; ++ip) {
        float *s = xavs + (size_t)ip * ld, *s1 = xavs1 + (size_t)ip * ld;
        for (int j = 1; j <= npt2; ++j) s1[j] = s1[j] * dmax;
        s[npt] = 0.0f;
        s1[npt] = 0.0f;
        float x1 = xstar[npt], xts1 = s1[npt];
        for (int j = 1; j <= npt2; ++j) {
            const int jref = npt - j;
            const float x2 = xstar[jref], xts2 = s1[jref];
            s[jref] = s[jref + 1] - 0.5f * (x1 - x2) * (xts1 + xts2);
            x1 = x2;
            xts1 = xts2;
        }
        for (int j = 1; j <= npt2; ++j) s[j] = s[j] * wfac[j];
    }
    /* abs_energy_ep ato_manipulation_rev4.py:4128-4157 and the potential factor (:5950-5962) */
    float energabs = 0.0f;
    for (int k = 0; k < nsets; ++k) {
        float lo = 0.0f, hi = 0.0f;
        for (int i = 2; i <= nterms; ++i) {
            const float t = pcoefp[(size_t)k * w + i];
            lo = fminf(lo, t);
            hi = fmaxf(hi, t);
        }
        energabs = fmaxf(energabs, hi - lo);
    }
    const float absolute_energy = par[0], erequnit = par[1], ereqstep = par[2], potfacamp = par[3];
    float pressfac = 1.0f;
    if (fabsf(absolute_energy) == 0.0f) {
        pressfac = 0.0f;
        energabs = 0.0f;
    } else if (fabsf(energabs) > 0.0f) {
        if (fabsf(energabs) < fabsf(erequnit)) {
            pressfac = fabsf(erequnit) / fabsf(energabs);
        } else {
            pressfac = fabsf(absolute_energy) / fabsf(energabs);
            if (pressfac > 1.0f && ereqstep == 0.0f) pressfac = 1.0f;
        }
    }
    /* multiply_pot_coeffs :5215 (once per pair, so a set shared by pairs is scaled again) */
    for (int ip = 0; ip < npairs; ++ip)
        for (int ic = 2; ic <= nterms; ++ic) pcoefp[(size_t)iref[ip] * w + ic] *= pressfac;
    /* scaled EP, total potential and both gradients (:5964-5985) */
    for (int ip = 0; ip < npairs; ++ip) {
        float *s = xavs + (size_t)ip * ld, *s1 = xavs1 + (size_t)ip * ld;
        float *t = xavtot + (size_t)ip * ld, *t1 = xavtot1 + (size_t)ip * ld;
        const float *ec = ecoul + (size_t)ip * ld;
        for (int j = 1; j <= npt2; ++j) {
            s[j] = s[j] * pressfac;
            t[j] = ec[j] + s[j];
        }
        float sums1 = s[1], sumtot1 = t[1], x1 = xstar[1];
        for (int j = 2; j <= npt; ++j) {
            const float x2 = xstar[j], xdif = x2 - x1;
            const float sums2 = s[j], sumtot2 = t[j];
            s1[j - 1] = (sums2 - sums1) / xdif;
            t1[j - 1] = (sumtot2 - sumtot1) / xdif;
            x1 = x2;
            sums1 = sums2;
            sumtot1 = sumtot2;
        }
        s1[npt] = 0.0f;
        t1[npt] = 0.0f;
    }
    /* the step of the potential factor (:5987-5995) */
    if (changepotfac && absolute_energy > 0.0f) {
        if (*potfac > 0.000001f && potfacamp > 0.0f) {
            float absediff = (absolute_energy - energabs) / fabsf(potfacamp * absolute_energy);
            if (fabsf(absediff) > 0.1f) absediff = copysignf(0.1f, absediff);
            float pf = *potfac * (1.0f + absediff);
            pf = fmaxf(pf, 0.000001f);
            pf = fminf(pf, 1.0f);
            *potfac = pf;
        }
    }
    out2[0] = energabs;
    out2[1] = pressfac;
}

/* calc_pwrexpr_grad epsr_standalone_rev3.py:5230-5309 (with fctrln lngamma_mod.py:16-32 and
 * dnext :5312-5326): expr [lpt][nterms] from xin[1..lpt]; returns ncfirst, or -1 when a term
 * needs a log-factorial beyond the table (an index error in the reference). */
int oracle_calc_pwrexpr_grad(int lpt, int nterms, float dmin, float dstep, float dmax, float sigmab, float rho,
                             const float *xin, float *expr, float rmin, int ncfirst, float fbroad, float rbroad) {
    const float pi = 3.141592653f, expmax = 25.0f;
    const int ntmax = (int)(dmax / sigmab + 3.0f);
    double *gamln = (double *)malloc(sizeof(double) * (size_t)(ntmax + 2));
    double g = 0.0, a = 0.0;
    for (int i = 1; i <= ntmax + 1; ++i) {
        gamln[i] = g;
        a = a + 1.0;
        g = g + log(a);
    }
    float d = dstep, rootd = 1.0f;
    for (int m = 1; m <= nterms; ++m) {
        if (d < rmin) ncfirst = m + 1;
        const float sigma = rootd * fbroad * sigmab;
        const int n = (sigma <= d && sigma > 0.0f && m > 1) ? (int)(d / sigma - 1.0f) : 0;
        const int nref = n + 3;
        if (nref > ntmax + 1) {
            free(gamln);
            return -1;
        }
        const float gfac = 4.0f * pi * rho * sigma * sigma * sigma;
        float sigln = (float)(gamln[nref] + (double)logf(gfac));
        if (m == 1) sigln = sigln - rmin / sigma;
        for (int i = 1; i <= lpt; ++i) {
            const float r = xin[i], rsigma = r / sigma;
            float fact = rbroad * r, expon;
            if (r > 0.0f) {
                expon = (float)n * logf(rsigma) - rsigma - sigln - fact;
                fact = (float)n / r - 1.0f / sigma - rbroad;
            } else if (n == 0 || n == 1) {
                expon = -rsigma - sigln - fact;
                fact = n == 0 ? -(1.0f / sigma + rbroad) : 1.0f / sigma;
            } else {
                expon = -2.0f * expmax;
                fact = 0.0f;
            }
            expr[(size_t)(i - 1) * nterms + (m - 1)] = expon > -expmax ? fact * expf(expon) : 0.0f;
        }
        float dn = d + dstep;
        const float dtest = d * dmin;
        if (dtest > dn) {
            dn = dtest;
            rootd = rootd * sqrtf(dmin);
        }
        d = dn;
    }
    free(gamln);
    return ncfirst;
}

/* ------------------------------------------------------------------ stog */
/* ato_manipulation_rev4.py:4067-4121. sofq [npairs][ldq] (i 1-based), q [ldq], r [nr+1]
 * (1-based), gofr out [npairs][nr+1]. */
static float lorch(float x, float pi) {
    if (x == 0.0f) return 1.0f;
    if (x < pi) return sinf(x) / x;
    return 0.0f;
}

void oracle_stog(float rho, const float *q, const float *sofq, int ldq, const float *r, float *gofr,
                 const int32_t *nqmin, const int32_t *nqmax, int nr, int npairs, const float *xwt) {
    const float pi = 3.14159265358979323846f;
    const float qstep = q[4] - q[3];
    const float sfac = 0.5f * qstep / pi / pi / rho;
    for (int j = 1; j <= nr; ++j) {
        const float rr = r[j];
        for (int in = 0; in < npairs; ++in) {
            const float qmax = pi / q[nqmax[in]];
            const float *s = sofq + (size_t)in * ldq;
            float sumi = 0.0f;
            for (int i = nqmin[in]; i <= nqmax[in]; ++i) {
                const float qq = q[i];
                float prod;
                if (rr > 0.0f) {
                    float qr = qq * rr;
                    prod = qq * sinf(qr) * lorch(qmax * qq, pi);
                } else {
                    prod = qq * qq * lorch(qmax * qq, pi);
                }
                sumi = sumi + s[i] * prod;
            }
            float g;
            if (rr > 0.0f) g = xwt[in] + sfac * sumi / rr;
            else g = xwt[in] + sfac * sumi;
            gofr[(size_t)in * (nr + 1) + j] = g;
        }
    }
}

/* ------------------------------------------------------------------ fit_expansion */
/* epsr_standalone_rev3.py:4806-4940 and smoop auxiliary_routines.py:744-763.
 * yin [npt+1], expr [npt*nterms+1] (1-based flat), yout [npt+1], wt/wtold [nterms+1].
 * scal[4] in/out = {stepr, acceptr, rejrat, chisqnew}.  Returns the number of trials. */
static float expand(int nterms, int j, const float *expr, const float *coeff, float summax) {
    float sum = 0.0f;
    const float *e = expr + (size_t)(j - 1) * nterms + 1;
    for (int i = 0; i < nterms; ++i) {
        sum = sum + e[i] * coeff[i + 1];
        if (fabsf(sum) > summax) sum = f_sign(summax, sum);
    }
    return sum;
}

static void smoop(int nqmin, int nqmax, int nsmoo, float *diff) {
    int n1 = nqmin, n2 = nqmax;
    if (n2 - 2 < n1 || nsmoo == 0) return;
    for (int it = 0; it < nsmoo; ++it) {
        float sm = 0.0f, sn = diff[n1];
        float sum1 = 0.25f * (sm + sn);
        for (int i = n1; i <= n2; ++i) {
            sm = sn;
            int j = i + 1;
            sn = j <= n2 ? diff[j] : 0.0f;
            float sum2 = 0.25f * (sm + sn);
            diff[i] = sum1 + sum2;
            sum1 = sum2;
        }
    }
}

/* chi^2 over rows nmin..npt of (yin - expand)^2: the reference's sequential float sum, or
 * (fast) the same float32 squares summed in double and rounded once to float32 -- the
 * summation the device's fast fit mode uses inside its trial loop. */
static float fit_chisq(const float *yin, const float *expr, const float *wt, int nmin, int npt, int nterms,
                       float summax, int fast) {
    if (fast) {
        double c = 0.0;
        for (int i = nmin; i <= npt; ++i) {
            float term = yin[i] - expand(nterms, i, expr, wt, summax);
            c += (double)(term * term);
        }
        return (float)c;
    }
    float c = 0.0f;
    for (int i = nmin; i <= npt; ++i) {
        float term = yin[i] - expand(nterms, i, expr, wt, summax);
        c = c + term * term;
    }
    return c;
}

int64_t oracle_fit_expansion_mode(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                                  float *scal, int nmin, int npt, int ncfirst, int nterms, int nits, int nfreq,
                                  oracle_ran1_state *R, int fast);

int64_t oracle_fit_expansion(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                             float *scal, int nmin, int npt, int ncfirst, int nterms, int nits, int nfreq,
                             oracle_ran1_state *R) {
    return oracle_fit_expansion_mode(yin, expr, yout, wt, wtold, scal, nmin, npt, ncfirst, nterms, nits, nfreq, R,
                                     0);
}

int64_t oracle_fit_expansion_mode(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                                  float *scal, int nmin, int npt, int ncfirst, int nterms, int nits, int nfreq,
                                  oracle_ran1_state *R, int fast) {
    const float summax = expf(25.0f);
    const int nstep = 100, ntry = 150;
    float stepr = scal[0];
    float acceptr = 0.05f;
    float rejrat = scal[2];
    float chisqnew = scal[3];
    const int npoints = npt - nmin + 1;
    int64_t trials = 0;
    float wtmax = 0.0f;
    for (int it = 1; it <= nterms; ++it) {
        wt[it] = wtold[it];
        float a = fabsf(wt[it]);
        wtmax = (a >= wtmax) ? a : wtmax;
    }
    if (stepr < 1.0e-6f * wtmax) stepr = 2.0e-6f * wtmax;
    if (nits > 0) {
        float chisqold;
        int icount = 0;
        chisqnew = fit_chisq(yin, expr, wt, nmin, npt, nterms, summax, fast);
        chisqold = chisqnew;
        float chisqtest = -1.0f, chisqfinish = 0.0f;
        int itry = 0;
        while (itry < 10 || (itry < ntry && chisqtest < 1.0e-4f)) {
            itry++;
            float accept = acceptr * chisqold / (float)npoints;
            rejrat = 0.0f;
            float chisqstart = chisqold / (float)npoints;
            for (int it = 1; it <= nstep; ++it) {
                trials++;
                for (int ic = ncfirst; ic <= nterms; ++ic) {
                    if (fabsf(wtold[ic]) < 1.0f)
                        wt[ic] = wtold[ic] + stepr * (2.0f * oracle_ran1(R) - 1.0f);
                    else
                        wt[ic] = wtold[ic] * (1.0f + stepr * (2.0f * oracle_ran1(R) - 1.0f));
                }
                chisqnew = fit_chisq(yin, expr, wt, nmin, npt, nterms, summax, fast);
                float exponent = (chisqnew - chisqold) / accept;
                float test;
                if (exponent > 0.0f && exponent <= 20.0f) test = expf(-exponent) - oracle_ran1(R);
                else if (exponent > 20.0f) test = -1.0f;
                else test = 1.0f;
                if (test >= 0.0f) {
                    icount++;
                    if (icount == nfreq) {
                        icount = 0;
                        smoop(ncfirst, nterms, 1, wt);
                        chisqnew = fit_chisq(yin, expr, wt, nmin, npt, nterms, summax, fast);
                    }
                    chisqold = chisqnew;
                    for (int ic = 1; ic <= nterms; ++ic) wtold[ic] = wt[ic];
                } else {
                    rejrat = rejrat + 1.0f;
                }
            }
            rejrat = rejrat / (float)nstep;
            chisqfinish = chisqold / (float)npoints;
            if (chisqstart > 0.0f) chisqtest = (chisqfinish - chisqstart) / chisqstart;
            else chisqtest = chisqfinish - chisqstart;
            float rejfac = rejrat > 0.0f ? 0.75f / rejrat : 2.0f;
            stepr = stepr * rejfac;
        }
        for (int ic = 1; ic <= nterms; ++ic) wt[ic] = wtold[ic];
    }
    chisqnew = 0.0f;
    for (int i = 1; i <= npt; ++i) {
        float term = expand(nterms, i, expr, wt, summax);
        yout[i] = term;
        if (i >= nmin) {
            float d = yin[i] - term;
            chisqnew = chisqnew + d * d;
        }
    }
    scal[0] = stepr;
    scal[1] = acceptr;
    scal[2] = rejrat;
    scal[3] = chisqnew;
    return trials;
}

/* FP64 en_mole_pair at the current coordinates; out2 = {energy, sum of |terms|}. */
void oracle_en_mole_pair64(const oracle_sys *S, int im, int jm, double *out2) {
    double sc = 0.0;
    const int a0 = S->naf[im];
    out2[0] = en_mole_pair64(S, im, S->xa + a0, S->ya + a0, S->za + a0, S->xadd[im], S->yadd[im], S->zadd[im], jm,
                             &sc);
    out2[1] = sc;
}
