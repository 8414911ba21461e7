/*
 * epsr_gpu.h -- C ABI of the B200 (sm_100a) EPSR minimum-image pair path.
 *
 * Every entry point takes device pointers and sizes, a CUDA stream (as void*, NULL = the
 * legacy default stream) and returns an int status: 0 on success, >0 on an error (text via
 * epsr_last_error()).  Host pointers appear only where an argument's name ends in _host and
 * in the host-side table builders (epsr_calc_pwrexpr_grad, epsr_calc_gaussr_grad,
 * epsr_generate_rp), which take no stream.  No C++ or framework types cross this boundary.  Calls are
 * asynchronous on the given stream unless stated otherwise; the reference's routines are
 * synchronous, so the host bindings synchronise before returning to the reference loop.
 *
 * Index conventions: molecules, atoms, types and pairs are 0-based.  The r-grid index iz
 * and the Q index keep the reference's 1-based meaning: tables are [pair][ld] with iz in
 * 1..npt (element 0 unused) because the bin arithmetic ifix(d/stepcl)+2 depends on it.
 * Coordinates are float32 box-fraction units (x_A/dmax) as in the reference.
 *
 * Each declaration names the reference routine (IzzyRodger-edb/EPSR_python_translation,
 * package src/epsr26) it replaces.
 */
#ifndef EPSR_GPU_H
#define EPSR_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPSR_OK 0
#define EPSR_ERR_ARG 1        /* bad argument (null pointer, size out of range) */
#define EPSR_ERR_CUDA 2       /* a CUDA runtime call failed */
#define EPSR_ERR_CAPACITY 3   /* a caller-sized buffer is too small */
#define EPSR_ERR_UNSUPPORTED 4/* a feature outside the pair path (see epsr_last_error) */
#define EPSR_ERR_TIMEOUT 5    /* a bounded device wait gave up */

/* ------------------------------------------------------------------ shared structs */

/* One periodic box.  All pointers are device pointers. */
typedef struct {
    int32_t nmol, natom, ntype, npairs, nmoltype;
    const int32_t *naf;      /* [nmol] first atom of each molecule */
    const int32_t *nato;     /* [nmol] atoms per molecule */
    const int32_t *mtype;    /* [nmol] molecule type */
    const int32_t *itype;    /* [natom] atom type */
    float *xa, *ya, *za;     /* [natom] atom offsets from the molecule centre */
    float *xadd, *yadd, *zadd; /* [nmol] molecule centres */
    float *pos;              /* [4*natom] scratch: absolute positions (xa+xadd, ..., type bits) */
    const int32_t *npairref; /* [ntype*ntype] pair index of a type pair */
    const float *xstar;      /* [ld] r grid / dmax, 1-based */
    const float *tab;        /* [4*npairs*ld] packed {xavs, xavs1, ecoul, ecoul1} per (pair, iz) */
    int32_t ld;              /* table leading dimension (npt+1) */
    int32_t npt2;            /* last usable table index (epsr16.npt2) */
    int32_t izcut;           /* last iz at which any table entry is nonzero (<= npt2) */
    float stepcl;            /* cellst/dmax */
    int32_t cubic;           /* 1: cubic minimum image; 0: triclinic via lat */
    float lat[6];            /* alatx, blatx, clatx, blaty, claty, clatz (box units) */
    int32_t maxat;           /* largest nato, or 0 (unknown: taken as 64); sizes shared-memory staging */
} epsr_box_t;

/* Cell list (CSR).  cell_mols in cell order is also the molfit visit order. */
typedef struct {
    int32_t ncelldiva, ncelldivb, ncelldivc, ncell, ncellneighb, maxcellno;
    int32_t *molcellno;   /* [nmol] 1-based cell number (atomcellno) */
    int32_t *cell_start;  /* [ncell+1] */
    int32_t *cell_mols;   /* [nmol] */
    int32_t *offsets;     /* [3*ncell] (ia, ib, ic) neighbour-cell offsets, first ncellneighb used */
    int32_t nnbrefmax;    /* largest neighbour-region size (get_nnbrefmax), written by epsr_cell_list */
} epsr_cells_t;

/* Pair-energy store of module ergpairreference (ergpairreference.py:63-210). */
typedef struct {
    int32_t nnbrefmax;    /* slots per molecule (M) */
    int32_t capacity;     /* size of ergpair */
    int32_t *nergpairm;   /* [nmol] used slots */
    int32_t *molergpair;  /* [nmol*M] partner molecule of each slot */
    int32_t *ergpairref;  /* [nmol*M] 1-based index into ergpair */
    float *ergpair;       /* [capacity] shared pair energies */
    int32_t *nergpair;    /* [1] device counter: entries used */
    int32_t *mirror;      /* [nmol*M] or NULL: index (m*M+s) of the partner's entry that
                             shares the same energy slot, -1 for an intramolecular entry;
                             written by epsr_fmolec1, read by the fast molfit path */
} epsr_store_t;

/* ------------------------------------------------------------------ lifecycle / info */

/* Text of the last error on this host thread (static storage). */
const char *epsr_last_error(void);
/* Library version string. */
const char *epsr_version(void);
/* Number of sm_100 devices visible; <0 if the runtime failed. */
int epsr_device_count(void);

/* ------------------------------------------------------------------ ran1 */
/* ran1 auxiliary_routines.py:324-391.  state: device int32[35] = idum, iy, mcall, iv[32].
 * Writes n deviates to out (device) and advances the state by exactly n draws. */
int epsr_ran1_fill(int32_t *state, float *out, int64_t n, void *stream);

/* ------------------------------------------------------------------ cell list */
/* Host-only size computation of initialise_cellneighbourlist cellneighbourlist.py:36-44:
 * dims[4] = ncelldiva, ncelldivb, ncelldivc, ncell. lat6 as in epsr_box_t.lat. */
int epsr_cell_dims(int32_t nmolcell, int32_t nmol, const float *lat6_host, int32_t *dims_host);

/* initialise_cellneighbourlist cellneighbourlist.py:23-90 + makecellneighbourlist :97-183.
 * Counting sort of molecule centres into cells (stable: molecule order within a cell) and
 * the neighbour-cell offsets within rmax.  cells->cell_start/cell_mols/molcellno/offsets are
 * caller-allocated (sizes from epsr_cell_dims); scalar fields are written back on the host
 * (the call synchronises the stream).  lat9 = alatc[3], blatc[3], clatc[3] (host). */
int epsr_cell_list(const float *xadd, const float *yadd, const float *zadd, int32_t nmol, int32_t nmolcell,
                   float rmax, const float *lat6_host, const float *lat9_host, epsr_cells_t *cells,
                   int32_t *scratch_i32, int64_t scratch_len, void *stream);

/* get_nnbrefmax cellneighbourlist.py:211-233 (synchronous; returns the value via out;
 * scratch_i32: one device int). */
int epsr_nnbrefmax(const epsr_cells_t *cells, int32_t *out_host, int32_t *scratch_i32, void *stream);

/* ------------------------------------------------------------------ positions */
/* Refresh box->pos from xa/ya/za + xadd/yadd/zadd (the float adds of en_change
 * molfit.py:855-857).  Call after any host upload of coordinates. */
int epsr_box_positions(const epsr_box_t *box, void *stream);

/* ------------------------------------------------------------------ fmolec1 */
/* fmolec1 ato_manipulation_rev4.py:2374-2528 (intra energies given, no three-body /
 * coordination / container terms): builds the pair store exactly as the reference
 * (intra slot first when nonzero, pairs in cell-visit order, the second-neighbour start of
 * the store loop).  eintra: [nmol] en_mole_intra values.  scratch: device bytes (size from
 * epsr_fmolec1_scratch_bytes).  out2_host[2] = {ftest, ftestb} per molecule.
 * strict=1 sums ftest/ftestb sequentially in the reference's order (bit-identical);
 * strict=0 sums in double.  Synchronous. */
int64_t epsr_fmolec1_scratch_bytes(int32_t nmol, int32_t ncell, int32_t nnbrefmax);
int epsr_fmolec1(const epsr_box_t *box, const epsr_cells_t *cells, const float *eintra, epsr_store_t *store,
                 void *scratch, int64_t scratch_bytes, int32_t strict, float *out2_host, void *stream);

/* ------------------------------------------------------------------ molfit */
/* Step sizes, counters and Metropolis parameters of one molfit cycle. */
typedef struct {
    float simt, rejrate, stepr, stepm, trstepmax, trstepmin;
    int32_t ireset;
    float *wholerot, *wholetrans;   /* [nmoltype] device, updated */
    float *internrot, *interntrans; /* [nmoltype] device, updated (clamped only) */
    int32_t *nwhole, *nmovem;       /* [2*nmoltype] device: tries then rejections */
    int32_t *nstepreject;           /* [nmol] device */
    float *fadds;                   /* [1] device, updated: fadds += sum(accepted dE)/nmol */
    int32_t *ran1;                  /* [35] device ran1 state */
    const float *cos_override;      /* NULL, or [3*nmol] cos values to use instead of the
                                       device cosine (test hook for bit-identity) */
    float *trace_den;               /* NULL or [nmol]: en_change value per move */
    int32_t *trace_acc;             /* NULL or [nmol]: 1 accepted, 0 rejected */
    int32_t strict;                 /* 1: the sequential kernel, en_change summed in list
                                       order (bit-identical); 0: the fast path -- every
                                       proposal and pair energy of the cycle computed in
                                       parallel, decisions resolved in visit order, each
                                       move's change summed in double */
    int32_t *status;                /* [1] device: 0 ok, 1 a molecule exceeds 64 atoms,
                                       2 the fast path's resolver timed out (cycle not applied) */
    /* Internal rotations of rotational groups before each molecule's whole-molecule move
     * (molfit.py:295-360, rotati :589): set intra (NULL: none).  Groups of type ROT or DIH; the
     * dihedral terms of DIH groups (en_mole_dihedral :1353) come from the dihedral block of the
     * epsr_intra_t.  With intra set, every cycle runs the sequential kernel. */
    const void *intra;              /* host pointer to the epsr_intra_t of the intramolecular model (its ngrot) */
    const int32_t *rot_nrf, *rot_nrl;   /* [nmol] first and last group of each molecule (0-based) */
    const int32_t *rot_axis;        /* [ngroups*2] axis atoms (0-based); the rotation is about the first */
    const int32_t *rot_first, *rot_last;    /* [ngroups] range of the group's atoms in rot_atoms */
    const int32_t *rot_atoms;       /* atoms rotated (0-based) */
    float stepri;                   /* > 0 enables internal rotations */
    int32_t rotcycle;               /* nonzero in a cycle where nisum is a multiple of rotfreq */
    int32_t *ninter;                /* [2*nmoltype] device: internal-rotation tries then rejections */
    float *faddbs;                  /* [1] device or NULL: faddbs += sum(accepted intra changes)/nmol */
    /* Draws ahead (fast path only): NULL, or device int32 [80 + ahead_cap].  While a cycle runs,
     * a second stream walks the ran1 stream on from where the cycle's draws end and keeps the
     * values here with the states they start from and lead to; the next cycle takes them when
     * it starts from exactly that state, and walks the stream itself otherwise -- the values
     * are the same either way.  Word 2 counts the cycles that took them.  ahead_cap >= 7*nmol
     * enables it; zero the buffer once before the first cycle. */
    int32_t *ahead;
    int64_t ahead_cap;
} epsr_mc_t;

/* molfit molfit.py:52-541, whole-molecule branch (:268-448) and step adaptation
 * (:465-536): every molecule gets rotatm (:672) + movem (:733), en_change (:806) and the
 * Metropolis test (:401-408) in cell-visit order.  Unsupported (error 4): internal
 * rotations (ngrot>0 with stepri>0), shake cycles (nisum>=intra), tethering, three-body,
 * coordination constraints, container forces, coarse graining -- the host refuses those.
 * scratch: device bytes from epsr_molfit_scratch_bytes. */
int64_t epsr_molfit_scratch_bytes(int32_t nmol, int32_t natom, int32_t nnbrefmax);
/* Bytes of the per-cycle buffers of the fast path for nmoltype molecule types. */
int64_t epsr_molfit_spec_scratch_bytes(int32_t nmol, int32_t natom, int32_t nnbrefmax, int32_t nmoltype);
int epsr_molfit(const epsr_box_t *box, const epsr_cells_t *cells, epsr_store_t *store, epsr_mc_t *mc,
                void *scratch, int64_t scratch_bytes, void *stream);

/* en_change molfit.py:806-919 for one molecule at its current coordinates against its
 * stored list: ergnew out [nnbrefmax] (device; slots 1.. as the reference, slot 0 receives
 * the total), *out_host = dE.  Synchronous. */
int epsr_en_change(const epsr_box_t *box, const epsr_store_t *store, int32_t im, float *ergnew, float *out_host,
                   void *stream);

/* en_mole_pair molfit.py:1528-1578 for n (im, jm) pairs: out[k] = E(im[k], jm[k]). */
int epsr_en_mole_pair(const epsr_box_t *box, const int32_t *im, const int32_t *jm, int32_t n, float *out,
                      void *stream);

/* ------------------------------------------------------------------ intramolecular moves */

/* The intramolecular model of en_atom_intra molfit.py:923-1045 and en_mole_intra :1327
 * (molecom arrays; all pointers device, atoms 0-based).  The dihedral block carries the
 * rotational groups' dihedral angles (molecom labrotdih / ndihedralang / dihedralang): the
 * energy tempdih * simt * en_mole_dihedral (:1345-1348, :1353, DIH groups) of a molecule with
 * groups, and their atom pairs left out of the reference potential (:999-1020); grp_nrf NULL
 * (the block zeroed) for a model without dihedral angles. */
typedef struct {
    const int32_t *nbond;      /* [natom] bonds listed for each atom */
    const int32_t *iabond;     /* [natom*maxbond] 0-based partner atom of each bond */
    const float *tbond;        /* [natom*maxbond] bond length (box units); < 0: a bond-angle pair */
    int32_t maxbond;
    const int32_t *imageatom;  /* [natom] 0-based image atom, -1 for none */
    const int32_t *qtype;      /* [natom] */
    const float *amassa;       /* [ntype] atom masses (centreofmassi) */
    const float *amassr;       /* [npairs] bond weights */
    const float *xav, *xav1;   /* [npairs][box->ld] reference potential of non-bonded intra pairs */
    const int32_t *ngrot;      /* [nmol] rotational groups of each molecule */
    float stepcl;              /* cellst / dmaxmol */
    float sizefactor, tempb, tempang, simt;
    int32_t refine_intra;      /* 1: add refine_intra_fac x EP (box->tab) to non-q pairs */
    float refine_intra_fac;
    int32_t ndih;                       /* dihedral angles over all groups */
    const int32_t *grp_nrf, *grp_nrl;   /* [nmol] first and last group of each molecule (0-based) */
    const int32_t *grp_axis;            /* [ngroups*2] the two base atoms of each group (labaxi) */
    const int32_t *grp_dih0;            /* [ngroups+1] each group's range in dih_* */
    const int32_t *grp_isdih;           /* [ngroups] 1 for a group of type DIH */
    const int32_t *dih_atoms;           /* [ndih*2] orientation atoms io1 (by base atom 1), io2 (by 2) */
    const float *dih_cos, *dih_sin;     /* [ndih] cosf, sinf of the angle (the host C library, as the reference) */
    float tempdih;                      /* molecom.tempdih (tempdihwt * tempb) */
} epsr_intra_t;

/* The molecule centres put back in the box (minimagec minimagec.py:13-62 of xadd, yadd, zadd),
 * as runepsr17 does after an intramolecular cycle (epsr_standalone_rev3.py:1332-1335), and the
 * atom positions refreshed.  Asynchronous. */
int epsr_minimage_centres(const epsr_box_t *box, void *stream);

/* en_mole_intra molfit.py:1327-1350 of every molecule at its current coordinates: out [nmol]
 * device (the intramolecular energies fmolec1 stores first).  Bit-identical.  Asynchronous. */
int epsr_en_mole_intra(const epsr_box_t *box, const epsr_intra_t *intra, float *out, void *stream);

/* The intramolecular cycle of molfit (molfit.py:124-174, taken when nisum >= intra, then the
 * step adaptation :465-536): for every molecule of more than one atom (stepmi > 0) in order,
 * movei :545 (3 ran1 values per atom, z y x), en_change_intra :763 against the first stored
 * energy, the Metropolis test (one ran1 value) and, on acceptance, the store's first entry
 * and centreofmassi ato_manipulation_rev4.py:442.  mc: simt, rejrate, trstepmax/min, ireset,
 * the step arrays (interntrans adapted from this cycle's counts; internrot set to 0 for
 * molecule types without rotational groups), nwhole/nmovem zeroed, fadds, ran1.  nmovei
 * [2*nmoltype] device out (tries, then rejections); faddbs [1] device in/out.  A molecule
 * with an empty pair list before any loaded one compares against 0 (the reference uses
 * whatever its work array last held).  Molecules with rotational groups of type ROT
 * (molfit.py:124-267): in index order, each molecule's atom moves and then, when mc->stepri > 0,
 * its groups rotated (rotati :589, one ran1 value each, mc->cos_override consumed in order when
 * set) and tested on the intramolecular change against ergold(1) plus the intermolecular change
 * over its stored list (en_change :806, summed in list order); mc must then carry the groups
 * (rot_*), ninter (counted and used for internrot's adaptation) and nstepreject, else
 * EPSR_ERR_UNSUPPORTED before any change; fadds gains the accepted intermolecular changes.
 * Bit-identical with the reference's exp values (and, for rotations, its cos values).
 * Synchronous (reads the draw count); scratch from epsr_molfit_shake_scratch_bytes. */
int64_t epsr_molfit_shake_scratch_bytes(int32_t nmol, int32_t natom);
int epsr_molfit_shake(const epsr_box_t *box, epsr_store_t *store, epsr_mc_t *mc, const epsr_intra_t *intra,
                      float stepmi, int32_t *nmovei, float *faddbs, void *scratch, int64_t scratch_bytes,
                      void *stream);

/* ------------------------------------------------------------------ batched checkerboard MC
 * No counterpart in the reference: many independent cubic boxes advanced together by a
 * parallel Metropolis scheme whose sampled distribution is the reference method's (the same
 * tabulated pair energies, bin rule and temperature; molfit.py:401-408 for the test).  Each
 * sweep bins every box's molecule centres into a grid of ncell^3 cells shifted by a random
 * offset; the cells are coloured with stride^3 colours so that two cells of one colour are
 * at least (stride-1) cells apart (>= the box's interaction range rint).  A step moves, in
 * every box, one randomly chosen molecule in every cell of one colour; moves that take a
 * centre out of its cell are rejected.  Moves of one step never interact, so they run in
 * parallel and are exact.  The proposal is symmetric: a rotation by an angle uniform in
 * [-rotmax, rotmax] about a uniformly random axis through the centre, then a translation
 * uniform in [-transmax, transmax]^3 (box units).  Random numbers come from Philox4x32-10
 * keyed by the box and counted by (sweep, step, slot).
 * Delayed acceptance: with a surrogate, a move is first accepted with min(1, exp(-s)) where s
 * is the network's antisymmetric estimate of beta*dE from the radial histograms of the moved
 * molecule (64 bins of 0.125 A to 8 A, 10 element-pair classes, before and after the move),
 * and only then evaluated exactly and accepted with min(1, exp(-(beta*dE - s))), which leaves
 * the sampled distribution exactly that of the single-stage test. */
typedef struct {
    int32_t mol0, nmol, atom0, natom;            /* this box's molecules and atoms in the packed arrays */
    int32_t ncell, stride, cell0, slot0, nslot;  /* cells per side, colour stride, offsets, (ncell/stride)^3 */
    int32_t tab0, ld, izcut, npairref0, ntype, xstar0;   /* tables: float4 offset, ld, cutoff, pair map */
    int32_t nrange, nrange_feat;                 /* cells scanned on each side for energies / features */
    float stepcl, beta, dmax, rint, rfeat;       /* rint, rfeat: box units */
    float rfeat_c;                               /* centre distance beyond which no feature pair exists */
    float rotmax, transmax;                      /* radians, box units */
    uint32_t key0, key1;                         /* Philox key */
    float shift[3];                              /* written by each sweep's binning */
    int32_t colour_off;                          /* written by each sweep's binning */
    int64_t sweep;                               /* the sweep being run (written by the binning) */
} epsr_bmc_box_t;

typedef struct {
    int32_t nbox, nmol, natom, ncell, nslot;
    int32_t threads;              /* threads per move's CTA in propose and decide: 64, 128 or 256 */
    epsr_bmc_box_t *box;          /* [nbox] */
    const int32_t *slot_box;      /* [nslot] box of each slot */
    const int32_t *mol_box;       /* [nmol] box of each molecule */
    const int32_t *naf, *nato;    /* [nmol] first atom (packed index) and atom count (<= 64) */
    const int32_t *fclass;        /* [natom] element class 0..3 of each atom (features) */
    float *xa, *ya, *za;          /* [natom] offsets from the centre (box units) */
    float *xadd, *yadd, *zadd;    /* [nmol] centres in [-0.5, 0.5) */
    float *pos;                   /* [4*natom] absolute positions, w = atom type bits */
    const float *tab;             /* packed float4 tables {xavs, xavs1, ecoul, ecoul1} of every box */
    const float *xstar;           /* packed r grids / dmax */
    const int32_t *npairref;      /* packed type-pair maps */
    int32_t *cell_start;          /* [ncell + nbox] per box ncell^3+1 starts */
    int32_t *cell_mols;           /* [nmol] */
    int32_t *mol_cell;            /* [nmol + 2*ncell + nbox] scratch: cell of each molecule, bin cursors,
                                     then the box of each packed cell (host-written, after the cursors) */
    int32_t *slot_mol;            /* [nslot] molecule moved in the step, -1 none, -2 left its cell */
    float *slot_new;              /* [nslot*64*4] proposed absolute positions */
    float *slot_off;              /* [nslot*64*4] proposed offsets */
    float *slot_centre;           /* [nslot*4] proposed centre */
    double *energy;               /* [nbox] running total energy (kJ/mol) */
    double *emol;                 /* [nmol] scratch of the total-energy kernel */
    long long *counters;          /* [nbox*4] attempts, first-stage accepts, accepts, left-cell */
    int64_t *sweep_counter;       /* [1] sweeps begun */
    int32_t *status;
} epsr_bmc_t;

/* Partial g(r) histograms of every box over all atom pairs (atogen ato_manipulation_rev4.py:
 * 3640-3899 with every molecule an origin: intramolecular pairs once each (nint bin, weight 2
 * at normalisation), intermolecular pairs jm > im, close contacts d*dmax < |rminex|), counted
 * in 64-bit integers, then normalised in float32 as atogen does (:3857-3897, csampled = the
 * atoms of every molecule by type, addwav 2, ycoh 0).  One launch covers every box's pairs.
 * Offsets are per box; types and pairs are box-local indices into the packed arrays; at most
 * 64 pair types per box. */
typedef struct {
    int32_t nitems, tile, max_bins;  /* inter-pass work items, target atoms per item, shared bins per CTA */
    const int32_t *items;            /* [nitems*3] box, first target atom, first origin atom (box-local) */
    const int32_t *hist0;            /* [nbox] box's counts: [2][npairs][ldw] then potex [npairs] (uint64 units) */
    const int32_t *wav0;             /* [nbox] box's wav: [2][npairs][ldw] (float units) */
    const int32_t *npairs, *npt1, *ldw, *pair0, *type0;   /* [nbox] */
    const int32_t *n1extr, *n2extr;  /* packed pair -> box-local types */
    const int32_t *atom_mol;         /* [natom] molecule of each atom (packed index) */
    const float *rminex, *cfrac, *csampled;   /* packed per pair / per type */
    unsigned long long *counts;      /* zeroed inside */
    float *wav, *potex;              /* outputs; potex [sum npairs] */
    long long *pairs;                /* [nbox] pair-updates counted */
} epsr_bmc_hist_t;
int epsr_bmc_histograms(const epsr_bmc_t *b, const epsr_bmc_hist_t *h, int64_t counts_len, void *stream);

/* Bin every box's centres for a new sweep (random shift and colour order per box). */
int epsr_bmc_begin_sweep(const epsr_bmc_t *b, void *stream);
/* Step `step` of the sweep: propose a move per slot; with x (device BF16 [2*nslot][1280],
 * rows 2k and 2k+1 = slot k's features before|after and after|before) also the features. */
int epsr_bmc_propose(const epsr_bmc_t *b, int32_t step, void *x, void *stream);
/* Decide the step's moves.  mode 0: single-stage Metropolis; 1: delayed acceptance with the
 * network outputs y [2*nslot] (s = (y[2k]-y[2k+1])/2); 2: single-stage for training.  target
 * [nslot] (optional in modes 0 and 1, required in 2) receives beta*dE - s for every move that
 * was evaluated exactly (s = 0 outside mode 1) and NaN for the others. */
int epsr_bmc_decide(const epsr_bmc_t *b, int32_t step, int32_t mode, const float *y, float *target, void *stream);
/* The sweep counter advances (after the sweep's steps). */
int epsr_bmc_end_sweep(const epsr_bmc_t *b, void *stream);
/* Total energy of every box from scratch into energy[] (sum over molecule pairs within rint). */
int epsr_bmc_total_energy(const epsr_bmc_t *b, void *stream);

/* ------------------------------------------------------------------ surrogate network
 * No counterpart in the reference: the first-stage screen of the delayed-acceptance Monte
 * Carlo (learned.py) -- a 1280 -> 128 -> 128 -> 1 perceptron with SiLU activations, BF16
 * weights and activations, FP32 accumulation, evaluated and trained by hand-written tcgen05
 * GEMM kernels (TMA-staged operands, accumulators in tensor memory).  All pointers are device
 * memory.  w1 [128][1280], b1 [128], w2 [128][128] (row = output unit), b2 [128], w3 [128],
 * b3 [1] are the FP32 master weights; w1h, w2h (BF16 copies) and w2th (BF16 w2 transposed)
 * are what the kernels read (epsr_mlp_sync_weights refreshes them from the masters; the
 * training step keeps them current).  dw1..db3 are FP32 gradient accumulators of the same
 * shapes (zero before the first training step; each step leaves them zero); m1 and v1 the Adam
 * moments of all parameters packed in the order w1, b1, w2, b2, w3, b3 (165,633 floats
 * each).  status [1]: set to 1 when a bounded wait inside a kernel gave up. */
typedef struct {
    float *w1, *b1, *w2, *b2, *w3, *b3;
    void *w1h, *w2h, *w2th;
    float *dw1, *db1, *dw2, *db2, *dw3, *db3;
    float *m1, *v1;
    int32_t *status;
} epsr_mlp_t;

/* D = A . B^T on the tensor cores, for tests: a [m][k] and b [n][k] row-major BF16 (k a
 * multiple of 64), out [m][ldo] FP32, stored (accumulate = 0) or added atomically (1), with the
 * k range split over kslices CTAs. */
int epsr_umma_gemm_f32(const void *a, int32_t m, const void *b, int32_t n, int32_t k, int32_t kslices, float *out,
                       int32_t ldo, int32_t accumulate, int32_t *status, void *stream);
/* device bytes of the work area for `rows` rows (forward or one training step) */
int64_t epsr_mlp_work_bytes(int32_t rows);
int epsr_mlp_sync_weights(const epsr_mlp_t *net, void *stream);
/* y[r] = net(x[r]) for x [rows][1280] BF16 (16-byte aligned rows). */
int epsr_mlp_forward(const epsr_mlp_t *net, const void *x, int32_t rows, float *y, void *work, int64_t work_bytes,
                     void *stream);
/* One Adam step (lr, bias correction for step >= 1) on rows row0..row0+rows-1 of x [.][1280]
 * (rows and row0 multiples of 128; row pairs 2p, 2p+1 hold the features of one move in both
 * orders) with xt = x transposed ([1280][ldxt] BF16).  The loss is the mean over pairs of
 * ((y(2p) - y(2p+1))/2 - target[row0/2 + p])^2; *loss_out (device, may be null) receives the
 * summed squared error of the batch. */
int epsr_mlp_train_step(const epsr_mlp_t *net, const void *x, const void *xt, int64_t ldxt, int32_t row0,
                        int32_t rows, const float *target, float lr, int32_t step, float *loss_out, void *work,
                        int64_t work_bytes, void *stream);

/* ------------------------------------------------------------------ kernel timing
 * For measurement; no counterpart in the reference.  While enabled, the library brackets each
 * launch of its main kernels (spec_energy_kernel, spec_corr_kernel, spec_resolve_kernel,
 * molfit_seq_kernel, fm_count_kernel, ag_inter_kernel, fitexp_cluster_kernel) with CUDA events
 * recorded on the launch stream.  epsr_timing_enable(1) clears earlier records and starts;
 * epsr_timing_enable(0) stops.  epsr_timing_read waits for the recorded events of one kernel
 * and returns the summed device time and the launch count.  Records are shared by all host
 * threads of the process. */
int epsr_timing_enable(int32_t on);
int epsr_timing_read(const char *kernel, double *total_ms, int64_t *launches);

/* ------------------------------------------------------------------ atogen */
/* atogen ato_manipulation_rev4.py:3640-3899 (no coarse graining, no container forces).
 * wav: device [2*npairs*ldw] (wav(1,iz,ic) at [ic*ldw+iz], wav(2,..) at [(npairs+ic)*ldw+iz]),
 * potex [npairs]; counts: device uint64 [2*npairs*ldw + npairs] integer histogram scratch
 * (zeroed inside).  rminex [npairs] (already through irefpcof), cfrac [ntype], ycoh [ldw].
 * ran1: device state (one draw per origin candidate, as the reference).
 * *ngrsamples_io (host) in/out as the reference's argument.  Synchronous. */
int epsr_atogen(const epsr_box_t *box, int32_t npt1, float sizefactor, float dmax, const float *rminex,
                const float *cfrac, const float *ycoh, const int32_t *n1extr, const int32_t *n2extr,
                int32_t natomr, int32_t *ngrsamples_io, int32_t *ran1, float *wav, int32_t ldw, float *potex,
                unsigned long long *counts, void *scratch, int64_t scratch_bytes, void *stream);
int64_t epsr_atogen_scratch_bytes(int32_t nmol, int32_t natom, int32_t nmoltype, int32_t ntype);
/* pair-updates counted by the last epsr_atogen call on this thread */
int64_t epsr_atogen_last_pair_updates(void);

/* epsr_atogen without caller scratch.  No counterpart in the reference: it exists for callers
 * that cannot allocate device memory for the library -- a plain C, Fortran or ctypes host
 * with no device allocator of its own, or a host whose device memory belongs to another
 * allocator that must not be bypassed.  Arguments and results are those of epsr_atogen
 * minus counts/scratch/scratch_bytes; the results are identical to epsr_atogen's.
 * Working memory is one file-scope device array of 8 MiB per device (4 MiB of histogram counts
 * plus 4 MiB of work space), so the call allocates nothing.  Limits: nmol <= 50000, natom <= 150000 and
 * 2*npairs*ldw + npairs <= 524288; larger boxes return EPSR_ERR_CAPACITY with the limits in
 * epsr_last_error.  Nothing needs to start at zero: the counts are cleared inside each call.
 * Every call looks up the array's address in the current device's context (the device the
 * call runs on must be current); the first call on a device may load the library's device
 * code there, so make that first call before any stream capture.  The array is shared by every call on the
 * device, so two calls that overlap in time (other streams or host threads) race on it and
 * give wrong results: serialise them. */
int epsr_atogen_noalloc(const epsr_box_t *box, int32_t npt1, float sizefactor, float dmax, const float *rminex,
                        const float *cfrac, const float *ycoh, const int32_t *n1extr, const int32_t *n2extr,
                        int32_t natomr, int32_t *ngrsamples_io, int32_t *ran1, float *wav, int32_t ldw,
                        float *potex, void *stream);

/* ------------------------------------------------------------------ press */
/* press ato_manipulation_rev4.py:3903-4062 over the stored pairs (no three-body terms, no
 * coordination constraints): for every molecule but the last and every stored partner
 * jm > im, the energy and virial of all atom pairs with bin iz <= npt1, summed in store
 * order.  sums_host[2] = {sumc (a float32 value), presst}; the caller forms the energy
 * sumc/nmol and the pressure as the reference's closing lines do (:4051-4056).  strict=1
 * sums sumc in float32 and presst in double sequentially (bit-identical); strict=0 sums
 * both in double in parallel.  scratch: device bytes from epsr_press_scratch_bytes.
 * Synchronous. */
int64_t epsr_press_scratch_bytes(int32_t nmol, int32_t nnbrefmax);
int epsr_press(const epsr_box_t *box, const epsr_store_t *store, int32_t npt1, void *scratch,
               int64_t scratch_bytes, int32_t strict, double *sums_host, void *stream);

/* ------------------------------------------------------------------ gensq / stog */
/* gensq epsr_standalone_rev3.py:4731-4802.  fq(j,i) = foqols[j*fq_sj + i*fq_si] (j = r
 * index 1..npt1, i = Q index 1..nq).  sofq out [2*npairs*(nq+1)]: sofq(1,i,ic) at
 * [ic*(nq+1)+i], sofq(2,i,ic) at [(npairs+ic)*(nq+1)+i]. natomsphere [ntype]. */
int epsr_gensq(int32_t nq, int32_t npairs, int32_t npt1, const float *wav, int32_t ldw, const float *foqols,
               int64_t fq_sj, int64_t fq_si, const float *ycoh, const int32_t *n2extr, const float *natomsphere,
               float *sofq, void *stream);

/* ptgnsq epsr_standalone_rev3.py:3844-3867 (the simulated fit of each data set, for the
 * potential refinement): out[d][i] = -(data[d][i] - sum_ic cwt[d][ic] * qwind[ic][i]), the
 * sum sequential over atom pairs ic with the reference's real*8 weights: each step
 * sum = real(dble(sum) + cwt * dble(qwind)).  data, out: [ndata][nq+1] float; cwt:
 * [ndata][npairs] double; qwind: [npairs][nq+1] (the intermolecular S(Q) of gensq).  The Q
 * window of :3856-3867 when q [nq+1] (1-based) is given: per data set nqmin, nqmax [ndata]
 * and szeros [ndata] (each may be NULL: 1, nq, 0) and qmin (the reference's qminptemp: qminp,
 * or qminm when qminp <= 0); with q NULL, out = -(data - sum) at every point.  X-ray data
 * sets (:3850-3852): where xray[d] != 0 the pair weights are wq[d][ic][i] (double,
 * [ndata][npairs][nq+1], x_rayf0.weightx of the set's X-ray file) instead of cwt[d][ic]; wq
 * and xray may be NULL.  Device pointers; asynchronous on `stream`.  Bit-identical. */
int epsr_ptgnsq_difference(int32_t ndata, int32_t npairs, int32_t nq, const float *data, const double *cwt,
                           const float *qwind, const float *q, const int32_t *nqmin, const int32_t *nqmax,
                           const float *szeros, float qmin, const double *wq, const int32_t *xray, float *out,
                           void *stream);

/* stog ato_manipulation_rev4.py:4067-4121 (+ lorch :4113).  q [ldq] 1-based, sofq
 * [npairs*ldq] (sofq(i,in) at [in*ldq+i]), r [nr+1] 1-based, gofr out [npairs*(nr+1)],
 * nqmin/nqmax (device, [npairs] each), xwt [npairs].  scratch: device bytes from
 * epsr_stog_scratch_bytes.  The limits are checked on the device (error via the return of
 * the next synchronising call is not needed: out-of-range limits are clamped to 1..ldq-1). */
int64_t epsr_stog_scratch_bytes(int32_t npairs, int32_t ldq);
int epsr_stog(float rho, const float *q, int32_t ldq, const float *sofq, const float *r, int32_t nr,
              int32_t npairs, const int32_t *nqmin, const int32_t *nqmax, const float *xwt, float *gofr,
              void *scratch, int64_t scratch_bytes, void *stream);

/* ------------------------------------------------------------------ fit_expansion */
/* fit_expansion epsr_standalone_rev3.py:4806-4921 (+ expand :4924, smoop
 * auxiliary_routines.py:744).  yin [npt+1], expr [npt*nterms+1] (1-based flat, row-major by
 * Q row as the reference), yout [npt+1], wt/wtold [nterms+1] (device, 1-based).
 * scal_host[4] in/out = {stepr, acceptr, rejrat, chisqnew}; returns trials via
 * *trials_host.  ran1: device state.  strict=1 sums chi^2 in the reference's row order
 * (bit-identical); strict=0 in double.  Runs on one thread-block cluster whose CTAs keep the
 * basis rows in shared memory (up to 8 CTAs, one row per worker thread: npt <= 8*480).
 * Returns EPSR_ERR_TIMEOUT if a bounded device wait gave up.  Synchronous. */
int epsr_fit_expansion(const float *yin, const float *expr, float *yout, float *wt, float *wtold,
                       float *scal_host, int32_t nmin, int32_t npt, int32_t ncfirst, int32_t nterms, int32_t nits,
                       int32_t nfreq, int32_t *ran1, void *scratch, int64_t scratch_bytes, int32_t strict,
                       int64_t *trials_host, void *stream);
int64_t epsr_fit_expansion_scratch_bytes(int32_t npt, int32_t nterms);

/* fit_expansion for nprob data sets in one launch, in order, on one ran1 stream -- what the
 * reference's successive calls for each data set do (ptgnsq epsr_standalone_rev3.py:3936-3944).
 * yin, yout [nprob*(npt+1)], wt, wtold [nprob*(nterms+1)], scal_host [nprob*4],
 * trials_host [nprob]; expr and the other arguments as epsr_fit_expansion.  Returns
 * EPSR_ERR_TIMEOUT if a bounded device wait gave up.  Synchronous. */
int epsr_fit_expansion_batch(int32_t nprob, const float *yin, const float *expr, float *yout, float *wt,
                             float *wtold, float *scal_host, int32_t nmin, int32_t npt, int32_t ncfirst,
                             int32_t nterms, int32_t nits, int32_t nfreq, int32_t *ran1, void *scratch,
                             int64_t scratch_bytes, int32_t strict, int64_t *trials_host, void *stream);
int64_t epsr_fit_expansion_batch_scratch_bytes(int32_t nprob, int32_t npt, int32_t nterms);

/* ------------------------------------------------------------------ running averages */

/* sumgr epsr_standalone_rev3.py:3578-3637: folds the new partial g(r) (wav/ycoh, 0 where
 * ycoh <= 0) into the running means and error bars, weights fc2 (old) and fc1 (new) as
 * runepsr17 sets them (:1614-1618), and recomputes the zero limit entsig.  wav
 * [2][npairs][ldw]; ycoh [ldw]; gorintra, gorinter, gr2intra, gr2inter, entsig
 * [npairs][ldw] (r index 1-based, points 2..nz updated), in place.  Bit-identical. */
int epsr_sumgr(int32_t nz, int32_t npairs, const float *wav, int32_t ldw, const float *ycoh, double fc1,
               double fc2, float *gorintra, float *gorinter, float *gr2intra, float *gr2inter, float *entsig,
               void *stream);
/* sumsq epsr_standalone_rev3.py:3642-3677: the same for the partial S(Q).  qwind
 * [2][npairs][ldq] (gensq's intra and inter S(Q)); soqintra, soqinter, sq2intra, sq2inter
 * [npairs][ldq] (Q index 1-based, points 1..nq), in place.  Bit-identical. */
int epsr_sumsq(int32_t nq, int32_t npairs, const float *qwind, int32_t ldq, double fc1, double fc2,
               float *soqintra, float *soqinter, float *sq2intra, float *sq2inter, void *stream);

/* ------------------------------------------------------------------ empirical potential */

/* generate_ep epsr_standalone_rev3.py:5876-6022 from the basis matrix the reference builds
 * at its start (calc_pwrexpr_grad / calc_gaussr_grad, below): for every pair, the EP gradient
 * on r points 1..npt2 (expand :4924, clamped at +-exp(25) after every term) x pcoefp(1) x
 * dmax, the potential integrated from the last point, x wfac, x pressfac (abs_energy_ep
 * ato_manipulation_rev4.py:4128 and the rules of :5966-5977), + ecoul, and both
 * forward-difference gradients; multiply_pot_coeffs (:6493) by pressfac; pwtold = the last
 * pair's coefficients with pwtold(1) = 0; and, if changepotfac, the step of *potfac
 * (:6015-6022).  Bit-identical.
 *   expgr    device [npt2][nterms] (the reference's expgr(1..npt2*nterms))
 *   pcoefp   device [nsets][ldc], coefficient ic of set k at [k*ldc + ic] (ic 1..nterms),
 *            updated in place
 *   irefpcof_host  host [npairs]: 0-based coefficient set of each pair (npairs <= 960)
 *   xstar, wfac    device [ld] (1-based r index); ecoul device [npairs][ld]
 *   xavs, xavs1, xavtot, xavtot1  device [npairs][ld], updated in place (the call also reads
 *            entries it does not rewrite, as the reference: xavs1(npt-1), xavtot(npt2+1..npt))
 *   pwtold   device [nterms+1]; potfac device [1] in/out; result device [2] = {energabs,
 *            pressfac}.  1 <= npt2 <= npt-1, npt+1 <= ld.  Asynchronous on `stream`. */
int epsr_generate_ep(int32_t npairs, int32_t npt, int32_t npt2, int32_t nterms, const float *expgr, float *pcoefp,
                     int32_t nsets, int32_t ldc, const int32_t *irefpcof_host, float dmax, const float *xstar,
                     const float *wfac, const float *ecoul, float *xavs, float *xavs1, float *xavtot, float *xavtot1,
                     int32_t ld, float *pwtold, float absolute_energy, float erequnit, float ereqstep,
                     float potfacamp, float *potfac, int32_t changepotfac, float *result, void *stream);

/* The coefficient increment of ptgnsq epsr_standalone_rev3.py:3948-3962 after the fits of all
 * ndata data sets: for each data set id in turn, each coefficient ic = 2..nterms and each pair
 * ip in order, pcoefp(ic, k) += ((pfact * efacp(k)) * cwtpot(ip, id)) * pwtold_id(ic) with k the
 * pair's set: cwtpot is real*8, so the increment is formed in double and rounded once to
 * float32 per step (bit-identical).  pfact is the reference's potadd (= potfac).
 *   pcoefp   device [nsets][ldc] in place; irefpcof_host host [npairs] (0-based sets,
 *            npairs <= 960); efacp device [nsets]; cwtpot device double [ndata][npairs];
 *   pwtold   device [ndata][ldw] (each data set's fitted coefficients, 1-based).
 * Asynchronous on `stream`. */
int epsr_ep_update(int32_t ndata, int32_t npairs, int32_t nterms, float *pcoefp, int32_t nsets, int32_t ldc,
                   const int32_t *irefpcof_host, const float *efacp, const double *cwtpot, const float *pwtold,
                   int32_t ldw, float pfact, void *stream);

/* The packed tables of epsr_box_t.tab from the four tables: tab[(pair*ld + j)*4 + {0,1,2,3}] =
 * {xavs, xavs1, ecoul, ecoul1}[pair*ld + j] (device, [npairs][ld] each; tab 16-byte aligned).
 * No reference counterpart: the reference reads the four arrays directly.  Asynchronous. */
int epsr_pack_tables(int32_t npairs, int32_t ld, const float *xavs, const float *xavs1, const float *ecoul,
                     const float *ecoul1, float *tab, void *stream);

/* The reference potential tables, host pointers throughout: generate_mp ato_manipulation_rev4.py:
 * 2816-2902 (the WCA core xav of intramolecular pairs) then generate_rp epsr_standalone_rev3.py:
 * 5675-5873 (n-6 Lennard-Jones + charged-sphere Coulomb, Gaussians or gauss6pot's modified
 * Morse, the repulsive core, forward-difference gradients).  Tables [npairs][ld] with the r
 * index 1-based; sets are 0-based (irefpcof).  Pairs whose set has rmaxex > 0 (container
 * forces) are outside this path.  Host computation with the C library's single-precision
 * functions, bit-identical. */
typedef struct {
    int32_t npairs, npt, npt2, ld;
    const float *x, *xstar, *wfac, *wfacc;     /* [ld] */
    float power, ecore, dcore, sizefactor, refpotfac, expecf, expecfpwr;
    int32_t harmonic;                          /* repulsive core: 0 exponential, 1 harmonic */
    int32_t modmorse;                          /* addpotential == "modmorse" */
    int32_t coul_intra;
    float coul_intra_fac;
    const int32_t *n1extr, *n2extr;            /* [npairs] 0-based atom types */
    const int32_t *irefpcof;                   /* [npairs] 0-based sets */
    const float *qradius;                      /* [ntype] */
    const float *ecor, *qcor, *dcor;           /* [npairs] */
    const float *coulfac, *pcoefex, *rminex;   /* [nsets] */
    const int32_t *npgauss;                    /* [nsets] */
    int32_t maxgauss;
    const float *wpgauss, *rpgauss, *hpgauss;  /* [nsets][maxgauss] */
    float *epot, *epot1, *ecoul, *ecoul1, *xav, *xav1;   /* out, [npairs][ld] */
} epsr_rp_t;
int epsr_generate_rp(const epsr_rp_t *rp);

/* calc_pwrexpr_grad epsr_standalone_rev3.py:5230-5309 (the power-exponential basis, with the
 * spacing of dnext :5312) and calc_gaussr_grad :5046-5096 (the Gaussian basis): host
 * functions, the C library's logf/expf as the reference.  xin host [lpt+1] (1-based), expr
 * host out [lpt][nterms] (the reference's expr(1..lpt*nterms)); *ncfirst in/out. */
int epsr_calc_pwrexpr_grad(int32_t lpt, int32_t nterms, float dmin, float dstep, float dmax, float sigmab, float rho,
                           const float *xin, float *expr, float rmin, int32_t *ncfirst, float fbroad, float rbroad);
int epsr_calc_gaussr_grad(int32_t lpt, int32_t nterms, float dstep, float dmax, float sigmab, float rho,
                          const float *xin, float *expr, float rmin, int32_t *ncfirst, float fbroad, float rbroad);

/* ------------------------------------------------------------------ one iteration */

/* One EPSR iteration of the path on one box, driven from native code: the iteration body of
 * runepsr17 (epsr_standalone_rev3.py:1235-1842) restricted to this path -- cell list,
 * fmolec1, ntimes molfit cycles, atogen, gensq, the per-data-set differences of ptgnsq,
 * press, fit_expansion over all data sets, the EP refinement (optional), the running averages
 * sumsq and sumgr, stog --
 * each stage the routine of that name
 * above, launched on `stream` from the calling thread.  The caller owns every buffer. */
typedef struct {
    const epsr_box_t *box;
    epsr_mc_t *mc;                    /* mc->ran1: the one ran1 stream of every stage */
    /* cell list */
    int32_t nmolcell;
    float rmax;                       /* sepmax (epsr_standalone_rev3.py:1259), box units */
    float lat6[6], lat9[9];           /* host */
    int32_t *cell_molcellno, *cell_start, *cell_mols, *cell_offsets;
    int32_t *cell_scratch;            /* int32 elements, see epsr_cell_list */
    int64_t cell_scratch_n;
    /* pair store: rows of store_m slots, store_capacity shared energies */
    int32_t store_m, store_capacity;
    int32_t *nergpairm, *molergpair, *ergpairref, *mirror, *nergpair;
    float *ergpair;
    const float *eintra;              /* [nmol] intramolecular energies */
    int32_t ntimes;                   /* molfit cycles per iteration */
    /* atogen */
    int32_t npt1, natomr, ngrsamples;
    float sizefactor, dmax;
    const float *rminex, *cfrac, *ycoh;
    const int32_t *n1extr, *n2extr;
    float *wav;                       /* [2][npairs][ldw] */
    int32_t ldw;
    float *potex;                     /* [npairs] */
    unsigned long long *counts;       /* [2*npairs*ldw + npairs] */
    /* gensq and the data-set differences */
    int32_t nq, ndata;
    const float *foqols;
    int64_t foqols_sj, foqols_si;
    const float *natomsphere;
    float *sofq;                      /* [2][npairs][nq+1] */
    const float *data;                /* [ndata][nq+1] */
    const double *cwt;                /* [ndata][npairs] (real*8, as the reference's weights) */
    float *dt;                        /* [ndata][nq+1] -(data - weighted S(Q)) */
    /* fit_expansion */
    const float *expr;
    int32_t nterms, ncfirst, nits, nfreq;
    float *fit_wt, *fit_wtold, *fit_yout;   /* [ndata][nterms+1], same, [ndata][nq+1] */
    float *fit_scal_host;             /* [ndata][4] host: stepr in/out; acceptr, rejrat, chisq out */
    int64_t *fit_trials_host;         /* [ndata] host */
    /* stog */
    float rho;
    const float *q;                   /* [nq+1] */
    const float *r;                   /* [nr+1] */
    int32_t nr;
    const int32_t *nqmin, *nqmax;     /* [npairs] */
    const float *xwt;                 /* [npairs] */
    float *gofr;                      /* [npairs][nr+1] */
    /* running averages (sumsq, sumgr): nsum is the accumulation count including this step
     * (runepsr17 :1611-1615: fc1 = 1/nsum, fc2 = (nsum-1)*fc1) */
    int32_t nsum;
    float *soqintra, *soqinter, *sq2intra, *sq2inter;           /* [npairs][nq+1] */
    float *gorintra, *gorinter, *gr2intra, *gr2inter, *entsig;  /* [npairs][ldw] */
    /* EP refinement after the fits, when refine != 0: ptgnsq's coefficient increment
     * (:3948-3962, epsr_ep_update) with pfact = potadd, generate_ep(.false.) (:4014) and the
     * repacked box->tab for the next iteration.  Tables [npairs][box->ld]; box->izcut must be
     * box->npt2 (a refined EP's gradient is nonzero at the last table point). */
    int32_t refine;
    float *pcoefp;                    /* [nsets][ldc] */
    int32_t nsets, ldc;
    const int32_t *irefpcof_host;     /* [npairs] host, 0-based */
    const float *efacp;               /* [nsets] */
    const double *cwtpot;             /* [ndata][npairs] (real*8) */
    const float *expgr, *wfac;        /* [npt2][nterms] basis, [ld] truncation */
    const float *ecoul, *ecoul1;      /* [npairs][ld] */
    float *xavs, *xavs1, *xavtot, *xavtot1;   /* [npairs][ld] */
    float *ep_pwtold, *potfac, *ep_result;    /* [nterms+1], [1], [2] = {energabs, pressfac} */
    float pfact, absolute_energy, erequnit, ereqstep, potfacamp;
    float *tab;                       /* box->tab, written */
    /* intramolecular cycles, when intra > 0: molfit's branch when nisum >= intra (molfit.py:
     * 124-174, epsr_molfit_shake) in place of a whole-molecule cycle, nisum kept as the
     * reference's counter (nisum in, rep->nisum out), and after each intramolecular cycle the
     * molecule centres put back in the box and the pair store rebuilt (runepsr17 :1328-1345).
     * With intra > 0 the stored intramolecular energies are intra_model's (epsr_en_mole_intra
     * into eintra_work) instead of eintra. */
    int32_t intra, nisum;
    float stepmi;
    const epsr_intra_t *intra_model;
    float *faddbs;                    /* [1] device */
    float *eintra_work;               /* [nmol] device */
    int32_t *nmovei;                  /* [2*nmoltype] device: the last intramolecular cycle's counts */
    /* one scratch block shared by the stages (epsr_iteration_scratch_bytes) */
    void *scratch;
    int64_t scratch_bytes;
    int32_t strict;
    void *stage_events[20];           /* NULL or CUDA events recorded at the start and end of
                                         cells, fmolec1, molfit, atogen, gensq, press, fit, ep,
                                         sums, stog */
    int32_t rotfreq;                  /* > 0 with mc's rotational groups: internal rotations in the
                                         whole-molecule cycles where nisum is a multiple of rotfreq */
} epsr_iteration_t;

typedef struct {
    int32_t nnbrefmax;                /* region size of this iteration's cell list */
    float ftest[2];                   /* fmolec1's ftest, ftestb */
    int32_t ngrsamples;               /* atogen's sampled origins */
    int64_t pair_updates;             /* atogen's pair-updates */
    double press[2];                  /* press sums: float32 energy sum, double virial sum */
    int32_t nisum;                    /* molfit's counter after the cycles (intra > 0) */
} epsr_iteration_report_t;

int64_t epsr_iteration_scratch_bytes(const epsr_iteration_t *it);
/* Returns EPSR_ERR_CAPACITY, before anything of the box has changed, when this iteration's
 * cell list needs more than store_m slots per molecule (rep->nnbrefmax says how many). */
int epsr_iteration_step(const epsr_iteration_t *it, epsr_iteration_report_t *rep, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* EPSR_GPU_H */
