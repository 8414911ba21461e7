"""CPU model of the speculative molfit cycle (csrc/mc_spec.cu) against the reference.

The device path computes every proposal and every pair energy of a cycle up front and then
only resolves the accept decisions in visit order.  This model follows the same phases with
the oracle's pair energies and checks that the resolved cycle reproduces the reference's
cycle (golden coordinates, stored energies, decisions, counters) -- i.e. that the decomposition
itself (which partner position and which stored energy each move sees, and which move's value
a shared energy slot keeps) is exact.
"""

import numpy as np
import pytest

from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
from oracle import oracle
from tests import goldens
from tests.goldens import assert_bits_equal

f32 = np.float32
W = 32


def model_cycle(box, cells, st, mc, ran1, cosv):
    N, M = box.nmol, st["nnbrefmax"]
    visit = cells["cell_mols"]
    vpos = np.empty(N, np.int64)
    vpos[visit] = np.arange(N)
    nmt = box.nmoltype
    rot = [(mc["stepr"] > 0 and box.nato[m] > 1) for m in visit]
    nd = np.array([(3 if r else 0) + (3 if mc["stepm"] > 0 else 0) + 1 for r in rot])
    off = np.concatenate([[0], np.cumsum(nd)])
    draws, ran1_next = oracle.ran1_fill(ran1, int(off[-1]))
    tmax, tmin = trsteps(box.natomr)
    rotstep = mc["wholerot"].astype(f32).copy()
    transstep = mc["wholetrans"].astype(f32).copy()
    for t in range(nmt):
        ms = [m for m in visit if box.mtype[m] == t]
        if ms and mc["stepr"] > 0 and box.nato[ms[0]] > 1 and rotstep[t] <= 0:
            rotstep[t] = f32(1e-5)
        if ms and mc["stepm"] > 0 and transstep[t] <= 0:
            transstep[t] = tmin
    pi = f32(np.pi)
    # proposals
    new_off = {}
    new_c = {}
    kr = 0
    for k, m in enumerate(visit):
        a0, n, t = box.naf[m], box.nato[m], box.mtype[m]
        x, y, z = box.xa[a0:a0 + n].copy(), box.ya[a0:a0 + n].copy(), box.za[a0:a0 + n].copy()
        u = draws[off[k]:off[k + 1]]
        q = 0
        if rot[k]:
            for ax in range(3):
                phi = pi * rotstep[t] * (f32(2.0) * u[q] - f32(1.0))
                q += 1
                c = cosv[3 * kr + ax]
                s = f32(np.copysign(np.sqrt(f32(1.0) - c * c, dtype=f32), phi))
                if ax == 0:
                    x, y = x * c - y * s, x * s + y * c
                elif ax == 1:
                    z, x = z * c - x * s, z * s + x * c
                else:
                    y, z = y * c - z * s, y * s + z * c
            kr += 1
        cx, cy, cz = box.xadd[m], box.yadd[m], box.zadd[m]
        stt = transstep[t]
        cz = cz + stt * (f32(2.0) * u[q] - f32(1.0))
        cy = cy + stt * (f32(2.0) * u[q + 1] - f32(1.0))
        cx = cx + stt * (f32(2.0) * u[q + 2] - f32(1.0))
        new_off[m] = (x.astype(f32), y.astype(f32), z.astype(f32))
        new_c[m] = (f32(cx), f32(cy), f32(cz))

    def energy(m, p, p_new):
        b = box.copy()
        a0, n = b.naf[m], b.nato[m]
        b.xa[a0:a0 + n], b.ya[a0:a0 + n], b.za[a0:a0 + n] = new_off[m]
        b.xadd[m], b.yadd[m], b.zadd[m] = new_c[m]
        if p_new:
            a0, n = b.naf[p], b.nato[p]
            b.xa[a0:a0 + n], b.ya[a0:a0 + n], b.za[a0:a0 + n] = new_off[p]
            b.xadd[p], b.yadd[p], b.zadd[p] = new_c[p]
        return f32(f32(0.0) + oracle.en_mole_pair(b, m, p))

    mol, ref, erg = st["molergpair"], st["ergpairref"], st["ergpair"]
    nn = st["nergpairm"]
    # mirror entries: the partner's slot that references the same energy
    owner = {}
    for m in range(N):
        for s in range(nn[m]):
            owner.setdefault(int(ref[m, s]), []).append((m, s))
    A, B = {}, {}
    for k, m in enumerate(visit):
        for s in range(1, nn[m]):
            p = int(mol[m, s])
            A[(m, s)] = energy(m, p, False)
            if vpos[p] < k:
                B[(m, s)] = energy(m, p, True)
    acc = np.zeros(N, bool)
    fd = np.zeros(N, f32)
    scale = np.zeros(N)
    temp = f32(1.0) / box.simt
    for k, m in enumerate(visit):
        tot = 0.0
        for s in range(1, nn[m]):
            p = int(mol[m, s])
            S = float(erg[ref[m, s] - 1])
            if vpos[p] < k and acc[vpos[p]]:
                (pm, ps), = [o for o in owner[int(ref[m, s])] if o[0] == p]
                old = float(A[(p, ps)]) if ps >= 1 else S
                new = float(B[(m, s)])
            else:
                old, new = S, float(A[(m, s)])
            tot += new - old
            scale[k] += abs(new) + abs(old)
        fd[k] = f32(tot)
        ediff = (fd[k] + f32(0.0)) * temp
        u = draws[off[k + 1] - 1]
        etest = f32(10.0) if ediff <= 0 else (f32(np.exp(-np.float64(ediff))) if ediff < 20 else f32(0.0))
        acc[k] = u < etest
    # commit
    for k, m in enumerate(visit):
        if acc[k]:
            a0, n = box.naf[m], box.nato[m]
            box.xa[a0:a0 + n], box.ya[a0:a0 + n], box.za[a0:a0 + n] = new_off[m]
            box.xadd[m], box.yadd[m], box.zadd[m] = new_c[m]
    for m in range(N):
        km = vpos[m]
        if not acc[km]:
            continue
        for s in range(1, nn[m]):
            p = int(mol[m, s])
            kp = vpos[p]
            (pm, ps), = [o for o in owner[int(ref[m, s])] if o[0] == p]
            p_writes = acc[kp] and ps >= 1
            if p_writes and kp > km:
                continue
            erg[ref[m, s] - 1] = B[(m, s)] if (kp < km and acc[kp]) else A[(m, s)]
    return acc, fd, scale, ran1_next


@pytest.mark.parametrize("case", ["c1_water", "silica", "mix_small"])
def test_speculative_cycle_model_matches_reference(case):
    z = goldens.load(case)
    box = BoxArrays.from_golden(z)
    cells = oracle.cell_list(box, int(z["in_nmolcell"]), f32(z["in_sepmax"]))
    st = oracle.fmolec1(box, cells, z["in_eintra"])
    mc = dict(stepr=f32(z["in_stepr"]), stepm=f32(z["in_stepm"]), wholerot=z["in_wholerot"],
              wholetrans=z["in_wholetrans"])
    ran1 = Ran1State.from_golden(z, "mf_ran1_before_")
    acc, fd, scale, _ = model_cycle(box, cells, st, mc, ran1, z["mf0_cos"])
    for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
        assert_bits_equal(getattr(box, k), z["mf0_" + k], k)
    assert_bits_equal(st["ergpair"][: st["nergpair"]], z["mf0_ergpair"], "ergpair")
    tol = 1e-5 * scale + 1e-6
    assert np.all(np.abs(fd - z["mf0_den"]) <= tol)
