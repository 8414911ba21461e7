"""The batched checkerboard Monte Carlo (csrc/batch.cu) against its NumPy restatement
(oracle/batch_ref.py) and the C oracle's FP64 pair energies, on three small boxes of
different kinds packed together (100 water, 240-atom SiO2-like, 20 DMSO + 40 water):

* the cell grid of every box keeps cells of one colour at least the interaction range apart;
* the binning, every proposal (molecule picked, rotation, translation, left-cell flag) and the
  radial-histogram features are bit-identical to the restatement;
* every energy change is within 1e-5 of the FP64 change (relative to the sum of |pair
  energies|), every decision is the Metropolis rule on the device's own change and the slot's
  draw, and a decision differs from the FP64 one only where the draw sits within that
  tolerance of the threshold; the coordinates after the step are the restatement's;
* the running total energy follows the from-scratch total over many sweeps, and the sweep
  replayed from a CUDA graph continues the same chain as the direct launches."""

import math

import numpy as np
import pytest
import torch

from oracle import batch_ref, oracle

pytestmark = pytest.mark.gpu
f32 = np.float32
RTOL = 1e-5


def _systems():
    from epsr_python_translation_b200 import configs
    return [configs.c1_water(seed=11), configs.silica(seed=12, natom=240),
            configs.c2_mixture(seed=13, ndmso=20, nwater=40)]


def _desc(bb, b):
    d = bb.descs[b]
    return dict(key0=d.key0, key1=d.key1, ncell=d.ncell, stride=d.stride, rotmax=d.rotmax, transmax=d.transmax,
                rfeat=d.rfeat, dmax=d.dmax, beta=d.beta, nslot=d.nslot, slot0=d.slot0)


def _box_arrays(s, co, b, bb):
    ms, as_ = bb.box_slices(b)
    return dict(xa=co["xa"][as_], ya=co["ya"][as_], za=co["za"][as_], xadd=co["xadd"][ms], yadd=co["yadd"][ms],
                zadd=co["zadd"][ms], naf=s.naf, nato=s.nato)


_TEMPLATES = {}


def _pair_energy64(s, posA, posB, tA, tB):
    """FP64 energy of two molecules' atoms through the C oracle's restatement (a two-molecule
    stand-in box sharing the system's tables)."""
    import dataclasses

    from epsr_python_translation_b200.box import BoxArrays
    if id(s) not in _TEMPLATES:
        _TEMPLATES[id(s)] = BoxArrays.from_system(s)
    nA, nB = posA.shape[0], posB.shape[0]
    p = np.concatenate([posA, posB]).astype(f32)
    box = dataclasses.replace(_TEMPLATES[id(s)], naf=np.array([0, nA], np.int32), nato=np.array([nA, nB], np.int32),
                              mtype=np.zeros(2, np.int32), itype=np.concatenate([tA, tB]).astype(np.int32),
                              xa=p[:, 0].copy(), ya=p[:, 1].copy(), za=p[:, 2].copy(), xadd=np.zeros(2, f32),
                              yadd=np.zeros(2, f32), zadd=np.zeros(2, f32))
    return oracle.en_mole_pair64(box, 0, 1)


@pytest.fixture(scope="module")
def bb():
    from epsr_python_translation_b200.batch import BatchBoxes
    return BatchBoxes(_systems(), rot_deg=20.0, trans_A=0.6, seed=5)


def test_grid_colours_are_independent(bb):
    for b, d in enumerate(bb.descs):
        s = bb.systems[b]
        a = 1.0 / d.ncell
        assert d.ncell % d.stride == 0
        # two cells of one colour are (stride-1) cells apart: beyond the cutoff and both radii
        assert (d.stride - 1) * a >= (d.izcut + 1) * d.stepcl - 1e-7
        assert d.nslot == (d.ncell // d.stride) ** 3 >= 1, (s.name, d.ncell, d.stride)


def test_total_energy_matches_fp64(bb):
    e = bb.total_energy().cpu().numpy()
    bb.check_status()
    for b, s in enumerate(bb.systems):
        from epsr_python_translation_b200.box import BoxArrays
        box = BoxArrays.from_system(s)
        tot, scale = 0.0, 0.0
        for i in range(s.nmol):
            for j in range(i + 1, s.nmol):
                v, sc = oracle.en_mole_pair64(box, i, j)
                tot += v
                scale += sc
        assert abs(e[b] - tot) <= RTOL * scale + 1e-6, (s.name, e[b], tot)


def test_step_proposals_features_decisions(bb):
    """Eight steps of one sweep, each checked in full (every box has few slots, so several
    steps are needed to see many moves)."""
    torch.cuda.synchronize()
    sweep = int(bb.sweep_counter.item())
    bb.begin_sweep()
    x, y = bb.feature_buffers()
    seen = 0
    for step in range(8):
        seen += _check_step(bb, sweep, step, x)
    bb.end_sweep()
    assert seen >= 6, seen


def _check_step(bb, sweep, step, x):
    co = bb.download()
    bb.propose(step, x)
    torch.cuda.synchronize()
    bb.check_status()
    slot_mol = bb.slot_mol.cpu().numpy()
    slot_new = bb.slot_new.cpu().numpy().reshape(bb.nslot, 64, 4)
    slot_off = bb.slot_off.cpu().numpy().reshape(bb.nslot, 64, 4)
    slot_centre = bb.slot_centre.cpu().numpy().reshape(bb.nslot, 4)
    feats = x.float().cpu().numpy()
    props = {}
    for b, s in enumerate(bb.systems):
        d = _desc(bb, b)
        shift, coff = batch_ref.begin(d, sweep)
        box = _box_arrays(s, co, b, bb)
        cells = batch_ref.bin_cells(d, shift, box["xadd"], box["yadd"], box["zadd"])
        ms, as_ = bb.box_slices(b)
        pos = co["pos"][as_, :3]
        fclass = bb.fclass.cpu().numpy()[as_]
        for j in range(d["nslot"]):
            k = d["slot0"] + j
            ix, iy, iz = batch_ref.slot_cell(d, coff, step, j)
            n = d["ncell"]
            members = cells[(ix * n + iy) * n + iz]
            pr = batch_ref.propose(d, sweep, step, k, members, box)
            if pr is None:
                assert slot_mol[k] == -1
                continue
            left = batch_ref.left_cell(d, shift, pr, (ix, iy, iz))
            assert slot_mol[k] == (-2 if left else pr["mol"] + ms.start), (s.name, k)
            na = pr["new"].shape[0]
            assert np.array_equal(slot_new[k, :na, :3].view(np.uint32), pr["new"].view(np.uint32)), (s.name, k)
            assert np.array_equal(slot_off[k, :na, :3].view(np.uint32), pr["off"].view(np.uint32))
            assert np.array_equal(slot_centre[k, :3].view(np.uint32), pr["centre"].view(np.uint32))
            if left:
                assert not np.any(feats[2 * k])
                continue
            # features against every other molecule of the box (the device scans cells in
            # range; molecules beyond 8 A contribute nothing)
            h = batch_ref.features(d, pr, box, pos, fclass, range(s.nmol))
            assert np.array_equal(feats[2 * k], (h * 0.25).astype(f32)), (s.name, k)
            assert np.array_equal(feats[2 * k + 1], np.concatenate([h[640:], h[:640]]).astype(f32) * f32(0.25))
            props[k] = (b, pr)
    # decisions: the FP64 energy change of each move against every other molecule
    e0 = bb.energy.clone()
    bb.decide(step, 0)
    torch.cuda.synchronize()
    bb.check_status()
    co2 = bb.download()
    parted = False
    for k, (b, pr) in props.items():
        s = bb.systems[b]
        d = _desc(bb, b)
        ms, as_ = bb.box_slices(b)
        box = _box_arrays(s, co, b, bb)
        mol = pr["mol"]
        a0, na = int(s.naf[mol]), int(s.nato[mol])
        pos = co["pos"][as_, :3]
        de, scale = 0.0, 0.0
        for jm in range(s.nmol):
            if jm == mol:
                continue
            b0, nb = int(s.naf[jm]), int(s.nato[jm])
            en, sn = _pair_energy64(s, pr["new"], pos[b0:b0 + nb], s.itype[a0:a0 + na], s.itype[b0:b0 + nb])
            eo, so = _pair_energy64(s, pos[a0:a0 + na], pos[b0:b0 + nb], s.itype[a0:a0 + na], s.itype[b0:b0 + nb])
            de += en - eo
            scale += sn + so
        _, u2 = batch_ref.decide_draw(d, sweep, step, k)
        x64 = d["beta"] * de
        acc64 = x64 <= 0 or u2 < math.exp(-x64)
        moved = not np.array_equal(co2["xadd"][ms.start + mol:ms.start + mol + 1],
                                   co["xadd"][ms.start + mol:ms.start + mol + 1]) or \
            not np.array_equal(co2["pos"][as_][a0:a0 + na], co["pos"][as_][a0:a0 + na])
        if moved != acc64:
            thr = -math.log(u2) / d["beta"] if u2 > 0 else math.inf
            assert abs(de - thr) <= RTOL * scale + 1e-6, ("decision away from the threshold", s.name, k, de, thr)
            parted = True
            continue
        if moved:
            assert np.array_equal(co2["pos"][as_][a0:a0 + na, :3].view(np.uint32), pr["new"].view(np.uint32))
            assert np.array_equal(co2["xa"][as_][a0:a0 + na].view(np.uint32), pr["off"][:, 0].view(np.uint32))
    # the running energy moved by the accepted changes only
    de_run = (bb.energy - e0).cpu().numpy()
    assert np.all(np.isfinite(de_run))
    del parted
    return len(props)




def test_running_energy_and_graph_replay(bb):
    for _ in range(3):
        bb.sweep("plain")
    run = bb.energy.clone()
    fresh = bb.total_energy().clone()
    bb.check_status()
    scale = np.abs(fresh.cpu().numpy()) + 1.0
    assert np.all(np.abs((run - fresh).cpu().numpy()) <= 1e-5 * scale * 50), (run, fresh)
    # a captured sweep continues the chain exactly as direct launches do
    from epsr_python_translation_b200.batch import BatchBoxes
    a = BatchBoxes(_systems(), rot_deg=20.0, trans_A=0.6, seed=9)
    b = BatchBoxes(_systems(), rot_deg=20.0, trans_A=0.6, seed=9)
    a.total_energy()
    b.total_energy()
    for _ in range(2):
        a.sweep("plain")
    g = b.capture("plain")      # the capture's warm-up runs one sweep directly
    g.replay()
    torch.cuda.synchronize()
    ca, cb = a.download(), b.download()
    for k in ("xadd", "yadd", "zadd", "xa", "pos"):
        assert np.array_equal(ca[k].view(np.uint32), cb[k].view(np.uint32)), k
    c = a.counters_host()
    assert c[:, 0].sum() > 0 and c[:, 2].sum() > 0 and np.all(c[:, 2] <= c[:, 0])


def test_histograms_match_oracle_atogen_all_origins(bb):
    """One launch over every box's atom pairs: the integer counts, normalised as atogen does
    with every molecule an origin, equal the oracle's atogen of each box bit for bit (wav over
    the r grid and potex)."""
    from epsr_python_translation_b200.box import BoxArrays, Ran1State
    for _ in range(2):
        bb.sweep("plain")
    out, pairs = bb.histograms(rminex=-2.0)
    torch.cuda.synchronize()
    co = bb.download()
    for b, s in enumerate(bb.systems):
        ms, as_ = bb.box_slices(b)
        box = BoxArrays.from_system(s)
        for k in ("xa", "ya", "za"):
            getattr(box, k)[:] = co[k][as_]
        for k in ("xadd", "yadd", "zadd"):
            getattr(box, k)[:] = co[k][ms]
        wav, potex, ngr, _ = oracle.atogen(box, s.nmol, Ran1State(idum=-1), np.full(s.npairs, -2.0, f32))
        assert ngr == s.nmol
        dw, dp = out[b]
        npt1 = s.grid["npt1"]
        got = dw.cpu().numpy()
        from tests.goldens import assert_bits_equal
        assert_bits_equal(got[:, :, 1:npt1 + 1], wav[:, :, 1:npt1 + 1], f"{s.name} wav")
        assert_bits_equal(dp.cpu().numpy(), potex, f"{s.name} potex")
        n = s.natom
        intra = int(sum(int(x) * (int(x) - 1) // 2 for x in s.nato))
        assert int(pairs[b].item()) == intra + sum(int(s.nato[i]) * int(np.sum(s.nato[i + 1:])) for i in range(s.nmol))
        del n
