#!/usr/bin/env python
"""Benchmark of the EPSR pair path on B200: MC molecule-moves/s (+ g(r) pair-updates/s).

One step = one EPSR iteration of the hot path on configuration C2 (200 DMSO + 400 water,
3200 atoms, 21 pair types) for each of R independent boxes on the GPU (``--replicas``,
default 16): cell list, fmolec1, 5 molfit cycles (3000 whole-molecule moves), atogen over
all 5,118,400 atom pairs, gensq, press, fit_expansion for three datasets, stog.  Each box has its
own ran1 seed, CUDA stream and host thread; a box's chain is sequential (Metropolis, one
ran1 stream), so independent boxes are how one GPU is filled.  ``value`` = molecule moves
of all boxes per second of device time, inputs resident in HBM; ``single_box`` reports one
box alone (its stage breakdown feeds the roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--replicas R] [--impl ours|reference]

Under torchrun each rank advances its own R boxes: there is no data-path collective, so
``scaling`` is "weak".  ``--impl reference`` times the reference's algorithm (the C
restatement in oracle/, single-threaded per process) on all host cores with one
independent box per core.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC molecule-moves/s"
# dram__bytes_read.sum + dram__bytes_write.sum of one fitexp_cluster_kernel launch on the C2
# fit, from an ncu --set full capture of one launch (independent of the trial count: the
# basis is read from HBM once per launch)
FIT_DRAM_BYTES_PER_LAUNCH = 409856
# SM cycles per ran1 value of the warp shuffle chain (two shuffles a step) on an otherwise
# idle SM (clock64 timing of 640,000 values)
FIT_CHAIN_CYCLES_PER_VALUE = 40.0
UNIT = "moves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2_mixture")
    ap.add_argument("--replicas", type=int, default=16, help="independent boxes per GPU (one stream each)")
    ap.add_argument("--strict", action="store_true", help="bit-identical sequential sums")
    ap.add_argument("--cpu-sample-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--intra", type=int, default=0,
                    help="flexible molecules: an intramolecular molfit cycle every INTRA cycles (0: rigid)")
    ap.add_argument("--python-driver", action="store_true",
                    help="drive each iteration's routines from Python instead of epsr_iteration_step")
    return ap.parse_args()


# ----------------------------------------------------------------------------- CPU side
def _cpu_worker(args):
    config, seed, steps, warmup, intra = args
    from epsr_python_translation_b200 import configs
    from oracle.workload import CpuIteration
    wl = configs.make_workload(config, intra=intra)
    it = CpuIteration(wl, ran1_seed=seed)
    for _ in range(warmup):
        it.step()
    t0 = time.perf_counter()
    per = []
    for _ in range(steps):
        a = time.perf_counter()
        it.step()
        per.append(time.perf_counter() - a)
    return time.perf_counter() - t0, per, it.stage_s, it.pair_updates, wl.ntimes * wl.system.nmol


def cpu_info():
    model = ""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count() or 1


def cpu_baseline(config, steps, intra=0):
    """Single core: the oracle (C restatement of the reference) on a bounded sample of the
    same workload."""
    wall, per, stages, pairs, moves = _cpu_worker((config, -7, steps, 1, intra))
    model, n = cpu_info()
    ms = 1000.0 * statistics.mean(per)
    return {"value": moves / statistics.mean(per), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} full EPSR iterations of {config} ({moves} moves each) after 1 warm-up, "
                      f"single-threaded C oracle, {ms:.0f} ms/iteration; pair-updates/s "
                      f"{pairs / stages.get('atogen', 1e9):.3e}; host {model}, nproc {n}",
            "stage_s": {k: round(v, 4) for k, v in stages.items()}}


def reference_arm(a):
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    model, ncpu = cpu_info()
    nproc = max(1, ncpu)
    steps, warmup = a.steps, a.warmup
    # bounded: a few minutes at most (one C2 iteration is about 1.4 s on one core)
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_cpu_worker, [(a.config, -(11 + i), steps, warmup, a.intra) for i in range(nproc)])
    wall = time.perf_counter() - t0
    moves = res[0][4]
    slowest = max(r[0] for r in res)
    value = nproc * steps * moves / slowest
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": steps,
        "warmup": warmup, "ms_per_step": 1000.0 * slowest / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded C2 mixture box)",
        "config": {"workload": a.config, "moves_per_step_per_replica": moves, "replicas": nproc,
                   "stages": "cells+fmolec1+5 molfit+atogen+gensq+ptgnsq differences+press+fit_expansion+"
                             "EP refinement+sums+stog"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port",
                         "sample": f"{nproc} independent replicas x {steps} iterations (+{warmup} warm-up) of the "
                                   f"single-threaded C restatement, one process per core; host {model}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 2),
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- GPU side
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = str(index)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9 or f[0] != self.index:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def box_seed(rank, boxes, r):
    """ran1 seed of box r of a rank: distinct over every box of every rank."""
    return -(1 + rank * boxes + r)


def max_over_ranks(x, dist, device):
    """The largest value of x over all ranks (x itself when not distributed)."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gpu_arm(a):
    import threading

    import numpy as np  # noqa: F401
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.iteration import STAGES, EpsrIteration

    wl = configs.make_workload(a.config, intra=a.intra)
    R = max(1, a.replicas)
    # independent boxes (own ran1 seeds), each driven by its own host thread on its own stream
    streams = [torch.cuda.Stream() for _ in range(R)]
    its = []
    for r in range(R):
        with torch.cuda.stream(streams[r]):
            its.append(EpsrIteration(wl, strict=a.strict, ran1_seed=box_seed(rank, R, r), native=not a.python_driver))
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2
    main = torch.cuda.current_stream()

    class Boxes:
        """R persistent host threads, one per box; run(body) advances every box by one step
        concurrently and returns the device time of that round (ms)."""

        def __init__(self):
            self.go = [threading.Event() for _ in range(R)]
            self.fin = [threading.Event() for _ in range(R)]
            self.body = None
            self.e0 = None
            self.done = [torch.cuda.Event() for _ in range(R)]
            self.err = []
            self.th = [threading.Thread(target=self._loop, args=(r,), daemon=True) for r in range(R)]
            for t in self.th:
                t.start()

        def _loop(self, r):
            while True:
                self.go[r].wait()
                self.go[r].clear()
                if self.body is None:
                    return
                try:
                    with torch.cuda.stream(streams[r]):
                        streams[r].wait_event(self.e0)
                        self.body(r)
                        self.done[r].record(streams[r])
                except Exception as e:  # reported by run()
                    self.err.append(e)
                self.fin[r].set()

        def run(self, body):
            self.body = body
            self.e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            self.e0.record(main)
            for ev in self.go:
                ev.set()
            for ev in self.fin:
                ev.wait()
                ev.clear()
            if self.err:
                raise self.err[0]
            for ev in self.done:
                main.wait_event(ev)
            e1.record(main)
            e1.synchronize()
            return self.e0.elapsed_time(e1)

        def close(self):
            self.body = None
            for ev in self.go:
                ev.set()
            for t in self.th:
                t.join()

    boxes = Boxes()
    run_round = boxes.run

    for _ in range(max(3, a.warmup)):
        run_round(lambda r: its[r].step())
    torch.cuda.synchronize()

    # ---------------- device-resident timing (value): R boxes x K steps
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    idx = vis.split(",")[local] if vis else str(local)
    clocks = ClockSampler(idx)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    # every box advances through its K iterations independently (no barrier between the boxes'
    # iterations, as replicas of a production run do), each iteration preceded on the box's own
    # stream by a 256 MB write that flushes L2 (inside the timed region)
    flush_box = [torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") for _ in range(R)]

    def free_steps(r):
        for k in range(a.steps):
            flush_box[r].fill_(float(k))
            its[r].step()

    round_ms = [run_round(free_steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    tmax_ms = max_over_ranks(sum(round_ms), dist, "cuda")
    moves = its[0].moves_per_step
    value = world * R * a.steps * moves / (tmax_ms / 1000.0)

    # ---------------- one box alone: stage breakdown and the roofline of the dominant kernel
    it = its[0]
    stage_tot = {k: 0.0 for k in STAGES}
    single_ms = 0.0
    with torch.cuda.stream(streams[0]):
        for k in range(a.steps):
            flush.fill_(float(k))
            streams[0].wait_stream(main)
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record()
            it.step()
            s1.record()
            for st, v in it.stage_ms().items():
                stage_tot[st] += v
            single_ms += s0.elapsed_time(s1)
    torch.cuda.synchronize()

    # ---------------- end to end through the public API with host buffers
    pinned, d2h = [], [0] * R
    for r in range(R):
        co = its[r].d.download_coords()
        pinned.append([torch.from_numpy(co[k]).pin_memory() for k in ("xa", "ya", "za", "xadd", "yadd", "zadd")])
    h2d = sum(p.numel() * 4 for p in pinned[0])

    def e2e_body(r):
        d = its[r].d
        for name, p in zip(("xa", "ya", "za", "xadd", "yadd", "zadd"), pinned[r]):
            getattr(d, name).copy_(p, non_blocking=True)
        d.refresh_positions()
        its[r].step()
        _, d2h[r] = its[r].download_outputs()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    def e2e_free(r):
        for k in range(a.steps):
            flush_box[r].fill_(float(k))
            e2e_body(r)

    e2e_ms = max_over_ranks(run_round(e2e_free), dist, "cuda")
    e2e_value = world * R * a.steps * moves / (e2e_ms / 1000.0)

    boxes.close()
    intra = intra_cycle(it, wl, a) if rank == 0 else None
    stage_ms = {k: v / a.steps for k, v in stage_tot.items()}
    roof, extra = roofline(it, stage_ms, a)
    launches = kernel_launches(it, wl)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": tmax_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": f"synthetic (seeded {a.config} boxes, synthetic data sets)",
            "config": {"workload": a.config, "nmol": it.box.nmol, "natom": it.box.natom, "npairs": it.box.npairs,
                       "molecules": "flexible: every %d-th molfit cycle intramolecular" % a.intra if a.intra > 0
                       else "rigid (whole-molecule moves only)",
                       "moves_per_step_per_box": moves, "boxes_per_gpu": R,
                       "pair_updates_per_step_per_box": it.pair_updates,
                       "stages": f"cells+fmolec1+{wl.ntimes} molfit+atogen+gensq+ptgnsq differences+press+"
                                 f"fit_expansion ({wl.data.shape[0]} data sets)+"
                                 f"{'EP refinement (coefficient increment, generate_ep, packed tables)+' if wl.ep else ''}"
                                 "sums (sumsq, sumgr)+stog",
                       "step": f"one EPSR iteration of each of the {R} independent boxes on this GPU, each box on "
                               "its own stream and host thread; the boxes advance through the K steps independently "
                               "(no barrier between their iterations)",
                       "l2": "flushed before every box iteration by a 256 MB write on the box's stream, inside the "
                             "timed region", "sums": "strict" if a.strict else "fast",
                       "parallelism": f"replicas: {R} boxes per GPU x {world} GPU(s)"},
            "single_box": {"ms_per_step": single_ms / a.steps,
                           "moves_per_s": moves / (single_ms / a.steps / 1000.0),
                           "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
                           "pair_updates_per_s": it.pair_updates / (stage_ms["atogen"] / 1000.0),
                           "mc_moves_per_s_molfit_only": moves / (stage_ms["molfit"] / 1000.0),
                           "fit_trials_per_step": it.fit_trials},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": R * h2d,
                    "d2h_bytes_per_step": sum(d2h)},
            "roofline": roof, **extra,
            "intra_cycle": intra,
            "gpu_launches": launches * a.steps * R,
            "clocks": clk,
        }
        if not a.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(a.config, a.cpu_sample_steps, a.intra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def intra_cycle(it, wl, a):
    """The intramolecular branch of molfit (molfit.py:124-174) on box 0 after the timed steps:
    device time of one cycle over every molecule (CUDA events, after 3 warm-up cycles), and the
    single-threaded C oracle on the same starting state."""
    import numpy as np
    import torch

    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.intra import IntraModel
    from oracle import oracle
    s = wl.system
    m = configs.intra_model(s)
    d = it.d
    model = IntraModel(d, **m)
    stepmi = 1.0
    faddbs = torch.zeros(1, dtype=torch.float32, device=d.dev)
    # start state for the oracle (coordinates, store, steps, ran1) before the timed cycles
    box = it.box.copy()
    for k, v in d.download_coords().items():
        getattr(box, k)[:] = v
    st = d.download_store()
    st = dict(nnbrefmax=st["nnbrefmax"], nergpair=st["nergpair"], nergpairm=st["nergpairm"].astype(np.int32),
              molergpair=np.ascontiguousarray(st["molergpair"], np.int32).reshape(-1),
              ergpairref=np.ascontiguousarray(st["ergpairref"], np.int32).reshape(-1),
              ergpair=st["ergpair"].astype(np.float32).copy())
    mc0 = d.download_mc()
    for _ in range(3):
        model.molfit_shake(stepmi, faddbs)
    torch.cuda.synchronize()
    n = max(3, a.steps)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(n):
        model.molfit_shake(stepmi, faddbs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    moved = int(np.sum(box.nato > 1))
    out = {"ms": ms, "moves_per_s": moved / (ms / 1000.0), "molecules_moved": moved,
           "workload": f"one intramolecular cycle of box 0 ({a.config}: every molecule of more than one atom, "
                       "harmonic bonds and bond-angle pairs of the templates)"}
    if not a.no_cpu_baseline:
        mc = {k: np.array(mc0[k], np.float32) for k in ("wholerot", "wholetrans", "internrot", "interntrans")}
        mc.update(rejrate=np.float32(wl.rejrate), ireset=0)
        t0 = time.perf_counter()
        oracle.molfit_shake(box, st, mc, m, stepmi, mc0["ran1"], 0.0, 0.0)
        out["cpu_ms"] = 1000.0 * (time.perf_counter() - t0)
        out["cpu_kind"] = "port (single-threaded C oracle)"
    return out


def kernel_launches(it, wl):
    """Own kernels launched per step, by stage (matches the ncu launch list of one iteration)."""
    n = 5             # cell list: assign, scan, scatter, sort, offsets
    n += 1            # region count (nnbrefmax)
    n += 12           # fmolec1: positions, radius, regions, count, 2 scans, intra, write, sort, sums, mirror x2
    n += 11 * wl.ntimes  # molfit cycle: plan, ran1 fill + copy, propose, energy, corr, resolve, 2 commits,
    #                      epilogue, sequential retry (launched always, runs only if flagged)
    n += 8            # atogen: positions, ran1, select, intra, molecule map, origin atoms, inter, norm
    n += 2            # gensq, data-set differences (ptgnsq)
    n += 3            # press: positions, pair terms, sums
    n += 1            # fit_expansion: one cluster launch for every data set
    if wl.ep is not None:
        n += 4        # EP refinement: coefficient increment, per-pair rebuild, coefficient scaling, pack
    n += 2            # running averages: sumsq, sumgr
    n += 2            # stog: lorch + stog
    return n


def roofline(it, stage_ms, a):
    """Roofline of the dominant stage (largest share of the step)."""
    import json as _j

    import numpy as np
    peaks = {}
    try:
        peaks = _j.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        src = "of measured"
    except (OSError, ValueError):
        src = "of fallback"
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    fp32_peak = 148 * 128 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12  # Top/s, 1 op/lane/clock
    dom = max(stage_ms, key=stage_ms.get)
    b = it.box
    wl = it.wl
    extra = {"dominant_stage": dom}
    if dom == "molfit":
        # algorithmic bytes of one sweep: per move its stored list (partner, ref, old energy,
        # new energy write: 16 B/entry) and the coordinates of every neighbour atom (16 B/atom)
        st = it.d.download_store()
        nn = st["nergpairm"].astype(np.int64)
        nato = b.nato.astype(np.int64)
        atoms_per_mol = np.array([int(np.sum(nato[st["molergpair"][m, 1:nn[m]]])) for m in range(b.nmol)])
        bytes_sweep = int(np.sum(16 * np.maximum(nn - 1, 0)) + np.sum(16 * atoms_per_mol))
        pairs_sweep = int(np.sum(atoms_per_mol * nato))
        per_launch_ms = stage_ms["molfit"] / wl.ntimes
        ach = bytes_sweep / (per_launch_ms / 1000.0) / 1e9
        extra["fp32_issue"] = {"achieved_Tops": pairs_sweep * 26 / (per_launch_ms / 1000.0) / 1e12,
                               "peak_Tops": fp32_peak, "ops_per_atom_pair": 26,
                               "atom_pairs_per_sweep": pairs_sweep}
        return {"bound": "hbm", "kernel": "molfit_seq_kernel", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": None, "peak_source": src,
                "algorithmic_bytes_per_launch": bytes_sweep, "launch_ms": per_launch_ms}, extra
    if dom == "fit_expansion":
        # one cluster launch per step fits every data set; per trial the basis is read once
        # (npt * nterms * 4 bytes, from shared memory after the first load)
        per_launch_ms = stage_ms["fit_expansion"]
        byt = it.fit_trials * wl.nq * wl.nterms * 4
        ach = byt / (per_launch_ms / 1000.0) / 1e9
        us_trial = 1000.0 * per_launch_ms / max(it.fit_trials, 1)
        extra["fit_us_per_trial"] = us_trial
        # The kernel is latency-bound: every trial consumes nterms+1 ran1 values from one
        # sequential shuffle chain, measured at 40 SM cycles per value on an otherwise idle SM.
        chain_us = (wl.nterms + 1) * FIT_CHAIN_CYCLES_PER_VALUE / (float(peaks.get("sm_max_mhz", 1965.0)))
        extra["fit_chain_bound"] = {"us_per_trial": chain_us, "frac": chain_us / us_trial,
                                    "cycles_per_value": FIT_CHAIN_CYCLES_PER_VALUE}
        return {"bound": "hbm", "kernel": "fitexp_cluster_kernel", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": FIT_DRAM_BYTES_PER_LAUNCH, "peak_source": src,
                "algorithmic_bytes_per_launch": byt, "launch_ms": per_launch_ms}, extra
    if dom == "atogen":
        per_launch_ms = stage_ms["atogen"]
        byt = 16 * b.natom * max(1, b.natom // 256)
        ach = byt / (per_launch_ms / 1000.0) / 1e9
        extra["fp32_issue"] = {"achieved_Tops": it.pair_updates * 17 / (per_launch_ms / 1000.0) / 1e12,
                               "peak_Tops": fp32_peak}
        return {"bound": "hbm", "kernel": "ag_inter_kernel", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": None, "peak_source": src, "algorithmic_bytes_per_launch": byt,
                "launch_ms": per_launch_ms}, extra
    per_launch_ms = stage_ms[dom]
    return {"bound": "hbm", "kernel": dom, "achieved": None, "peak": hbm, "unit": "GB/s", "frac": None,
            "traffic": None, "peak_source": src, "launch_ms": per_launch_ms}, extra


def c4_arm(a):
    """Configuration C4: 64 independent boxes of uneven size (300-30,000 atoms, water and SiO2,
    298-1500 K).  A step is, for every box, its cell list, pair store (fmolec1), one molfit
    sweep (the speculative cycle) and atogen over every origin (int64 histogram counts).  The
    boxes are spread over host threads by size (longest first onto the least-loaded thread),
    each thread driving its boxes in turn on its own stream; the threads advance through the K
    steps independently, each box step preceded by an L2-flushing 256 MB write on its stream."""
    import threading

    import numpy as np
    import torch

    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
    from epsr_python_translation_b200.device import DeviceBox
    from oracle import oracle
    torch.cuda.set_device(0)
    systems = configs.c4_batch(seed=1)
    nthreads = max(1, min(a.replicas, len(systems)))
    order = sorted(range(len(systems)), key=lambda i: -systems[i].natom)
    load, groups = [0] * nthreads, [[] for _ in range(nthreads)]
    for i in order:
        t = load.index(min(load))
        groups[t].append(i)
        load[t] += systems[i].natom
    streams = [torch.cuda.Stream() for _ in range(nthreads)]
    boxes = [None] * len(systems)
    eintra = [configs.intra_energies(s) for s in systems]
    for t in range(nthreads):
        with torch.cuda.stream(streams[t]):
            for i in groups[t]:
                s = systems[i]
                d = DeviceBox(BoxArrays.from_system(s))
                tmax, tmin = trsteps(d.host.natomr)
                nmt = s.nmoltype
                d.mc_setup(rejrate=0.75, stepr=1.0, stepm=1.0, wholerot=np.full(nmt, 10.0 / 180.0, np.float32),
                           wholetrans=np.full(nmt, 0.5, np.float32) / np.float32(s.dmax), ran1=Ran1State(idum=-(i + 1)),
                           trstepmax=tmax, trstepmin=tmin)
                boxes[i] = d
    rminex = [torch.full((s.npairs,), -2.0, dtype=torch.float32, device="cuda") for s in systems]
    flush = [torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") for _ in range(nthreads)]
    pupd = [0] * len(systems)

    def box_step(i, k, t):
        d = boxes[i]
        flush[t].fill_(float(k))
        d.cell_list(10, d.host.sepmax)
        d.fmolec1(eintra[i], strict=False)
        d.molfit(strict=False)
        d.atogen(0, d.m_ran1, rminex[i])
        pupd[i] = d.last_pair_updates

    def run(nsteps, k0):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        main = torch.cuda.current_stream()
        e0.record(main)
        errs = []

        def worker(t):
            try:
                with torch.cuda.stream(streams[t]):
                    streams[t].wait_event(e0)
                    for k in range(nsteps):
                        for i in groups[t]:
                            box_step(i, k0 + k, t)
            except Exception as e:   # reported below
                errs.append(e)
        th = [threading.Thread(target=worker, args=(t,)) for t in range(nthreads)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        if errs:
            raise errs[0]
        for s_ in streams:
            main.wait_stream(s_)
        e1.record(main)
        e1.synchronize()
        return e0.elapsed_time(e1)

    run(max(3, a.warmup), 0)
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(vis.split(",")[0] if vis else "0")
    clocks.start()
    time.sleep(0.3)
    ms = run(a.steps, 100)
    clk = clocks.stop()
    moves = sum(s.nmol for s in systems)
    value = a.steps * moves / (ms / 1000.0)
    pairs = sum(pupd)
    fp32_peak = 148 * 128 * 1965.0e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (64 seeded boxes: water and SiO2-like, log-uniform sizes)",
        "config": {"workload": "c4_batch", "boxes": len(systems), "atoms": int(sum(s.natom for s in systems)),
                   "atoms_min_max": [int(min(s.natom for s in systems)), int(max(s.natom for s in systems))],
                   "moves_per_step": moves, "host_threads": nthreads,
                   "step": "every box: cell list, fmolec1, one molfit sweep, atogen over every origin",
                   "l2": "flushed before every box step by a 256 MB write on its stream, inside the timed region",
                   "deviation": "boxes on concurrent streams, not one persistent launch per sweep"},
        "pair_updates_per_s": a.steps * pairs / (ms / 1000.0),
        "fp32_issue_atogen_lower_bound": {"achieved_Tops": 17.0 * a.steps * pairs / (ms / 1000.0) / 1e12,
                                          "peak_Tops": fp32_peak / 1e12, "ops_per_pair_update": 17,
                                          "note": "whole step time charged to atogen's 17 FP32 ops per pair-update"},
        "roofline": None, "clocks": clk,
    }
    if not a.no_cpu_baseline:
        small = sorted(range(len(systems)), key=lambda i: systems[i].natom)[:4]
        t0 = time.perf_counter()
        mv = 0
        for i in small:
            s = systems[i]
            ob = BoxArrays.from_system(s)
            oc = oracle.cell_list(ob, 10, ob.sepmax)
            st = oracle.fmolec1(ob, oc, eintra[i])
            nmt = s.nmoltype
            omc = dict(rejrate=np.float32(0.75), stepr=np.float32(1.0), stepm=np.float32(1.0),
                       wholerot=np.full(nmt, 10.0 / 180.0, np.float32),
                       wholetrans=np.full(nmt, 0.5, np.float32) / np.float32(s.dmax), internrot=np.zeros(nmt, np.float32),
                       interntrans=np.zeros(nmt, np.float32), ireset=0)
            _, _, r = oracle.molfit(ob, oc, st, omc, Ran1State(idum=-(i + 1)), record_cos=False)
            oracle.atogen(ob, 0, r, np.full(s.npairs, -2.0, np.float32))
            mv += s.nmol
        wall = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": mv / wall, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"one step (cell list, fmolec1, sweep, full atogen) of the 4 smallest boxes "
                                          f"({mv} molecules), single-threaded C oracle"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return reference_arm(a)
    if a.config == "c4_batch":
        return c4_arm(a)
    return gpu_arm(a)


if __name__ == "__main__":
    import numpy as np  # noqa: F401  (used by roofline)
    sys.exit(main())
