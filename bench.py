#!/usr/bin/env python
"""Benchmark of the EPSR pair path on B200: MC molecule-moves/s and g(r) pair-updates/s.

Headline workload: configuration C3, 20,000 rigid water (60,000 atoms, L = 84.3 A, EP on,
g(r) bin 0.03 A).  One step = one EPSR iteration of the hot path for each of R independent
boxes on the GPU (``--replicas``): cell list, fmolec1, 100 molfit sweeps (2,000,000
whole-molecule moves), atogen over 1,000 sampled origin molecules, gensq, ptgnsq's
difference, press, fit_expansion against one synthetic S(Q) (1,000 Q points), the EP
refinement, the running averages and stog.  Each box has its own ran1 seed, CUDA stream and
host thread; a box's chain is sequential (Metropolis, one ran1 stream), so independent boxes
are how one GPU is filled.  ``value`` = molecule moves of all boxes per second of device
time, inputs resident in HBM; ``pair_updates_per_s`` the atogen pair-updates of all boxes
per second of the same time; ``single_box`` reports one box alone.  A secondary line
(``secondary``) measures configuration C2 (200 DMSO + 400 water, 16 boxes, 5 sweeps per
iteration) the same way.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c3_water|c2_mixture|c4_batch]
                    [--replicas R] [--sweeps S] [--impl ours|reference]

Under torchrun each rank advances its own R boxes: there is no data-path collective, so
``scaling`` is "weak".  ``--impl reference`` times the reference's algorithm (the C
restatement in oracle/, single-threaded per process) on all host cores with one
independent box per core; at C3 each of its steps is one sweep, and the iteration time is
the sampled sweeps scaled to the iteration's sweep count plus the other stages timed once.
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

METRIC = "MC molecule-moves/s (+ g(r) pair-updates/s)"
# dram__bytes_read.sum + dram__bytes_write.sum of one fitexp_cluster_kernel launch on the C2
# fit, from an ncu --set full capture of one launch (independent of the trial count: the
# basis is read from HBM once per launch)
FIT_DRAM_BYTES_PER_LAUNCH = 409856
# SM cycles per ran1 value of the warp shuffle chain (two shuffles a step) on an otherwise
# idle SM (clock64 timing of 640,000 values)
FIT_CHAIN_CYCLES_PER_VALUE = 40.0
# FP32 operations per atom pair of a pair energy (3 sub, 6 minimum image, 5 d^2, 1 sqrt,
# 2 div, 4 table arithmetic, 2 adds, 1 scale, 2 more) and per atogen pair-update
# dram__bytes_read.sum + dram__bytes_write.sum per atom pair of one spec_energy_kernel launch
# (an ncu capture of one launch), or None while no capture has been taken
SPEC_ENERGY_TRAFFIC_PER_PAIR = None
OPS_PER_ENERGY_PAIR = 26
OPS_PER_PAIR_UPDATE = 17
UNIT = "moves/s"
DEFAULT_SWEEPS = {"c3_water": 100}          # molfit sweeps per iteration (others: 5)
DEFAULT_REPLICAS = {"c3_water": 4, "c2_mixture": 16}
# kernels the library brackets with CUDA events while timing is enabled
TIMED_KERNELS = ("spec_energy_kernel", "spec_corr_kernel", "spec_resolve_kernel", "molfit_seq_kernel",
                 "fm_count_kernel", "ag_inter_kernel", "fitexp_cluster_kernel", "ahead_fill_kernel",
                 "ran1_fill_kernel", "spec_plan_kernel", "spec_propose_kernel", "spec_commit_kernel")
# the ordered walk of spec_resolve_kernel on its own (one warp, rows in shared memory, no far
# parts to wait for), measured on B200: the latency floor of a resolved move
RESOLVE_WALK_CYCLES_PER_MOVE = 88.5
# a dependent warp shuffle on B200 (the step of the ran1 walk)
RAN1_SHUFFLE_CYCLES = 32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3_water")
    ap.add_argument("--replicas", type=int, default=None,
                    help="independent boxes per GPU (one stream each; default 2 at C3, 16 at C2)")
    ap.add_argument("--sweeps", type=int, default=None, help="molfit sweeps per iteration (default 100 at C3, else 5)")
    ap.add_argument("--no-secondary", action="store_true", help="skip the secondary C2 x 16 measurement")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned delayed-acceptance comparison on C5 (learned vs plain ESS/s)")
    ap.add_argument("--c5-boxes", type=int, default=16, help="C5 boxes advanced together by the batched arms")
    ap.add_argument("--c5-spec-boxes", type=int, default=4,
                    help="C5 boxes advanced at once on the reference-order (speculative) path")
    ap.add_argument("--c5-sweeps", type=int, default=200, help="timed sweeps of each C5 arm")
    ap.add_argument("--c5-pairs", type=int, default=1000000, help="(features, beta dE) pairs the surrogate trains on")
    ap.add_argument("--strict", action="store_true", help="bit-identical sequential sums")
    ap.add_argument("--cpu-sample-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--intra", type=int, default=0,
                    help="flexible molecules: an intramolecular molfit cycle every INTRA cycles (0: rigid)")
    ap.add_argument("--python-driver", action="store_true",
                    help="drive each iteration's routines from Python instead of epsr_iteration_step")
    a = ap.parse_args()
    if a.sweeps is None:
        a.sweeps = DEFAULT_SWEEPS.get(a.config, 5)
    if a.replicas is None:
        a.replicas = DEFAULT_REPLICAS.get(a.config, 16)
    return a


# ----------------------------------------------------------------------------- CPU side
SAMPLED_SWEEPS_ABOVE = 5   # iterations with more sweeps than this are timed as a bounded sample


def _cpu_worker(args):
    """One process, one core: the oracle (the C restatement of the reference) on one box.
    Returns (seconds per iteration, stage seconds of one iteration, pair-updates per
    iteration, moves per iteration, sample description).  Iterations of at most
    SAMPLED_SWEEPS_ABOVE sweeps run whole (warmup, then steps timed); longer ones run one
    iteration with a single sweep (its other stages timed once), then warmup + steps single
    sweeps, and the iteration time is those stages plus the mean sweep x the sweep count."""
    config, seed, steps, warmup, intra, sweeps = args
    from epsr_python_translation_b200 import configs
    from oracle.workload import CpuIteration
    wl = configs.make_workload(config, intra=intra, ntimes=sweeps)
    it = CpuIteration(wl, ran1_seed=seed)
    moves = wl.ntimes * wl.system.nmol
    if sweeps <= SAMPLED_SWEEPS_ABOVE:
        for _ in range(warmup):
            it.step()
        per = []
        for _ in range(steps):
            a = time.perf_counter()
            it.step()
            per.append(time.perf_counter() - a)
        return (statistics.mean(per), dict(it.stage_s), it.pair_updates, moves,
                f"{steps} full EPSR iterations of {config} ({moves} moves each) after {warmup} warm-up")
    it.step(sample_sweeps=1)
    fixed = {k: v for k, v in it.stage_s.items() if k != "molfit"}
    for _ in range(warmup):
        it.sweep()
    per = []
    for _ in range(steps):
        a = time.perf_counter()
        it.sweep()
        per.append(time.perf_counter() - a)
    sw = statistics.mean(per)
    stages = dict(fixed, molfit=sw * wl.ntimes)
    return (sum(stages.values()), stages, it.pair_updates, moves,
            f"one {config} iteration sampled: its stages other than molfit timed once, {steps} molfit sweeps "
            f"({wl.system.nmol} moves each) timed after {warmup} warm-up, the iteration = those stages + "
            f"{wl.ntimes} x the mean sweep ({sw:.2f} s)")


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


def cpu_baseline(config, steps, intra=0, sweeps=5):
    """Single core: the oracle (C restatement of the reference) on a bounded sample of the
    same workload."""
    if sweeps > SAMPLED_SWEEPS_ABOVE:
        steps = min(steps, 2)
    t_iter, stages, pairs, moves, sample = _cpu_worker((config, -7, steps, 1, intra, sweeps))
    model, n = cpu_info()
    return {"value": moves / t_iter, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{sample}; single-threaded C oracle, {1000.0 * t_iter:.0f} ms/iteration; pair-updates/s "
                      f"{pairs / stages.get('atogen', 1e9):.3e} (atogen alone); host {model}, nproc {n}",
            "pair_updates_per_s": pairs / t_iter,
            "stage_s": {k: round(v, 4) for k, v in stages.items()}}


def reference_arm(a):
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    model, ncpu = cpu_info()
    nproc = max(1, ncpu)
    steps, warmup = a.steps, a.warmup
    # bounded: a few minutes at most (one C2 iteration is about 1 s on one core; a C3 sweep
    # about 1.3 s, plus about 40 s of set-up and the other stages once)
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_cpu_worker, [(a.config, -(11 + i), steps, warmup, a.intra, a.sweeps) for i in range(nproc)])
    wall = time.perf_counter() - t0
    moves = res[0][3]
    slowest = max(r[0] for r in res)
    value = nproc * moves / slowest
    pairs = nproc * res[0][2] / slowest
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": steps,
        "warmup": warmup, "ms_per_step": 1000.0 * slowest, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {a.config} box per core)",
        "config": {"workload": a.config, "moves_per_step_per_box": moves, "boxes_per_gpu": nproc,
                   "sweeps_per_iteration": a.sweeps,
                   "stages": f"cells+fmolec1+{a.sweeps} molfit+atogen+gensq+ptgnsq differences+press+fit_expansion+"
                             "EP refinement+sums+stog",
                   "parallelism": f"replicas: one box per host core ({nproc})"},
        "pair_updates_per_s": pairs,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port",
                         "sample": f"{nproc} independent boxes, one process per core, each: {res[0][4]}; "
                                   f"the slowest box's iteration time counts; host {model}"},
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


class Replicas:
    """R independent boxes of one workload, each with its own ran1 seed, CUDA stream and
    persistent host thread.  run(body) advances every box by body(r) concurrently and returns
    the device time of that round (ms): events on a common stream that every box stream waits
    on at the start and that waits on every box stream at the end."""

    def __init__(self, wl, R, rank, strict, native):
        import threading

        import torch

        from epsr_python_translation_b200.iteration import EpsrIteration
        self.R = R
        self.streams = [torch.cuda.Stream() for _ in range(R)]
        self.its = []
        for r in range(R):
            with torch.cuda.stream(self.streams[r]):
                self.its.append(EpsrIteration(wl, strict=strict, ran1_seed=box_seed(rank, R, r), native=native))
        torch.cuda.synchronize()
        self.main = torch.cuda.current_stream()
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
        import torch
        while True:
            self.go[r].wait()
            self.go[r].clear()
            if self.body is None:
                return
            try:
                with torch.cuda.stream(self.streams[r]):
                    self.streams[r].wait_event(self.e0)
                    self.body(r)
                    self.done[r].record(self.streams[r])
            except Exception as e:  # reported by run()
                self.err.append(e)
            self.fin[r].set()

    def run(self, body):
        import torch
        self.body = body
        self.e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.e0.record(self.main)
        for ev in self.go:
            ev.set()
        for ev in self.fin:
            ev.wait()
            ev.clear()
        if self.err:
            raise self.err[0]
        for ev in self.done:
            self.main.wait_event(ev)
        e1.record(self.main)
        e1.synchronize()
        return self.e0.elapsed_time(e1)

    def close(self):
        self.body = None
        for ev in self.go:
            ev.set()
        for t in self.th:
            t.join()


def kernel_times(lib):
    """{kernel: (total ms, launches)} of the kernels the library timed."""
    import ctypes as C
    out = {}
    for k in TIMED_KERNELS:
        ms, n = C.c_double(0.0), C.c_int64(0)
        if lib.epsr_timing_read(k.encode(), C.byref(ms), C.byref(n)) == 0 and n.value > 0:
            out[k] = (ms.value, int(n.value))
    return out


def gpu_arm(a):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from epsr_python_translation_b200 import _lib, configs
    from epsr_python_translation_b200.iteration import STAGES
    lib = _lib.load(require_device=True)

    wl = configs.make_workload(a.config, intra=a.intra, ntimes=a.sweeps)
    R = max(1, a.replicas)
    reps = Replicas(wl, R, rank, a.strict, not a.python_driver)
    its, streams, main = reps.its, reps.streams, reps.main
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    for _ in range(max(3, a.warmup)):
        reps.run(lambda r: its[r].step())
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
    # stream by a 256 MB write that flushes L2 (inside the timed region); the library brackets
    # its main kernels with events on their streams meanwhile (kernel_ms)
    flush_box = [torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") for _ in range(R)]

    def free_steps(r):
        for k in range(a.steps):
            flush_box[r].fill_(float(k))
            its[r].step()

    lib.epsr_timing_enable(1)
    round_ms = reps.run(free_steps)
    torch.cuda.synchronize()
    lib.epsr_timing_enable(0)
    ktimes = kernel_times(lib)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    tmax_ms = max_over_ranks(round_ms, dist, "cuda")
    moves = its[0].moves_per_step
    value = world * R * a.steps * moves / (tmax_ms / 1000.0)
    pair_value = world * R * a.steps * its[0].pair_updates / (tmax_ms / 1000.0)

    # ---------------- one box alone: stage breakdown
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

    e2e_ms = max_over_ranks(reps.run(e2e_free), dist, "cuda")
    e2e_value = world * R * a.steps * moves / (e2e_ms / 1000.0)

    reps.close()
    intra = intra_cycle(it, wl, a) if rank == 0 and a.config != "c3_water" else None
    stage_ms = {k: v / a.steps for k, v in stage_tot.items()}
    roof, extra = roofline(it, ktimes, a)
    launches = kernel_launches(it, wl)
    pairs_box, fit_trials = it.pair_updates, it.fit_trials
    secondary = None
    if rank == 0 and world == 1 and a.config != "c2_mixture" and not a.no_secondary:
        del reps, its, it
        torch.cuda.empty_cache()
        secondary = secondary_c2(a)
    learned = None
    if rank == 0 and world == 1 and not a.no_learned:
        torch.cuda.empty_cache()
        learned = learned_c5(a)

    if rank == 0:
        b = wl.system
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": tmax_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": f"synthetic (seeded {a.config} boxes, synthetic data sets)",
            "pair_updates_per_s": pair_value,
            "config": {"workload": a.config, "nmol": int(b.nmol), "natom": int(b.natom), "npairs": int(b.npairs),
                       "molecules": "flexible: every %d-th molfit cycle intramolecular" % a.intra if a.intra > 0
                       else "rigid (whole-molecule moves only)",
                       "sweeps_per_iteration": wl.ntimes, "moves_per_step_per_box": moves, "boxes_per_gpu": R,
                       "pair_updates_per_step_per_box": pairs_box,
                       "stages": f"cells+fmolec1+{wl.ntimes} molfit+atogen+gensq+ptgnsq differences+press+"
                                 f"fit_expansion ({wl.data.shape[0]} data set{'s' if wl.data.shape[0] > 1 else ''})+"
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
                           "pair_updates_per_s_atogen": pairs_box / (stage_ms["atogen"] / 1000.0),
                           "mc_moves_per_s_molfit_only": moves / (stage_ms["molfit"] / 1000.0),
                           "fit_trials_per_step": fit_trials},
            "kernel_ms": {k: {"total_ms": round(v[0], 3), "launches": v[1], "mean_us": round(1000 * v[0] / v[1], 2)}
                          for k, v in ktimes.items()},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": R * h2d,
                    "d2h_bytes_per_step": sum(d2h)},
            "roofline": roof, **extra,
            "intra_cycle": intra,
            "gpu_launches": launches * a.steps * R,
            "clocks": clk,
        }
        if secondary is not None:
            line["secondary"] = secondary
        if learned is not None:
            line["learned_c5"] = learned
        if not a.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(a.config, a.cpu_sample_steps, a.intra, a.sweeps)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def secondary_c2(a):
    """Configuration C2 (200 DMSO + 400 water, 3,200 atoms, 5 sweeps per iteration) on 16
    independent boxes, timed as the headline (no L2 flush difference, same rules)."""
    import torch

    from epsr_python_translation_b200 import configs
    wl = configs.make_workload("c2_mixture", ntimes=5)
    R = 16
    reps = Replicas(wl, R, 0, a.strict, not a.python_driver)
    its = reps.its
    for _ in range(3):
        reps.run(lambda r: its[r].step())
    flush_box = [torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") for _ in range(R)]
    steps = max(5, min(a.steps, 20))

    def free_steps(r):
        for k in range(steps):
            flush_box[r].fill_(float(k))
            its[r].step()

    ms = reps.run(free_steps)
    reps.close()
    moves = its[0].moves_per_step
    return {"workload": "c2_mixture", "boxes_per_gpu": R, "sweeps_per_iteration": 5, "steps": steps,
            "value": R * steps * moves / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
            "pair_updates_per_s": R * steps * its[0].pair_updates / (ms / 1000.0)}


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


def _peaks():
    import json as _j
    try:
        peaks = _j.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        src = "of measured"
    except (OSError, ValueError):
        peaks, src = {}, "of fallback"
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    # FP32 CUDA-core issue peak: 148 SMs x 128 FP32 lanes x the SM clock, one operation per
    # lane per clock (no FMA contraction: the path is built with -fmad=false).  No measured
    # FP32 figure exists for this pool, so this one is nominal.
    fp32 = 148 * 128 * mhz * 1e6 / 1e12
    return hbm, fp32, mhz, src


def spec_energy_pairs(it):
    """Atom pairs one spec_energy_kernel launch evaluates on box ``it`` as it stands: for every
    move k (molecule m in visit order) and stored partner p, E(new m, old p) always and
    E(new m, new p) when p is earlier in the visit order -- na(m) x na(p) atom pairs each.
    Returns (those pairs, stored entries, partner atoms over the entries, atom pairs with each
    entry evaluated once)."""
    import numpy as np
    d = it.d
    st = d.download_store()
    cells = d.download_cells()
    nato = it.box.nato.astype(np.int64)
    visit = cells["cell_mols"][: it.box.nmol]
    vpos = np.empty_like(visit)
    vpos[visit] = np.arange(visit.size)
    nn = st["nergpairm"].astype(np.int64)
    M = st["nnbrefmax"]
    cols = np.arange(M)[None, :]
    valid = (cols >= 1) & (cols < nn[:, None])
    part = np.where(valid, st["molergpair"], 0)
    pa = nato[part] * valid
    earlier = (vpos[part] < vpos[:, None]) & valid
    per_mol = (pa + pa * earlier).sum(axis=1) * nato
    entries = int(valid.sum())
    once = int((pa.sum(axis=1) * nato).sum())
    return int(per_mol.sum()), entries, int(pa.sum()), once


def roofline(it, ktimes, a):
    """Roofline of the kernel with the largest device time in the timed region (the library's
    per-launch events), against the bound that applies to it."""
    import numpy as np  # noqa: F401
    hbm, fp32, mhz, src = _peaks()
    extra = {}
    if not ktimes:
        return None, extra
    dom = max(ktimes, key=lambda k: ktimes[k][0])
    tot, n = ktimes[dom]
    launch_ms = tot / n
    extra["dominant_kernel"] = dom
    extra["kernel_share_of_timed"] = {k: round(v[0] / sum(x[0] for x in ktimes.values()), 4)
                                      for k, v in ktimes.items()}
    wl = it.wl
    if dom in ("spec_energy_kernel", "molfit_seq_kernel"):
        pairs, entries, partner_atoms, once = spec_energy_pairs(it)
        if dom == "molfit_seq_kernel":
            pairs = once          # the sequential kernel evaluates E(new m, cur p) once per entry
        ops = OPS_PER_ENERGY_PAIR * pairs
        ach = ops / (launch_ms / 1000.0) / 1e12
        # bytes the kernel must move at least: per stored entry its partner index and reference
        # (8 B) and the energy written (4 B), per partner atom its float4 position (16 B) for the
        # old and, when earlier in the visit order, the new position
        byt = 12 * entries + 16 * partner_atoms
        extra["hbm_algorithmic"] = {"bytes_per_launch": byt, "achieved_GBs": byt / (launch_ms / 1000.0) / 1e9,
                                    "peak_GBs": hbm, "frac": byt / (launch_ms / 1000.0) / 1e9 / hbm,
                                    "peak_source": src}
        return {"bound": "fp32", "kernel": dom, "achieved": ach, "peak": fp32, "unit": "Tops/s (FP32 issue)",
                "frac": ach / fp32, "traffic": SPEC_ENERGY_TRAFFIC_PER_PAIR and int(SPEC_ENERGY_TRAFFIC_PER_PAIR * pairs),
                "peak_source": "nominal (148 SMs x 128 lanes x %.0f MHz)" % mhz,
                "ops_per_launch": ops, "atom_pairs_per_launch": pairs, "ops_per_atom_pair": OPS_PER_ENERGY_PAIR,
                "launch_ms": launch_ms, "launches": n}, extra
    if dom == "spec_resolve_kernel":
        ns = 1e6 * launch_ms / it.box.nmol
        floor_ns = RESOLVE_WALK_CYCLES_PER_MOVE / mhz * 1000.0
        fill = ktimes.get("ahead_fill_kernel")
        if fill:
            extra["ran1_fill_ns_per_move"] = 1e6 * fill[0] / fill[1] / it.box.nmol
        return {"bound": "latency (ordered walk)", "kernel": dom, "achieved": floor_ns / ns, "peak": 1.0,
                "unit": "walk floor / measured time per move", "frac": floor_ns / ns, "traffic": None,
                "ns_per_move": ns, "floor_ns_per_move": floor_ns,
                "floor_source": "the walk alone on B200, %.1f cycles per move at %.0f MHz" % (RESOLVE_WALK_CYCLES_PER_MOVE, mhz),
                "launch_ms": launch_ms, "launches": n}, extra
    if dom in ("ahead_fill_kernel", "ran1_fill_kernel"):
        # the next cycle's ran1 values: 7 a move (3 rotation, 3 translation, 1 acceptance), one
        # dependent warp shuffle per value
        values = 7 * it.box.nmol
        floor_ms = values * RAN1_SHUFFLE_CYCLES / mhz / 1000.0
        return {"bound": "latency (ran1 shuffle chain)", "kernel": dom, "achieved": floor_ms / launch_ms, "peak": 1.0,
                "unit": "chain floor / measured time per launch", "frac": floor_ms / launch_ms, "traffic": None,
                "values_per_launch": values, "floor_ms": floor_ms,
                "floor_source": "one dependent warp shuffle per value, %d cycles on B200 at %.0f MHz" % (RAN1_SHUFFLE_CYCLES, mhz),
                "launch_ms": launch_ms, "launches": n}, extra
    if dom == "fitexp_cluster_kernel":
        trials = max(it.fit_trials, 1)
        flops = 2.0 * wl.nq * wl.nterms * trials
        ach = flops / (launch_ms / 1000.0) / 1e12
        us_trial = 1000.0 * launch_ms / trials
        chain_us = (wl.nterms + 1) * FIT_CHAIN_CYCLES_PER_VALUE / mhz
        extra["fit_chain_bound"] = {"us_per_trial": chain_us, "measured_us_per_trial": us_trial,
                                    "frac": chain_us / us_trial, "cycles_per_value": FIT_CHAIN_CYCLES_PER_VALUE}
        return {"bound": "ran1 chain (latency)", "kernel": dom, "achieved": ach, "peak": fp32,
                "unit": "Tops/s (FP32 issue)", "frac": ach / fp32, "traffic": FIT_DRAM_BYTES_PER_LAUNCH,
                "peak_source": "nominal (148 SMs x 128 lanes x %.0f MHz)" % mhz, "launch_ms": launch_ms,
                "launches": n}, extra
    if dom == "ag_inter_kernel":
        pu = it.pair_updates
        ops = OPS_PER_PAIR_UPDATE * pu
        ach = ops / (launch_ms / 1000.0) / 1e12
        return {"bound": "fp32", "kernel": dom, "achieved": ach, "peak": fp32, "unit": "Tops/s (FP32 issue)",
                "frac": ach / fp32, "traffic": None, "peak_source": "nominal (148 SMs x 128 lanes x %.0f MHz)" % mhz,
                "pair_updates_per_launch": pu, "launch_ms": launch_ms, "launches": n}, extra
    return {"bound": "unknown", "kernel": dom, "achieved": None, "peak": None, "unit": None, "frac": None,
            "traffic": None, "launch_ms": launch_ms, "launches": n}, extra


def c4_arm(a):
    """Configuration C4: 64 independent boxes of uneven size (300-30,000 atoms, water and
    SiO2-like, 298-1500 K) advanced together by the batched checkerboard scheme.  A step is one
    sweep of every box -- one CUDA graph launch whose kernels each cover every box (binning,
    then per step one propose and one decide launch) -- and the partial g(r) histograms of every
    box over all atom pairs (int64 counts, one launch).  Launch shapes come from the project's
    autotuner.  Each step is preceded by a 256 MB L2-flushing write inside the timed region."""
    import numpy as np
    import torch

    import torch.distributed as dist

    from epsr_python_translation_b200 import autotune, configs
    from epsr_python_translation_b200.batch import BatchBoxes, partition_boxes
    from epsr_python_translation_b200.box import BoxArrays, Ran1State
    from oracle import oracle
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    all_systems = configs.c4_batch(seed=1)
    # the boxes are independent: each rank advances its share, split greedily by atom count,
    # with no exchange during a sweep
    mine = partition_boxes([s.natom for s in all_systems], world)[rank]
    systems = [all_systems[i] for i in mine]
    bb = BatchBoxes(systems, rot_deg=10.0, trans_A=0.5, seed=1 + 1000 * rank)
    bb.total_energy()
    choice = autotune.tune(bb, "plain")
    g = bb.capture("plain")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for k in range(max(3, a.warmup)):
        flush.fill_(float(k))
        g.replay()
        bb.histograms()
    torch.cuda.synchronize()
    c0 = bb.counters.clone()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = ClockSampler(vis.split(",")[0] if vis else "0")
    clocks.start()
    time.sleep(0.3)
    import ctypes as C
    bb.lib.epsr_timing_enable(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pairs = torch.zeros(1, dtype=torch.int64, device="cuda")
    e0.record()
    for k in range(a.steps):
        flush.fill_(float(k))
        g.replay()
        _, hp = bb.histograms()
        pairs += hp.sum()
    e1.record()
    torch.cuda.synchronize()
    bb.lib.epsr_timing_enable(0)
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    clk = clocks.stop()
    bb.check_status()
    kt = {}
    for kname in ("bmc_propose_kernel", "bmc_decide_kernel", "bmc_hist_inter_kernel"):
        tms, n = C.c_double(0.0), C.c_int64(0)
        bb.lib.epsr_timing_read(kname.encode(), C.byref(tms), C.byref(n))
        if n.value:
            kt[kname] = {"total_ms": round(tms.value, 3), "launches": int(n.value),
                         "mean_us": round(1000 * tms.value / n.value, 2)}
    cnt = (bb.counters - c0).cpu().numpy().reshape(bb.nbox, 4)
    tot = torch.tensor([float(cnt[:, 0].sum()), float(pairs.item()), float(cnt[:, 2].sum())], dtype=torch.float64,
                       device="cuda")
    if world > 1:   # the moves and pair-updates of every rank's boxes
        dist.all_reduce(tot)
    moves, npairs, accepted = int(tot[0].item()), int(tot[1].item()), float(tot[2].item())
    value = moves / (ms / 1000.0)
    hbm, fp32, mhz, src = _peaks()
    hist_ms = kt.get("bmc_hist_inter_kernel", {}).get("total_ms", 0.0)
    launches_per_step = 6 + 2 * bb.steps_per_sweep + 3
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (64 seeded boxes: water and SiO2-like, log-uniform sizes)",
        "pair_updates_per_s": npairs / (ms / 1000.0),
        "config": {"workload": "c4_batch", "boxes": len(all_systems), "atoms": int(sum(s.natom for s in all_systems)),
                   "atoms_min_max": [int(min(s.natom for s in all_systems)), int(max(s.natom for s in all_systems))],
                   "boxes_per_gpu": "split over %d GPU(s) greedily by atom count, no exchange during a sweep" % world,
                   "moves_per_step": moves // a.steps, "steps_per_sweep": bb.steps_per_sweep,
                   "launches_per_step": launches_per_step, "launches_depend_on_box_count": False,
                   "autotuned": {"threads": choice["threads"], "hist_tile": choice["tile"]},
                   "step": "one graph launch per sweep of every box (checkerboard scheme) + all-pairs g(r) "
                           "histograms of every box (int64 counts) in one launch",
                   "l2": "flushed before every step by a 256 MB write, inside the timed region"},
        "acceptance": accepted / max(moves, 1), "kernel_ms": kt,
        "roofline": {"bound": "fp32", "kernel": "bmc_hist_inter_kernel",
                     "achieved": (OPS_PER_PAIR_UPDATE * npairs / (hist_ms / 1000.0) / 1e12) if hist_ms else None,
                     "peak": fp32, "unit": "Tops/s (FP32 issue)",
                     "frac": (OPS_PER_PAIR_UPDATE * npairs / (hist_ms / 1000.0) / 1e12 / fp32) if hist_ms else None,
                     "traffic": None, "peak_source": "nominal (148 SMs x 128 lanes x %.0f MHz)" % mhz},
        "gpu_launches": launches_per_step * a.steps, "clocks": clk,
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    if not a.no_cpu_baseline and world == 1:
        small = sorted(range(len(systems)), key=lambda i: systems[i].natom)[:4]
        t0 = time.perf_counter()
        mv = 0
        for i in small:
            s = systems[i]
            ob = BoxArrays.from_system(s)
            oc = oracle.cell_list(ob, 10, ob.sepmax)
            st = oracle.fmolec1(ob, oc, configs.intra_energies(s))
            nmt = s.nmoltype
            omc = dict(rejrate=np.float32(0.75), stepr=np.float32(1.0), stepm=np.float32(1.0),
                       wholerot=np.full(nmt, 10.0 / 180.0, np.float32),
                       wholetrans=np.full(nmt, 0.5, np.float32) / np.float32(s.dmax), internrot=np.zeros(nmt, np.float32),
                       interntrans=np.zeros(nmt, np.float32), ireset=0)
            _, _, r = oracle.molfit(ob, oc, st, omc, Ran1State(idum=-(i + 1)), record_cos=False)
            oracle.atogen(ob, s.nmol, r, np.full(s.npairs, -2.0, np.float32))
            mv += s.nmol
        wall = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": mv / wall, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"one step (cell list, fmolec1, one reference-order sweep, all-pairs atogen) "
                                          f"of the 4 smallest boxes ({mv} molecules), single-threaded C oracle"}
    print(json.dumps(line), flush=True)
    return 0


def learned_c5(a, steps=None):
    """Configuration C5 (2,700 DMSO + 5,300 water, 8,000 molecules): decorrelated moves per
    second of (1) the plain GPU path in the reference's visit order (the speculative molfit
    cycle on one box, the path the headline measures), (2) the plain single-stage test on
    ``--c5-boxes`` boxes advanced together by the batched checkerboard scheme, one CUDA graph
    per sweep, and (3) the same boxes with the learned delayed-acceptance first stage, its
    network trained on the batched plain run's (features, beta dE) pairs by the tcgen05
    kernels.  ESS of the total energy from its integrated autocorrelation time per box, summed
    over boxes; every arm starts from the same equilibrated configuration."""
    import numpy as np
    import torch

    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.learned import RMSE_BOUND, LearnedMC, ess
    nsw = a.c5_sweeps
    s0 = configs.c5_learned(seed=1)
    B = max(1, a.c5_boxes)
    t0 = time.perf_counter()
    lm = LearnedMC([s0] * B, rot_deg=10.0, trans_A=0.5, seed=11)
    lm.run(100, "plain")                                       # equilibration from the random start
    out = {"workload": "c5_learned", "nmol": s0.nmol, "natom": s0.natom, "boxes": B,
           "grid": {"stride": lm.bb.grid[0][0], "ncell": lm.bb.grid[0][1], "moves_in_parallel_per_box":
                    lm.bb.descs[0].nslot, "steps_per_sweep": lm.bb.steps_per_sweep},
           "proposal": "rotation <= 10 deg about a random axis + translation <= 0.5 A (every arm)"}
    # (2) batched plain
    sp, ms_p, cp, _ = lm.run(nsw, "plain")
    e_p, tau_p = ess(sp[1:])
    mv_p = int(cp[:, 0].sum())
    out["batched_plain"] = {"sweeps": nsw, "ms": ms_p, "moves_per_s": mv_p / (ms_p / 1e3),
                            "acceptance": float(cp[:, 2].sum() / max(cp[:, 0].sum(), 1)),
                            "left_cell": float(cp[:, 3].sum() / max(cp[:, 0].sum(), 1)),
                            "tau_sweeps_median": float(np.median(tau_p)), "ess": float(e_p.sum()),
                            "ess_per_s": float(e_p.sum() / (ms_p / 1e3))}
    # (3) learned: record, train, run
    tr0 = time.perf_counter()
    x, t = lm.collect(a.c5_pairs)
    torch.cuda.synchronize()
    rec_s = time.perf_counter() - tr0
    rep = lm.train(x, t, epochs=24, batch=2048, lr=1e-3)
    del x, t
    torch.cuda.empty_cache()
    sd, ms_d, cd, mode = lm.run(nsw, "da")
    e_d, tau_d = ess(sd[1:])
    mv_d = int(cd[:, 0].sum())
    out["learned"] = {"mode": mode, "sweeps": nsw, "ms": ms_d, "moves_per_s": mv_d / (ms_d / 1e3),
                      "first_stage_accept": float(cd[:, 1].sum() / max(cd[:, 0].sum() - cd[:, 3].sum(), 1)),
                      "acceptance": float(cd[:, 2].sum() / max(cd[:, 0].sum(), 1)),
                      "tau_sweeps_median": float(np.median(tau_d)), "ess": float(e_d.sum()),
                      "ess_per_s": float(e_d.sum() / (ms_d / 1e3)),
                      "training": {k: v for k, v in rep.items()}, "record_s": rec_s,
                      "heldout_bound_kT": RMSE_BOUND, "residual_rmse_last_step_kT": lm.residual_rmse()}
    # (1) the reference-order plain GPU path on one box from box 0's configuration, and (4) on
    # R boxes at once (boxes 0..R-1 of the batched run), each on its own stream and host thread
    nref = max(20, nsw // 4)
    r1 = reference_order_boxes(lm, s0, 1, nref)
    out["reference_order_plain"] = dict(r1, note="the speculative molfit cycle, fast sums, adaptive steps as molfit")
    R = max(1, min(a.c5_spec_boxes, B))
    rR = reference_order_boxes(lm, s0, R, nref)
    out["reference_order_plain_concurrent"] = dict(
        rR, note="the same path on %d boxes at once (own stream and host thread each); ESS summed over boxes" % R)
    base = out["reference_order_plain"]["ess_per_s"]
    out["learned_vs_plain_ess_per_s"] = out["learned"]["ess_per_s"] / base if base > 0 else None
    out["batched_plain_vs_plain_ess_per_s"] = out["batched_plain"]["ess_per_s"] / base if base > 0 else None
    out["learned_vs_batched_plain_ess_per_s"] = (out["learned"]["ess_per_s"] / out["batched_plain"]["ess_per_s"]
                                                 if out["batched_plain"]["ess_per_s"] > 0 else None)
    out["concurrent_plain_vs_plain_ess_per_s"] = out["reference_order_plain_concurrent"]["ess_per_s"] / base if base > 0 else None
    out["wall_s"] = time.perf_counter() - t0
    return out


def reference_order_boxes(lm, s0, R, nref):
    """The speculative molfit cycle on R C5 boxes at once, started from boxes 0..R-1 of the
    batched run: nref timed sweeps of every box after 5 untimed ones, each box on its own stream
    and host thread; device time from events on a common stream that every box stream joins at
    both ends.  ESS of each box's energy series (molfit's running fadds), summed over boxes."""
    import threading

    import numpy as np
    import torch

    from epsr_python_translation_b200 import configs
    from epsr_python_translation_b200.box import BoxArrays, Ran1State, trsteps
    from epsr_python_translation_b200.device import DeviceBox
    from epsr_python_translation_b200.learned import ess
    co = lm.bb.download()
    main = torch.cuda.current_stream()
    streams = [torch.cuda.Stream() for _ in range(R)]
    boxes, sers = [], []
    for r in range(R):
        ms_, as_ = lm.bb.box_slices(r)
        box = BoxArrays.from_system(s0)
        for k in ("xa", "ya", "za", "xadd", "yadd", "zadd"):
            getattr(box, k)[:] = co[k][as_ if k in ("xa", "ya", "za") else ms_]
        with torch.cuda.stream(streams[r]):
            d = DeviceBox(box)
            d.cell_list(10, box.sepmax)
            d.fmolec1(configs.intra_energies(s0), strict=False)
            tmax, tmin = trsteps(box.natomr)
            nmt = box.nmoltype
            d.mc_setup(rejrate=np.float32(0.75), stepr=1.0, stepm=1.0,
                       wholerot=np.full(nmt, 10.0 / 180.0, np.float32),
                       wholetrans=np.full(nmt, 0.5, np.float32) / np.float32(s0.dmax), ran1=Ran1State(idum=-5 - r),
                       trstepmax=tmax, trstepmin=tmin)
            for _ in range(5):
                d.molfit(strict=False)
            sers.append(torch.zeros(nref, dtype=torch.float32, device="cuda"))
        boxes.append(d)
    torch.cuda.synchronize()
    errs = []

    def body(r):
        try:
            with torch.cuda.stream(streams[r]):
                streams[r].wait_event(ev0)
                for i in range(nref):
                    boxes[r].molfit(strict=False)
                    sers[r][i] = boxes[r].m_fadds[0]
        except Exception as e:  # noqa: BLE001  (re-raised on the main thread)
            errs.append(e)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(main)
    th = [threading.Thread(target=body, args=(r,)) for r in range(R)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    for st in streams:
        main.wait_stream(st)
    ev1.record(main)
    torch.cuda.synchronize()
    for d in boxes:
        d.check_status()
    ms_r = ev0.elapsed_time(ev1)
    e_r, tau_r = ess(torch.stack(sers, 1).cpu().numpy().astype(np.float64))
    return {"boxes": R, "sweeps": nref, "ms": ms_r, "moves_per_s": R * nref * s0.nmol / (ms_r / 1e3),
            "tau_sweeps": [float(t) for t in tau_r], "ess": float(e_r.sum()), "ess_per_s": float(e_r.sum() / (ms_r / 1e3))}


def c5_arm(a):
    import torch
    torch.cuda.set_device(0)
    r = learned_c5(a)
    line = {"metric": "ESS/s of total energy (learned delayed-acceptance vs plain)", "value": r["learned"]["ess_per_s"],
            "unit": "effective samples/s", "n_gpus": 1, "steps": a.c5_sweeps, "warmup": 100,
            "ms_per_step": r["learned"]["ms"] / a.c5_sweeps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (surrogate bf16/f32)", "data": "synthetic (seeded c5_learned boxes)",
            "config": {"workload": "c5_learned", "boxes": r["boxes"]}, "c5": r}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return reference_arm(a)
    if a.config == "c4_batch":
        return c4_arm(a)
    if a.config == "c5_learned":
        return c5_arm(a)
    return gpu_arm(a)


if __name__ == "__main__":
    import numpy as np  # noqa: F401  (used by roofline)
    sys.exit(main())
