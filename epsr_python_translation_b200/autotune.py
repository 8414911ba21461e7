"""Autotuner of the batched engine's launch shapes.

For a given batch of boxes (batch.BatchBoxes) it times, on the device, every candidate of the
shapes that do not change results:
  * threads per move's CTA of the propose and decide kernels (64, 128, 256): a small molecule
    with a short partner list runs best on fewer threads, many boxes of large ones on more;
  * target atoms per work item of the all-pairs histogram pass (256 ... 4096): larger tiles
    amortise the shared-histogram clear and merge, smaller ones balance uneven boxes;
and keeps the fastest.  Results are cached per batch signature (box count and each box's size
class and composition), in memory and optionally in a JSON file.

Each candidate is timed with CUDA events after one untimed launch, over a copy of the batch's
state that is restored afterwards, so tuning leaves the chain where it was.
"""

from __future__ import annotations

import json
import os

import torch

THREADS = (64, 128, 256)
TILES = (256, 512, 1024, 2048, 4096)
_CACHE = {}


def signature(bb):
    """Batch key: per box its size class (log2 of the atom count) and molecule count."""
    return "|".join(f"{max(s.natom, 1).bit_length()}:{s.nmol}:{s.ntype}" for s in bb.systems)


def _state(bb):
    names = ("xa", "ya", "za", "xadd", "yadd", "zadd", "pos", "energy", "counters", "sweep_counter")
    return {k: getattr(bb, k).clone() for k in names}


def _restore(bb, st):
    for k, v in st.items():
        getattr(bb, k).copy_(v)


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune(bb, mode="plain", net=None, path=None, hist=True):
    """Choose bb.c.threads (sweep kernels) and the histogram tile; returns the choice and the
    timings.  ``path``: JSON cache file (read first, updated after tuning)."""
    key = f"{signature(bb)}#{mode}"
    if path and os.path.exists(path) and key not in _CACHE:
        try:
            _CACHE.update(json.load(open(path)))
        except (OSError, ValueError):
            pass
    if key in _CACHE:
        ch = _CACHE[key]
        bb.c.threads = int(ch["threads"])
        if hist:
            bb._hist = None
            bb.hist_tile = int(ch["tile"])
        return ch
    st = _state(bb)
    times = {"threads": {}, "tile": {}}
    for t in THREADS:
        bb.c.threads = t
        times["threads"][t] = _time(lambda: bb.sweep(mode, net), reps=2)
        _restore(bb, st)
    best_t = min(times["threads"], key=times["threads"].get)
    bb.c.threads = best_t
    best_tile = 1024
    if hist:
        for tl in TILES:
            bb._hist = None
            times["tile"][tl] = _time(lambda: bb.histograms(tile=tl), reps=3)
        best_tile = min(times["tile"], key=times["tile"].get)
        bb._hist = None
        bb.hist_tile = best_tile
    _restore(bb, st)
    ch = {"threads": best_t, "tile": best_tile, "times_ms": {k: {str(a): b for a, b in v.items()}
                                                              for k, v in times.items()}}
    _CACHE[key] = ch
    if path:
        try:
            with open(path, "w") as f:
                json.dump(_CACHE, f, indent=1)
        except OSError:
            pass
    return ch
