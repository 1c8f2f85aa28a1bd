"""Schedule autotuner of the island solver.

The persistent island launch has three schedule knobs: the vertex counts
above which an island gets a whole 1024-thread CTA (``mid``) or a 256-thread
sub-team instead of one warp (``small``), and how many CTAs start with the
small-island classes (``rev_ctas``, which keeps long-lived small islands out
of the launch's tail). The best choice depends on the batch's island-size
distribution and on the device, so ``tune`` times short ARAP and LSCM runs
of the batch itself under each candidate (CUDA events, UVs restored after
every trial) and applies the fastest. Results are cached per device and
size signature; ``tune`` is meant for a warm-up, not for a timed region.
"""
from __future__ import annotations

import itertools

import numpy as np
import torch

from . import _lib

CANDIDATES = {
    "mid": (1024, 2048),
    "small": (128, 256),
    "rev_ctas": (0, 24, 48),
}

_cache = {}


def signature(db):
    """Device name and a coarse histogram of island sizes (log2 buckets)."""
    return _signature(db.plan, db.dev)


def _signature(plan, dev):
    nv = np.diff(plan.vofs.astype(np.int64))
    hist = np.bincount(np.minimum(np.log2(np.maximum(nv, 1)).astype(int), 24), minlength=25)
    # bucket counts rounded to 2 significant bits so near-identical batches share a key
    key = tuple(int(2 ** np.floor(np.log2(h))) if h else 0 for h in hist)
    return torch.cuda.get_device_name(dev), key


def lookup(plan, dev):
    """The schedule ``tune`` chose earlier for batches of this signature on
    this device, or None. DeviceBatch applies it to every new batch."""
    if not _cache:
        return None
    return _cache.get(_signature(plan, dev))


def _time(fn, dev):
    s = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1)


def tune(db, arap_iters=3, candidates=None, use_cache=True):
    """Choose (mid, small, rev_ctas) for DeviceBatch ``db``; returns the
    chosen setting and the measured milliseconds of every candidate."""
    cand = dict(CANDIDATES, **(candidates or {}))
    sig = signature(db)
    if use_cache and sig in _cache:
        best = _cache[sig]
        db.set_classes(best["mid"], best["small"])
        db.rev_ctas = best["rev_ctas"]
        return best, {}
    U0 = db.U.clone()
    results = {}
    for mid, small, rev in itertools.product(cand["mid"], cand["small"], cand["rev_ctas"]):
        db.set_classes(mid, small)
        ms = _time(lambda: db.lscm(rev_ctas=rev), db.dev)
        ms += _time(lambda: db.arap(iters=arap_iters, rev_ctas=rev), db.dev)
        results[(mid, small, rev)] = ms
        db.U.copy_(U0)
    (mid, small, rev), _ = min(results.items(), key=lambda kv: kv[1])
    best = {"mid": mid, "small": small, "rev_ctas": rev}
    db.set_classes(mid, small)
    db.rev_ctas = rev
    db.U.copy_(U0)
    _cache[sig] = best
    return best, results
