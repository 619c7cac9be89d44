"""Autotuner for the batched tensor-core Signal.

The persistent launch splits every problem into work units of (run, row tile,
column tile, node range).  Two knobs shape the units (fm_tc_tuning): the
nodes per unit along the node range, and the most kz values per tile of a
factored run.  Fewer, longer units pay less per-unit setup (phase tables,
the last accumulator fold, the split sums); more, shorter units balance the
persistent blocks better across the 148 SMs.  The best point depends on the
batch's shape, so the tuner times the candidates on the batch itself (CUDA
events, after a warm-up call) and caches the winner per shape class, in
memory and, when FEELMRI_B200_TUNING names a file, on disk.

A problem's result depends on the tuning (its node splits fix the FP32
summation order), never on the other problems of the batch.
"""
from __future__ import annotations

import json
import math
import os
import threading

import torch

from . import ops

__all__ = ["CANDIDATES", "shape_class", "tune", "cached"]

CANDIDATES = tuple(ops.Tuning(split_nodes=s, kz_cap=k) for s in (0, 8192, 16384, 32768, 65536) for k in (0, 16))

_lock = threading.Lock()
_cache: dict[str, ops.Tuning] = {}


def _cache_file() -> str | None:
    return os.environ.get("FEELMRI_B200_TUNING") or None


def _load() -> None:
    path = _cache_file()
    if not path or not os.path.exists(path):
        return
    try:
        with open(path) as f:
            for k, v in json.load(f).items():
                _cache.setdefault(k, ops.Tuning(**v))
    except (OSError, ValueError, TypeError):
        pass


def _store() -> None:
    path = _cache_file()
    if not path:
        return
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump({k: {"split_nodes": v.split_nodes, "kz_cap": v.kz_cap} for k, v in _cache.items()}, f, indent=1)
    os.replace(tmp, path)


def shape_class(problems) -> str:
    """Key of a batch: problem count, log2 buckets of total and largest node
    count and sample count, the widest column count and the kz depth."""
    ns = [int(inp.r0.shape[0]) for inp, _, _ in problems]
    ss = [int(inp.kx.numel()) for inp, _, _ in problems]
    vs = [int(inp.Mxy.shape[1]) for inp, _, _ in problems]
    kz = [int(inp.kx.shape[2]) for inp, _, _ in problems]
    b = lambda x: int(round(math.log2(max(x, 1))))  # noqa: E731
    return (f"n{len(problems)}-N{b(sum(ns))}-Nmax{b(max(ns))}-S{b(sum(ss))}-Smax{b(max(ss))}"
            f"-V{max(vs)}-kz{b(max(kz))}")


def cached(problems) -> ops.Tuning | None:
    with _lock:
        if not _cache:
            _load()
        return _cache.get(shape_class(problems))


def _time(batch: ops.SignalBatch, reps: int) -> float:
    batch.run()  # warm-up (and error check)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(reps):
        batch.enqueue()
    end.record()
    end.synchronize()
    batch.status()
    return start.elapsed_time(end) / reps


def tune(problems, candidates=CANDIDATES, reps: int = 3, force: bool = False) -> tuple[ops.Tuning, dict]:
    """Best tuning for the batch `problems` ((inputs, motion, out) triples):
    the cached one for its shape class unless `force`, else the fastest
    candidate.  Returns (tuning, {tuning: ms per launch} of this search)."""
    key = shape_class(problems)
    if not force:
        hit = cached(problems)
        if hit is not None:
            return hit, {}
    times = {}
    for cand in candidates:
        times[cand] = _time(ops.SignalBatch(problems, cand), reps)
    best = min(times, key=times.get)
    with _lock:
        _cache[key] = best
        _store()
    return best, times
