"""Autotuner for the forward pencil-beam kernel.

The forward kernel exists in several shapes (block threads x voxels per
thread over an 8x8x8 tile, and the number of spots each thread culls per
compaction round; ``pb_dose_variant_name`` lists them), and the batched
persistent launch also takes a number of resident blocks per SM.  Which is
fastest depends on the grid size, the spot density and the beam count.  The
tuner times every candidate with CUDA events on the workload at hand (after
one warm-up run) and keeps the winner in a JSON cache keyed by GPU name and
a size class, so that later plans of the same class skip the search.

Cache file: $DOSECUDA_B200_TUNE_CACHE, else
~/.cache/dosecuda_b200/autotune.json.
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Callable, Dict, Iterable, Optional, Tuple

import torch

from . import _lib

_LOCK = threading.Lock()


def cache_path() -> str:
    env = os.environ.get("DOSECUDA_B200_TUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "dosecuda_b200", "autotune.json")


def _load(path: str) -> Dict[str, list]:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path: str, key: str, value) -> None:
    with _LOCK:
        data = _load(path)
        data[key] = value
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
        except OSError:
            pass


def size_class(n_vox: int, n_spots: int, n_beams: int) -> str:
    """Power-of-two buckets of voxels and spots, and the beam count."""
    v = int(round(math.log2(max(n_vox, 1))))
    s = int(round(math.log2(max(n_spots, 1))))
    return f"V2^{v}_S2^{s}_B{n_beams}"


def variants() -> Tuple[str, ...]:
    n = _lib.lib.pb_dose_variant_count()
    return tuple(_lib.lib.pb_dose_variant_name(v).decode() for v in range(n))


def threads_of(name: str) -> int:
    return int(name.split("_")[0][1:])


def best(candidates: Iterable, run: Callable, reps: int = 3, device=None):
    """Time run(c) for each candidate (one warm-up, then `reps` runs timed
    with CUDA events) and return (best candidate, {candidate: ms})."""
    stream = torch.cuda.current_stream(device)
    times = {}
    for c in candidates:
        run(c)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            run(c)
        b.record(stream)
        b.synchronize()
        times[c] = a.elapsed_time(b) / reps
    return min(times, key=times.get), times


def tune_plan(dp, reps: int = 3, use_cache: bool = True) -> int:
    """Forward variant for a DevicePlan (its WET must be computed)."""
    name = torch.cuda.get_device_name(dp.device)
    key = f"{name}|plan|{size_class(dp.n_vox, dp.n_spots, dp.n_beams)}"
    path = cache_path()
    if use_cache:
        hit = _load(path).get(key)
        if hit is not None:
            return int(hit[0])
    out = torch.empty(dp.n_vox, dtype=torch.float32, device=dp.device)
    v, times = best(range(len(variants())), lambda c: dp.forward_variant(c, out=out), reps,
                    dp.device)
    _store(path, key, [v, {str(k): t for k, t in times.items()}])
    return v


def rounds_of(name: str) -> int:
    """Rounds of spots a kernel shape culls at once (t<threads>_v<vpt>_c<k>)."""
    return int(name.split("_")[2][1:])


def max_blocks_per_sm(name: str) -> int:
    """Resident blocks per SM a kernel shape is compiled for: 6 for 128
    threads with one round, 5 for other 128-thread shapes, 3 for 256."""
    if threads_of(name) != 128:
        return 3
    return 6 if rounds_of(name) == 1 else 5


def batch_candidates():
    """(variant, blocks per SM) pairs the batch launch accepts."""
    out = []
    for v, name in enumerate(variants()):
        for bps in range(2, max_blocks_per_sm(name) + 1):
            out.append((v, bps))
    return out


def tune_batch(batch, reps: int = 2, use_cache: bool = True) -> Tuple[int, int]:
    """(variant, blocks per SM) for a BatchPlans' persistent forward."""
    name = torch.cuda.get_device_name(batch.device)
    key = (f"{name}|batch|{size_class(batch.n_vox, batch.n_spots, batch.n_plans)}")
    path = cache_path()
    if use_cache:
        hit = _load(path).get(key)
        if hit is not None:
            return int(hit[0]), int(hit[1])
    (v, bps), times = best(batch_candidates(),
                           lambda c: batch.run(_lib.PB_BATCH_DOSE, variant=c[0],
                                               blocks_per_sm=c[1]), reps, batch.device)
    _store(path, key, [v, bps, {f"{k[0]},{k[1]}": t for k, t in times.items()}])
    return v, bps
