"""Autotuner for the forward pencil-beam kernel.

The forward kernel exists in several shapes (``pb_dose_variant_name``
lists them), in two families:
  t<threads>_v<voxels per thread>_c<k>   8x8x8 voxel tiles, each thread a
                                         set of voxels evaluated one by one;
  l8x<TY>x<TZ>_c<k>                      8 x TY x TZ voxel tiles, each thread
                                         a line of 8 voxels along x;
with k the spots each thread culls per compaction round.  The batched
persistent launch takes the shapes whose tiles divide an 8x8x8 block, and a
number of resident blocks per SM.  Which is fastest depends on the grid
size, the spot density and the beam count.  The
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


def default_variant() -> int:
    """The shape pb_dose uses."""
    return int(_lib.lib.pb_dose_variant_default())


def default_batch_variant() -> int:
    """The shape the batch uses before tuning: the default when the batch
    takes it, else the first batch shape of the default's family."""
    names = variants()
    d = default_variant()
    if batch_shape(names[d]):
        return d
    fam = shape_of(names[d])[0]
    return next(v for v, n in enumerate(names) if shape_of(n)[0] == fam and batch_shape(n))


def shape_of(name: str) -> Tuple[str, Tuple[int, int, int], int, int]:
    """(family "t" or "l", voxel tile (x, y, z), block threads, spots culled
    per thread per round) of a kernel shape."""
    parts = name.split("_")
    k = int(parts[-1][1:])
    if name.startswith("l"):
        tile = tuple(int(v) for v in parts[0][1:].split("x"))
        return "l", tile, tile[1] * tile[2], k
    return "t", (8, 8, 8), int(parts[0][1:]), k


def threads_of(name: str) -> int:
    return shape_of(name)[2]


def round_size(name: str) -> int:
    """Spots a kernel shape culls per compaction round (threads x k)."""
    _, _, nt, k = shape_of(name)
    return nt * k


def same_decisions(a: str, b: str) -> bool:
    """Two shapes whose doses are equal bit for bit: the same family and
    tile (the same culling decisions and per-voxel arithmetic) and the same
    round size (the same order of each layer's spots)."""
    fa, ta, _, _ = shape_of(a)
    fb, tb, _, _ = shape_of(b)
    return fa == fb and ta == tb and round_size(a) == round_size(b)


def batch_shape(name: str) -> bool:
    """The persistent batch takes tiles that divide 8x8x8 blocks."""
    _, (_, ty, tz), _, _ = shape_of(name)
    return 8 % ty == 0 and 8 % tz == 0


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


def max_blocks_per_sm(name: str) -> int:
    """Resident blocks per SM a kernel shape is compiled for.  8x8x8
    family: 6 for 128 threads with one spot per thread per round, 5 for the
    other 128-thread shapes, 3 for 256.  Line family: 20 of 32 threads, 10
    of 64, 5 of 128."""
    fam, _, nt, k = shape_of(name)
    if fam == "l":
        return {32: 20, 64: 10, 128: 5}[nt]
    if nt != 128:
        return 3
    return 6 if k == 1 else 5


def batch_candidates():
    """(variant, blocks per SM) pairs the batch launch accepts."""
    out = []
    for v, name in enumerate(variants()):
        if not batch_shape(name):
            continue
        top = max_blocks_per_sm(name)
        lo = 2 if shape_of(name)[0] == "t" else max(1, top // 4)
        step = 1 if shape_of(name)[0] == "t" else max(1, top // 4)
        out += [(v, bps) for bps in range(lo, top + 1, step)]
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
