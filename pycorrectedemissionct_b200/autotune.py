"""Kernel-variant autotuner with an on-disk cache.

The fp kernel has two shared-memory staging variants with identical results: load/store
staging (default) and TMA bulk-tensor staging (``CCT_VARIANT_FP_TMA``).  Which is faster
depends on n, the angle count, the map type and the batch, so ``tune`` times both on the
actual shape (CUDA events, a few launches over a batch of the real size) and caches the
winner per (GPU, n, angles, detectors, slices, map dtype) in a JSON file
(``$CCT_AUTOTUNE_CACHE`` or ``~/.cache/corrct_b200/autotune.json``).
"""

from __future__ import annotations

import json
import os
import threading

import torch

from . import _lib
from .core import XrfCore

_LOCK = threading.Lock()
VARIANTS = (0, _lib.CCT_VARIANT_FP_TMA)


def cache_path() -> str:
    return os.environ.get("CCT_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "corrct_b200", "autotune.json"))


def _load() -> dict:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(cache: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as fh:
            json.dump(cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def key(core: XrfCore, n_slices: int, maps_dtype: torch.dtype) -> str:
    name = torch.cuda.get_device_name(core.device).replace(" ", "_")
    return f"{name}|n{core.n}|a{core.n_angles}|d{core.n_det}|s{n_slices}|{str(maps_dtype).split('.')[-1]}"


def time_fp(core: XrfCore, vol: torch.Tensor, maps: torch.Tensor, variant: int, reps: int = 3) -> float:
    """Mean fp launch time (ms) of one variant on the given batch."""
    old = core.variant
    core.variant = variant
    try:
        out = core.fp(vol, maps)  # warm-up (also loads the kernel)
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            core.fp(vol, maps, out=out)
        stop.record()
        stop.synchronize()
        return start.elapsed_time(stop) / reps
    finally:
        core.variant = old


def tune(core: XrfCore, vol: torch.Tensor, maps: torch.Tensor, force: bool = False) -> int:
    """Pick the faster fp variant for this shape (cached); sets and returns ``core.variant``."""
    k = key(core, vol.shape[0], maps.dtype)
    with _LOCK:
        cache = _load()
        if not force and k in cache:
            core.variant = int(cache[k]["variant"])
            return core.variant
        times = {}
        for v in VARIANTS:
            if v == _lib.CCT_VARIANT_FP_TMA and core.n % 8 != 0:
                continue
            times[v] = time_fp(core, vol, maps, v)
        best = min(times, key=times.get)
        cache[k] = {"variant": best, "ms": {str(v): t for v, t in times.items()}}
        _store(cache)
        core.variant = best
        return best
