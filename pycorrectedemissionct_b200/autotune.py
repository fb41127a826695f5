"""Kernel-variant autotuner with an on-disk cache.

The fp kernel has three variants with identical results: one slice per CTA with load/store
staging (default) or TMA bulk-tensor staging (``CCT_VARIANT_FP_TMA``), and two slices per CTA
sharing the sample coordinates (``CCT_VARIANT_FP_SLICES2``).  Which is
faster depends on n, the angle count, the map type, the batch and whether the maps are an
angle range of a larger array (the TMA variant needs dense maps), so ``tune`` times every
applicable variant on the actual call (CUDA events, a few launches over a batch of the real
size) and caches the winner per (GPU, n, angles, detectors, slices, map dtype, layout) in a
JSON file (``$CCT_AUTOTUNE_CACHE`` or ``~/.cache/corrct_b200/autotune.json``).
"""

from __future__ import annotations

import json
import os
import threading

import torch

from . import _lib
from .core import XrfCore

_LOCK = threading.Lock()
VARIANTS = (0, _lib.CCT_VARIANT_FP_TMA, _lib.CCT_VARIANT_FP_SLICES2)


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


def key(core: XrfCore, n_slices: int, maps_dtype: torch.dtype, dense: bool = True) -> str:
    name = torch.cuda.get_device_name(core.device).replace(" ", "_")
    layout = "" if dense else "|strided"
    return f"{name}|n{core.n}|a{core.n_angles}|d{core.n_det}|s{n_slices}|{str(maps_dtype).split('.')[-1]}{layout}"


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
    dense = maps is None or maps.is_contiguous()
    k = key(core, vol.shape[0], None if maps is None else maps.dtype, dense)
    with _LOCK:
        cache = _load()
        if not force and k in cache and int(cache[k]["variant"]) in VARIANTS:
            core.variant = int(cache[k]["variant"])
            return core.variant
        times = {}
        for v in VARIANTS:
            if v == _lib.CCT_VARIANT_FP_TMA and (core.n % 8 != 0 or not dense):
                continue
            if v == _lib.CCT_VARIANT_FP_SLICES2 and vol.shape[0] < 2:
                continue
            times[v] = time_fp(core, vol, maps, v)
        best = min(times, key=times.get)
        cache[k] = {"variant": best, "ms": {str(v): t for v, t in times.items()}}
        _store(cache)
        core.variant = best
        return best
