"""Kernel-variant and pass-size autotuner with an on-disk cache.

The fp kernel has three variants with identical results: one slice per CTA with load/store
staging (default) or TMA bulk-tensor staging (``CCT_VARIANT_FP_TMA``), and two slices per CTA
sharing the sample coordinates (``CCT_VARIANT_FP_SLICES2``).  Which is
faster depends on n, the angle count, the map type, the batch and whether the maps are an
angle range of a larger array (the TMA variant needs dense maps), so ``tune`` times every
applicable variant on the actual call (CUDA events, a few launches over a batch of the real
size, with the fused MLEM epilogue the solvers launch) and caches the winner per (GPU, n, angles,
detectors, slices, map dtype, layout) in a
JSON file (``$CCT_AUTOTUNE_CACHE`` or ``~/.cache/corrct_b200/autotune.json``).

``tune_maps`` does the same for ``compute_maps``: how many entries (angles, or half-turn pairs)
one pass of the scan and resample kernels covers, i.e. the workspace size, timed within a memory
budget (larger passes keep more of the GPU busy per launch; their rotated-frame workspace spills
from L2 either way).  ``maps_entries`` returns a cached choice without timing (the ragged stream
consults it for each of its groups).
"""

from __future__ import annotations

import json
import os
import threading

import numpy as np
import torch

from . import _lib, core
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
    return f"{name}|n{core.n}|a{core.n_angles}|d{core.n_det}|s{n_slices}|{str(maps_dtype).split('.')[-1]}{layout}|mlem-fp"


def time_fp(core: XrfCore, vol: torch.Tensor, maps: torch.Tensor, variant: int, reps: int = 3,
            epilogue: str = "mlem") -> float:
    """Mean fp launch time (ms) of one variant on the given batch: the fused MLEM fp (ratio and KL
    residual, ``cct_mlem_fp``, what the solvers launch) or the plain projection (``"store"``)."""
    import ctypes

    from .engine import BatchedSolver

    old = core.variant
    core.variant = variant
    try:
        out = core.fp(vol, maps)  # warm-up (also loads the kernel)
        if epilogue == "mlem":
            sv = BatchedSolver(core, maps, out, "mlem", x0=vol)
            h = core_stream(core)

            def launch():
                _lib.call("cct_mlem_fp", ctypes.byref(sv.desc), sv._maps_ptr, ctypes.byref(sv.state), h)
        else:
            def launch():
                core.fp(vol, maps, out=out)
        launch()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            launch()
        stop.record()
        stop.synchronize()
        return start.elapsed_time(stop) / reps
    finally:
        core.variant = old


def core_stream(c: XrfCore):
    return core.stream_handle(c.device)


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


MAPS_ENTRIES = (4, 8, 16, 32)


def maps_key(device, n: int, n_angles: int, n_det: int, n_slices: int, maps_dtype: str, quads: bool = False) -> str:
    name = torch.cuda.get_device_name(device).replace(" ", "_")
    return f"maps|{name}|n{n}|a{n_angles}|d{n_det}|s{n_slices}|{maps_dtype}" + ("|quads" if quads else "")


def maps_entries(device, n: int, n_angles: int, n_det: int, n_slices: int, maps_dtype: str = "float32",
                 quads: bool = False) -> int | None:
    """The cached entries per pass of ``tune_maps`` for this shape, or None."""
    hit = _load().get(maps_key(device, n, n_angles, n_det, n_slices, maps_dtype, quads))
    return None if hit is None else int(hit["entries"])


def tune_maps(mu_in: torch.Tensor, mu_out: torch.Tensor, angles_rad32, det_angles=(np.pi / 2,),
              maps_dtype: str = "float32", budget_bytes: int = 4 << 30, out: torch.Tensor | None = None,
              force: bool = False, emitted_scale: float | None = None) -> int:
    """Entries per pass of ``compute_maps`` for this batch (cached): times every choice of
    ``MAPS_ENTRIES`` whose workspace fits ``budget_bytes`` (two calls each, CUDA events)."""
    ref = mu_in if mu_in is not None else mu_out
    s, n = ref.shape[0], ref.shape[-1]
    n_det = len(np.atleast_1d(det_angles))
    n_angles = len(np.atleast_1d(angles_rad32))
    k = maps_key(ref.device, n, n_angles, n_det, s, maps_dtype, emitted_scale is not None)
    with _LOCK:
        cache = _load()
        if not force and k in cache:
            return int(cache[k]["entries"])
        per_entry = core.maps_entry_bytes(n, s, n_det, 1, mu_in is not None, mu_out is not None)
        choices = [e for e in MAPS_ENTRIES if e * per_entry <= budget_bytes] or [1]
        times = {}
        for e in choices:
            ws = torch.empty(e * per_entry, dtype=torch.uint8, device=ref.device)
            out = core.compute_maps(mu_in, mu_out, angles_rad32, det_angles, maps_dtype=maps_dtype, workspace=ws,
                                    out=out, emitted_scale=emitted_scale)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(2):
                core.compute_maps(mu_in, mu_out, angles_rad32, det_angles, maps_dtype=maps_dtype, workspace=ws, out=out,
                                  emitted_scale=emitted_scale)
            stop.record()
            stop.synchronize()
            times[e] = start.elapsed_time(stop) / 2
            del ws
        best = min(times, key=times.get)
        cache[k] = {"entries": best, "ms": {str(e): t for e, t in times.items()}}
        _store(cache)
        return best

