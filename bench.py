"""Benchmark: converged slices/s of attenuated XRF MLEM on 512x512-pixel, 720-angle slices,
plain (cold start) vs warm start.

One step = the hot path over one batch of synthetic slices already resident in HBM:
``compute_maps`` (incident + emitted attenuation maps) followed by MLEM with the reference's
KL-residual stopping rule, run until every slice reaches the residual that the plain solver
reaches after 200 iterations (calibrated once, untimed).  Paths:

* plain: MLEM from the default start;
* subsets (the headline): ordered-subsets EM passes (90 subsets x 2 passes, then 18 x 1; each pass
  costs one MLEM iteration), then MLEM to the residual, which judges every slice;
* learned: on the learned part's own data (textured slices at 1e4 peak counts), the learned
  start (one ordered-subsets pass keeping 10 snapshots, the tensor-core encoder-decoder, one pass
  per ordered-subsets level) then MLEM to the residual, timed beside plain MLEM and the
  ordered-subsets passes on the same slices.

``value`` = slices converged per second over the timed steps of the headline path (``--method``,
default the ordered-subsets warm start); the other paths are reported beside it.  Max over ranks;
weak scaling (each rank owns its own slices, no collective on the data path).

``e2e`` repeats the headline step through the public API from pinned host buffers (mu and the
data copied in, the reconstruction copied out inside the timed region); ``dropin_e2e`` times the
call a corrct user makes (projector from mu + MLEM with a tolerance, numpy in and out).
``--impl reference`` times the reference algorithm's CPU implementation (the oracle port in
``oracle/``) on the host cores on a bounded sample of the same workload.  Other workloads:
``--workload ragged`` (mixed sizes), ``waves`` (512 slices of plain MLEM in HBM-sized waves, FP32
and BF16 maps), ``channels`` (8 fluorescence channels of 1024x1024x1440 slices, PDHG-TV).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged slices/s, XRF MLEM 512²x720 to fixed residual: plain vs warm start"
UNIT = "slices/s"
# fp variants (cct_xrf_desc.variant): the label, the kernel and the DRAM bytes per slice of one
# ncu capture at 512^2 x 720 FP32 maps (read + write)
FP_VARIANT_NAMES = {0: "ldg", 1: "tma", 2: "slices2"}
FP_KERNEL_NAMES = {0: "fp_kernel", 1: "fp_tma_kernel", 2: "fp_pair_kernel"}
FP_TRAFFIC_PER_SLICE = {0: 2.8680e9 / 4, 1: 2.9200e9 / 4, 2: 2.7911e9 / 4}
WEIGHTS = os.path.join(ROOT, "pycorrectedemissionct_b200", "weights", "warmstart.pt")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slices", type=int, default=32, help="slices per GPU")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--angles", type=int, default=720)
    ap.add_argument("--iters", type=int, default=200, help="plain MLEM iterations that define the residual")
    ap.add_argument("--maps-dtype", default="float32", choices=["float32", "bfloat16"])
    ap.add_argument("--peak", type=float, default=1e5)
    ap.add_argument("--seed", type=int, default=20240)
    ap.add_argument("--method", default="auto", choices=["auto", "plain", "subsets"],
                    help="headline path (auto: ordered subsets); the others are timed beside it")
    ap.add_argument("--learned-peak", type=float, default=1e4, help="learned leg: Poisson peak counts of its textured slices")
    ap.add_argument("--subsets", default="90:2,18:1", help="ordered-subsets schedule subsets:passes,...")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-legs", action="store_true",
                    help="skip the drop-in e2e, BF16-maps and FP64-error legs")
    ap.add_argument("--no-learned-leg", action="store_true", help="skip the learned warm-start leg")
    ap.add_argument("--fp64-angle-step", type=int, default=24,
                    help="FP64 oracle check of the headline slice on every k-th angle")
    ap.add_argument("--fp-variant", default="auto", choices=["auto", "ldg", "tma", "slices2"],
                    help="fp staging variant: the autotuner's choice (auto) or a fixed one")
    ap.add_argument("--workload", default="batch", choices=["batch", "ragged", "waves", "channels"],
                    help="batch: the 512x720 benchmark (default); ragged: the mixed-size stream; waves: "
                         "512 slices of plain MLEM in HBM-sized waves, FP32 and BF16 maps; channels: "
                         "8 fluorescence channels of 1024x1024x1440 slices, PDHG-KL-TV")
    ap.add_argument("--field-slices", type=int, default=1, help="channels workload: field slices per wave")
    ap.add_argument("--wave-slices", type=int, default=512)
    ap.add_argument("--ragged-slices", type=int, default=400)
    ap.add_argument("--ragged-legs", default="subsets,learned,plain",
                    help="ragged workload: MLEM starts to time (subsets, learned, plain), comma-separated")
    ap.add_argument("--cpu-sample-angles", type=int, default=144)
    return ap.parse_args()


def workload_name(a) -> str:
    return f"XRF MLEM {a.n}x{a.n}, {a.angles} angles, batch of {a.slices} slices/GPU, {a.maps_dtype} maps"


def make_inputs(a, rank: int):
    """Seeded phantoms and attenuation (mu in [0, 0.01], mu_out = mu_in), float32, host."""
    from pycorrectedemissionct_b200 import phantoms

    xs, mus = [], []
    for k in range(a.slices):
        rng = phantoms.slice_rng(a.seed, rank * a.slices + k)
        xs.append(phantoms.ellipse_phantom(a.n, rng, 12))
        mus.append(phantoms.disk_attenuation(a.n, rng, 0.01))
    return np.stack(xs), np.stack(mus)


# ----------------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int):
        # the raw samples go to $CCT_CLOCKS_DIR (default: the temp directory); the summary is in
        # the JSON line
        out = os.environ.get("CCT_CLOCKS_DIR", tempfile.gettempdir())
        self.path = os.path.join(out, f"cct_clocks_rank{index}_{os.getpid()}.csv")
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait (at most 3 s) for its first sample, so that the
        # timed region that follows is covered from its start
        t_end = time.time() + 3.0
        while time.time() < t_end and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1", "0x1"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------- cpu baseline
def cpu_baseline(a, iterations_per_slice: float) -> dict:
    """Oracle port (the reference algorithm, float32 like the reference's default run) on the host
    cores: maps, one fp and one bp on a bounded sample of the angles, extrapolated to one slice."""
    from oracle import port
    from pycorrectedemissionct_b200 import phantoms

    workers = os.cpu_count() or 1
    rng = phantoms.slice_rng(a.seed, 0)
    x = phantoms.ellipse_phantom(a.n, rng, 12)
    mu = phantoms.disk_attenuation(a.n, rng, 0.01)
    angles = phantoms.angles(a.angles)
    sample = max(1, min(a.cpu_sample_angles, a.angles))
    rad32, deg32 = port.backend_angles(angles[:: max(1, a.angles // sample)][:sample])
    t0 = time.perf_counter()
    maps = port.compute_maps(mu, mu, rad32, dtype=np.float32, workers=workers)
    t1 = time.perf_counter()
    sino = port.fp_xrf(x, maps, deg32, workers=workers)
    t2 = time.perf_counter()
    port.bp_xrf(sino, maps, deg32, workers=workers)
    t3 = time.perf_counter()
    scale = a.angles / len(rad32)
    t_slice = scale * ((t1 - t0) + iterations_per_slice * ((t2 - t1) + (t3 - t2)))
    return {
        "value": 1.0 / t_slice,
        "unit": UNIT,
        "cores": workers,
        "kind": "port",
        "sample": (
            f"numpy/float32 oracle port of the reference's scikit-image path on {workers} threads: compute_maps, "
            f"one attenuated fp and one bp over {len(rad32)} of {a.angles} angles of one {a.n}x{a.n} slice "
            f"({t3 - t0:.1f} s), scaled to {a.angles} angles and {iterations_per_slice:.1f} plain MLEM iterations per slice"
        ),
        "seconds_per_slice": t_slice,
        "sample_seconds": t3 - t0,
    }


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    iters = float(a.iters)
    for _ in range(max(0, a.warmup)):
        cpu_baseline(a, iters)
    samples = [cpu_baseline(a, iters) for _ in range(max(1, a.steps))]
    v = float(np.median([s["value"] for s in samples]))
    cb = dict(samples[-1])
    cb["value"] = v
    # a step is one bounded sample (maps, one fp and one bp over a subset of the angles of one
    # slice); the value extrapolates it to whole slices solved by plain MLEM
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * float(np.mean([s["sample_seconds"] for s in samples])), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded ellipse phantoms, disk attenuation)",
        "config": {"workload": workload_name(a), "n": a.n, "angles": a.angles, "mlem_iterations": a.iters,
                   "solver": "plain MLEM (the reference has no warm start)"},
        "impl": "reference", "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------- ours
def run_ours(a):
    import torch

    from pycorrectedemissionct_b200 import autotune, core, distributed, engine
    rank, world, local = distributed.env_ranks()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    distributed.init("nccl", dev)

    xs_h, mus_h = make_inputs(a, rank)
    angles = np.linspace(0, 2 * np.pi, a.angles, endpoint=False)
    S, n = a.slices, a.n
    schedule = parse_schedule(a.subsets)
    perm = engine.subset_permutation(a.angles, [k for k, _ in schedule])
    perm_t = torch.from_numpy(perm).to(dev)
    c = core.XrfCore(n, angles, device=dev)                 # natural angle order (plain, learned)
    c_os = core.XrfCore(n, angles[perm], device=dev)        # subset-major order (ordered subsets)
    mu_in = torch.from_numpy(mus_h).to(dev)
    mu_out = mu_in.clone()  # mu_out = mu_in for this workload
    x_true = torch.from_numpy(xs_h).to(dev)
    tdt = torch.float32 if a.maps_dtype == "float32" else torch.bfloat16
    maps = torch.empty((S, a.angles, 1, n, n), dtype=tdt, device=dev)  # recomputed by every step, in its order
    # maps workspace: the entries per pass (half-turn pairs of angles) the autotuner picks for this
    # batch within 6 GB
    entries = autotune.tune_maps(mu_in, mu_out, c.angles_rad32, maps_dtype=a.maps_dtype, budget_bytes=6 << 30,
                                 out=maps, emitted_scale=1.0)
    ws = torch.empty(entries * core.maps_entry_bytes(n, S), dtype=torch.uint8, device=dev)

    # mu_out = mu_in in this workload: each emitted line integral is the incident one of the angle
    # a quarter turn on (compute_maps' quarter-turn quads)
    def maps_natural():
        core.compute_maps(mu_in, mu_out, c.angles_rad32, maps_dtype=a.maps_dtype, workspace=ws, out=maps,
                          emitted_scale=1.0)

    def maps_subsets():
        core.compute_maps(mu_in, mu_out, c_os.angles_rad32, maps_dtype=a.maps_dtype, workspace=ws, out=maps,
                          emitted_scale=1.0)

    maps_natural()
    passes = core.compute_maps.last_passes  # two kernels per pass
    if a.fp_variant == "auto":
        variant = autotune.tune(c, x_true, maps)
    else:
        variant = {"ldg": 0, "tma": core._lib.CCT_VARIANT_FP_TMA, "slices2": core._lib.CCT_VARIANT_FP_SLICES2}[
            a.fp_variant]
        c.variant = variant
    c_os.variant = variant
    clean = c.fp(x_true, maps)
    gen = torch.Generator(device=dev)
    gen.manual_seed(a.seed + rank)
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * a.peak, generator=gen)
    del clean
    b_os = b[:, :, perm_t].contiguous()

    # calibration (untimed): the plain solver's residual after `iters` iterations defines the target
    calib = engine.BatchedSolver(c, maps, b, "mlem")
    calib.run(a.iters, check_every=a.iters, use_graph=False)
    torch.cuda.synchronize(dev)
    tol_np = calib.residuals.cpu().numpy() * (1 + 1e-9)
    del calib
    max_iters = 2 * a.iters

    plain = engine.BatchedSolver(c, maps, b, "mlem", tolerance=tol_np)
    subsets = engine.OrderedSubsets(c_os, maps, b_os, schedule)
    judge = engine.BatchedSolver(c_os, maps, b_os, "mlem", tolerance=tol_np, x_shared=subsets.x)
    launches_os_pass = sum(k * 3 * p for k, p in schedule)

    fp_ms, bp_ms, launches = [], [], [0]

    def solve_to_tol(solver, timed: bool, budget: int, block: int = 10) -> int:
        its, active = 0, S
        while its < budget and active > 0:
            evs = []
            for _ in range(block):
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                solver.step_timed(*e)
                evs.append(e)
            its += block
            launches[0] += 3 * block
            block_full = active == S
            active = int(solver.active.sum().item())  # synchronises the stream
            if timed and block_full:
                # kernel times only from blocks in which every slice was active (full-batch launches)
                for e in evs:
                    fp_ms.append(e[0].elapsed_time(e[1]))
                    bp_ms.append(e[1].elapsed_time(e[2]))
        return its

    def step_plain(timed: bool) -> float:
        maps_natural()
        launches[0] += 2 * passes
        plain.reset()
        solve_to_tol(plain, timed, max_iters)
        return float(plain.iterations.float().mean().item())

    phase_ms = []  # (maps, passes, judge) of timed ordered-subsets steps

    def step_subsets(timed: bool) -> float:
        # NVTX ranges name the phases for a profiler (ncu --nvtx --nvtx-include "subset_passes/")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        torch.cuda.nvtx.range_push("compute_maps")
        maps_subsets()
        torch.cuda.nvtx.range_pop()
        ev[1].record()
        launches[0] += 2 * passes + launches_os_pass
        torch.cuda.nvtx.range_push("subset_passes")
        subsets.reset()
        subsets.run()
        torch.cuda.nvtx.range_pop()
        ev[2].record()
        torch.cuda.nvtx.range_push("judge_mlem")
        judge.reset(subsets.x)
        solve_to_tol(judge, False, max_iters, block=2)
        torch.cuda.nvtx.range_pop()
        ev[3].record()
        if timed:
            phase_ms.append(ev)
        return float((judge.iterations.float() + subsets.passes).mean().item())

    def timed_steps(fn, k: int) -> tuple[float, float]:
        distributed.barrier(dev)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        its = [fn(True) for _ in range(k)]
        t1.record()
        distributed.barrier(dev)
        return t0.elapsed_time(t1) / 1e3, float(np.mean(its))

    paths = {"plain": step_plain, "subsets": step_subsets}
    headline = {"auto": "subsets", "plain": "plain", "subsets": "subsets"}[a.method]
    if headline not in paths:
        raise RuntimeError(f"path {headline!r} is unavailable")
    for _ in range(a.warmup):
        for fn in paths.values():
            fn(False)

    results = {}
    fp_keep, bp_keep = [], []
    for name, fn in paths.items():
        if name == headline:
            continue
        fp_ms.clear(); bp_ms.clear()
        secs, its = timed_steps(fn, a.steps)
        secs = distributed.max_over_ranks(secs, dev)
        results[name] = {"value": S * a.steps * world / secs, "unit": UNIT, "mean_iterations": its,
                         "ms_per_step": secs / a.steps * 1e3}
        if name == "plain":
            fp_keep, bp_keep = list(fp_ms), list(bp_ms)
    # the headline path, with the clock sampler running
    clocks = ClockSampler(local)
    clocks.start()
    launches[0] = 0
    fp_ms.clear(); bp_ms.clear()
    head_s, head_its = timed_steps(paths[headline], a.steps)
    head_s = distributed.max_over_ranks(head_s, dev)
    clk = clocks.stop()
    head_launches = launches[0]
    result = {"plain": plain, "subsets": judge}[headline]
    converged = int((result.residuals.cpu().numpy() <= tol_np).sum())
    total_slices = S * a.steps * world
    value = total_slices / head_s
    if headline == "plain":
        fp_keep, bp_keep = list(fp_ms), list(bp_ms)

    # ---- e2e: the headline step from pinned host buffers, copies inside the timed region.  A
    # step's inputs (mu, copied once: mu_out = mu_in here, and the data) go host -> device on a side
    # stream into staging buffers while the previous step computes; the step moves them into its
    # working buffers with a device copy, and its reconstruction comes back to pinned memory.
    mu_h = torch.from_numpy(mus_h).pin_memory()
    b_h = b.cpu().pin_memory()
    x_h = torch.empty((S, n, n), dtype=torch.float32).pin_memory()
    side = torch.cuda.Stream(dev)
    mu_stage, b_stage = torch.empty_like(mu_in), torch.empty_like(b)
    pipe = {"staged": None, "free": torch.cuda.Event(), "left": 0}
    pipe["free"].record()

    def stage_inputs():
        side.wait_event(pipe["free"])
        with torch.cuda.stream(side):
            mu_stage.copy_(mu_h, non_blocking=True)
            b_stage.copy_(b_h, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(side)
        pipe["staged"] = ev

    def e2e_step(_timed):
        if pipe["staged"] is None:
            stage_inputs()
        cur = torch.cuda.current_stream(dev)
        cur.wait_event(pipe["staged"])
        mu_in.copy_(mu_stage)
        mu_out.copy_(mu_stage)
        b.copy_(b_stage)
        pipe["free"].record(cur)
        pipe["staged"] = None
        pipe["left"] -= 1
        if pipe["left"] > 0:
            stage_inputs()  # the next step's inputs, overlapping this step's compute
        if headline == "subsets":
            torch.index_select(b, 2, perm_t, out=b_os)
            subsets.set_data(b_os)
        its = paths[headline](False)
        x_h.copy_(result.x, non_blocking=True)
        return its

    pipe["left"] = 1
    e2e_step(False)  # warm-up: no copy carried into the timed steps
    pipe["left"] = a.steps
    e2e_s, _ = timed_steps(e2e_step, a.steps)
    e2e_s = distributed.max_over_ranks(e2e_s, dev)
    h2d = S * (n * n + a.angles * n) * 4
    d2h = S * n * n * 4

    extra = {}
    if rank == 0 and not a.no_extra_legs:
        extra = extra_legs(a, dev, c, maps, mus_h, xs_h, b, tol_np, max_iters, variant)
    learned_leg = None
    if os.path.exists(WEIGHTS) and not a.no_learned_leg:
        learned_leg = run_learned_leg(a, dev, rank, world, maps, ws, variant, schedule)

    # ---- roofline of the dominant kernel (attenuated fp with the fused MLEM epilogue, plain path)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    else:
        peak = 6650.0
        peak_src = "fallback"
    map_bytes = 4 if a.maps_dtype == "float32" else 2
    fp_bytes = S * (a.angles * n * n * map_bytes + n * n * 4 + 2 * a.angles * n * 4)
    fp_avg_s = float(np.mean(fp_keep)) / 1e3 if fp_keep else float("nan")
    bp_avg_s = float(np.mean(bp_keep)) / 1e3 if bp_keep else float("nan")
    achieved = fp_bytes / fp_avg_s / 1e9
    solver_desc = {
        "plain": "plain MLEM (cold start)",
        "subsets": f"MLEM warm-started by ordered-subsets EM passes {schedule} (subsets, passes), then MLEM to the residual",
    }
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": head_s / a.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded ellipse phantoms, disk attenuation, Poisson 1e5 peak counts)",
        "config": {
            "workload": workload_name(a), "n": n, "angles": a.angles, "slices_per_gpu": S, "maps_dtype": a.maps_dtype,
            "target": f"KL residual of plain MLEM after {a.iters} iterations (per slice)",
            "solver": solver_desc[headline],
            "parallelism": f"slices sharded over {world} GPU(s), no collective on the data path",
            "l2": "inputs larger than L2 (maps %.0f MB per slice)" % (a.angles * n * n * map_bytes / 1e6),
            "mean_iterations": head_its, "converged_slices_last_step": converged,
            "fp_variant": FP_VARIANT_NAMES[variant],
        },
        "roofline": {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            # DRAM read + write bytes per launch from one ncu capture of each variant on 4 slices
            # (fp_kernel 2.8680 GB, fp_tma_kernel 2.9200 GB, fp_pair_kernel 2.7911 GB), scaled by the
            # slices per launch; only for the captures' own configuration
            "traffic": (FP_TRAFFIC_PER_SLICE[variant] * S)
            if (n == 512 and a.angles == 720 and a.maps_dtype == "float32") else None,
            "kernel": FP_KERNEL_NAMES[variant] + "<MLEM> (attenuated fp + ratio + KL residual)",
            "peak_source": peak_src, "fp_launch_us": fp_avg_s * 1e6, "bp_launch_us": bp_avg_s * 1e6,
            "algorithmic_bytes_per_launch": fp_bytes,
        },
        "e2e": {"value": total_slices / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": head_launches,
        "clocks": clk,
    }
    if headline == "subsets" and phase_ms:
        torch.cuda.synchronize(dev)
        ph = np.array([[e[i].elapsed_time(e[i + 1]) for i in range(3)] for e in phase_ms])
        line["phases_ms_per_step"] = dict(zip(("compute_maps", "subset_passes", "judge_mlem"), ph.mean(axis=0).tolist()))
    for name, r in results.items():
        line[name] = dict(r, solver=solver_desc[name])
    if learned_leg is not None:
        line["learned"] = learned_leg
    line.update(extra)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        plain_its = results.get("plain", {}).get("mean_iterations", float(a.iters))
        line["cpu_baseline"] = cpu_baseline(a, plain_its)
        cpu_v = line["cpu_baseline"]["value"]
        # like for like: the same algorithm (plain MLEM to the plain residual) on both sides; the
        # headline ratio also contains the ordered-subsets warm start's algorithmic gain
        line["vs_cpu"] = {
            "plain_gpu_over_cpu": results["plain"]["value"] / cpu_v if "plain" in results else None,
            "dropin_e2e_over_cpu": (extra["dropin_e2e"]["value"] / cpu_v) if "dropin_e2e" in extra else None,
            "headline_over_cpu": value / cpu_v,
            "note": "plain_gpu_over_cpu and dropin_e2e_over_cpu compare plain MLEM with plain MLEM; "
                    "headline_over_cpu also counts the ordered-subsets warm start (fewer passes)",
        }
    if rank == 0:
        print(json.dumps(line), flush=True)
    distributed.finalize()


def run_learned_leg(a, dev, rank, world, maps, ws, variant, schedule) -> dict:
    """The learned warm start on the learned part's own data at the benchmark shape: seeded textured
    phantoms (5-20 ellipses with a Gaussian-random-field texture), disk
    attenuation with mu in [0, 0.02] and emitted mu = 0.7 incident mu, Poisson data at 1e4 peak
    counts, held-out seeds.  Three paths on the same slices, each step = compute_maps + the solve
    until every slice reaches the KL residual plain MLEM reaches after 200 iterations: plain MLEM,
    the ordered-subsets passes alone, and the learned start (a snapshot pass, the network, one
    pass per ordered-subsets level) followed by MLEM, which judges every slice."""
    import torch

    from pycorrectedemissionct_b200 import core, distributed, engine
    from pycorrectedemissionct_b200 import train_warmstart as tw
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    net = WarmStartNet(device=dev)
    net.load(WEIGHTS)
    S, n, A = a.slices, a.n, a.angles
    levels = net.os_levels(A)
    if not levels:
        return {"unavailable": "the committed network reads MLEM iterates, not ordered-subsets snapshots"}
    seeds = [a.seed + 500_000 + rank * S + k for k in range(S)]
    c4, maps4, b4, _, mu4 = tw.synth_batch(n, A, seeds, 0.02, a.learned_peak, dev, subsets=levels, return_mu=True)
    c4.variant = variant
    del maps4
    maps4 = maps  # the shared maps buffer, recomputed by every step in this leg's angle order
    mu4_out = 0.7 * mu4

    def maps_step():
        core.compute_maps(mu4, mu4_out, c4.angles_rad32, maps_dtype=a.maps_dtype, workspace=ws, out=maps4,
                          emitted_scale=0.7)

    maps_step()
    calib = engine.BatchedSolver(c4, maps4, b4, "mlem")
    calib.run(a.iters, check_every=a.iters, use_graph=False)
    tol = calib.residuals.cpu().numpy() * (1 + 1e-9)
    del calib
    plain = engine.BatchedSolver(c4, maps4, b4, "mlem", tolerance=tol)
    os_ = engine.OrderedSubsets(c4, maps4, b4, [(levels[0], 1), (levels[1], 1)])
    judge = engine.BatchedSolver(c4, maps4, b4, "mlem", tolerance=tol, x_shared=os_.x)
    tau = plain.tau

    def run_judge(block):
        its = 0
        while its < 2 * a.iters and int(judge.active.sum().item()) > 0:
            for _ in range(block):
                judge.step()
            its += block
        return judge.iterations

    def step_plain():
        maps_step()
        plain.reset()
        plain.run(2 * a.iters, check_every=10)
        return float(plain.iterations.float().mean().item()), int(plain.iterations.max().item())

    graphs = {}

    def graphed(name, fn):
        """fn's launches as one CUDA graph: eager on the first call (every kernel loaded), captured
        on the second, replayed from then on (both warm starts alike)."""
        g = graphs.get(name)
        if g is None:
            fn()
            graphs[name] = "eager"
            return
        if g == "eager":
            torch.cuda.synchronize(dev)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                fn()
            graphs[name] = g
        g.replay()

    def subsets_start():
        os_.reset()
        os_.run_level(0, 2)
        os_.run_level(1)

    def learned_start():
        os_.reset()
        tw.learned_start(net, os_, c4, b4, tau)

    def step_subsets():
        maps_step()
        graphed("subsets", subsets_start)
        judge.reset(os_.x)
        it = run_judge(1)
        return float(it.float().mean().item()) + 3, int(it.max().item()) + 3

    def step_learned():
        maps_step()
        graphed("learned", learned_start)
        judge.reset(os_.x)
        it = run_judge(1)
        return float(it.float().mean().item()) + 3, int(it.max().item()) + 3

    out = {}
    for name, fn, k in (("plain", step_plain, 1), ("subsets", step_subsets, a.steps), ("learned", step_learned, a.steps)):
        for _ in range(1 if name == "plain" else max(1, a.warmup)):
            fn()
        distributed.barrier(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        its = [fn() for _ in range(k)]
        e1.record()
        distributed.barrier(dev)
        secs = distributed.max_over_ranks(e0.elapsed_time(e1) / 1e3, dev)
        out[name] = {"value": S * k * world / secs, "unit": UNIT, "ms_per_step": secs / k * 1e3,
                     "mean_passes": float(np.mean([i[0] for i in its])), "max_passes": max(i[1] for i in its)}
    res = {
        "value": out["learned"]["value"], "unit": UNIT, "ms_per_step": out["learned"]["ms_per_step"],
        "mean_passes": out["learned"]["mean_passes"], "max_passes": out["learned"]["max_passes"],
        "solver": (f"learned start (one ordered-subsets pass over {levels[0]} subsets keeping 10 snapshots, the "
                   f"encoder-decoder, one pass over {levels[0]} and one over {levels[1]} subsets), then MLEM to the "
                   "plain residual"),
        "data": (f"textured slices at {n}x{n}x{A}: {S} held-out seeds, textured phantoms, mu in [0, 0.02], "
                 f"emitted mu 0.7 incident, Poisson {a.learned_peak:g} peak counts"),
        "same_data": {"plain": out["plain"], "subsets": dict(out["subsets"], schedule=[(levels[0], 2), (levels[1], 1)])},
        "learned_over_plain": out["learned"]["value"] / out["plain"]["value"],
        "learned_over_subsets": out["learned"]["value"] / out["subsets"]["value"],
    }
    del plain, judge, os_, b4
    return res


def fp64_errors(a, c, maps, mu0, x0, dev) -> dict:
    """Relative L2 errors of the GPU maps, attenuated fp and reference bp of one headline slice
    against the FP64 oracle, on every k-th angle of the full set (the oracle needs minutes per
    slice for all 720)."""
    import torch

    from oracle import port
    from pycorrectedemissionct_b200 import core

    step = max(1, a.fp64_angle_step)
    idx = np.arange(0, c.n_angles, step)
    rad32 = c.angles_rad32[idx]
    _, deg32 = port.backend_angles(rad32)
    workers = os.cpu_count() or 1
    t0 = time.perf_counter()
    mu64 = mu0.astype(np.float64)
    ref_maps = port.compute_maps(mu64, mu64, rad32, workers=workers)
    x64 = x0.astype(np.float64)
    ref_fp = port.fp_xrf(x64, ref_maps, deg32, workers=workers)
    y = ref_fp / ref_fp.max()
    ref_bp = port.bp_uncorrected(y, deg32, c.n, workers=workers)
    sub = core.XrfCore(c.n, rad32, device=dev)
    sub.variant = c.variant
    m_sub = maps[0:1, torch.from_numpy(idx).to(dev)].contiguous()
    xs = torch.from_numpy(x0).to(dev)[None]

    def rel(u, v):
        u = np.asarray(u, np.float64)
        return float(np.linalg.norm(u - v) / np.linalg.norm(v))

    out = {
        "maps": rel(m_sub[0].float().cpu().numpy(), ref_maps),
        "maps_then_fp": rel(sub.fp(xs, m_sub)[0, 0].cpu().numpy(), ref_fp),
        "fp_on_fp64_maps": rel(sub.fp(xs, torch.from_numpy(ref_maps.astype(np.float32)).to(dev)[None])[0, 0].cpu().numpy(),
                               ref_fp),
        "bp_reference": rel(sub.bp(torch.from_numpy(y.astype(np.float32)).to(dev)[None, None], "reference")[0].cpu().numpy(),
                            ref_bp),
        "sample": f"slice 0 of the batch, {len(idx)} of {c.n_angles} angles (every {step}th), FP64 oracle port "
                  f"({time.perf_counter() - t0:.1f} s on {workers} host threads)",
        "bound": 1e-5,
        # kept for the BF16 leg (removed before printing)
        "_ref": (idx, ref_maps, ref_fp, sub, xs),
    }
    return out


def extra_legs(a, dev, c, maps, mus_h, xs_h, b, tol_np, max_iters, variant) -> dict:
    """Legs reported beside the headline: the drop-in call (numpy in and out) end to end, FP64
    errors of the headline slice, and plain MLEM with BF16-stored maps."""
    import torch

    from pycorrectedemissionct_b200 import autotune, core, engine, projectors, solvers

    out = {}
    n, S = a.n, a.slices
    angles = np.linspace(0, 2 * np.pi, a.angles, endpoint=False)
    mu_t = torch.from_numpy(mus_h).to(dev)
    # the shared maps buffer holds the last timed path's angle order: natural order again
    core.compute_maps(mu_t, mu_t, c.angles_rad32, out=maps)
    # ---- the drop-in call a corrct user makes: maps from mu on the GPU, plain MLEM to the
    # plain residual, numpy in and out, timed end to end on the host clock
    mu0, b0, tol0 = mus_h[0], b[0, 0].cpu().numpy(), float(tol_np[0])

    def dropin_once():
        p = projectors.ProjectorAttenuationXRF((n, n), angles, att_in=mu0, att_out=mu0, verbose=False)
        x, info = solvers.MLEM(tolerance=tol0)(p, b0, iterations=max_iters)
        return info.iterations, x

    dropin_once()
    reps = max(1, min(3, a.steps))
    t0 = time.perf_counter()
    its = [dropin_once()[0] for _ in range(reps)]
    dt = (time.perf_counter() - t0) / reps
    out["dropin_e2e"] = {
        "value": 1.0 / dt, "unit": UNIT, "mean_iterations": float(np.mean(its)), "seconds_per_slice": dt,
        "h2d_bytes_per_step": 2 * n * n * 4 + a.angles * n * 4, "d2h_bytes_per_step": n * n * 4,
        "call": "projectors.ProjectorAttenuationXRF((n, n), angles, att_in=mu, att_out=mu) + "
                "solvers.MLEM(tolerance)(p, b, iterations) on one numpy slice (plain MLEM, host clock)",
    }
    # ---- FP64 oracle errors of the headline slice
    try:
        out["fp64_error"] = fp64_errors(a, c, maps, mus_h[0], xs_h[0], dev)
    except Exception as exc:  # the oracle is a checker: report, never fail the bench on it
        out["fp64_error"] = {"unavailable": repr(exc)}
    # ---- BF16-stored maps: map error against FP32 maps, plain MLEM (200 iterations) speed
    m16 = torch.empty((S, a.angles, 1, n, n), dtype=torch.bfloat16, device=dev)
    ws = torch.empty(16 * core.maps_entry_bytes(n, S), dtype=torch.uint8, device=dev)
    core.compute_maps(mu_t, mu_t, c.angles_rad32, maps_dtype="bfloat16", workspace=ws, out=m16)
    torch.cuda.synchronize(dev)
    e16 = float(((m16[0].float() - maps[0].float()).double().norm() / maps[0].double().norm()).item())
    c16 = core.XrfCore(n, angles, device=dev)
    bf16_variant = autotune.tune(c16, torch.from_numpy(xs_h).to(dev), m16)
    bf16_fp64 = {}
    ref = out.get("fp64_error", {}).pop("_ref", None)
    if ref is not None:
        idx, ref_maps, ref_fp, sub, xs = ref
        m16_sub = m16[0:1, torch.from_numpy(idx).to(dev)].contiguous()
        bf16_fp64 = {
            "maps_rel_l2_vs_fp64": float(np.linalg.norm(m16_sub[0].float().cpu().numpy() - ref_maps)
                                         / np.linalg.norm(ref_maps)),
            "maps_then_fp_rel_l2_vs_fp64": float(np.linalg.norm(sub.fp(xs, m16_sub)[0, 0].cpu().numpy() - ref_fp)
                                                 / np.linalg.norm(ref_fp)),
        }
        del m16_sub
    sv = engine.BatchedSolver(c16, m16, b, "mlem")
    sv.step()
    fps, bps = [], []
    for _ in range(10):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        sv.step_timed(*e)
        torch.cuda.synchronize(dev)
        fps.append(e[0].elapsed_time(e[1]))
        bps.append(e[1].elapsed_time(e[2]))
    sv.reset()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    core.compute_maps(mu_t, mu_t, c.angles_rad32, maps_dtype="bfloat16", workspace=ws, out=m16)
    sv.run(a.iters, check_every=a.iters, use_graph=True)
    ev[1].record()
    torch.cuda.synchronize(dev)
    secs = ev[0].elapsed_time(ev[1]) / 1e3
    res_ratio = (sv.residuals.cpu().numpy() / tol_np).tolist()
    out["bf16_maps"] = {
        "plain_mlem_slices_per_s": S / secs, "iterations": a.iters,
        "fp_launch_us": 1e3 * float(np.median(fps)), "bp_launch_us": 1e3 * float(np.median(bps)),
        "maps_rel_l2_vs_fp32": e16, **bf16_fp64, "fp_variant": FP_VARIANT_NAMES[bf16_variant],
        "final_residual_over_fp32_target": [float(np.min(res_ratio)), float(np.max(res_ratio))],
        "note": "maps stored in bfloat16 (8-bit mantissa), FP32 arithmetic; errors against the FP64 oracle on the "
                "fp64_error sample",
    }
    del m16, ws, sv
    return out


def run_waves(a):
    """Independent slices in HBM-sized waves: --wave-slices independent 512x512 slices over 720 angles, plain MLEM for
    200 iterations with all slices of a wave in one launch per operator and each block of
    iterations in a CUDA graph; waves sized to HBM; FP32 and BF16 maps.  Data synthesis is
    untimed; each wave's timed work is compute_maps + 200 MLEM iterations."""
    import torch

    from pycorrectedemissionct_b200 import core, engine, phantoms

    dev = torch.device("cuda", 0)
    n, A = a.n, a.angles
    angles = np.linspace(0, 2 * np.pi, A, endpoint=False)
    c = core.XrfCore(n, angles, device=dev)
    out = {}
    for dtype, mb in (("float32", 4), ("bfloat16", 2)):
        free = torch.cuda.mem_get_info(dev)[0]
        per_slice = A * n * n * mb + 8 * A * n * 4 + 6 * n * n * 4
        wave = max(1, min(a.wave_slices, int(0.8 * free // per_slice)))
        tdt = torch.float32 if dtype == "float32" else torch.bfloat16
        total_s, done = 0.0, 0
        ws = torch.empty(16 * core.maps_entry_bytes(n, wave), dtype=torch.uint8, device=dev)
        maps = torch.empty((wave, A, 1, n, n), dtype=tdt, device=dev)
        for w0 in range(0, a.wave_slices, wave):
            k = min(wave, a.wave_slices - w0)
            xs, mus = [], []
            for s in range(w0, w0 + k):
                r = phantoms.slice_rng(a.seed, s)
                xs.append(phantoms.ellipse_phantom(n, r, 12))
                mus.append(phantoms.disk_attenuation(n, r, 0.01))
            x = torch.from_numpy(np.stack(xs)).to(dev)
            mu = torch.from_numpy(np.stack(mus)).to(dev)
            mk = maps[:k]
            core.compute_maps(mu, mu, c.angles_rad32, maps_dtype=dtype, workspace=ws, out=mk)
            clean = c.fp(x, mk)
            gen = torch.Generator(device=dev)
            gen.manual_seed(a.seed + w0)
            bb = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * a.peak, generator=gen)
            del clean
            sv = engine.BatchedSolver(c, mk, bb, "mlem")
            torch.cuda.synchronize(dev)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record()
            core.compute_maps(mu, mu, c.angles_rad32, maps_dtype=dtype, workspace=ws, out=mk)
            sv.run(a.iters, check_every=10, use_graph=True)
            ev[1].record()
            torch.cuda.synchronize(dev)
            total_s += ev[0].elapsed_time(ev[1]) / 1e3
            done += k
            del sv, bb, x, mu
        out[dtype] = {"slices": done, "wave": wave, "seconds": total_s, "slices_per_s": done / total_s}
        del maps, mk, ws  # mk views maps: release both before the next map type's buffer
        torch.cuda.empty_cache()
    line = {"metric": f"plain MLEM slices/s, {a.wave_slices} slices of {n}x{n}x{A} in HBM-sized waves",
            "value": out["float32"]["slices_per_s"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "config": {"workload": "independent 512x512x720 slices in HBM-sized waves, 200 MLEM iterations, FP32 vs BF16 maps",
                       "iterations": a.iters}, "float32": out["float32"], "bfloat16": out["bfloat16"],
            "data": "synthetic", "dtype": "f32"}
    print(json.dumps(line), flush=True)


def run_channels(a):
    """Fluorescence channels c = 0..7 whose emitted attenuation is s_c times the incident
    one (s_c in {0.5, 0.75, 1, 1.25, 1.5, 2, 2.5, 3}), 1024 x 1024 slices over 1440 angles, Poisson
    data at 1e4 peak counts, PDHG with the KL data term and isotropic TV (lambda 1e-2) for 300
    iterations.  The maps are line-integral fields (L_in and L_out: two planes per angle and
    field slice, shared by its 8 channels).  One wave of --field-slices field slices is solved in
    full; the full configuration (64 field slices, 6 TB of FP32 maps or 0.8 TB of fields) runs as
    64 / field_slices such waves.  Timed: compute_maps (fields) + 300 PDHG iterations; data
    synthesis untimed."""
    import torch

    from pycorrectedemissionct_b200 import core, engine, phantoms

    dev = torch.device("cuda", 0)
    n, A, F, iters = 1024, 1440, max(1, a.field_slices), 300
    scales = np.array([0.5, 0.75, 1.0, 1.25, 1.5, 2.0, 2.5, 3.0], dtype=np.float32)
    C = len(scales)
    angles = np.linspace(0, 2 * np.pi, A, endpoint=False)
    c = core.XrfCore(n, angles, device=dev)
    c.set_channels(scales)
    xs, mus = [], []
    for f in range(F):
        r = phantoms.slice_rng(a.seed + 31, f)
        mus.append(phantoms.disk_attenuation(n, r, 0.01))
        for ch in range(C):
            xs.append(phantoms.ellipse_phantom(n, phantoms.slice_rng(a.seed + 37, f * C + ch), 12))
    mu = torch.from_numpy(np.stack(mus)).to(dev)
    x_true = torch.from_numpy(np.stack(xs)).to(dev)
    ws = torch.empty(8 * core.maps_entry_bytes(n, F), dtype=torch.uint8, device=dev)
    fields = core.compute_maps(mu, mu, c.angles_rad32, maps_dtype="fields-float32", workspace=ws)
    clean = c.fp(x_true, fields)
    gen = torch.Generator(device=dev)
    gen.manual_seed(a.seed)
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * 1e4, generator=gen)
    del clean
    # fp launch time (the PDHG step's fp reads x_relax with the same fields)
    out = torch.empty_like(b)
    c.fp(x_true, fields, out=out)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(3):
        c.fp(x_true, fields, out=out)
    ev[1].record()
    torch.cuda.synchronize(dev)
    fp_s = ev[0].elapsed_time(ev[1]) / 3 / 1e3
    del out
    sv = engine.BatchedSolver(c, fields, b, "pdhg", tv_lambda=1e-2)
    sv.run(10, check_every=10, use_graph=True)
    torch.cuda.synchronize(dev)
    sv = engine.BatchedSolver(c, fields, b, "pdhg", tv_lambda=1e-2)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    core.compute_maps(mu, mu, c.angles_rad32, maps_dtype="fields-float32", workspace=ws, out=fields)
    sv.run(iters, check_every=10, use_graph=True)
    ev[1].record()
    torch.cuda.synchronize(dev)
    secs = ev[0].elapsed_time(ev[1]) / 1e3
    # FP64 oracle: channel maps and fp of field slice 0's channel s_c = 3 on every 60th angle
    err = {}
    try:
        from oracle import port

        idx = np.arange(0, A, 60)
        rad32 = c.angles_rad32[idx]
        _, deg32 = port.backend_angles(rad32)
        mu64 = mus[0].astype(np.float64)
        ref = port.compute_maps(mu64, float(scales[-1]) * mu64, rad32, workers=os.cpu_count() or 1)
        f0 = fields[0, torch.from_numpy(idx).to(dev)].double().cpu().numpy()
        got = np.exp(-(f0[:, 0] + np.float64(scales[-1]) * f0[:, 1]))[:, None]
        err["channel_maps_s3"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        sub = core.XrfCore(n, rad32, device=dev)
        sub.set_channels(scales[-1:])
        fsub = fields[0:1, torch.from_numpy(idx).to(dev)].contiguous()
        fp = sub.fp(x_true[C - 1:C], fsub)[0, 0].cpu().numpy()
        ref_fp = port.fp_xrf(xs[C - 1].astype(np.float64), ref, deg32, workers=os.cpu_count() or 1)
        err["channel_fp_s3"] = float(np.linalg.norm(fp - ref_fp) / np.linalg.norm(ref_fp))
        err["sample"] = f"field slice 0, channel s_c = 3, {len(idx)} of {A} angles, FP64 oracle port"
    except Exception as exc:
        err["unavailable"] = repr(exc)
    S = F * C
    map_once = A * 2 * n * n * 4 * F                      # the two planes, read once per field slice
    per_channel = S * (n * n * 4 + A * n * 4)             # x read, sinogram written
    line = {
        "metric": "slices x channels per s, PDHG-KL-TV 300 iterations, 1024x1024x1440, 8 channels",
        "value": S / secs, "unit": "slice-channels/s", "n_gpus": 1, "higher_is_better": True,
        "ms_per_step": secs * 1e3, "dtype": "f32", "data": "synthetic (seeded ellipse phantoms, disk attenuation)",
        "config": {"workload": f"{F} field slice(s) x {C} channels per wave (the full 64 field slices run as "
                               f"{-(-64 // F)} waves)", "n": n, "angles": A, "channel_scales": scales.tolist(),
                   "iterations": iters, "tv_lambda": 1e-2, "maps": "line-integral fields, 2 planes per angle"},
        "fp_roofline": {"fp_launch_us": fp_s * 1e6, "algorithmic_bytes": map_once + per_channel,
                        "achieved_GBps": (map_once + per_channel) / fp_s / 1e9,
                        "note": "fields counted once per field slice (channels share them through L2)"},
        "fp64_error": err,
    }
    print(json.dumps(line), flush=True)


def run_ragged(a):
    """Ragged stream (a seeded sample of the mixed-size workload): slices with sides drawn from
    {128, 256, 384, 512, 768, 1024} and angle counts uniform in [90, 1440], half SIRT (150
    iterations), half MLEM to the residual plain MLEM reaches after 200 iterations (calibrated,
    untimed), solved by ``RaggedStream`` with the ordered-subsets warm start and, for
    comparison, from the cold start.  Data synthesis is untimed."""
    import torch

    from pycorrectedemissionct_b200 import core, phantoms, stream

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(a.seed)
    sizes = (128, 256, 384, 512, 768, 1024)
    jobs = []
    for k in range(a.ragged_slices):
        n = int(rng.choice(sizes))
        n_ang = int(rng.integers(90, 1441))
        r = phantoms.slice_rng(a.seed + 7, k)
        x = phantoms.ellipse_phantom(n, r, 12)
        mu = phantoms.disk_attenuation(n, r, 0.02)
        peak = float(10 ** rng.uniform(3, 5))
        angles = np.linspace(0, 2 * np.pi, n_ang, endpoint=False)
        c = core.XrfCore(n, angles, device=dev)
        mu_t = torch.from_numpy(mu).to(dev)[None]
        maps = core.compute_maps(mu_t, 0.7 * mu_t, c.angles_rad32)
        clean = c.fp(torch.from_numpy(x).to(dev)[None], maps)
        gen = torch.Generator(device=dev)
        gen.manual_seed(a.seed + k)
        b = torch.poisson(clean / clean.max() * peak, generator=gen)[0, 0].cpu().numpy()
        del maps, clean
        jobs.append(stream.Job(n, angles, mu, 0.7 * mu, b, method="sirt" if k % 2 else "mlem"))
    mlem = [j for j in jobs if j.method == "mlem"]
    stream.RaggedStream(dev, warm_start=False).solve(mlem, max_iterations=a.iters)  # calibration
    for j in mlem:
        j.tolerance = j.extra["residual"] * (1 + 1e-9)

    def reset():
        for j in jobs:
            j.x, j.iterations_done, j.finished_s = None, 0, 0.0

    net = None
    legs = [x.strip() for x in a.ragged_legs.split(",") if x.strip()]
    if "learned" in legs:
        if os.path.exists(WEIGHTS):
            from pycorrectedemissionct_b200.warmstart import WarmStartNet

            net = WarmStartNet(device=dev)
            net.load(WEIGHTS)
        else:
            legs.remove("learned")
    out = {}
    for name in legs:
        warm = {"subsets": True, "learned": "learned", "plain": False}[name]
        reset()
        st = stream.RaggedStream(dev, warm_start=warm, net=net)  # schedules follow each slice's angle count
        r = st.solve(jobs, max_iterations=3 * a.iters)  # room for a fallback restart after 200
        r["launches"] = st.launches
        r["mlem_mean_passes"] = float(np.mean([j.iterations_done for j in mlem]))
        r["converged"] = int(sum(j.extra["residual"] <= j.tolerance for j in mlem))
        r["restarted"] = int(sum(bool(j.extra.get("restarted")) for j in mlem))
        out[name] = r
    head = "learned" if "learned" in out else legs[0]
    line = {
        "metric": "ragged stream slices/s (mixed sizes and angle counts, half SIRT 150, half MLEM to residual)",
        "value": out[head]["slices_per_s"], "unit": "slices/s", "n_gpus": 1, "higher_is_better": True,
        "config": {"workload": f"{a.ragged_slices} slices, sides {list(sizes)}, angles U[90, 1440], mu <= 0.02, "
                               "peaks log-U[1e3, 1e5]", "ragged": "one launch per operator over all groups of a wave",
                   "headline_start": head},
        "p50_s": out[head]["p50_s"], "p99_s": out[head]["p99_s"], **out,
        "data": "synthetic", "dtype": "f32",
    }
    print(json.dumps(line), flush=True)


def parse_schedule(text: str) -> list[tuple[int, int]]:
    """'30:10,10:10' -> [(30, 10), (10, 10)] (subsets, passes)."""
    out = []
    for part in text.split(","):
        k, p = part.split(":")
        out.append((int(k), int(p)))
    return out


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "ragged":
        run_ragged(a)
    elif a.workload == "waves":
        run_waves(a)
    elif a.workload == "channels":
        run_channels(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
