"""Benchmark: converged slices/s of attenuated XRF MLEM on 512x512-pixel, 720-angle slices.

One step = the hot path over one batch of synthetic slices already resident in HBM:
``compute_maps`` (incident + emitted attenuation maps) followed by MLEM with the reference's
KL-residual stopping rule, run until every slice reaches the residual that the plain solver
reaches after 200 iterations (calibrated once, untimed).  ``value`` = slices converged per
second over the timed steps (max over ranks; weak scaling, each rank owns its own slices).

``e2e`` repeats the step through the public API from pinned host buffers (mu_in, mu_out and the
data copied in, the reconstruction copied out inside the timed region).  ``--impl reference``
times the reference algorithm's CPU implementation (the oracle port in ``oracle/``) on the host
cores on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged slices/s, XRF MLEM 512²x720 to fixed residual: plain vs warm start"
UNIT = "slices/s"


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
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv") if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else f"/tmp/cct_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL,
            )
        except (OSError, FileNotFoundError):
            self.proc = None

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
    rad32, deg32 = port.backend_angles(angles[:: a.angles // sample][:sample])
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
            f"({t3 - t0:.1f} s), scaled to {a.angles} angles and {iterations_per_slice:.1f} MLEM iterations per slice"
        ),
        "seconds_per_slice": t_slice,
    }


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    iters = float(a.iters)
    samples = []
    for _ in range(max(1, a.warmup)):
        cpu_baseline(a, iters)
    for _ in range(max(1, a.steps)):
        samples.append(cpu_baseline(a, iters))
    v = float(np.median([s["value"] for s in samples]))
    cb = dict(samples[-1])
    cb["value"] = v
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded ellipse phantoms, disk attenuation)",
        "config": {"workload": workload_name(a), "n": a.n, "angles": a.angles, "mlem_iterations": a.iters},
        "impl": "reference", "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------- ours
def run_ours(a):
    import torch

    from pycorrectedemissionct_b200 import core, engine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    xs_h, mus_h = make_inputs(a, rank)
    angles = np.linspace(0, 2 * np.pi, a.angles, endpoint=False)
    rad32 = np.array(angles, dtype=np.float32)
    S, n = a.slices, a.n
    c = core.XrfCore(n, angles, device=dev)
    mu_in = torch.from_numpy(mus_h).to(dev)
    mu_out = mu_in.clone()  # mu_out = mu_in for this workload
    x_true = torch.from_numpy(xs_h).to(dev)
    tdt = torch.float32 if a.maps_dtype == "float32" else torch.bfloat16
    maps = torch.empty((S, a.angles, 1, n, n), dtype=tdt, device=dev)
    # maps workspace: ~16 angles of the whole batch per pass (2 x 2.1 MB per angle and slice)
    ws = torch.empty(max(core.DEFAULT_MAPS_WORKSPACE, 16 * 2 * (a.n + 2 * ((int(np.ceil(np.sqrt(2) * a.n)) - a.n + 1) // 2)) ** 2 * 4 * S),
                     dtype=torch.uint8, device=dev)
    core.compute_maps(mu_in, mu_out, rad32, maps_dtype=a.maps_dtype, workspace=ws, out=maps)
    from pycorrectedemissionct_b200 import autotune

    variant = autotune.tune(c, x_true, maps)
    clean = c.fp(x_true, maps)
    gen = torch.Generator(device=dev)
    gen.manual_seed(a.seed + rank)
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * a.peak, generator=gen)
    del clean

    # calibration (untimed): the plain solver's residual after `iters` iterations defines the target
    solver = engine.BatchedSolver(c, maps, b, "mlem", history_len=a.iters + 1)
    solver.run(a.iters, check_every=a.iters, use_graph=False)
    torch.cuda.synchronize(dev)
    tol = solver.residuals.clone()
    tol_np = tol.cpu().numpy()
    solver = engine.BatchedSolver(c, maps, b, "mlem", tolerance=tol_np * (1 + 1e-9), history_len=2 * a.iters + 2)
    max_iters = 2 * a.iters

    passes = int(getattr(core.compute_maps, "last_passes", 1))
    fp_ms, bp_ms, launches = [], [], [0]

    def one_step(timed: bool):
        core.compute_maps(mu_in, mu_out, rad32, maps_dtype=a.maps_dtype, workspace=ws, out=maps)
        launches[0] += 2 * passes
        solver.reset()
        its, active = 0, S
        while its < max_iters and active > 0:
            evs = []
            for _ in range(10):
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                solver.step_timed(*e)
                evs.append(e)
            its += 10
            launches[0] += 30
            block_full = active == S
            active = int(solver.active.sum().item())  # synchronises the stream
            if timed and block_full:
                # kernel times only from blocks in which every slice was active (full-batch launches)
                for e in evs:
                    fp_ms.append(e[0].elapsed_time(e[1]))
                    bp_ms.append(e[1].elapsed_time(e[2]))
        return its

    for _ in range(a.warmup):
        one_step(False)
    barrier()
    fp_ms.clear(); bp_ms.clear(); launches[0] = 0
    clocks = ClockSampler(local)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    barrier()
    t0.record()
    its_total = 0
    for _ in range(a.steps):
        its_total += one_step(True)
    t1.record()
    barrier()
    clk = clocks.stop()
    elapsed_s = t0.elapsed_time(t1) / 1e3
    iterations = solver.iterations.cpu().numpy()
    converged = int((solver.residuals.cpu().numpy() <= tol_np * (1 + 1e-9)).sum())
    elapsed_max = max_over_ranks(elapsed_s)
    total_slices = S * a.steps * world
    value = total_slices / elapsed_max

    # ---- e2e: the same step from pinned host buffers, copies inside the timed region
    mu_h = torch.from_numpy(mus_h).pin_memory()
    b_h = b.cpu().pin_memory()
    x_h = torch.empty((S, n, n), dtype=torch.float32).pin_memory()
    def e2e_step():
        mu_in.copy_(mu_h, non_blocking=True)
        mu_out.copy_(mu_h, non_blocking=True)
        solver.b.copy_(b_h, non_blocking=True)
        one_step(False)
        x_h.copy_(solver.x, non_blocking=True)
    e2e_step()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        e2e_step()
    e1.record()
    barrier()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    h2d = S * (2 * n * n + a.angles * n) * 4
    d2h = S * n * n * 4

    # ---- roofline of the dominant kernel (attenuated fp with the fused MLEM epilogue)
    import json as _json

    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = float(_json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    else:
        peak = 6650.0
        peak_src = "fallback"
    map_bytes = 4 if a.maps_dtype == "float32" else 2
    fp_bytes = S * (a.angles * n * n * map_bytes + n * n * 4 + 2 * a.angles * n * 4)
    fp_avg_s = float(np.mean(fp_ms)) / 1e3 if fp_ms else float("nan")
    bp_avg_s = float(np.mean(bp_ms)) / 1e3 if bp_ms else float("nan")
    achieved = fp_bytes / fp_avg_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": elapsed_max / a.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded ellipse phantoms, disk attenuation, Poisson 1e5 peak counts)",
        "config": {
            "workload": workload_name(a), "n": n, "angles": a.angles, "slices_per_gpu": S, "maps_dtype": a.maps_dtype,
            "target": f"KL residual of plain MLEM after {a.iters} iterations (per slice)", "solver": "plain MLEM (cold start)",
            "parallelism": f"slices sharded over {world} GPU(s), no collective on the data path",
            "l2": "inputs larger than L2 (maps %.0f MB per slice)" % (a.angles * n * n * map_bytes / 1e6),
            "mean_iterations": float(np.mean(iterations)), "converged_slices_last_step": converged,
            "fp_variant": "tma" if variant else "ldg",
        },
        "roofline": {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            # DRAM bytes per launch from one ncu capture of this kernel on 2 slices (1.4366 GB), scaled
            # by the slices per launch; only for the capture's own configuration
            "traffic": (1.4366e9 / 2 * S) if (n == 512 and a.angles == 720 and a.maps_dtype == "float32") else None,
            "kernel": "fp_kernel<MLEM> (attenuated fp + ratio + KL residual)",
            "peak_source": peak_src, "fp_launch_us": fp_avg_s * 1e6, "bp_launch_us": bp_avg_s * 1e6,
            "algorithmic_bytes_per_launch": fp_bytes,
        },
        "e2e": {"value": total_slices / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches[0],
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(a, float(np.mean(iterations)))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
