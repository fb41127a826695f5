"""Ragged streams: many slices of different sizes and angle counts, solved in waves.

Every slice is a job: its side n, its rotation angles, its incident / emitted attenuation and its
data, solved either by SIRT for a fixed number of iterations or by MLEM to a data-residual
tolerance (the reference's stopping rule).  Jobs are packed into waves whose device memory (maps
and solver buffers) fits a budget; inside a wave, jobs with the same (n, angles, method) form a
uniform group, and every operator of every iteration runs as ONE ragged launch over all groups
(``cct_ragged_step``): SIRT groups together, MLEM groups together, and for the MLEM warm start
every ordered-subsets step over all groups' subset m together.  With ``warm_start=False`` MLEM
starts from the reference's default (the plain cold-start path); with ``warm_start="learned"``
each MLEM group starts from the learned start (``train_warmstart.learned_start``: one
ordered-subsets pass keeping snapshots, the warm-start network, one pass per ordered-subsets
level of ``WarmStartNet.os_levels``), run per group, and the ragged MLEM iterations then judge
every slice as for the other starts.

The per-slice arithmetic is that of ``BatchedSolver`` (and so of corrct's solvers), which the
ragged kernels reproduce bit for bit.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import autotune
from . import core as _core
from .engine import BatchedSolver, OrderedSubsets, RaggedSolvers, subset_permutation


@dataclass
class Job:
    """One slice.  ``b`` is (A, n) float32 data in the order of ``angles``."""

    n: int
    angles: np.ndarray
    mu_in: np.ndarray | None
    mu_out: np.ndarray | None
    b: np.ndarray
    method: str = "mlem"          # "mlem" (to `tolerance`) or "sirt" (`iterations`)
    tolerance: float | None = None
    iterations: int = 150
    # results
    x: np.ndarray | None = None
    iterations_done: int = 0
    finished_s: float = 0.0
    extra: dict = field(default_factory=dict)


def job_bytes(job: Job, maps_bytes: int = 4) -> int:
    """Device bytes a job holds while its wave runs (maps, data and solver buffers)."""
    a, n = len(job.angles), job.n
    return a * n * n * maps_bytes + 6 * a * n * 4 + 8 * n * n * 4


def default_schedule(n_angles: int, angles_per_subset: int = 12) -> list[tuple[int, int]]:
    """Ordered-subsets schedule for a slice of ``n_angles`` angles: 3 passes over subsets of about
    ``angles_per_subset`` angles (an even count), then 2 passes over half as many subsets (twice
    the angles); 720 angles give [(60, 3), (30, 2)]."""
    k = max(2, (n_angles // angles_per_subset) // 2 * 2)
    return [(k, 3), (k // 2, 2)]


def pack_waves(jobs: list[Job], memory_budget: int, maps_bytes: int = 4) -> list[list[Job]]:
    """Jobs sorted by (method, n, angles) and cut into consecutive waves of at most
    ``memory_budget`` bytes (``job_bytes``); a job larger than the budget is a wave of its own."""
    order = sorted(jobs, key=lambda j: (j.method, j.n, len(j.angles)))
    out, cur, used = [], [], 0
    for j in order:
        need = job_bytes(j, maps_bytes)
        if cur and used + need > memory_budget:
            out.append(cur)
            cur, used = [], 0
        cur.append(j)
        used += need
    if cur:
        out.append(cur)
    return out


class _Group:
    def __init__(self, jobs: list[Job], device, maps_dtype: str, schedule, warm, workspace: torch.Tensor, net=None):
        j0 = jobs[0]
        self.jobs = jobs
        self.method = j0.method
        angles = np.asarray(j0.angles, dtype=np.float64)
        # the learned start's ordered-subsets levels, when the network has them for this angle count
        # (the encoder-decoder halves the side three times: n a multiple of 8)
        self.learned = (warm == "learned" and j0.method == "mlem" and net is not None and j0.n % 8 == 0
                        and bool(net.os_levels(len(angles))))
        if self.learned:
            schedule = [(k, 1) for k in net.os_levels(len(angles))]
        if schedule is None:
            schedule = default_schedule(len(angles))
        self.schedule = None if schedule is None else [(int(k), int(p)) for k, p in schedule]
        levels = [k for k, _ in self.schedule]
        self.perm = None
        if self.method == "mlem" and warm:
            self.perm = subset_permutation(len(angles), levels)
            angles = angles[self.perm]
        self.core = _core.XrfCore(j0.n, angles, device=device)
        self.restarted = False
        self.judge_its = self.spent = 0
        f32 = dict(dtype=torch.float32, device=device)
        mu_in = None if j0.mu_in is None else torch.from_numpy(np.stack([j.mu_in for j in jobs])).to(**f32)
        mu_out = None if j0.mu_out is None else torch.from_numpy(np.stack([j.mu_out for j in jobs])).to(**f32)
        # the pass size the autotuner chose for this group's shape, when it has one
        entries = autotune.maps_entries(device, j0.n, len(angles), 1, len(jobs), maps_dtype)
        if entries is not None:
            per_entry = _core.maps_entry_bytes(j0.n, len(jobs))
            workspace = workspace[: min(workspace.numel(), entries * per_entry)]
        self.maps = _core.compute_maps(mu_in, mu_out, self.core.angles_rad32, maps_dtype=maps_dtype,
                                       workspace=workspace)
        b = np.stack([j.b for j in jobs])[:, None]
        if self.perm is not None:
            b = b[:, :, self.perm]
        self.b = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float32)).to(device)
        if self.method == "sirt":
            self.solver = BatchedSolver(self.core, self.maps, self.b, "sirt")
            self.subsets = None
        else:
            tol = np.array([j.tolerance for j in jobs], dtype=np.float64)
            self.subsets = OrderedSubsets(self.core, self.maps, self.b, self.schedule) if warm else None
            x_shared = None if self.subsets is None else self.subsets.x
            self.solver = BatchedSolver(self.core, self.maps, self.b, "mlem", tolerance=tol, x_shared=x_shared)

    def warm_passes(self) -> int:
        """Full-data passes of the warm start (the learned start's snapshot pass included)."""
        if self.subsets is None:
            return 0
        return self.subsets.passes + (1 if self.learned else 0)


class RaggedStream:
    """Solve a list of jobs in waves of at most ``memory_budget`` device bytes.

    schedule : ordered-subsets warm start of the MLEM jobs, [(subsets, passes), ...] for every
        job, or None for ``default_schedule`` of each job's angle count.
    check_every : MLEM iterations between two host checks of the stopping flags.
    fallback_after : judging MLEM iterations after which a warm-started group that has not met
        its residual restarts from the default start (plain MLEM is the fallback).
    """

    def __init__(self, device=None, memory_budget: int = 100 << 30, schedule=None,
                 maps_dtype: str = "float32", warm_start=True, check_every: int = 2, fallback_after: int = 200,
                 net=None):
        self.device = _core.require_cuda(device)
        self.memory_budget = int(memory_budget)
        self.schedule = None if schedule is None else [(int(k), int(p)) for k, p in schedule]
        self.maps_dtype = maps_dtype
        if warm_start not in (True, False, "subsets", "learned"):
            raise ValueError(f"warm_start must be True / 'subsets', 'learned' or False, got {warm_start!r}")
        if warm_start == "learned" and net is None:
            raise ValueError("warm_start='learned' needs the warm-start network (net=WarmStartNet with weights)")
        self.warm = warm_start if warm_start == "learned" else bool(warm_start)
        self.net = net
        self.check_every = int(check_every)
        self.fallback_after = int(fallback_after)
        self.launches = 0

    def waves(self, jobs: list[Job]) -> list[list[Job]]:
        return pack_waves(jobs, self.memory_budget, 2 if self.maps_dtype == "bfloat16" else 4)

    def solve(self, jobs: list[Job], max_iterations: int = 1000) -> dict:
        """Solve every job (results in ``job.x``, ``job.iterations_done``, ``job.finished_s`` =
        seconds from the start of the stream to the slice's completion).  Returns totals."""
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        # maps workspace: 4x the default, so that the few slices of a small group still fill the
        # GPU with enough angles per pass (outside the wave budget)
        ws = torch.empty(4 * _core.DEFAULT_MAPS_WORKSPACE, dtype=torch.uint8, device=self.device)
        for wave in self.waves(jobs):
            groups = {}
            for j in wave:
                if j.method not in ("mlem", "sirt"):
                    raise ValueError(f"unknown method {j.method!r}")
                key = (j.method, j.n, len(j.angles), tuple(np.round(np.asarray(j.angles, np.float64), 9)))
                groups.setdefault(key, []).append(j)
            gs = [_Group(js, self.device, self.maps_dtype, self.schedule, self.warm, ws, self.net)
                  for js in groups.values()]
            self._run_sirt([g for g in gs if g.method == "sirt"], t0)
            self._run_mlem([g for g in gs if g.method == "mlem"], t0, max_iterations)
            del gs
        torch.cuda.synchronize(self.device)
        total = time.perf_counter() - t0
        done = np.array([j.finished_s for j in jobs])
        return dict(seconds=total, slices=len(jobs), slices_per_s=len(jobs) / total,
                    p50_s=float(np.percentile(done, 50)), p99_s=float(np.percentile(done, 99)))

    def _finish(self, g: _Group, t0: float) -> None:
        x = g.solver.x.cpu().numpy()
        its = g.solver.iterations.cpu().numpy()
        res = g.solver.residuals.cpu().numpy()
        for k, j in enumerate(g.jobs):
            j.x = x[k]
            j.extra["residual"] = float(res[k])
            j.iterations_done = int(its[k]) + (g.spent if g.restarted else g.warm_passes())
            j.extra["restarted"] = g.restarted
            if j.finished_s == 0.0:
                j.finished_s = time.perf_counter() - t0

    def _run_sirt(self, gs: list[_Group], t0: float) -> None:
        if not gs:
            return
        rag = RaggedSolvers([g.solver for g in gs])
        iters = max(j.iterations for g in gs for j in g.jobs)
        for _ in range(iters):
            rag.step()
            self.launches += 3
        torch.cuda.synchronize(self.device)
        for g in gs:
            self._finish(g, t0)
        rag.close()

    def _run_mlem(self, gs: list[_Group], t0: float, max_iterations: int) -> None:
        if not gs:
            return
        learned = [g for g in gs if g.learned]
        if learned:
            from .train_warmstart import learned_start

            for g in learned:
                learned_start(self.net, g.subsets, g.core, g.b, g.solver.tau)
                self.launches += 1
        others = [g for g in gs if g.subsets is not None and not g.learned]
        if others:
            # step t of a level applies subset t mod k_g of every group g still in its passes, all
            # groups in one ragged launch per operator
            for li in range(max(len(g.schedule) for g in others)):
                live = [g for g in others if li < len(g.schedule)]
                steps = max(g.schedule[li][0] * g.schedule[li][1] for g in live)
                for t in range(steps):
                    members = [g.subsets.levels[li][t % g.schedule[li][0]] for g in live
                               if t < g.schedule[li][0] * g.schedule[li][1]]
                    p = RaggedSolvers(members)
                    p.step()
                    self.launches += 3
                    p.close()
        rag = RaggedSolvers([g.solver for g in gs])
        its = 0
        pending = list(gs)
        for g in gs:
            g.judge_its, g.spent = 0, 0
        while pending and its < max_iterations:
            for _ in range(self.check_every):
                rag.step()
                self.launches += 3
            its += self.check_every
            # the plain solver is the fallback: a warm-started group whose slices have not met their
            # residual after `fallback_after` judging iterations restarts from the default start
            for g in pending:
                g.judge_its += self.check_every
                if self.warm and g.subsets is not None and g.judge_its >= self.fallback_after and not g.restarted:
                    if int(g.solver.active.sum().item()) > 0:
                        g.spent = g.warm_passes() + g.judge_its
                        g.solver.reset()
                        g.restarted = True
            flags = torch.cat([g.solver.active for g in pending]).cpu().numpy()  # one copy per check
            now = time.perf_counter() - t0
            still, pos = [], 0
            for g in pending:
                act = flags[pos : pos + len(g.jobs)]
                pos += len(g.jobs)
                for k, j in enumerate(g.jobs):
                    if act[k] == 0 and j.finished_s == 0.0:
                        j.finished_s = now
                if act.any():
                    still.append(g)
                else:
                    self._finish(g, t0)
            pending = still
        for g in pending:
            self._finish(g, t0)
        rag.close()
