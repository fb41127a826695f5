"""Batched, device-resident solver engine: MLEM / SIRT / PDHG over many slices at once.

Each iteration is one ``cct_*_step`` call (a fused fp + residual + stopping test +
bp + update sequence of kernels on the current stream).  Slices that meet their
tolerance stop updating inside the kernels (per-slice ``active`` flags); the host
only polls the flags every ``check_every`` iterations.  Blocks of iterations can be
captured once in a CUDA graph and replayed.

The update equations are the reference's (``corrct``: ``src/corrct/solvers.py``):
MLEM ``:725-805``, SIRT ``:895-984`` with ``compute_diagonal_scaling`` ``:60-117``,
PDHG ``:1099-1206`` with the KL data term and isotropic TV2D.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .core import XrfCore, _maps_stride, stream_handle

_BP_MODE_CODES = {"reference": _lib.CCT_BP_REFERENCE, "symmetric": _lib.CCT_BP_SYMMETRIC}


class BatchedSolver:
    """State of one batched solve.

    Parameters
    ----------
    core : XrfCore
        Geometry (n, angles, detectors, weights).
    maps : (S, A, D, n, n) tensor or None
        Attenuation maps (float32 or bfloat16); None for the uncorrected projector.
    b : (S, D, A, n) float32 tensor
        Data.
    method : "mlem" | "sirt" | "pdhg"
    tolerance : (S,) array, float, or None
        Stop a slice when ``tolerance > residual`` (the reference's rule).
    x_mask : (n, n) or (S, n, n) tensor or None
    b_mask, b_test_mask : (S, D, A, n) tensors (or broadcastable) or None
        Data mask (masks the residual and its norm, SIRT's update, PDHG's dual and the scaling
        tau) and cross-validation mask (MLEM / SIRT: its residual per iterate goes to
        ``residuals_test`` / ``history_test``), as the reference's ``b_mask`` / ``b_test_mask``
        after ``_initialize_b_masks``.
    x_shared : (S, n, n) tensor or None
        MLEM only: use this tensor as the iterate, in place and without initialising it.
    scaling : (sigma, tau) or None
        SIRT / PDHG: scalar step sizes instead of the diagonal scaling (the reference's
        ``precondition=False``).
    joint_stop : bool
        The S slices are one 3-D volume: a single stopping test on the residual summed over the
        slices (the reference's norm over the whole volume, compared with ``tolerance[0]``); the
        per-iteration volume residual is row 0 of ``history``.
    """

    def __init__(
        self,
        core: XrfCore,
        maps: torch.Tensor | None,
        b: torch.Tensor,
        method: str = "mlem",
        tolerance=None,
        x0: torch.Tensor | None = None,
        x_mask: torch.Tensor | None = None,
        lower_limit: float | None = None,
        upper_limit: float | None = None,
        relaxation: float | None = None,
        tv_lambda: float = 1e-2,
        bp_mode: str = "reference",
        background: float | None = None,
        history_len: int = 0,
        joint_stop: bool = False,
        x_shared: torch.Tensor | None = None,
        b_mask: torch.Tensor | None = None,
        b_test_mask: torch.Tensor | None = None,
        scaling: tuple[float, float] | None = None,
    ):
        self.core = core
        self.device = core.device
        self.method = method.lower()
        if self.method not in ("mlem", "sirt", "pdhg"):
            raise ValueError(f"Unknown method {method!r}: expected 'mlem', 'sirt' or 'pdhg'")
        n, s = core.n, b.shape[0]
        self.n_slices = s
        self.maps = maps
        self.maps_dtype = _lib.CCT_DTYPE_F32
        if maps is not None:
            self.maps_dtype = core._check_maps(maps, s)
        if bp_mode not in _BP_MODE_CODES:
            raise ValueError(f"bp_mode must be one of {sorted(_BP_MODE_CODES)}")
        self.bp_mode = bp_mode
        expect = (s, core.n_det, core.n_angles, n)
        if tuple(b.shape) != expect or b.dtype != torch.float32 or b.device != self.device:
            raise ValueError(f"b must be a float32 CUDA tensor of shape {expect}")
        self.b = b.contiguous()
        dev = self.device
        f32 = dict(dtype=torch.float32, device=dev)
        if self.method == "pdhg" and b_test_mask is not None:
            raise NotImplementedError("the PDHG step keeps no test residual: evaluate A x apart")
        self.b_mask = None if b_mask is None else b_mask.to(**f32).expand(expect).contiguous()
        self.b_test_mask = None if b_test_mask is None else b_test_mask.to(**f32).expand(expect).contiguous()

        bp_maps = maps if bp_mode == "symmetric" else None
        if self.method == "mlem":
            # tau = A^T 1 (solvers.py:734-737); the default XRF bp ignores maps, so tau is shared
            if self.b_mask is None:
                ones = torch.ones((1, core.n_det, core.n_angles, n), **f32)
                self.tau = core.bp(ones, "reference")[0].contiguous()
                self.tau_shared = 1
            else:
                # tau = A^T b_mask per slice (solvers.py:734-737)
                self.tau = core.bp(self.b_mask, "reference").contiguous()
                self.tau_shared = 0
            self.sigma = None
            if x_shared is not None:
                # iterate owned by the caller (ordered subsets share one x between subset solvers)
                if tuple(x_shared.shape) != (s, n, n) or x_shared.dtype != torch.float32 or not x_shared.is_contiguous():
                    raise ValueError(f"x_shared must be a contiguous float32 tensor of shape {(s, n, n)}")
                self.x = x_shared
            else:
                self.x = torch.ones((s, n, n), **f32) if x0 is None else x0.to(**f32).clone().contiguous()
                if x_mask is not None:
                    self.x *= x_mask
        elif scaling is not None:
            # scalar (sigma, tau), e.g. compute_Lipschitz_scaling (solvers.py:120-158)
            self.tau = torch.full((s, n, n), float(scaling[1]), **f32)
            self.tau_shared = 0
            self.sigma = torch.full(tuple(self.b.shape), float(scaling[0]), **f32)
            self.x = torch.zeros((s, n, n), **f32) if x0 is None else x0.to(**f32).clone().contiguous()
        else:
            relax = relaxation if relaxation is not None else (1.95 if self.method == "sirt" else 0.95)
            reg_tau = 4.0 if self.method == "pdhg" else 0.0
            ones_b = torch.ones_like(self.b) if self.b_mask is None else self.b_mask.clone()
            tau = core.bp(ones_b, bp_mode, bp_maps).abs_()
            tau += reg_tau
            # the reference scales by the maximum over its whole volume: per slice for independent
            # 2-D slices, over the stack for one 3-D volume (solvers.py:90-117)
            tmax = tau.amax() if joint_stop else tau.amax(dim=(1, 2), keepdim=True)
            tau = torch.where(tau / tmax < 1e-5, torch.ones_like(tau), tau)
            self.tau = (relax / tau).contiguous()
            self.tau_shared = 0
            x_ones = torch.ones((s, n, n), **f32)
            if x_mask is not None:
                x_ones *= x_mask
            sig = core.fp(x_ones, maps).abs_()
            smax = sig.amax() if joint_stop else sig.amax(dim=(1, 2, 3), keepdim=True)
            sig = torch.where(sig / smax < 1e-5, torch.ones_like(sig), sig)
            sig_relax = relax if self.method == "pdhg" else 1.0
            self.sigma = (sig_relax / sig).contiguous()
            self.x = torch.zeros((s, n, n), **f32) if x0 is None else x0.to(**f32).clone().contiguous()
        self.x_relax = self.x.clone() if self.method == "pdhg" else None
        self.tv_dual = torch.zeros((s, 2, n, n), **f32) if self.method == "pdhg" else None
        self.sino_buf = torch.zeros_like(self.b)
        # PDHG with a detector PSF keeps the raw projection apart from the dual variable
        self.sino_tmp = torch.empty_like(self.b) if (self.method == "pdhg" and core.psf is not None) else None
        self.vol_buf = torch.empty((s, n, n), **f32)
        self.partials = torch.zeros(max(core.partials_count(s), 1), dtype=torch.float64, device=dev)
        self.residuals = torch.zeros(s, dtype=torch.float64, device=dev)
        self.active = torch.ones(s, dtype=torch.int32, device=dev)
        self.iterations = torch.zeros(s, dtype=torch.int32, device=dev)
        if tolerance is None:
            self.tolerance = None
        else:
            tol = np.broadcast_to(np.asarray(tolerance, dtype=np.float64), (s,)).copy()
            self.tolerance = torch.from_numpy(tol).to(dev)
        self.x_mask = None if x_mask is None else x_mask.to(**f32).contiguous()
        if self.x_mask is not None and tuple(self.x_mask.shape) not in ((n, n), (s, n, n)):
            raise ValueError(f"x_mask must have shape {(n, n)} or {(s, n, n)}")

        st = _lib.SolverState()
        st.x = self.x.data_ptr()
        st.x_relax = None if self.x_relax is None else self.x_relax.data_ptr()
        st.b = self.b.data_ptr()
        st.tau = self.tau.data_ptr()
        st.sigma = None if self.sigma is None else self.sigma.data_ptr()
        st.sino_buf = self.sino_buf.data_ptr()
        st.vol_buf = self.vol_buf.data_ptr()
        st.tv_dual = None if self.tv_dual is None else self.tv_dual.data_ptr()
        st.partials = self.partials.data_ptr()
        st.residuals = self.residuals.data_ptr()
        st.active = self.active.data_ptr()
        st.iterations = self.iterations.data_ptr()
        st.tolerance = None if self.tolerance is None else self.tolerance.data_ptr()
        st.x_mask = None if self.x_mask is None else self.x_mask.data_ptr()
        st.has_lower = int(lower_limit is not None)
        st.lower_limit = float(lower_limit) if lower_limit is not None else 0.0
        st.has_upper = int(upper_limit is not None)
        st.upper_limit = float(upper_limit) if upper_limit is not None else 0.0
        st.has_background = int(background is not None)
        st.background = float(background) if background is not None else 0.0
        st.tv_lambda = float(tv_lambda)
        st.tau_shared = self.tau_shared
        st.sino_tmp = None if self.sino_tmp is None else self.sino_tmp.data_ptr()
        self.history = torch.zeros((s, history_len), dtype=torch.float64, device=dev) if history_len > 0 else None
        st.residual_history = None if self.history is None else self.history.data_ptr()
        st.history_len = int(history_len)
        st.x_mask_per_slice = int(self.x_mask is not None and self.x_mask.dim() == 3)
        st.b_mask = None if self.b_mask is None else self.b_mask.data_ptr()
        self.residuals_test = self.history_test = self.partials_test = None
        if self.b_test_mask is not None:
            st.b_test_mask = self.b_test_mask.data_ptr()
            self.partials_test = torch.zeros_like(self.partials)
            self.residuals_test = torch.zeros(s, dtype=torch.float64, device=dev)
            st.partials_test = self.partials_test.data_ptr()
            st.residuals_test = self.residuals_test.data_ptr()
            if history_len > 0:
                self.history_test = torch.zeros((s, history_len), dtype=torch.float64, device=dev)
                st.history_test = self.history_test.data_ptr()
        st.joint_stop = int(joint_stop)
        self.joint_stop = bool(joint_stop)
        self.state = st
        self.desc = core.desc(s, self.maps_dtype)
        self.desc.maps_slice_stride = _maps_stride(maps)
        self._maps_ptr = None if maps is None else maps.data_ptr()
        self._graph: torch.cuda.CUDAGraph | None = None
        self._graph_steps = 0

    # --------------------------------------------------------------------------- stepping
    def step(self) -> None:
        """Queue one iteration on the current stream."""
        h = stream_handle(self.device)
        if self.method == "mlem":
            _lib.call("cct_mlem_step", ctypes.byref(self.desc), self._maps_ptr, ctypes.byref(self.state), h)
        elif self.method == "sirt":
            _lib.call(
                "cct_sirt_step", ctypes.byref(self.desc), self._maps_ptr, _BP_MODE_CODES[self.bp_mode],
                ctypes.byref(self.state), h,
            )
        else:
            _lib.call(
                "cct_pdhg_step", ctypes.byref(self.desc), self._maps_ptr, _BP_MODE_CODES[self.bp_mode],
                ctypes.byref(self.state), h,
            )

    def step_timed(self, ev_fp0, ev_fp1, ev_bp1) -> None:
        """One MLEM iteration with CUDA events recorded around its fp and bp halves."""
        if self.method != "mlem":
            raise ValueError("step_timed is only defined for MLEM")
        stream = torch.cuda.current_stream(self.device)
        h = stream.cuda_stream
        ev_fp0.record(stream)
        _lib.call("cct_mlem_fp", ctypes.byref(self.desc), self._maps_ptr, ctypes.byref(self.state), h)
        ev_fp1.record(stream)
        _lib.call("cct_mlem_update", ctypes.byref(self.desc), ctypes.byref(self.state), h)
        ev_bp1.record(stream)

    def reset(self, x0: torch.Tensor | None = None) -> None:
        """Restart the solve from x0 (default: the method's default start) keeping all buffers."""
        if x0 is None:
            self.x.fill_(1.0 if self.method == "mlem" else 0.0)
            if self.x_mask is not None and self.method == "mlem":
                self.x *= self.x_mask
        else:
            self.x.copy_(x0)
            if self.x_mask is not None and self.method == "mlem":
                self.x *= self.x_mask  # as __init__ (the reference masks x0 too, solvers.py:750-752)
        if self.x_relax is not None:
            self.x_relax.copy_(self.x)
        if self.tv_dual is not None:
            self.tv_dual.zero_()
        self.sino_buf.zero_()
        self.active.fill_(1)
        self.iterations.zero_()
        self.residuals.zero_()
        if self.history is not None:
            self.history.zero_()
        if self.residuals_test is not None:
            self.residuals_test.zero_()
        if self.history_test is not None:
            self.history_test.zero_()

    def capture(self, steps: int) -> None:
        """Capture `steps` iterations into a CUDA graph.  Call after at least one eager
        ``step()`` so every kernel is loaded before capture."""
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(steps):
                self.step()
        self._graph = g
        self._graph_steps = steps

    def run(self, iterations: int, check_every: int = 10, use_graph: bool = True) -> int:
        """Run up to `iterations` iterations; returns the number queued.

        The first block of `check_every` iterations runs eagerly; later full blocks replay
        one captured CUDA graph.  When a tolerance is set, the host checks the per-slice
        active flags after every block and stops once all slices are done.
        """
        done = 0
        while done < iterations:
            block = min(check_every, iterations - done)
            if use_graph and done > 0 and block == check_every:
                if self._graph is None or self._graph_steps != block:
                    self.capture(block)
                self._graph.replay()
            else:
                for _ in range(block):
                    self.step()
            done += block
            if self.tolerance is not None and int(self.active.sum().item()) == 0:
                break
        return done

    def results(self) -> dict:
        return dict(
            x=self.x,
            residuals=self.residuals,
            iterations=self.iterations,
            active=self.active,
        )


# ------------------------------------------------------------------------------ ordered subsets
def subset_permutation(n_angles: int, levels: list[int]) -> np.ndarray:
    """Angle order in which every subset of every level is one contiguous range.

    ``levels`` are subset counts, each dividing the one before (and none above ``n_angles``);
    a subset of k holds the angles a with a mod k equal to its index (every k-th angle; subsets
    differ in size by at most one when k does not divide ``n_angles``).  Angles are grouped by
    residue modulo the finest count, and those groups by residue modulo each coarser count, so
    the subsets of a coarser level are unions of consecutive finer ones.
    """
    levels = [int(k) for k in levels]
    if not levels or any(k < 1 or k > n_angles for k in levels):
        raise ValueError(f"subset counts must be in [1, {n_angles}]: {levels}")
    if any(levels[i] % levels[i + 1] for i in range(len(levels) - 1)):
        raise ValueError(f"each subset count must divide the previous one: {levels}")
    finest = levels[0]
    residues = sorted(range(finest), key=lambda r: tuple(r % k for k in reversed(levels)))
    return np.concatenate([np.arange(r, n_angles, finest) for r in residues])


def subset_ranges(n_angles: int, levels: list[int]) -> list[list[slice]]:
    """Per level, the ranges of ``subset_permutation(n_angles, levels)`` that hold its subsets."""
    perm = subset_permutation(n_angles, levels)
    out = []
    for k in levels:
        res = perm % k
        cuts = [0] + [i for i in range(1, n_angles) if res[i] != res[i - 1]] + [n_angles]
        out.append([slice(cuts[i], cuts[i + 1]) for i in range(len(cuts) - 1)])
        if len(out[-1]) != k:
            raise AssertionError("subset ranges are not contiguous")
    return out


class OrderedSubsets:
    """Ordered-subsets EM passes (H. M. Hudson and R. S. Larkin, "Accelerated image reconstruction
    using ordered subsets of projection data", IEEE TMI 13, 1994) as a warm start for MLEM.

    A pass visits the k subsets of a level in turn and applies the MLEM update of each subset,
    x *= A_m^T(b_m / A_m x) / A_m^T 1, with the fused MLEM kernels restricted to the subset's
    angles; one pass costs about one full MLEM iteration.  ``core``, ``maps`` and ``b`` must be in
    the angle order of ``subset_permutation(A, [k for k, _ in schedule])``.

    schedule : [(subsets, passes), ...], subset counts decreasing, each dividing the previous.
    """

    def __init__(self, core: XrfCore, maps: torch.Tensor | None, b: torch.Tensor, schedule, x0=None):
        self.core = core
        self.device = core.device
        self.schedule = [(int(k), int(p)) for k, p in schedule]
        ranges = subset_ranges(core.n_angles, [k for k, _ in self.schedule])  # validates the levels
        s, n = b.shape[0], core.n
        self.x = torch.ones((s, n, n), dtype=torch.float32, device=self.device)
        if x0 is not None:
            self.x.copy_(x0)
        self.levels: list[list[BatchedSolver]] = []
        self.ranges = ranges
        for level_ranges in ranges:
            solvers = []
            for rng in level_ranges:
                sub = core.angle_range(rng)
                sub_maps = None if maps is None else maps[:, rng]
                b_sub = b[:, :, rng].contiguous()
                solvers.append(BatchedSolver(sub, sub_maps, b_sub, "mlem", x_shared=self.x))
            self.levels.append(solvers)
        self._graphs: list[torch.cuda.CUDAGraph | None] = [None] * len(self.levels)

    def reset(self, x0: torch.Tensor | None = None) -> None:
        if x0 is None:
            self.x.fill_(1.0)
        else:
            self.x.copy_(x0)
        for solvers in self.levels:
            for sm in solvers:
                sm.active.fill_(1)
                sm.iterations.zero_()

    def set_data(self, b: torch.Tensor) -> None:
        """Refresh every subset's copy of the data from ``b`` (subset-major angle order)."""
        for level, level_ranges in zip(self.levels, self.ranges):
            for sm, rng in zip(level, level_ranges):
                sm.b.copy_(b[:, :, rng])

    def _pass(self, level: int) -> None:
        for sm in self.levels[level]:
            sm.step()

    def run_level(self, level: int, passes: int = 1) -> torch.Tensor:
        """``passes`` eager passes over the subsets of one level of the schedule (whatever the
        schedule's own pass counts); returns the shared iterate."""
        for _ in range(passes):
            self._pass(level)
        return self.x

    def run(self, use_graph: bool = True) -> torch.Tensor:
        """All passes of the schedule; returns the shared iterate."""
        for li, (_, passes) in enumerate(self.schedule):
            if passes <= 0:
                continue
            if not use_graph:
                for _ in range(passes):
                    self._pass(li)
                continue
            if self._graphs[li] is None:
                self._pass(li)  # eager first pass: every kernel is loaded before capture
                torch.cuda.synchronize(self.device)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._pass(li)
                self._graphs[li] = g
                todo = passes - 1
            else:
                todo = passes
            for _ in range(todo):
                self._graphs[li].replay()
        return self.x

    @property
    def passes(self) -> int:
        return sum(p for _, p in self.schedule)


# ------------------------------------------------------------------------------- ragged batches
class RaggedSolvers:
    """One iteration of many uniform batches (different n, angle counts, detectors) in three
    launches: the fp with its fused epilogue, the residuals and stopping tests, and the bp with
    its fused update run once over all groups' CTAs (``cct_ragged_step``).

    ``solvers``: BatchedSolver objects, all MLEM or all SIRT (same bp mode), one maps type, no
    PSF.  Each keeps its own buffers; their iterates, residuals and active flags evolve exactly
    as if each were stepped on its own.
    """

    def __init__(self, solvers: list[BatchedSolver]):
        if not solvers:
            raise ValueError("no solvers")
        methods = {sv.method for sv in solvers}
        if len(methods) != 1 or next(iter(methods)) not in ("mlem", "sirt"):
            raise ValueError("a ragged batch steps MLEM solvers or SIRT solvers, not a mix")
        self.solvers = list(solvers)
        self.method = next(iter(methods))
        self.device = solvers[0].device
        g = len(solvers)
        bp_modes = {sv.bp_mode for sv in solvers}
        if len(bp_modes) != 1:
            raise ValueError("every group must use the same back-projection mode")
        self.bp_mode = next(iter(bp_modes))
        lib = _lib.load()
        nbytes = ctypes.c_size_t(0)
        _lib.check(lib.cct_ragged_workspace_size(g, ctypes.byref(nbytes)))
        self.workspace = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=self.device)
        base = self.workspace.data_ptr()
        self._ws_ptr = (base + 255) & ~255
        descs = (_lib.XrfDesc * g)(*[sv.desc for sv in solvers])
        maps = (ctypes.c_void_p * g)(*[sv._maps_ptr for sv in solvers])
        states = (_lib.SolverState * g)(*[sv.state for sv in solvers])
        plan = ctypes.c_void_p(0)
        method = _lib.CCT_METHOD_MLEM if self.method == "mlem" else _lib.CCT_METHOD_SIRT
        _lib.check(
            lib.cct_ragged_plan_create(
                method, _BP_MODE_CODES[self.bp_mode], g, descs, maps, states, self._ws_ptr, int(nbytes.value),
                ctypes.byref(plan), stream_handle(self.device),
            )
        )
        self._plan = plan
        self._lib = lib

    def step(self) -> None:
        """One iteration of every group, queued on the current stream."""
        _lib.check(self._lib.cct_ragged_step(self._plan, stream_handle(self.device)))

    def active(self) -> int:
        return int(sum(int(sv.active.sum().item()) for sv in self.solvers))

    def close(self) -> None:
        if getattr(self, "_plan", None):
            self._lib.cct_ragged_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
