"""Solvers with the reference's interface running device-resident on the B200 projectors.

Mirrors ``corrct``: ``src/corrct/solvers.py`` — ``SolutionInfo`` (``:161-201``),
``MLEM`` (``:634-805``), ``SIRT`` (``:808-984``), ``PDHG`` (``:987-1206``, KL data term
with isotropic TV2D), ``SART`` (``:473-631``) and ``FISTA`` (``:1209-1513``, l2 data term,
no regularizer).  ``__call__(A, b, iterations, x0, lower_limit, upper_limit, x_mask, b_mask,
b_test_mask, ...)`` returns ``(x, SolutionInfo)`` like the reference, with the data masks of
``Solver._initialize_b_masks`` (``:333-343``) and the cross-validation residuals.  MLEM, SIRT
and PDHG run the fused ``cct_*_step`` kernels (the update equations of the reference); SART and
FISTA drive the projector's device fp / bp.
``A`` must be one of this package's projectors: the unchanged corrct solvers
remain available for any other operator (including these projectors).
"""

from __future__ import annotations

import numpy as np
import torch

from .engine import BatchedSolver
from .projectors import ProjectorAttenuationXRF, ProjectorUncorrected

eps = np.finfo(np.float32).eps


class SolutionInfo:
    """Reconstruction info (corrct ``solvers.py:161-201``)."""

    def __init__(self, method: str, max_iterations: int, tolerance, residual0: float = np.inf, residual0_cv: float = np.inf):
        self.method = method
        self.max_iterations = max_iterations
        self.tolerance = tolerance
        self.residual0 = residual0
        self.residual0_cv = residual0_cv
        self.residuals = np.zeros(max_iterations)
        self.residuals_cv = np.zeros(max_iterations)
        self.iterations = 0

    @property
    def residuals_rel(self):
        return self.residuals / self.residual0

    @property
    def residuals_cv_rel(self):
        return self.residuals_cv / self.residual0_cv


def _check_projector(A) -> None:
    if not isinstance(A, ProjectorUncorrected):
        raise TypeError(
            "the B200 solvers run on this package's projectors; use corrct's own solvers for other operators"
        )


def _data_term_name(data_term) -> tuple[str, float | None]:
    if isinstance(data_term, str):
        name = data_term.lower()
        if name not in ("l2", "kl"):
            raise ValueError(f"Unknown data term: '{data_term}', only accepted terms are: 'l2' | 'kl'.")
        return name, None
    name = getattr(data_term, "__data_fidelity_name__", "").lower()
    if name not in ("l2", "kl"):
        raise ValueError(f"Unsupported data term: '{data_term}', only 'kl' and 'l2' are supported.")
    bg = getattr(data_term, "background", None)
    return name, (None if bg is None else float(np.asarray(bg)))


def _tensor(v, dev) -> torch.Tensor:
    t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32))
    return t.to(dev, torch.float32)


def _as_batch(A, b, x0, x_mask):
    """Device tensors of one solve: b (Z, D, A, n), x0 (Z, n, n), mask (n, n) or (Z, n, n), maps.

    A 3-D volume of Z slices (data (D, Z, A, n) in the reference's order) is solved as Z slices
    with a joint stopping test."""
    dev = A.projector_backend.device
    n = int(A.vol_shape[-1])
    z = A.projector_backend.n_slices
    n_det = A._n_det() if isinstance(A, ProjectorAttenuationXRF) else 1
    n_ang = len(A.angles_rot_rad)
    as_np = not isinstance(b, torch.Tensor)
    bt = _tensor(b, dev).reshape(n_det, z, n_ang, n).permute(1, 0, 2, 3).contiguous()
    x0t = None if x0 is None else _tensor(x0, dev).reshape(z, n, n).contiguous()
    mt = None
    if x_mask is not None:
        mt = _tensor(x_mask, dev)
        mt = mt.reshape(n, n) if mt.numel() == n * n else mt.reshape(z, n, n)
        mt = mt.contiguous()
    maps = A.maps_device if isinstance(A, ProjectorAttenuationXRF) else None
    return bt, x0t, mt, maps, as_np


def _operator_norm(A, b, bt: torch.Tensor, bp_mode: str, maps) -> float:
    """``power_method`` (corrct ``solvers.py:26-57``, 5 iterations) with the device fp / bp.  Its
    start is ``np.random.rand`` in the data's own shape and dtype, the reference's draw."""
    shape = tuple(b.shape)
    dtype = b.dtype if isinstance(b, np.ndarray) else np.float32
    xr = np.random.rand(*shape).astype(dtype)
    xr /= np.linalg.norm(xr)
    s, n_det, n_ang, n = bt.shape
    x = _tensor(xr, bt.device).reshape(n_det, s, n_ang, n).permute(1, 0, 2, 3).contiguous()
    core = A.core
    bp_maps = maps if bp_mode == "symmetric" else None
    v = core.bp(x, bp_mode, bp_maps)
    v_norm = float(torch.linalg.norm(v.double()).item())
    L = v_norm
    for _ in range(5):
        v = (v / v_norm).contiguous()
        v = core.bp(core.fp(v, maps), bp_mode, bp_maps)
        v_norm = float(torch.linalg.norm(v.double()).item())
        L = float(np.sqrt(v_norm))
    return L


def _is_volume(A) -> bool:
    return len(A.vol_shape) == 3


def _finish(solver: BatchedSolver, info: SolutionInfo, iterations: int, as_np: bool, volume: bool = False):
    torch.cuda.current_stream(solver.device).synchronize()
    info.iterations = int(solver.iterations[0].item())
    if solver.history is not None:
        h = solver.history[0].cpu().numpy()
        k = min(info.iterations, iterations)
        info.residuals[:k] = h[:k]
    x = solver.x if volume else solver.x[0]
    return (x.cpu().numpy() if as_np else x.clone()), info


class Solver:
    """Base solver (corrct ``solvers.py:204-400``)."""

    def __init__(self, verbose: bool = False, leave_progress: bool = True, relaxation: float = 1.0, tolerance=None, data_term="l2", data_term_test=None):
        self.verbose = verbose
        self.leave_progress = leave_progress
        self.relaxation = relaxation
        self.tolerance = tolerance
        self.data_term, self.background = _data_term_name(data_term)
        if data_term_test is not None:
            name, bg = _data_term_name(data_term_test)
            if name != self.data_term:
                raise NotImplementedError("the cross-validation data term must be of the solver's data term type")
            # the reference gives the test term the solver's background (solvers.py:762-765)

    def info(self) -> str:
        return type(self).__name__

    def upper(self) -> str:
        return type(self).__name__.upper()

    def lower(self) -> str:
        return type(self).__name__.lower()

    @staticmethod
    def _masks(A, b_mask, b_test_mask):
        """Device (S, D, A, n) masks after ``_initialize_b_masks`` (solvers.py:333-343)."""
        if b_test_mask is not None and b_mask is None:
            b_mask = np.ones(1, dtype=np.float32)
        if b_mask is None:
            return None, None
        dev = A.projector_backend.device
        n = int(A.vol_shape[-1])
        z = A.projector_backend.n_slices
        n_det = A._n_det() if isinstance(A, ProjectorAttenuationXRF) else 1
        shape = (n_det, z, len(A.angles_rot_rad), n)

        def dev_mask(m):
            t = _tensor(m, dev)
            t = t.expand(shape) if t.numel() == 1 else t.reshape(shape)
            return t.permute(1, 0, 2, 3).contiguous()

        bm = dev_mask(b_mask)
        if b_test_mask is None:
            return bm, None
        bt = dev_mask(b_test_mask)
        return bm * (1 - bt), bt * bm

    @staticmethod
    def _cv_info(solver: BatchedSolver, info, iterations: int, volume: bool) -> None:
        if solver.history_test is None:
            return
        h = solver.history_test.sum(dim=0) if volume else solver.history_test[0]
        k = min(info.iterations, iterations)
        info.residuals_cv[:k] = h.cpu().numpy()[:k]


class MLEM(Solver):
    """MLEM with the KL data term (corrct ``solvers.py:634-805``)."""

    def __init__(self, verbose: bool = False, leave_progress: bool = True, tolerance=None, regularizer=None, data_term="kl", data_term_test=None):
        super().__init__(verbose=verbose, leave_progress=leave_progress, tolerance=tolerance, data_term=data_term, data_term_test=data_term_test)
        if regularizer is not None:
            raise NotImplementedError("MLEM regularizers are not supported by the B200 solvers")

    def __call__(self, A, b, iterations: int, x0=None, lower_limit=None, upper_limit=None, x_mask=None, b_mask=None, b_test_mask=None):
        _check_projector(A)
        if getattr(A, "is_symmetric", False) or getattr(A, "bp_mode", "reference") != "reference":
            raise NotImplementedError("the fused MLEM uses the reference (non-symmetric) back projection")
        bt, x0t, mt, maps, as_np = _as_batch(A, b, x0, x_mask)
        bm, btm = self._masks(A, b_mask, b_test_mask)
        solver = BatchedSolver(
            A.core, maps, bt, "mlem", tolerance=self.tolerance, x0=x0t, x_mask=mt,
            lower_limit=lower_limit, upper_limit=upper_limit, background=self.background, history_len=iterations,
            joint_stop=_is_volume(A), b_mask=bm, b_test_mask=btm,
        )
        info = SolutionInfo(self.info(), max_iterations=iterations, tolerance=self.tolerance)
        if self.tolerance is not None or btm is not None:
            ax0 = A.core.fp(solver.x, maps)
            if self.tolerance is not None:
                info.residual0 = _kl_residual_norm(ax0, bt, self.background, bm)
            if btm is not None:
                info.residual0_cv = _kl_residual_norm(ax0, bt, self.background, btm)
        solver.run(iterations, check_every=10 if self.tolerance is not None else max(iterations, 1))
        x, info = _finish(solver, info, iterations, as_np, _is_volume(A))
        self._cv_info(solver, info, iterations, _is_volume(A))
        return x, info


class SIRT(Solver):
    """SIRT with the l2 data term (corrct ``solvers.py:808-984``)."""

    def __init__(self, verbose: bool = False, leave_progress: bool = True, relaxation: float = 1.95, tolerance=None, regularizer=None, data_term="l2", data_term_test=None):
        super().__init__(verbose=verbose, leave_progress=leave_progress, relaxation=relaxation, tolerance=tolerance, data_term=data_term, data_term_test=data_term_test)
        if regularizer is not None:
            raise NotImplementedError("SIRT regularizers are not supported by the B200 solvers")
        if self.data_term != "l2":
            raise NotImplementedError("the fused SIRT uses the l2 data term")

    def __call__(self, A, b, iterations: int, x0=None, lower_limit=None, upper_limit=None, x_mask=None, b_mask=None, b_test_mask=None):
        _check_projector(A)
        bt, x0t, mt, maps, as_np = _as_batch(A, b, x0, x_mask)
        bm, btm = self._masks(A, b_mask, b_test_mask)
        bp_mode = "symmetric" if getattr(A, "is_symmetric", False) else "reference"
        solver = BatchedSolver(
            A.core, maps, bt, "sirt", tolerance=self.tolerance, x0=x0t, x_mask=mt, lower_limit=lower_limit,
            upper_limit=upper_limit, relaxation=self.relaxation, bp_mode=bp_mode, background=self.background,
            history_len=iterations, joint_stop=_is_volume(A), b_mask=bm, b_test_mask=btm,
        )
        info = SolutionInfo(self.info(), max_iterations=iterations, tolerance=self.tolerance)
        if self.tolerance is not None or btm is not None:
            r0 = bt - (A.core.fp(solver.x, maps) + (0.0 if self.background is None else self.background))
            if self.tolerance is not None:
                rm = r0 if bm is None else r0 * bm
                info.residual0 = float(torch.sum(rm.double() ** 2).item())
            if btm is not None:
                info.residual0_cv = float(torch.sum((r0 * btm).double() ** 2).item())
        solver.run(iterations, check_every=10 if self.tolerance is not None else max(iterations, 1))
        x, info = _finish(solver, info, iterations, as_np, _is_volume(A))
        self._cv_info(solver, info, iterations, _is_volume(A))
        return x, info


class PDHG(Solver):
    """Chambolle-Pock PDHG with the KL data term and optional isotropic TV2D (corrct ``solvers.py:987-1206``).

    ``regularizer`` is an object with ``__reg_name__ == "TV2D"`` (or a float TV weight).  With a
    ``tolerance`` or a ``b_test_mask`` every iterate is projected once more for its residuals, as
    the reference does (solvers.py:1192-1204).
    """

    def __init__(self, verbose: bool = False, leave_progress: bool = True, tolerance=None, relaxation: float = 0.95, regularizer=None, data_term="kl", data_term_test=None):
        super().__init__(verbose=verbose, leave_progress=leave_progress, relaxation=relaxation, tolerance=tolerance, data_term=data_term, data_term_test=data_term_test)
        if self.data_term != "kl":
            raise NotImplementedError("the fused PDHG uses the KL data term")
        self.tv_weight = _tv_weight(regularizer)

    def __call__(self, A, b, iterations: int, x0=None, lower_limit=None, upper_limit=None, x_mask=None, b_mask=None, b_test_mask=None, precondition: bool = True):
        _check_projector(A)
        bt, x0t, mt, maps, as_np = _as_batch(A, b, x0, x_mask)
        bm, btm = self._masks(A, b_mask, b_test_mask)
        bp_mode = "symmetric" if getattr(A, "is_symmetric", False) else "reference"
        if self.tv_weight is None:
            raise NotImplementedError("the fused PDHG needs a TV2D regularizer")
        scaling = None
        if not precondition:
            # compute_Lipschitz_scaling (solvers.py:120-158); the TV term adds 2 * ndims to tau
            L = _operator_norm(A, b, bt, bp_mode, maps)
            scaling = (self.relaxation / L, self.relaxation / (L + 4.0))
        solver = BatchedSolver(
            A.core, maps, bt, "pdhg", x0=x0t, x_mask=mt, lower_limit=lower_limit, upper_limit=upper_limit,
            relaxation=self.relaxation, tv_lambda=self.tv_weight, bp_mode=bp_mode, background=self.background,
            joint_stop=_is_volume(A), b_mask=bm, scaling=scaling,
        )
        info = SolutionInfo(self.info(), max_iterations=iterations, tolerance=self.tolerance)
        if self.tolerance is None and btm is None:
            solver.run(iterations, check_every=max(iterations, 1))
            x, info = _finish(solver, info, iterations, as_np, _is_volume(A))
            info.iterations = iterations
            return x, info

        def residuals(x):
            # KL residuals with the dual scaling sigma (data_terms.py:720-742, solvers.py:1137)
            ax = A.core.fp(x, maps)
            r = _kl_residual_norm(ax, bt, self.background, bm, solver.sigma)
            r_cv = None if btm is None else _kl_residual_norm(ax, bt, self.background, btm, solver.sigma)
            return r, r_cv

        info.residual0, r0_cv = residuals(solver.x)
        if r0_cv is not None:
            info.residual0_cv = r0_cv
        for ii in range(iterations):
            info.iterations += 1
            solver.step()
            info.residuals[ii], r_cv = residuals(solver.x)
            if r_cv is not None:
                info.residuals_cv[ii] = r_cv
            if self.tolerance is not None and self.tolerance > info.residuals[ii]:
                break
        x = solver.x if _is_volume(A) else solver.x[0]
        return (x.cpu().numpy() if as_np else x.clone()), info


def _tv_weight(regularizer):
    if regularizer is None:
        return None
    if isinstance(regularizer, (int, float)):
        return float(regularizer)
    if getattr(regularizer, "__reg_name__", "") == "TV2D":
        return float(np.max(np.asarray(regularizer.weight)))
    raise NotImplementedError("only the isotropic TV2D regularizer is supported by the B200 PDHG")


def _kl_residual_norm(ax: torch.Tensor, b: torch.Tensor, background, mask: torch.Tensor | None = None,
                      sigma: torch.Tensor | None = None) -> float:
    """||KL residual * mask||_1 in FP64 (corrct ``data_terms.py:720-742``; sigma = 1 unless given)."""
    proj = ax.double() if background is None else ax.double() + background
    r = torch.clamp(proj, min=float(eps))
    sd = 4 * torch.clamp(b.double(), min=0)
    if sigma is not None:
        r = r * sigma.double()
        sd = sd * sigma.double()
    res = (1 + r - torch.sqrt((r - 1) ** 2 + sd)) / 2
    if mask is not None:
        res = res * mask.double()
    return float(res.abs().sum().item())


class SART(Solver):
    """SART row-action solver on per-angle device projections (corrct ``solvers.py:473-631``)."""

    def __call__(self, A, b, iterations: int, A_num_rows=None, At=None, x0=None, lower_limit=None, upper_limit=None, x_mask=None, b_mask=None):
        _check_projector(A)
        dev = A.projector_backend.device
        n_ang = len(A.angles_rot_rad)
        as_np = not isinstance(b, torch.Tensor)
        bt = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float32) if as_np else b).to(dev, torch.float32)
        xrf = isinstance(A, ProjectorAttenuationXRF)
        fpa = lambda x, ii: A.fp_angle(x, ii)  # noqa: E731
        bpa = (lambda y, ii: A.bp_angle(y, ii, single_line=True)) if xrf else (lambda y, ii: A.bp_angle(y, ii))  # noqa: E731
        bm = None if b_mask is None else _tensor(b_mask, dev).expand(bt.shape).contiguous()
        b_ones = torch.ones_like(bt) if bm is None else bm.clone()
        tau = torch.stack([bpa(b_ones[..., ii, :].contiguous(), ii) for ii in range(n_ang)], dim=-2).abs()
        tau = torch.where(tau / tau.max() < 1e-5, torch.ones_like(tau), tau)
        tau = self.relaxation / tau
        vol_shape = tuple(int(v) for v in A.vol_shape)
        x_ones = torch.ones(vol_shape, device=dev)
        if x_mask is not None:
            x_ones = x_ones * _tensor(x_mask, dev)
        sigma = torch.stack([fpa(x_ones, ii) for ii in range(n_ang)], dim=-2).abs()
        sigma = torch.where(sigma / sigma.max() < 1e-5, torch.ones_like(sigma), sigma)
        sigma = 1 / sigma
        x = torch.zeros(vol_shape, device=dev) if x0 is None else _tensor(x0, dev).reshape(vol_shape).clone()
        mask = None if x_mask is None else _tensor(x_mask, dev)
        info = SolutionInfo(self.info(), max_iterations=iterations, tolerance=self.tolerance)

        def residual_norm(v):
            # compute_residual (solvers.py:476-508): all angles' projections minus the data, masked
            r = torch.stack([fpa(v, a) for a in range(n_ang)], dim=-2) - bt
            if bm is not None:
                r = r * bm
            return float(torch.linalg.norm(r.double()).item())

        if self.tolerance is not None:
            info.residual0 = residual_norm(x)
        rows_sequence = np.random.permutation(n_ang)
        for ii in range(iterations):
            info.iterations += 1
            for a in rows_sequence:
                res = fpa(x, int(a)) - bt[..., a, :]
                if bm is not None:
                    res = res * bm[..., a, :]
                x = x - bpa((res * sigma[..., a, :]).contiguous(), int(a)) * tau[..., a, :]
                if lower_limit is not None:
                    x = torch.clamp(x, min=lower_limit)
                if upper_limit is not None:
                    x = torch.clamp(x, max=upper_limit)
                if mask is not None:
                    x = x * mask
            if self.tolerance is not None:
                info.residuals[ii] = residual_norm(x)
                if self.tolerance > info.residuals[ii]:
                    break
        return (x.cpu().numpy() if as_np else x), info


class FISTA(Solver):
    """FISTA with the l2 data term and no regularizer (corrct ``solvers.py:1209-1513``)."""

    def __init__(self, verbose: bool = False, leave_progress: bool = True, tolerance=None, relaxation: float = 1.0, regularizer=None, data_term="l2", data_term_test=None, restart_period=None):
        super().__init__(verbose=verbose, leave_progress=leave_progress, relaxation=relaxation, tolerance=tolerance, data_term=data_term, data_term_test=data_term_test)
        if regularizer is not None:
            raise NotImplementedError("FISTA regularizers are not supported by the B200 solvers")
        if self.data_term != "l2":
            raise ValueError(f"Unknown data term: '{data_term}'. FISTA only accepts 'l2' and derivatives.")
        self.restart_period = restart_period

    def __call__(self, A, b, iterations: int, x0=None, lower_limit=None, upper_limit=None, x_mask=None, b_mask=None, b_test_mask=None, precondition: bool = True):
        _check_projector(A)
        bt, x0t, mt, maps, as_np = _as_batch(A, b, x0, x_mask)
        bm, btm = self._masks(A, b_mask, b_test_mask)
        core = A.core
        bp_mode = "symmetric" if getattr(A, "is_symmetric", False) else "reference"
        fp = lambda v: core.fp(v, maps)  # noqa: E731
        bp = lambda y: core.bp(y, bp_mode, maps if bp_mode == "symmetric" else None)  # noqa: E731
        n = core.n
        z = bt.shape[0]
        if precondition:
            # compute_diagonal_scaling (solvers.py:60-117), relaxation on tau
            tau = bp(torch.ones_like(bt) if bm is None else bm.clone()).abs()
            tau = torch.where(tau / tau.max() < 1e-5, torch.ones_like(tau), tau)
            tau = self.relaxation / tau
            x_ones = torch.ones((z, n, n), device=core.device)
            if mt is not None:
                x_ones = x_ones * mt
            sigma = fp(x_ones).abs()
            sigma = torch.where(sigma / sigma.max() < 1e-5, torch.ones_like(sigma), sigma)
            sigma = 1.0 / sigma
        else:
            # compute_Lipschitz_scaling (solvers.py:120-158) without regularizers
            L = _operator_norm(A, b, bt, bp_mode, maps)
            sigma, tau = 1.0 / L, self.relaxation / L
        x = torch.zeros((z, n, n), device=core.device) if x0t is None else x0t.clone()
        if mt is not None:
            x = x * mt
        y = x.clone()
        t = 1.0
        bg = 0.0 if self.background is None else self.background
        info = SolutionInfo(self.info(), max_iterations=iterations, tolerance=self.tolerance)
        track = self.tolerance is not None or btm is not None

        def residuals(v):
            # squared l2 norms of the masked residuals (data_terms.py:136-161)
            r = bt - (fp(v.contiguous()) + bg)
            rm = r if bm is None else r * bm
            r_cv = None if btm is None else float(torch.sum((r * btm).double() ** 2).item())
            return float(torch.sum(rm.double() ** 2).item()), r_cv

        if track:
            info.residual0, r_cv = residuals(x)
            if r_cv is not None:
                info.residual0_cv = r_cv
        for ii in range(iterations):
            info.iterations += 1
            residual = bt - (fp(y.contiguous()) + bg)
            if bm is not None:
                residual = residual * bm
            grad = bp((residual * sigma).contiguous())
            x_new = y + tau * grad
            if lower_limit is not None or upper_limit is not None:
                x_new = torch.clamp(x_new, min=lower_limit, max=upper_limit)
            if mt is not None:
                x_new = x_new * mt
            t_new = float(1.0 + np.sqrt(1.0 + 4.0 * t * t)) / 2.0
            if self.restart_period is not None and (ii + 1) % self.restart_period == 0:
                t_new = 1.0
            momentum = (t - 1.0) / t_new
            y = x_new + momentum * (x_new - x)
            x, t = x_new, t_new
            if track:
                info.residuals[ii], r_cv = residuals(x)
                if r_cv is not None:
                    info.residuals_cv[ii] = r_cv
                if self.tolerance is not None and self.tolerance > info.residuals[ii]:
                    break
        x = x if _is_volume(A) else x[0]
        return (x.cpu().numpy() if as_np else x), info
