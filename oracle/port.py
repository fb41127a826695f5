"""Standalone numpy port of the reference's attenuation-corrected XRF projection path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Every function names the
reference ``file:line`` (paths inside the ``corrct`` project) whose behaviour it
restates.  The scikit-image primitives come from ``oracle.skimage_restated``.
All arithmetic follows the dtype of the inputs: float64 inputs give the FP64
oracle; float32 inputs reproduce the reference's default float32 run.

This module is checked against golden fixtures produced by the reference's own
Python (``tests/golden/make_golden.py``); it is what the GPU parity tests
compare against at sizes beyond the fixtures, and what the CPU-baseline legs of
``bench.py`` time.
"""

from __future__ import annotations

import concurrent.futures as cf
from collections.abc import Sequence

import numpy as np
from numpy.typing import NDArray

from . import skimage_restated as skr

EPS32 = np.finfo(np.float32).eps  # solvers.py:20, data_terms.py:19


# --------------------------------------------------------------------------------------
# Geometry helpers
# --------------------------------------------------------------------------------------


def backend_angles(angles_rot_rad: Sequence[float] | NDArray) -> tuple[NDArray, NDArray]:
    """Backend angles: float32 radians and float32 degrees.

    ``_projector_backends.py:148`` casts the angles to float32 and
    ``_projector_backends.py:299`` converts them with ``np.rad2deg``.
    """
    rad = np.array(angles_rot_rad, ndmin=1, dtype=np.float32)
    return rad, np.rad2deg(rad)


def padded_size(n: int) -> tuple[int, int]:
    """Padding of ``compute_attenuation``: returns (edge, padded size) (``_projector_backends.py:75-77``)."""
    min_size = np.ceil(np.sqrt(2.0 * n * n))
    edge = int(np.ceil((min_size - n) / 2))
    return edge, n + 2 * edge


# --------------------------------------------------------------------------------------
# Attenuation maps
# --------------------------------------------------------------------------------------


def compute_attenuation(vol: NDArray, angle_rad: float, invert: bool = False) -> NDArray:
    """exp(-line integral) map of one 2-D slice for one direction.

    Restates ``_projector_backends.py:43-99``: zero-pad to the diagonal
    (``:62-65, 75-77, 83``), rotate by ``-angle`` (``:68``), add the rolled copy
    and cumulate half of it along rows (``:70-71``), rotate back (``:73``), crop
    (``:95``) and exponentiate (``:97``).  ``invert`` adds pi (``:79-80``).
    """
    n = vol.shape[-1]
    edge, _ = padded_size(n)
    if invert:
        angle_rad += np.pi
    rot_angle_deg = np.rad2deg(angle_rad)
    cum = np.pad(vol, ((edge, edge), (edge, edge)), mode="constant")
    cum = skr.rotate(cum, -rot_angle_deg, order=1, clip=False)
    cum += np.roll(cum, 1, axis=-2)
    cum = np.cumsum(cum / 2, axis=-2)
    cum = skr.rotate(cum, rot_angle_deg, order=1, clip=False)
    cum = cum[edge:-edge, edge:-edge]
    return np.exp(-cum)


def detector_sub_angles(surface_mm2: float, distance_mm: float, sub_sampling: int) -> NDArray:
    """Sub-angle offsets of a finite detector (``physics/xrf.py:243-258``, ``attenuation.py:111-114``)."""
    if surface_mm2 > 0.0:
        half_edge = np.sqrt(surface_mm2) / 2
        half_angle = np.arctan2(half_edge, distance_mm)
        sub = np.linspace(-half_angle, half_angle, sub_sampling + 1)
        return np.convolve(sub, np.ones(2), "valid") / 2
    return np.zeros(1)


def compute_maps(
    mu_in: NDArray | None,
    mu_out: NDArray | None,
    angles_rot_rad: NDArray,
    angles_det_rad: Sequence[float] | NDArray = (np.pi / 2,),
    dtype=np.float64,
    detector_surfaces_mm2: Sequence[float] | None = None,
    detector_distances_mm: Sequence[float] | None = None,
    emitted_sub_sampling: int = 1,
    workers: int = 1,
) -> NDArray:
    """Attenuation maps ``(A, D, N, N)`` = exp(-L_in) * mean_s exp(-L_out).

    Restates ``AttenuationVolume.compute_maps`` (``physics/attenuation.py:122-180``)
    with ``_compute_attenuation_angle_in`` (``:105-106``) and
    ``_compute_attenuation_angle_out`` (``:108-120``).  ``angles_rot_rad`` are the
    (float32) backend angles the projector passes in (``projectors.py:462``).
    ``workers > 1`` spreads angles over a thread pool like the reference
    (``attenuation.py:139-158``); results do not depend on it.
    """
    angles_rot_rad = np.array(angles_rot_rad, ndmin=1)
    det_angles = np.array(angles_det_rad, ndmin=1, dtype=np.float64)
    n_det = len(det_angles)
    surfaces = np.zeros(n_det) if detector_surfaces_mm2 is None else np.array(detector_surfaces_mm2, ndmin=1)
    distances = np.ones(n_det) if detector_distances_mm is None else np.array(detector_distances_mm, ndmin=1)
    ref = mu_in if mu_in is not None else mu_out
    if ref is None:
        raise ValueError("No attenuation volumes were given.")
    n_ang = len(angles_rot_rad)
    maps = np.ones([n_ang, n_det, *ref.shape], dtype=dtype)

    def one_angle(ii: int) -> None:
        a = angles_rot_rad[ii]
        if mu_in is not None:
            maps[ii] *= compute_attenuation(mu_in, a, invert=False)[None, ...]
        if mu_out is not None:
            angle_det = a + det_angles
            atts = np.zeros(maps.shape[1:], dtype=dtype)
            for dd, ad in enumerate(angle_det):
                subs = detector_sub_angles(surfaces[dd], distances[dd], emitted_sub_sampling)
                for a_s in subs:
                    atts[dd] += compute_attenuation(mu_out, ad + a_s, invert=True)
                atts[dd] /= len(subs)
            maps[ii] *= atts

    if workers > 1:
        with cf.ThreadPoolExecutor(max_workers=workers) as ex:
            list(ex.map(one_angle, range(n_ang)))
    else:
        for ii in range(n_ang):
            one_angle(ii)
    return maps


# --------------------------------------------------------------------------------------
# Projections
# --------------------------------------------------------------------------------------


def fp_angle(vol: NDArray, angle_deg32: np.floating) -> NDArray:
    """One sinogram line: ``skt.radon(vol, [deg])`` squeezed (``_projector_backends.py:333``)."""
    return np.squeeze(skr.radon(vol, np.asarray([angle_deg32])))


def bp_angle(line: NDArray, angle_deg32: np.floating, n: int) -> NDArray:
    """One-line back projection ``iradon(...)*2/pi`` (``_projector_backends.py:358-359``)."""
    vol = skr.iradon(line[:, np.newaxis], np.asarray([angle_deg32]), output_size=n, filter_name=None, circle=False)
    return vol * 2 / np.pi


def fp_uncorrected(vol: NDArray, angles_deg32: NDArray, workers: int = 1) -> NDArray:
    """Sinogram ``(A, N)`` of ``ProjectorBackendSKimage.fp`` (``_projector_backends.py:326-331``)."""
    out = np.empty((len(angles_deg32), vol.shape[-1]), dtype=vol.dtype)

    def one(ii: int) -> None:
        out[ii] = fp_angle(vol, angles_deg32[ii])

    _run(one, len(angles_deg32), workers)
    return out


def bp_uncorrected(sino: NDArray, angles_deg32: NDArray, n: int, workers: int = 1, intensities=None) -> NDArray:
    """Volume ``(N, N)`` of ``ProjectorBackendSKimage.bp`` (``_projector_backends.py:352-359``), after
    ``ProjectorUncorrected.bp``'s intensity scaling (``projectors.py:336-337``; the PSF adjoint is the
    identity for the default ``is_symm=False``)."""
    if intensities is not None:
        sino = sino * np.asarray(intensities)[:, None]
    parts = np.empty((len(angles_deg32), n, n), dtype=sino.dtype)

    def one(ii: int) -> None:
        parts[ii] = skr.iradon(
            sino[ii, :, np.newaxis], np.asarray([angles_deg32[ii]]), output_size=n, filter_name=None, circle=False
        )

    _run(one, len(angles_deg32), workers)
    return parts.sum(axis=0) * 2 / np.pi


def _run(func, count: int, workers: int) -> None:
    if workers > 1:
        with cf.ThreadPoolExecutor(max_workers=workers) as ex:
            list(ex.map(func, range(count)))
    else:
        for ii in range(count):
            func(ii)


def _weights(n_ang: int, n_det: int, weights_det, weights_angles) -> NDArray:
    """Per (angle, detector) weight ``w_det[d] * w_ang[a, d]`` (``projectors.py:439-459, 516``)."""
    wd = np.ones(n_det) if weights_det is None else np.array(weights_det, ndmin=1, dtype=np.float64)
    if n_det > 1 and len(wd) == 1:
        wd = np.tile(wd, [n_det])
    wa = np.ones((n_ang, n_det)) if weights_angles is None else np.array(weights_angles)
    return wd[None, :] * wa


def psf_convolve(line: NDArray, kernel: NDArray) -> NDArray:
    """Detector PSF of ``TransformConvolution._op_direct`` (``operators.py:472-483``) on one line:
    edge padding by (L-1)//2, scipy 'same' convolution, crop."""
    from scipy import signal

    kernel = np.asarray(kernel)
    pw = (len(kernel) - 1) // 2
    x = np.pad(line, pw, mode="edge")
    x = signal.convolve(x, kernel, mode="same")
    return x[pw:-pw] if pw else x


def _line(vol2d, deg32, ii_intensity, psf):
    """``ProjectorUncorrected.fp_angle`` (``projectors.py:259-279``): radon, intensity, PSF."""
    prj = fp_angle(vol2d, deg32)
    if ii_intensity is not None:
        prj = prj * ii_intensity
    if psf is not None:
        prj = psf_convolve(prj, psf)
    return prj


def fp_xrf(
    vol: NDArray,
    maps: NDArray,
    angles_deg32: NDArray,
    weights_det=None,
    weights_angles=None,
    workers: int = 1,
    intensities=None,
    psf=None,
) -> NDArray:
    """Attenuated forward projection (``ProjectorAttenuationXRF.fp``, ``projectors.py:502-531, 570-596``).

    Returns ``(D, A, N)``, squeezed to ``(A, N)`` for a single detector.
    """
    n_ang, n_det = maps.shape[:2]
    w = _weights(n_ang, n_det, weights_det, weights_angles)
    out = np.empty((n_det, n_ang, vol.shape[-1]), dtype=np.result_type(vol, maps))

    def one(ii: int) -> None:
        temp = vol * maps[ii]
        inten = None if intensities is None else intensities[ii]
        for dd in range(n_det):
            out[dd, ii] = w[ii, dd] * _line(temp[dd], angles_deg32[ii], inten, psf)

    _run(one, n_ang, workers)
    return out[0] if n_det == 1 else out


def bp_xrf(
    sino: NDArray,
    maps: NDArray,
    angles_deg32: NDArray,
    weights_det=None,
    weights_angles=None,
    is_symmetric: bool = False,
    workers: int = 1,
    intensities=None,
) -> NDArray:
    """Back projection of ``ProjectorAttenuationXRF.bp`` (``projectors.py:533-568, 598-622``).

    Default (``is_symmetric=False``): plain per-detector back projections summed,
    with neither maps nor weights (``:619-622``).  Symmetric: per angle, weighted
    per-detector back projections multiplied by the maps (``:553-568``).
    """
    n_ang, n_det = maps.shape[:2]
    n = maps.shape[-1]
    sino = np.reshape(sino, [n_det, n_ang, -1])
    if not is_symmetric:
        return np.sum(
            np.stack([bp_uncorrected(sino[d], angles_deg32, n, workers, intensities) for d in range(n_det)]), axis=0
        )
    w = _weights(n_ang, n_det, weights_det, weights_angles)
    if intensities is not None:
        w = w * np.asarray(intensities)[:, None]
    parts = np.empty((n_ang, n, n), dtype=np.result_type(sino, maps))

    def one(ii: int) -> None:
        acc = np.stack([w[ii, d] * bp_angle(sino[d, ii], angles_deg32[ii], n) for d in range(n_det)])
        acc *= maps[ii]
        parts[ii] = acc.sum(axis=0)

    _run(one, n_ang, workers)
    return parts.sum(axis=0)


def fp_xrf_adjoint(
    sino: NDArray, maps: NDArray | None, angles_deg32: NDArray, n: int, weights_det=None, weights_angles=None
) -> NDArray:
    """Exact transpose of ``fp_xrf`` (scatter of every bilinear tap).

    No reference counterpart: the reference's back projection is the unmatched
    ``iradon`` discretisation.  This is the definition the GPU ``adjoint`` mode is
    tested against.  ``maps=None`` gives the transpose of the uncorrected fp.
    """
    n_ang = len(angles_deg32)
    n_det = 1 if maps is None else maps.shape[1]
    sino = np.reshape(sino, [n_det, n_ang, n])
    w = _weights(n_ang, n_det, weights_det, weights_angles)
    out = np.zeros((n, n), dtype=np.float64)
    rr, cc = np.mgrid[:n, :n]
    for ii in range(n_ang):
        m = skr.radon_matrix(angles_deg32[ii], n).astype(np.float64)
        cols_in = m[0, 0] * cc + m[0, 1] * rr + m[0, 2]
        rows_in = m[1, 0] * cc + m[1, 1] * rr + m[1, 2]
        r0, c0 = np.floor(rows_in), np.floor(cols_in)
        r1, c1 = np.ceil(rows_in), np.ceil(cols_in)
        dr, dc = rows_in - r0, cols_in - c0
        for dd in range(n_det):
            vals = np.broadcast_to(sino[dd, ii][None, :] * w[ii, dd], (n, n))
            acc = np.zeros((n, n))
            for rt, ct, wt in (
                (r0, c0, (1 - dr) * (1 - dc)),
                (r0, c1, (1 - dr) * dc),
                (r1, c0, dr * (1 - dc)),
                (r1, c1, dr * dc),
            ):
                ri, ci = rt.astype(np.int64), ct.astype(np.int64)
                ok = (ri >= 0) & (ri < n) & (ci >= 0) & (ci < n)
                np.add.at(acc, (ri[ok], ci[ok]), (vals * wt)[ok])
            out += acc if maps is None else acc * maps[ii, dd]
    return out


# --------------------------------------------------------------------------------------
# Data terms, TV, solvers (update equations of solvers.py)
# --------------------------------------------------------------------------------------


def kl_residual(ax: NDArray, b: NDArray, sigma=1.0, background=None, mask=None) -> NDArray:
    """``DataFidelity_KL.compute_residual`` with the proximal (``data_terms.py:720-739``)."""
    proj = ax if background is None else ax + background
    proj = np.fmax(proj, EPS32)
    res = np.fmax(proj, EPS32) * sigma
    sigma_data = 4 * sigma * np.fmax(b, 0.0)
    res = (1 + res - np.sqrt((res - 1) ** 2 + sigma_data)) / 2
    if mask is not None:
        res = res * mask
    return -res


def kl_residual_norm(res: NDArray) -> float:
    """l1 norm of the KL residual (``data_terms.py:741-742``)."""
    return float(np.linalg.norm(res.flatten(), ord=1))


def l2_residual(ax: NDArray, b: NDArray, background=None, mask=None) -> NDArray:
    """``DataFidelityBase.compute_residual`` (``data_terms.py:136-161``)."""
    proj = ax if background is None else ax + background
    res = b - proj
    if mask is not None:
        res = res * mask
    return res


def gradient(x: NDArray) -> NDArray:
    """``TransformGradient.gradient`` with edge padding (``operators.py:796-816``)."""
    d = []
    for ax in (-2, -1):
        pad = [(0, 0)] * x.ndim
        pad[ax] = (0, 1)
        d.append(np.diff(np.pad(x, pad, mode="edge"), n=1, axis=ax))
    return np.stack(d, axis=0)


def divergence(q: NDArray) -> NDArray:
    """``TransformGradient.divergence`` with edge padding (``operators.py:818-844``)."""
    d = []
    for ii, ax in enumerate((-2, -1)):
        pad = [(0, 0)] * (q.ndim - 1)
        pad[ax] = (1, 0)
        d.append(np.diff(np.pad(q[ii], pad, mode="edge"), n=1, axis=ax))
    return np.sum(np.stack(d, axis=0), axis=0)


def diagonal_scaling(fp, bp, b: NDArray, x_shape, reg_tau: float = 0.0, relax_tau: float = 1.0, relax_sigma: float = 1.0, b_mask=None, x_mask=None):
    """``compute_diagonal_scaling`` (``solvers.py:60-117``) for one TV regularizer contribution ``reg_tau``."""
    b_ones = np.ones_like(b) if b_mask is None else np.ones_like(b) * b_mask
    tau = np.abs(bp(b_ones))
    tau = tau + reg_tau
    tau[(tau / np.max(tau)) < 1e-5] = 1
    tau = relax_tau / tau
    x_ones = np.ones(x_shape, dtype=tau.dtype) if x_mask is None else np.ones(x_shape, dtype=tau.dtype) * x_mask
    sigma = np.abs(fp(x_ones))
    sigma[(sigma / np.max(sigma)) < 1e-5] = 1.0
    sigma = relax_sigma / sigma
    return sigma, tau


def b_masks(b: NDArray, b_mask, b_test_mask):
    """``Solver._initialize_b_masks`` (``solvers.py:333-343``)."""
    if b_test_mask is not None:
        if b_mask is None:
            b_mask = np.ones_like(b)
        b_mask, b_test_mask = b_mask * (1 - b_test_mask), b_test_mask * b_mask
    return b_mask, b_test_mask


def power_method(fp, bp, b: NDArray, iterations: int = 5) -> float:
    """l2 norm of the operator by power iterations from a ``np.random.rand`` start (``solvers.py:26-57``)."""
    x = np.random.rand(*b.shape).astype(b.dtype)
    x /= np.linalg.norm(x)
    x = bp(x)
    x_norm = np.linalg.norm(x)
    L = x_norm
    for _ in range(iterations):
        x /= x_norm
        x = bp(fp(x))
        x_norm = np.linalg.norm(x)
        L = np.sqrt(x_norm)
    return float(L)


def lipschitz_scaling(fp, bp, b: NDArray, reg_tau: float = 0.0, relax_tau: float = 1.0, relax_sigma: float = 1.0):
    """``compute_Lipschitz_scaling`` (``solvers.py:120-158``): scalar (sigma, tau)."""
    L = power_method(fp, bp, b)
    return relax_sigma / L, relax_tau / (L + reg_tau)


def mlem(fp, bp, b: NDArray, iterations: int, x0=None, tolerance=None, lower_limit=None, upper_limit=None, x_mask=None,
         b_mask=None, b_test_mask=None, residuals_cv=None):
    """MLEM update loop of ``solvers.py:725-805`` (KL data term, no background).

    Returns (x, residuals list); the test-mask residuals go to the list ``residuals_cv``.
    """
    b = np.array(b)
    b_mask, b_test_mask = b_masks(b, b_mask, b_test_mask)
    tau = bp(np.ones_like(b) if b_mask is None else np.ones_like(b) * b_mask)
    x = np.ones_like(tau) if x0 is None else np.array(x0).copy()
    if x_mask is not None:
        x *= x_mask
    residuals = []
    for _ in range(iterations):
        ax = fp(x)
        if b_test_mask is not None and residuals_cv is not None:
            residuals_cv.append(kl_residual_norm(kl_residual(ax, b, mask=b_test_mask)))
        if tolerance is not None:
            r = kl_residual_norm(kl_residual(ax, b, mask=b_mask))
            residuals.append(r)
            if tolerance > r:
                break
        ax = ax.clip(EPS32, None)
        upd = bp(b / ax)
        x *= upd / tau
        if lower_limit is not None or upper_limit is not None:
            x = x.clip(lower_limit, upper_limit)
        if x_mask is not None:
            x *= x_mask
    return x, residuals


def sirt(fp, bp, b: NDArray, iterations: int, x_shape, relaxation: float = 1.95, x0=None, lower_limit=None, upper_limit=None, x_mask=None,
         b_mask=None, b_test_mask=None, residuals_cv=None):
    """SIRT update loop of ``solvers.py:895-984`` (l2 data term, no regularizer).

    The test-mask residuals (squared l2 norms) go to the list ``residuals_cv``.
    """
    b_mask, b_test_mask = b_masks(b, b_mask, b_test_mask)
    sigma, tau = diagonal_scaling(fp, bp, b, x_shape, relax_tau=relaxation, b_mask=b_mask, x_mask=x_mask)
    x = np.zeros_like(tau) if x0 is None else np.array(x0).copy()
    for _ in range(iterations):
        ax = fp(x)
        if b_test_mask is not None and residuals_cv is not None:
            residuals_cv.append(float(np.sum(l2_residual(ax, b, mask=b_test_mask) ** 2)))
        res = l2_residual(ax, b, mask=b_mask)
        x += bp(res * sigma) * tau
        if lower_limit is not None or upper_limit is not None:
            x = x.clip(lower_limit, upper_limit)
        if x_mask is not None:
            x *= x_mask
    return x


def pdhg_kl_tv(fp, bp, b: NDArray, iterations: int, x_shape, lam: float, relaxation: float = 0.95, lower_limit=None, upper_limit=None, x_mask=None,
               x0=None, b_mask=None, b_test_mask=None, tolerance=None, residuals=None, residuals_cv=None, precondition: bool = True):
    """PDHG with KL data term and isotropic TV2D (``solvers.py:1099-1206``).

    Dual KL prox ``data_terms.py:682-692``; TV via ``Regularizer_Grad``
    (``regularizers.py:260-273``, sigma = 0.5, tau contribution 2*ndims = 4) with
    the l12 dual prox (``data_terms.py:549-555, 607-608``).  With a tolerance or a test mask
    the KL residuals (with the dual scaling sigma) of every iterate go to the lists
    ``residuals`` / ``residuals_cv``.
    """
    b = np.array(b)
    b_mask, b_test_mask = b_masks(b, b_mask, b_test_mask)
    if precondition:
        sigma, tau = diagonal_scaling(fp, bp, b, x_shape, reg_tau=4.0, relax_tau=relaxation, relax_sigma=relaxation, x_mask=x_mask, b_mask=b_mask)
    else:
        sigma, tau = lipschitz_scaling(fp, bp, b, reg_tau=4.0, relax_tau=relaxation, relax_sigma=relaxation)
    x = np.zeros(x_shape, dtype=b.dtype) if x0 is None else np.array(x0).copy()
    x_relax = x.copy()
    sigma_data = 4 * sigma * np.fmax(b, 0.0)
    p = np.zeros_like(b)
    q = np.zeros((2, *x_shape), dtype=x.dtype)
    track = tolerance is not None or b_test_mask is not None
    for _ in range(iterations):
        p += fp(x_relax) * sigma
        p[:] = (1 + p - np.sqrt((p - 1) ** 2 + sigma_data)) / 2
        if b_mask is not None:
            p *= b_mask
        q += 0.5 * gradient(x_relax)
        qn = np.linalg.norm(q, ord=2, axis=0, keepdims=True)
        q /= np.fmax(qn, lam)
        q *= lam
        upd = bp(p) - divergence(q)
        x_new = x - upd * tau
        if lower_limit is not None or upper_limit is not None:
            x_new = x_new.clip(lower_limit, upper_limit)
        if x_mask is not None:
            x_new *= x_mask
        x_relax = x_new + (x_new - x)
        x = x_new
        if track:
            ax = fp(x)
            r = kl_residual_norm(kl_residual(ax, b, sigma, mask=b_mask))
            if residuals is not None:
                residuals.append(r)
            if b_test_mask is not None and residuals_cv is not None:
                residuals_cv.append(kl_residual_norm(kl_residual(ax, b, sigma, mask=b_test_mask)))
            if tolerance is not None and tolerance > r:
                break
    return x


def fista(fp, bp, b: NDArray, iterations: int, x_shape, relaxation: float = 1.0, x0=None, lower_limit=None, upper_limit=None,
          x_mask=None, b_mask=None, b_test_mask=None, tolerance=None, restart_period=None, residuals=None, residuals_cv=None,
          precondition: bool = True):
    """FISTA, l2 data term, no regularizer (``solvers.py:1395-1513``); diagonal or Lipschitz scaling."""
    b = np.array(b)
    b_mask, b_test_mask = b_masks(b, b_mask, b_test_mask)
    if precondition:
        sigma, tau = diagonal_scaling(fp, bp, b, x_shape, relax_tau=relaxation, x_mask=x_mask, b_mask=b_mask)
    else:
        sigma, tau = lipschitz_scaling(fp, bp, b, relax_tau=relaxation)
    x = np.zeros(x_shape, dtype=b.dtype) if x0 is None else np.array(x0).copy()
    if x_mask is not None:
        x *= x_mask
    y = x.copy()
    t = 1.0
    track = tolerance is not None or b_test_mask is not None
    for ii in range(iterations):
        grad = bp(l2_residual(fp(y), b, mask=b_mask) * sigma)
        x_new = y + tau * grad
        if lower_limit is not None or upper_limit is not None:
            x_new = x_new.clip(lower_limit, upper_limit)
        if x_mask is not None:
            x_new *= x_mask
        t_new = float(1.0 + np.sqrt(1.0 + 4.0 * t * t)) / 2.0
        if restart_period is not None and (ii + 1) % restart_period == 0:
            t_new = 1.0
        y = x_new + (t - 1.0) / t_new * (x_new - x)
        x, t = x_new, t_new
        if track:
            ax = fp(x)
            r = float(np.sum(l2_residual(ax, b, mask=b_mask) ** 2))
            if residuals is not None:
                residuals.append(r)
            if b_test_mask is not None and residuals_cv is not None:
                residuals_cv.append(float(np.sum(l2_residual(ax, b, mask=b_test_mask) ** 2)))
            if tolerance is not None and tolerance > r:
                break
    return x


# --------------------------------------------------------------------------------------
# Synthetic data
# --------------------------------------------------------------------------------------
def add_noise(
    img_clean: NDArray,
    num_photons: float,
    add_poisson: bool = False,
    readout_noise_std: float | None = None,
    background_avg: float | None = None,
    background_std: float | None = None,
    detection_efficiency: float = 1.0,
    dtype=np.float32,
) -> tuple[NDArray, NDArray, float]:
    """Noise model of ``testing.add_noise`` (``testing.py:266-320``) on numpy's global generator.

    Draw order and arithmetic follow the reference (a float32 image scaled by a Python float,
    float64 background and read-out terms added in place, the background mean taken before the
    Poisson draw), so after ``np.random.seed(s)`` it returns the reference's values.
    """
    scaled = num_photons * detection_efficiency * img_clean.copy().astype(dtype)
    noisy = scaled.copy()
    if background_avg is not None:
        std = background_avg * 5e-2 if background_std is None else background_std
        noisy += num_photons * detection_efficiency * np.abs(np.random.normal(background_avg, std, scaled.shape))
    background = float(np.mean((noisy - scaled).flatten()))
    if add_poisson:
        noisy = np.random.poisson(noisy).astype(dtype)
    if readout_noise_std is not None:
        noisy += np.random.normal(0, readout_noise_std, scaled.shape)
    return noisy, scaled, background
