"""Per-angle sampling matrices of the XRF path, built with the same numpy operations as the reference.

The kernels receive, per angle, the exact matrices scikit-image builds inside the
reference's scikit-image backend, so sample positions agree with the reference
to float32 rounding:

* ``fp_matrices`` — scikit-image ``radon`` (``circle=True``) inverse map per angle:
  ``np.deg2rad`` of the float32 backend degrees (``corrct``:
  ``src/corrct/_projector_backends.py:148, 299``), float32 ``cos``/``sin``, and the
  entries ``[[c, s, -C(c+s-1)], [-s, c, -C(c-s-1)]]`` with ``C = n // 2`` evaluated in
  float32.
* ``bp_trig`` — the float32 ``(cos, sin)`` that scikit-image ``iradon`` uses for the
  back projection of each angle.
* ``rotate_matrix`` — scikit-image ``rotate`` about ``((P-1)/2, (P-1)/2)`` composed in
  float64 from ``math.cos``/``math.sin`` of ``np.deg2rad(angle)``.
* ``attenuation_rotations`` — the two rotations (``-phi`` then ``+phi``) of every
  ``compute_attenuation`` call (``src/corrct/_projector_backends.py:67-80``) made by
  ``AttenuationVolume.compute_maps`` (``src/corrct/physics/attenuation.py:105-120``):
  incident angles are the float32 backend angles; emitted angles are
  ``angle + detector angle + sub-angle + pi`` in float64.
"""

from __future__ import annotations

import math
from collections.abc import Sequence

import numpy as np
from numpy.typing import NDArray


def backend_angles(angles_rot_rad) -> tuple[NDArray, NDArray]:
    """(float32 radians, float32 degrees) as the reference backend stores them."""
    rad = np.array(angles_rot_rad, ndmin=1, dtype=np.float32)
    return rad, np.rad2deg(rad)


def fp_matrices(angles_deg32: NDArray, n: int) -> NDArray:
    """``(A, 6)`` float32 radon inverse maps (M00, M01, M02, M10, M11, M12)."""
    out = np.empty((len(angles_deg32), 6), dtype=np.float32)
    center = n // 2
    for ii, th in enumerate(np.asarray(angles_deg32, dtype=np.float32)):
        angle = np.deg2rad(np.asarray([th]))[0]
        c, s = np.cos(angle), np.sin(angle)
        out[ii] = [c, s, -center * (c + s - 1), -s, c, -center * (c - s - 1)]
    return out


# Row strides the forward projection may use for its staged box, per kernel: (candidate
# strides, shared-memory banks per phase of the element size, lanes per phase).
FP_STRIDE_CHOICES = (
    (np.array([100]), 32, 32),         # one slice per CTA: fixed (immediate tap offsets)
    (80 + 2 * np.arange(5), 16, 16),   # two slices per CTA: 8-byte elements, even strides
)


def fp_box_strides(fp_mat: NDArray, patches: int = 8) -> NDArray:
    """``(A, 2)`` int32 row-stride selectors of the forward projection's staged box: column 0 for
    the one-slice kernel (always 0: its stride is fixed at 100 floats), column 1 for the two-slice
    kernel (``80 + 2 v`` elements of two floats, v in 0..4).

    A warp samples an 8 (columns) x 4 (rows) block of the rotated lattice (lane = 8 row-lane +
    column-lane) and reads each bilinear tap of a sample as one element; the shared-memory bank
    of an element is its index modulo the banks per phase (32 four-byte banks for 32 lanes, or
    16 eight-byte banks for each 16-lane half).  For each angle this counts, over a few lattice
    blocks, the wavefronts of every candidate stride (distinct elements per bank, the largest per
    phase) and keeps the cheapest.  Speed only: any choice gives the same results.
    """
    m = np.asarray(fp_mat, dtype=np.float64).reshape(-1, 6)
    a = m.shape[0]
    out = np.zeros((a, 2), dtype=np.int32)
    if a == 0:
        return out
    lane = np.arange(32)
    lc, lr = lane % 8, lane // 8
    p = np.arange(patches)
    c = (p[:, None] * 37 + 5) % 61 + lc[None, :]          # (P, 32) lattice columns
    r = (p[:, None] * 53 + 11) % 59 + lr[None, :]         # rows
    px = m[:, 0, None, None] * c + m[:, 1, None, None] * r + m[:, 2, None, None]
    py = m[:, 3, None, None] * c + m[:, 4, None, None] * r + m[:, 5, None, None]
    fx = np.floor(px).astype(np.int64)                    # (A, P, 32)
    fy = np.floor(py).astype(np.int64)
    for col, (strides, nb, lanes) in enumerate(FP_STRIDE_CHOICES):
        k = len(strides)
        cost = np.zeros((a, k))
        for dy, dx in ((0, 0), (0, 1), (1, 0), (1, 1)):
            e = (fy[:, None] + dy) * strides[None, :, None, None] + fx[:, None] + dx    # (A, K, P, 32)
            e = np.sort(e.reshape(a, k, patches, 32 // lanes, lanes), axis=-1)
            distinct = np.ones(e.shape, dtype=bool)
            distinct[..., 1:] = e[..., 1:] != e[..., :-1]
            groups = np.arange(e[..., 0].size).reshape(e.shape[:-1])
            key = (groups[..., None] * nb + np.mod(e, nb))[distinct]
            counts = np.bincount(key, minlength=groups.size * nb).reshape(*e.shape[:-1], nb)
            cost += counts.max(axis=-1).sum(axis=(-1, -2))
        out[:, col] = np.argmin(cost, axis=1)
    return out


def bp_trig(angles_deg32: NDArray) -> NDArray:
    """``(A, 2)`` float32 ``(cos, sin)`` of iradon per angle."""
    angle = np.deg2rad(np.asarray(angles_deg32, dtype=np.float32))
    return np.stack([np.cos(angle), np.sin(angle)], axis=1).astype(np.float32)


def padded_size(n: int) -> tuple[int, int]:
    """(edge, P) of ``compute_attenuation``'s zero padding (``_projector_backends.py:75-77``)."""
    min_size = np.ceil(np.sqrt(2.0 * n * n))
    edge = int(np.ceil((min_size - n) / 2))
    return edge, n + 2 * edge


def rotate_matrix(angle_deg, size: int) -> NDArray:
    """scikit-image ``rotate`` inverse map of a ``size x size`` image, as 6 float64 entries."""
    center = np.array((size, size)) / 2.0 - 0.5
    rot = np.deg2rad(angle_deg)
    c, s = math.cos(rot), math.sin(rot)
    t1 = np.array([[1.0, 0.0, center[0]], [0.0, 1.0, center[1]], [0.0, 0.0, 1.0]])
    r = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    t3 = np.array([[1.0, 0.0, -center[0]], [0.0, 1.0, -center[1]], [0.0, 0.0, 1.0]])
    m = t1 @ (r @ t3)
    return m[:2].reshape(6)


def _attenuation_pair(angle_rad, invert: bool, size: int) -> NDArray:
    if invert:
        angle_rad = angle_rad + np.pi
    deg = np.rad2deg(angle_rad)
    return np.stack([rotate_matrix(-deg, size), rotate_matrix(deg, size)])


def detector_sub_angles(surface_mm2: float, distance_mm: float, sub_sampling: int) -> NDArray:
    """Sub-angle offsets of a detector (``physics/xrf.py:243-258``, ``attenuation.py:111-114``)."""
    if surface_mm2 > 0.0:
        half_angle = np.arctan2(np.sqrt(surface_mm2) / 2, distance_mm)
        sub = np.linspace(-half_angle, half_angle, sub_sampling + 1)
        return np.convolve(sub, np.ones(2), "valid") / 2
    return np.zeros(1)


def attenuation_rotations(
    angles_rot_rad32: NDArray,
    det_angles: Sequence[float] | NDArray,
    n: int,
    surfaces_mm2: Sequence[float] | None = None,
    distances_mm: Sequence[float] | None = None,
    sub_sampling: int = 1,
) -> tuple[NDArray, NDArray, int]:
    """Rotation matrices ``rot_in (A, 2, 6)`` and ``rot_out (A, D, n_sub, 2, 6)`` (float64)."""
    _, size = padded_size(n)
    det_angles = np.array(det_angles, ndmin=1, dtype=np.float64)
    n_det = len(det_angles)
    surfaces = np.zeros(n_det) if surfaces_mm2 is None else np.array(surfaces_mm2, ndmin=1, dtype=np.float64)
    distances = np.ones(n_det) if distances_mm is None else np.array(distances_mm, ndmin=1, dtype=np.float64)
    subs = [detector_sub_angles(surfaces[d], distances[d], sub_sampling) for d in range(n_det)]
    n_sub = max(len(s) for s in subs)
    # a point detector next to finite ones has one direction: repeating it keeps one sub-angle
    # count for the kernels (the mean of identical factors is the factor, up to rounding)
    subs = [np.resize(sa, n_sub) if len(sa) == 1 else sa for sa in subs]
    if any(len(s) != n_sub for s in subs):
        raise ValueError("All detectors must use the same number of emitted sub-angles")
    angles = np.array(angles_rot_rad32, ndmin=1)
    rot_in = np.empty((len(angles), 2, 6))
    rot_out = np.empty((len(angles), n_det, n_sub, 2, 6))
    for ii, a in enumerate(angles):
        rot_in[ii] = _attenuation_pair(a, False, size)
        angle_det = a + det_angles
        for dd, ad in enumerate(angle_det):
            for kk, a_s in enumerate(subs[dd]):
                rot_out[ii, dd, kk] = _attenuation_pair(ad + a_s, True, size)
    return rot_in, rot_out, n_sub


def half_turn_pairs(angles_rot_rad32: NDArray, tol: float = 1e-6) -> NDArray | None:
    """(angle, partner) entries for the maps: partner = the angle that is ``angle + pi`` (within
    ``tol`` radians, which covers the float32 rounding of the two angles), -1 when there is none.

    Every angle appears once, as an entry's angle or as its partner.  None when no angle has a
    partner.  The maps of a partner come from its angle's rotations turned by a half turn (an
    exact permutation of the rotated lattice); the rotation angle then differs from the
    partner's own float32 angle by at most ``tol``.
    """
    a = np.mod(np.array(angles_rot_rad32, ndmin=1, dtype=np.float64), 2 * np.pi)
    order = np.argsort(a, kind="stable")
    srt = a[order]
    used = np.zeros(len(a), dtype=bool)
    entries = []
    for i in range(len(a)):
        if used[i]:
            continue
        used[i] = True
        partner = -1
        target = np.mod(a[i] + np.pi, 2 * np.pi)
        for t in (target, target - 2 * np.pi, target + 2 * np.pi):
            k = int(np.searchsorted(srt, t - tol))
            while k < len(srt) and srt[k] <= t + tol:
                j = int(order[k])
                if not used[j]:
                    partner = j
                    break
                k += 1
            if partner >= 0:
                break
        if partner >= 0:
            used[partner] = True
        entries.append((i, partner))
    if all(p < 0 for _, p in entries):
        return None
    return np.array(entries, dtype=np.int32)


def quarter_turn_quads(angles_rot_rad32: NDArray, pairs: NDArray | None, det_angle: float,
                       tol: float = 1e-6) -> NDArray | None:
    """(n_quads, 6) int32 quads of half-turn pair entries, or None when the angle set does not allow
    them.

    The emitted direction of angle a is a + det_angle + pi (``attenuation.py:108-120`` with the
    ``invert`` half turn of ``_projector_backends.py:79-80``).  When it is, within ``tol`` radians,
    the incident direction of another angle of the set, the emitted line integral of a is the
    incident one of that angle (times mu_out / mu_in).  For a detector at +-pi / 2 this closes over
    four angles, two half-turn pairs (e, e'): each row is (e, e', s0, s1, s2, s3) with the quad's
    angles k = (e's angle, e's partner, e''s angle, e''s partner) and s_k the index (0..3) of the one
    whose incident direction is angle k's emitted direction.  Every entry must have a partner and
    every entry must land in one quad; otherwise None.
    """
    if pairs is None or len(pairs) % 2 or (pairs[:, 1] < 0).any():
        return None
    a = np.mod(np.array(angles_rot_rad32, ndmin=1, dtype=np.float32).astype(np.float64), 2 * np.pi)
    entry_of = np.full(len(a), -1, dtype=np.int64)
    entry_of[pairs[:, 0]] = np.arange(len(pairs))
    entry_of[pairs[:, 1]] = np.arange(len(pairs))
    order = np.argsort(a, kind="stable")
    srt = a[order]

    def emitted(i: int) -> int:
        t = np.mod(a[i] + det_angle + np.pi, 2 * np.pi)
        for target in (t, t - 2 * np.pi, t + 2 * np.pi):
            k = int(np.searchsorted(srt, target - tol))
            if k < len(srt) and abs(srt[k] - target) <= tol:
                return int(order[k])
        return -1

    rows, used = [], np.zeros(len(pairs), dtype=bool)
    for e in range(len(pairs)):
        if used[e]:
            continue
        e2 = entry_of[emitted(int(pairs[e, 0]))] if emitted(int(pairs[e, 0])) >= 0 else -1
        if e2 < 0 or e2 == e or used[e2]:
            return None
        quad = [int(pairs[e, 0]), int(pairs[e, 1]), int(pairs[e2, 0]), int(pairs[e2, 1])]
        src = []
        for k in quad:
            m = emitted(k)
            if m not in quad:
                return None
            src.append(quad.index(m))
        used[e] = used[e2] = True
        rows.append([e, int(e2)] + src)
    return np.array(rows, dtype=np.int32)

