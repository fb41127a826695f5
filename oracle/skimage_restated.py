"""Restatement of the scikit-image primitives used by the reference's projection path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference calls three scikit-image functions on this path:

* ``skimage.transform.radon(vol, [deg])`` — forward projection of one angle
  (``src/corrct/_projector_backends.py:327-333``);
* ``skimage.transform.iradon(line[:, None], [deg], circle=False,
  output_size=N, filter_name=None)`` — unfiltered back projection of one
  sinogram line (``src/corrct/_projector_backends.py:350-358``);
* ``skimage.transform.rotate(img, deg, order=1, clip=False)`` — the two
  rotations inside ``compute_attenuation``
  (``src/corrct/_projector_backends.py:67-73``).

scikit-image is a third-party dependency of the reference (not vendored, no
pinned version; ``requirements.txt`` lists ``scikit-image[data]``) and is not
installed here.  The functions below restate its published algorithm:

``_warp_affine``
    scikit-image's ``warp`` fast path for a 3x3 affine matrix on a 2-D image
    (``_warp_fast``): for every output pixel (row ``r``, col ``c``) the input
    position is ``col_in = M00*c + M01*r + M02``, ``row_in = M10*c + M11*r +
    M12`` computed in the image's floating dtype (the matrix is first cast to
    that dtype), then sampled with bilinear interpolation where each of the
    four taps that falls outside the image reads ``cval = 0`` (scikit-image's
    ``get_pixel2d`` in constant mode; ``floor``/``ceil`` pick the taps, so an
    integral coordinate uses one tap with weight 1).
``radon``
    ``circle=True`` on a square image: centre ``C = N // 2``; per angle the
    float32 degrees are converted with ``np.deg2rad`` (float32), ``cos`` and
    ``sin`` are evaluated in float32, and the matrix
    ``[[c, s, -C(c+s-1)], [-s, c, -C(c-s-1)]]`` is built from those float32
    values; the rotated image is summed over rows.
``iradon`` (``filter_name=None``)
    the unit filter's FFT round trip is the identity up to round-off and is
    omitted; each output pixel ``(i, j)`` receives ``np.interp(t, k - K, line,
    left=0, right=0)`` with ``t = (j - R) cos - (i - R) sin``, ``R =
    output_size // 2`` and ``K = len(line) // 2``; the result is scaled by
    ``pi / (2 * n_angles)``.
``rotate``
    rotation about ``((cols - 1) / 2, (rows - 1) / 2)``; the angle goes through
    ``np.deg2rad`` (keeping its numpy dtype) and ``math.cos`` / ``math.sin``
    (double precision), and the matrix ``T(+c) R T(-c)`` is composed in float64
    before ``_warp_affine``.

All arithmetic follows the input dtype, so a float64 input reproduces the
FP64 oracle and a float32 input reproduces the reference's default float32
run.
"""

from __future__ import annotations

import math

import numpy as np
from numpy.typing import NDArray

__all__ = ["radon", "iradon", "rotate", "warp_affine", "bilinear_zero"]


def bilinear_zero(image: NDArray, rows: NDArray, cols: NDArray) -> NDArray:
    """Bilinear samples of ``image`` at (``rows``, ``cols``); out-of-image taps read 0.

    Follows scikit-image's ``bilinear_interpolation`` with ``mode='C'``:
    taps are ``floor``/``ceil`` of each coordinate, weights ``(1-d)`` and ``d``
    with ``d = coord - floor(coord)``, evaluated in the dtype of the inputs.
    """
    dtype = image.dtype
    rows = np.asarray(rows, dtype=dtype)
    cols = np.asarray(cols, dtype=dtype)
    h, w = image.shape

    r0 = np.floor(rows)
    c0 = np.floor(cols)
    r1 = np.ceil(rows)
    c1 = np.ceil(cols)
    dr = rows - r0
    dc = cols - c0

    def tap(rr: NDArray, cc: NDArray) -> NDArray:
        ri = rr.astype(np.int64)
        ci = cc.astype(np.int64)
        ok = (ri >= 0) & (ri < h) & (ci >= 0) & (ci < w)
        out = np.zeros(rows.shape, dtype=dtype)
        out[ok] = image[ri[ok], ci[ok]]
        return out

    one = dtype.type(1)
    top = (one - dc) * tap(r0, c0) + dc * tap(r0, c1)
    bottom = (one - dc) * tap(r1, c0) + dc * tap(r1, c1)
    return (one - dr) * top + dr * bottom


def warp_affine(image: NDArray, matrix: NDArray) -> NDArray:
    """Inverse-map affine warp (output shape = input shape), restating scikit-image ``warp``."""
    dtype = image.dtype
    m = np.asarray(matrix).astype(dtype)
    h, w = image.shape
    rr, cc = np.mgrid[:h, :w]
    x = cc.astype(dtype)
    y = rr.astype(dtype)
    cols_in = m[0, 0] * x + m[0, 1] * y + m[0, 2]
    rows_in = m[1, 0] * x + m[1, 1] * y + m[1, 2]
    return bilinear_zero(image, rows_in, cols_in)


def radon_matrix(theta_deg: np.floating, n: int) -> NDArray:
    """Per-angle inverse map of scikit-image ``radon`` (``circle=True``), float32-built entries."""
    angle = np.deg2rad(np.asarray([theta_deg]))[0]
    cos_a, sin_a = np.cos(angle), np.sin(angle)
    center = n // 2
    return np.array(
        [
            [cos_a, sin_a, -center * (cos_a + sin_a - 1)],
            [-sin_a, cos_a, -center * (cos_a - sin_a - 1)],
            [0, 0, 1],
        ]
    )


def radon(image: NDArray, theta: NDArray | list, circle: bool = True) -> NDArray:
    """Restated ``skimage.transform.radon`` for square images and ``circle=True``.

    Returns an array of shape ``(N, len(theta))`` in the image dtype.
    """
    if image.ndim != 2 or image.shape[0] != image.shape[1]:
        raise ValueError("The restated radon only supports square 2-D images")
    if not circle:
        raise NotImplementedError("Only circle=True is used by the reference backend")
    theta = np.asarray(theta)
    n = image.shape[0]
    out = np.zeros((n, len(theta)), dtype=image.dtype)
    for ii, th in enumerate(theta):
        rotated = warp_affine(image, radon_matrix(th, n))
        out[:, ii] = rotated.sum(0)
    return out


def iradon_matrix_terms(theta_deg: np.floating) -> tuple[np.floating, np.floating]:
    """(cos, sin) of one iradon angle, as scikit-image evaluates them (dtype of theta)."""
    angle = np.deg2rad(np.asarray([theta_deg]))[0]
    return np.cos(angle), np.sin(angle)


def iradon(
    radon_image: NDArray,
    theta: NDArray | list,
    output_size: int | None = None,
    filter_name: str | None = "ramp",
    circle: bool = True,
) -> NDArray:
    """Restated ``skimage.transform.iradon`` for ``filter_name=None``, ``circle=False``, linear interpolation."""
    if filter_name is not None:
        raise NotImplementedError("Only filter_name=None is used by the reference backend")
    if circle:
        raise NotImplementedError("Only circle=False is used by the reference backend")
    theta = np.asarray(theta)
    if radon_image.shape[1] != len(theta):
        raise ValueError("The given ``theta`` does not match the number of projections in ``radon_image``.")
    dtype = radon_image.dtype
    img_shape = radon_image.shape[0]
    if output_size is None:
        output_size = int(np.floor(np.sqrt((img_shape) ** 2 / 2.0)))
    reconstructed = np.zeros((output_size, output_size), dtype=dtype)
    radius = output_size // 2
    xpr, ypr = np.mgrid[:output_size, :output_size] - radius
    x = np.arange(img_shape) - img_shape // 2
    for col, th in zip(radon_image.T, theta):
        cos_a, sin_a = iradon_matrix_terms(th)
        t = ypr * cos_a - xpr * sin_a
        reconstructed += np.interp(t, x, col, left=0, right=0)
    return reconstructed * np.pi / (2 * len(theta))


def rotate_matrix(angle_deg: float | np.floating, rows: int, cols: int) -> NDArray:
    """Inverse map of scikit-image ``rotate`` (``resize=False``, default centre), float64."""
    center = np.array((cols, rows)) / 2.0 - 0.5
    rot = np.deg2rad(angle_deg)
    c, s = math.cos(rot), math.sin(rot)
    t1 = np.array([[1.0, 0.0, center[0]], [0.0, 1.0, center[1]], [0.0, 0.0, 1.0]])
    r = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    t3 = np.array([[1.0, 0.0, -center[0]], [0.0, 1.0, -center[1]], [0.0, 0.0, 1.0]])
    return t1 @ (r @ t3)


def rotate(
    image: NDArray,
    angle: float | np.floating,
    resize: bool = False,
    center=None,
    order: int | None = None,
    mode: str = "constant",
    cval: float = 0,
    clip: bool = True,
    preserve_range: bool = False,
) -> NDArray:
    """Restated ``skimage.transform.rotate`` for ``order=1``, ``mode='constant'``, ``cval=0``, no resize."""
    if resize or center is not None or (order not in (None, 1)) or mode != "constant" or cval != 0:
        raise NotImplementedError("Only the reference's rotate arguments are restated")
    if clip:
        raise NotImplementedError("The reference always passes clip=False")
    if image.ndim != 2:
        raise ValueError("Only 2-D images are restated")
    rows, cols = image.shape
    return warp_affine(image, rotate_matrix(angle, rows, cols))
