"""Seeded synthetic inputs for the XRF projection path.

There is no public dataset on this path; the workloads are seeded synthetic
slices with the shapes and value ranges of the benchmark configurations:

* emission phantom: ``k`` ellipses with values ``U[0, 1]``, each overwriting
  the earlier ones, all inside the inscribed circle (scikit-image's ``radon``
  with ``circle=True`` assumes zero signal outside it);
* attenuation: ``d`` disks with a per-disk ``mu ~ U[0, mu_max]`` (1/pixel), zero
  elsewhere, also inside the inscribed circle;
* data: the attenuated forward projection scaled so that its maximum equals the
  peak count, then Poisson-sampled (``testing.add_noise``,
  ``src/corrct/testing.py:266-320``, with ``add_poisson=True``).

Angles follow ``np.linspace(start, end, A, endpoint=False)`` like
``testing.create_sino`` (``src/corrct/testing.py:381``).
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

__all__ = ["angles", "ellipse_phantom", "disk_attenuation", "poisson_data", "slice_rng"]


def slice_rng(base_seed: int, slice_id: int) -> np.random.Generator:
    """PCG64 generator of one slice: seed = base + slice id."""
    return np.random.default_rng(np.random.PCG64(base_seed + slice_id))


def angles(num_angles: int, start: float = 0.0, end: float = 2 * np.pi) -> NDArray:
    """Rotation angles in radians, ``endpoint=False``."""
    return np.linspace(start, end, num_angles, endpoint=False)


def _grid(n: int) -> tuple[NDArray, NDArray]:
    c = (n - 1) / 2
    yy, xx = np.mgrid[:n, :n]
    return (yy - c) / (n / 2), (xx - c) / (n / 2)


def ellipse_phantom(n: int, rng: np.random.Generator, num_ellipses: int = 12, dtype=np.float32) -> NDArray:
    """``num_ellipses`` random ellipses (values ``U[0, 1]``) inside 85 % of the inscribed circle."""
    yy, xx = _grid(n)
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(num_ellipses):
        a = rng.uniform(0.06, 0.4)
        b = rng.uniform(0.06, 0.4)
        rmax = 0.85 - max(a, b)
        rad = rng.uniform(0.0, max(rmax, 0.0))
        ang = rng.uniform(0, 2 * np.pi)
        cy, cx = rad * np.sin(ang), rad * np.cos(ang)
        phi = rng.uniform(0, np.pi)
        cp, sp = np.cos(phi), np.sin(phi)
        u = (xx - cx) * cp + (yy - cy) * sp
        v = -(xx - cx) * sp + (yy - cy) * cp
        inside = (u / a) ** 2 + (v / b) ** 2 <= 1.0
        img[inside] = rng.uniform(0.0, 1.0)
    img[(xx**2 + yy**2) > 0.9**2] = 0
    return img.astype(dtype)


def disk_attenuation(n: int, rng: np.random.Generator, mu_max: float, num_disks: int = 5, dtype=np.float32) -> NDArray:
    """``num_disks`` random disks with ``mu ~ U[0, mu_max]`` inside 85 % of the inscribed circle."""
    yy, xx = _grid(n)
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(num_disks):
        r = rng.uniform(0.1, 0.45)
        rad = rng.uniform(0.0, max(0.85 - r, 0.0))
        ang = rng.uniform(0, 2 * np.pi)
        cy, cx = rad * np.sin(ang), rad * np.cos(ang)
        inside = (xx - cx) ** 2 + (yy - cy) ** 2 <= r * r
        img[inside] = rng.uniform(0.0, mu_max)
    return img.astype(dtype)


def poisson_data(sino_clean: NDArray, peak_counts: float, rng: np.random.Generator, dtype=np.float32) -> NDArray:
    """Scale to ``max == peak_counts`` and draw Poisson counts."""
    scale = peak_counts / max(float(np.max(sino_clean)), 1e-30)
    return rng.poisson(np.clip(sino_clean, 0, None) * scale).astype(dtype)
