"""Attenuation maps with the reference's ``AttenuationVolume`` interface, computed on the GPU.

Mirrors ``corrct``: ``src/corrct/physics/attenuation.py:32-331`` (constructor checks,
``compute_maps``, ``get_maps``, ``get_projector_args``) and ``DetectorXRF``
(``src/corrct/physics/xrf.py:218-258``).  The maps are computed by
``cct_compute_maps`` and stay on the device (``maps_device``); ``maps`` gives the
reference's host array ``(A, D, *vol_shape)`` on demand.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass

import numpy as np
import torch

from . import core as _core
from . import geometry


@dataclass
class DetectorXRF:
    """Simple XRF detector model (corrct ``physics/xrf.py:218-258``)."""

    surface_mm2: float = 0.0
    distance_mm: float = 1.0
    angle_rad: float = np.pi / 2

    def __post_init__(self):
        if self.surface_mm2 < 0.0:
            raise ValueError(f"Surface cannot be negative, but {self.surface_mm2} was passed")
        if self.distance_mm <= 0.0:
            raise ValueError(f"The distance needs to be positive, but {self.distance_mm} was passed")

    @property
    def solid_angle_sr(self) -> float:
        return self.surface_mm2 / (4 * np.pi * self.distance_mm**2)

    @property
    def angle_range_rad(self) -> tuple[float, float]:
        half_edge = np.sqrt(self.surface_mm2) / 2
        half_angle = np.arctan2(half_edge, self.distance_mm)
        return (-half_angle, half_angle)


class AttenuationVolume:
    """Attenuation volume computation class (corrct ``physics/attenuation.py:32-331``).

    Extra keyword ``maps_dtype`` ("float32" or "bfloat16") selects the device storage
    type of the maps; ``device`` selects the CUDA device.
    """

    def __init__(
        self,
        incident_local,
        emitted_local,
        angles_rot_rad,
        angles_det_rad=np.pi / 2,
        emitted_sub_sampling: int = 1,
        dtype=np.float32,
        maps_dtype: str = "float32",
        device=None,
    ):
        self.incident_local = incident_local
        self.emitted_local = emitted_local
        self.angles_rot_rad = np.array(angles_rot_rad, ndmin=1)
        self.detectors: list[DetectorXRF] = []
        if isinstance(angles_det_rad, (int, float, DetectorXRF)):
            angles_det_rad = [angles_det_rad]
        for a in angles_det_rad:
            if isinstance(a, DetectorXRF):
                self.detectors.append(a)
            elif isinstance(a, float):
                self.detectors.append(DetectorXRF(surface_mm2=0, distance_mm=1, angle_rad=a))
            else:
                raise ValueError(
                    f"Input parameter {angles_det_rad = } should be one of: float | NDArray | Sequence[float | DetectorXRF]"
                )
        self.dtype = dtype
        self.maps_dtype = maps_dtype
        self.device = device

        if self.incident_local is not None:
            self.vol_shape_zyx = np.array(_shape(self.incident_local))
            if self.emitted_local is not None and np.any(self.vol_shape_zyx != _shape(self.emitted_local)):
                raise ValueError(
                    f"Incident volume shape ({_shape(self.incident_local)}) does not"
                    + f" match the emitted volume shape ({_shape(self.emitted_local)})"
                )
        elif self.emitted_local is not None:
            self.vol_shape_zyx = np.array(_shape(self.emitted_local))
        else:
            raise ValueError("No attenuation volumes were given.")
        self.emitted_sub_sampling = emitted_sub_sampling
        self.vol_shape_zyx = np.array(self.vol_shape_zyx, ndmin=1)
        num_dims = len(self.vol_shape_zyx)
        if num_dims not in [2, 3]:
            raise ValueError(f"Maps can only be 2D or 3D Arrays. A {num_dims}-dimensional was passed ({self.vol_shape_zyx}).")
        if self.vol_shape_zyx[-1] != self.vol_shape_zyx[-2]:
            raise ValueError(f"Only square slices are supported, got {self.vol_shape_zyx}")
        self.maps_device: torch.Tensor | None = None
        self._maps_host: np.ndarray | None = None

    def _get_detector_angles(self) -> np.ndarray:
        return np.array([det.angle_rad for det in self.detectors], ndmin=1)

    def _to_device(self, vol) -> torch.Tensor | None:
        if vol is None:
            return None
        dev = _core.require_cuda(self.device if self.device is not None else getattr(vol, "device", None))
        t = torch.as_tensor(np.asarray(vol) if not isinstance(vol, torch.Tensor) else vol)
        t = t.to(device=dev, dtype=torch.float32)
        if t.ndim == 2:
            t = t[None]
        return t.contiguous()

    def compute_maps(self, use_multithreading: bool = True, verbose: bool = True) -> None:
        """Compute the correction maps for each angle on the GPU (corrct ``attenuation.py:122-180``).

        ``use_multithreading`` and ``verbose`` are accepted for signature compatibility.
        """
        mu_in = self._to_device(self.incident_local)
        mu_out = self._to_device(self.emitted_local)
        subs = self.emitted_sub_sampling if any(d.surface_mm2 > 0 for d in self.detectors) else 1
        if self.emitted_sub_sampling > 1 and verbose:
            for ii, det in enumerate(self.detectors):
                sub = geometry.detector_sub_angles(det.surface_mm2, det.distance_mm, self.emitted_sub_sampling)
                print(f"Detector #{ii}: Super-sampling outgoing sub-angles: {np.round(np.rad2deg(sub), decimals=3)} deg")
        # equal incident and emitted attenuation (mu_out = 1 * mu_in) lets compute_maps derive the
        # emitted line integrals from the incident ones where the geometry allows it
        same = mu_in is not None and mu_out is not None and mu_in.shape == mu_out.shape and torch.equal(mu_in, mu_out)
        self.maps_device = _core.compute_maps(
            mu_in,
            mu_out,
            self.angles_rot_rad,
            self._get_detector_angles(),
            surfaces_mm2=[d.surface_mm2 for d in self.detectors],
            distances_mm=[d.distance_mm for d in self.detectors],
            sub_sampling=subs,
            maps_dtype=self.maps_dtype,
            emitted_scale=1.0 if same else None,
        )
        self._maps_host = None

    @property
    def maps(self) -> np.ndarray:
        """Host copy ``(A, D, *vol_shape)`` in ``dtype`` (the reference's ``self.maps``)."""
        if self.maps_device is None:
            raise AttributeError("maps have not been computed: call compute_maps()")
        if self._maps_host is None:
            m = self.maps_device.float()  # (Z, A, D, n, n)
            if len(self.vol_shape_zyx) == 2:
                m = m[0]
            else:
                m = m.permute(1, 2, 0, 3, 4)
            self._maps_host = m.cpu().numpy().astype(self.dtype, copy=False)
        return self._maps_host

    def get_maps(self, roi=None, rot_ind=None, det_ind=None, binning: int = 1) -> np.ndarray:
        """Return the attenuation maps (corrct ``attenuation.py:253-297``)."""
        maps = self.maps
        if rot_ind is not None:
            if isinstance(rot_ind, int):
                rot_ind = slice(rot_ind, rot_ind + 1, 1)
            maps = maps[rot_ind, ...]
        if det_ind is not None:
            if isinstance(det_ind, int):
                det_ind = slice(det_ind, det_ind + 1, 1)
            maps = maps[:, det_ind, ...]
        if roi is not None:
            raise NotImplementedError("Extracting a region of interest is not supported, yet.")
        if binning > 1:
            maps = bin_maps(maps, binning, len(self.vol_shape_zyx))
        return maps

    def get_projector_args(self, roi=None, rot_ind=None, det_ind=None, binning: int = 1) -> dict:
        """Projector arguments (corrct ``attenuation.py:299-331``)."""
        if det_ind is None:
            det_angles = self._get_detector_angles()
        else:
            det_angles = self.detectors[det_ind].angle_rad
        return dict(att_maps=self.get_maps(roi=roi, rot_ind=rot_ind, det_ind=det_ind, binning=binning), angles_detectors_rad=det_angles)


def bin_maps(maps: np.ndarray, binning, n_axes: int) -> np.ndarray:
    """Integer binning of the last ``n_axes`` axes (the volume's) of ``maps`` by block means, after
    cropping each of those axes to a multiple of ``binning`` (the excess split between both ends,
    the larger half at the start): the integer branch of corrct's ``bin_imgs(..., auto_crop=True)``
    (``processing/pre.py:180-231``) as ``get_maps`` calls it (``physics/attenuation.py:292-293``)."""
    if int(binning) != binning:
        raise NotImplementedError("Only integer binning of the maps is supported by the B200 backend.")
    binning = int(binning)
    axes = list(range(maps.ndim - n_axes, maps.ndim))
    slicing = [slice(None)] * maps.ndim
    for ax in axes:
        excess = maps.shape[ax] % binning
        if excess:
            slicing[ax] = slice(excess - excess // 2, maps.shape[ax] - excess // 2)
    maps = maps[tuple(slicing)]
    shape = []
    for ax, size in enumerate(maps.shape):
        shape += [size // binning, binning] if ax in axes else [size]
    mean_axes = tuple(i + 1 + k for k, i in enumerate(axes))
    return maps.reshape(shape).mean(axis=mean_axes, dtype=np.float64).astype(maps.dtype)


def _shape(vol) -> tuple:
    return tuple(vol.shape)
