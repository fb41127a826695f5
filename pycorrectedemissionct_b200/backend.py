"""The B200 projector backend, with the reference's backend plug-in interface.

``ProjectorBackendB200`` follows ``ProjectorBackend`` / ``ProjectorBackendSKimage``
(``corrct``: ``src/corrct/_projector_backends.py:102-359``): ``initialize_geometry``,
``get_vol_shape``, ``get_prj_shape``, ``make_ready``, ``dispose``, ``fp(vol,
angle_ind=None)`` and ``bp(prj, angle_ind=None)``, with the scikit-image backend's
geometry (2-D slices, or 3-D volumes as stacks of independent slices; no
rotation-axis shift, no ``ProjectionGeometry``) and discretisation.  An instance can be passed as ``backend=`` to the reference's own
``ProjectorUncorrected`` / ``ProjectorAttenuationXRF`` (``projectors.py:175-186``
accept backend instances), or used through this package's projectors.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import core as _core


@dataclass
class VolumeGeometry:
    """Volume geometry subset used on this path (corrct ``models.py:421-550``)."""

    _vol_shape_xyz: np.ndarray
    vox_size: float = 1.0

    def __post_init__(self):
        self._vol_shape_xyz = np.array(self._vol_shape_xyz, ndmin=1)

    def is_square(self) -> bool:
        return self._vol_shape_xyz[0] == self._vol_shape_xyz[1]

    @property
    def shape_xyz(self) -> np.ndarray:
        return self._vol_shape_xyz

    @property
    def shape_zxy(self) -> np.ndarray:
        vol_shape_zyx = np.flip(self._vol_shape_xyz)
        return np.array([*vol_shape_zyx[:-2], vol_shape_zyx[-1], vol_shape_zyx[-2]], dtype=int)

    def is_3D(self) -> bool:
        return len(self._vol_shape_xyz) == 3 and self._vol_shape_xyz[-1] > 1


def get_vol_geom_from_volume(volume) -> VolumeGeometry:
    """Default geometry of a (.., Y, X) volume (corrct ``models.py:776-793``)."""
    shape_zxy = tuple(volume.shape)
    if len(shape_zxy) < 2:
        raise ValueError(f"The volume should be at least 2-dimensional, but the following shape was passed: {shape_zxy}")
    return VolumeGeometry(np.array([shape_zxy[-2], shape_zxy[-1], *np.flip(shape_zxy[:-2])]))


class ProjectorBackendB200:
    """sm_100a projector backend with the scikit-image backend's geometry and discretisation."""

    def __init__(self, device=None) -> None:
        self.is_initialized = False
        self.is_ready = True
        self.device = _core.require_cuda(device)

    def initialize_geometry(
        self, vol_geom, angles_rot_rad, rot_axis_shift_pix=None, prj_geom=None, create_single_projs: bool = False
    ):
        """Initialize the geometry (corrct ``_projector_backends.py:121-160, 259-299``).

        A 3-D geometry is a stack of independent slices along Z, each projected with the 2-D
        discretisation (projections ``(Z, A, n)``, the reference's V-W-U order)."""
        if rot_axis_shift_pix is not None:
            raise ValueError("With the B200 backend, rotation axis shifts are not supported!")
        if prj_geom is not None:
            raise ValueError("With the B200 backend, `ProjectionGeometry` is not supported!")
        self.vol_geom = vol_geom
        self.vol_shape_zxy = vol_geom.shape_zxy
        self.angles_w_rad = np.array(angles_rot_rad, ndmin=1, dtype=np.float32)
        self.vol_eff_shape_zxy = np.floor(self.vol_shape_zxy * vol_geom.vox_size).astype(int)
        self.prj_shape_vwu = np.array(
            [*self.vol_eff_shape_zxy[:-2], len(self.angles_w_rad), self.vol_eff_shape_zxy[-1]], dtype=int
        )
        self.prj_shape_vu = np.array([*self.vol_eff_shape_zxy[:-2], 1, self.vol_eff_shape_zxy[-1]], dtype=int)
        self.has_individual_projs = create_single_projs
        self.angles_w_deg = np.rad2deg(self.angles_w_rad)
        n = int(self.vol_shape_zxy[-1])
        if int(self.vol_shape_zxy[-2]) != n:
            raise ValueError("With the B200 backend, only square slices are allowed!")
        self.n_slices = int(np.prod(self.vol_shape_zxy[:-2])) if len(self.vol_shape_zxy) > 2 else 1
        self.core = _core.XrfCore(n, self.angles_w_rad, n_det=1, device=self.device)
        self.is_initialized = True

    def get_vol_shape(self) -> np.ndarray:
        return self.vol_shape_zxy

    def get_prj_shape(self) -> np.ndarray:
        return self.prj_shape_vwu

    def make_ready(self) -> None:
        self.is_ready = True

    def dispose(self) -> None:
        self.is_ready = False

    def __repr__(self) -> str:
        name = f"{self.__class__.__name__}: "
        if self.is_initialized:
            return name + "{\n" + f"  Shape vol ZXY: {self.get_vol_shape()}\n  Shape prj VWU: {self.get_prj_shape()}\n}}"
        return name + "{ Not initialized! }"

    def _in(self, x):
        if isinstance(x, torch.Tensor):
            if x.device.type != "cuda":
                raise ValueError("torch inputs must live on a CUDA device")
            return x.to(device=self.device, dtype=torch.float32).contiguous(), False
        return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(self.device), True

    def fp(self, vol, angle_ind: int | None = None):
        """Forward projection of the whole sinogram or one line (corrct ``_projector_backends.py:312-333``).

        Shapes: (n, n) -> (A, n) or (n,); a stack (Z, n, n) -> (Z, A, n) or (Z, n)."""
        v, as_np = self._in(vol)
        n = self.core.n
        z = self.n_slices
        v = v.reshape(z, n, n)
        d = self.core.n_det
        self.core.n_det = 1
        try:
            if angle_ind is None:
                out = self.core.fp(v)[:, 0]
            else:
                a = int(angle_ind)
                out = self.core.fp(v, angles=slice(a, a + 1))[:, 0, 0]
        finally:
            self.core.n_det = d
        if z == 1 and len(self.vol_shape_zxy) == 2:
            out = out[0]
        return out.cpu().numpy() if as_np else out

    def bp(self, prj, angle_ind: int | None = None):
        """Back projection of the whole sinogram or one line (corrct ``_projector_backends.py:335-359``).

        Shapes: (A, n) or (n,) -> (n, n); a stack (Z, A, n) or (Z, n) -> (Z, n, n)."""
        y, as_np = self._in(prj)
        n = self.core.n
        z = self.n_slices
        d = self.core.n_det
        self.core.n_det = 1
        try:
            if angle_ind is None:
                out = self.core.bp(y.reshape(z, 1, self.core.n_angles, n), "reference")
            else:
                a = int(angle_ind)
                out = self.core.bp(y.reshape(z, 1, 1, n), "reference", angles=slice(a, a + 1))
        finally:
            self.core.n_det = d
        if z == 1 and len(self.vol_shape_zxy) == 2:
            out = out[0]
        return out.cpu().numpy() if as_np else out
