"""Projectors with the reference's interface whose fp / bp run as fused sm_100a kernels.

Mirrors ``corrct``: ``src/corrct/projectors.py`` — ``ProjectorUncorrected``
(``:103-341``) and ``ProjectorAttenuationXRF`` (``:344-622``) keep their constructor
arguments, ``fp`` / ``bp`` / ``fp_angle`` / ``bp_angle``, the context manager and
``collapse_detectors``.  The attenuation multiply, the detector and angle weights
and the rotate-and-sum are one kernel (``cct_fp``); the back projection is
``cct_bp`` in the reference's discretisation (or the exact adjoint with
``bp_mode="adjoint"``).

Arrays: numpy inputs are copied to the device and results come back as numpy
arrays (the reference's behaviour); CUDA tensors stay on the device and results
are CUDA tensors.  There is no CPU computation path.
"""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np
import torch

from . import core as _core
from .attenuation import AttenuationVolume
from .backend import ProjectorBackendB200, VolumeGeometry
from .operators import ProjectorOperator

_BACKEND_NAMES = ("b200", "cuda", "astra", "skimage")


def _to_device(x, device: torch.device) -> tuple[torch.Tensor, bool]:
    """(float32 contiguous CUDA tensor, input-was-numpy)."""
    if isinstance(x, torch.Tensor):
        if x.device.type != "cuda":
            raise ValueError("torch inputs must live on a CUDA device")
        return x.to(device=device, dtype=torch.float32).contiguous(), False
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(device), True


def _out(t: torch.Tensor, as_numpy: bool, dtype=np.float32):
    return t.cpu().numpy().astype(dtype, copy=False) if as_numpy else t


class ProjectorUncorrected(ProjectorOperator):
    """Base projection class (corrct ``projectors.py:103-341``)."""

    def __init__(
        self,
        vol_geom,
        angles_rot_rad,
        rot_axis_shift_pix=None,
        *,
        prj_geom=None,
        prj_intensities=None,
        psf=None,
        backend="b200",
        create_single_projs: bool = False,
    ):
        if not isinstance(vol_geom, VolumeGeometry):
            vol_geom = VolumeGeometry(_vol_shape_xyz=np.array(vol_geom))
        self.vol_geom = vol_geom
        self.prj_geom = prj_geom
        if len(self.vol_geom.shape_xyz) not in (2, 3):
            raise ValueError(f"Only 2D or 3D volumes are valid, following volume geometry passed instead: {self.vol_geom}")
        if not self.vol_geom.is_square():
            raise ValueError(f"Only square volumes are valid, following volume geometry passed instead: {self.vol_geom}")
        if isinstance(backend, str):
            if backend.lower() not in _BACKEND_NAMES:
                raise ValueError(f"Unknown backend: {backend}. Available options are: {', '.join(_BACKEND_NAMES)}.")
            self.projector_backend = ProjectorBackendB200()
        elif isinstance(backend, ProjectorBackendB200):
            self.projector_backend = backend
        else:
            raise ValueError("backend must be a backend name or a ProjectorBackendB200 instance")
        self.projector_backend.initialize_geometry(
            vol_geom=vol_geom,
            angles_rot_rad=angles_rot_rad,
            rot_axis_shift_pix=rot_axis_shift_pix,
            prj_geom=prj_geom,
            create_single_projs=create_single_projs,
        )
        if prj_intensities is not None:
            prj_intensities = np.array(prj_intensities, dtype=np.float64)
        self.prj_intensities = prj_intensities
        self.projector_backend.core.set_intensities(prj_intensities)
        self._set_psf(psf)
        self.vol_shape = np.array(self.projector_backend.get_vol_shape(), ndmin=1)
        self.prj_shape = np.array(self.projector_backend.get_prj_shape(), ndmin=1)
        super().__init__()

    def _set_psf(self, psf) -> None:
        """Detector PSF along u (corrct ``projectors.py:229-244``); 2-D volumes take a 1-D PSF."""
        if psf is not None:
            psf = np.squeeze(np.array(psf, dtype=np.float64))
            if psf.ndim >= len(self.vol_geom.shape_xyz):
                raise ValueError(
                    "PSF should either be 1D (for 2D and 3D reconstructions) or 2D (for 3D reconstructions)."
                    + f" Passed PSF has shape: {psf.shape}, and the reconstruction is {len(self.vol_geom.shape_xyz)}D."
                )
            psf = np.atleast_1d(psf)
            if psf.ndim > 1:
                raise NotImplementedError("the B200 projectors apply 1-D PSFs (along the detector) only")
        self.psf = psf
        self.projector_backend.core.set_psf(psf)

    @property
    def angles_rot_rad(self) -> np.ndarray:
        return self.projector_backend.angles_w_rad

    @property
    def core(self) -> _core.XrfCore:
        return self.projector_backend.core

    def __enter__(self):
        self.projector_backend.make_ready()
        return self

    def __exit__(self, *args):
        self.projector_backend.dispose()

    def fp_angle(self, vol, angle_ind: int):
        return self.projector_backend.fp(vol, angle_ind)

    def bp_angle(self, prj_vu, angle_ind: int):
        return self.projector_backend.bp(prj_vu, angle_ind)

    def fp(self, vol):
        return self.projector_backend.fp(vol)

    def bp(self, prj_vwu):
        return self.projector_backend.bp(prj_vwu)


class ProjectorAttenuationXRF(ProjectorUncorrected):
    """Attenuation corrected XRF projector with multi-detector support (corrct ``projectors.py:344-622``).

    Extra keywords (no reference counterpart): ``maps_dtype`` ("float32" | "bfloat16")
    for the device copy of the maps, and ``bp_mode`` ("reference" | "adjoint") to
    select the iradon discretisation or the exact transpose of ``fp``.
    """

    def __init__(
        self,
        vol_geom,
        angles_rot_rad,
        rot_axis_shift_pix=None,
        *,
        prj_geom=None,
        prj_intensities=None,
        backend="b200",
        att_maps=None,
        att_in=None,
        att_out=None,
        angles_detectors_rad=(np.pi / 2),
        weights_detectors=None,
        psf=None,
        is_symmetric: bool = False,
        weights_angles=None,
        use_multithreading: bool = True,
        data_type=np.float32,
        verbose: bool = True,
        maps_dtype: str = "float32",
        bp_mode: str = "reference",
    ):
        ProjectorUncorrected.__init__(
            self,
            vol_geom=vol_geom,
            angles_rot_rad=angles_rot_rad,
            rot_axis_shift_pix=rot_axis_shift_pix,
            prj_geom=prj_geom,
            psf=psf,
            prj_intensities=prj_intensities,
            backend=backend,
            create_single_projs=True,
        )
        if bp_mode not in ("reference", "adjoint"):
            raise ValueError("bp_mode must be 'reference' or 'adjoint'")
        self.data_type = data_type
        self.use_multithreading = use_multithreading
        self.verbose = verbose
        self.is_symmetric = is_symmetric
        self.bp_mode = bp_mode
        self.maps_dtype = maps_dtype

        self.angles_det_rad = np.array(angles_detectors_rad, ndmin=1)
        num_det_angles = len(self.angles_det_rad)
        if weights_detectors is None:
            weights_detectors = np.ones_like(self.angles_det_rad)
        self.weights_det = np.array(weights_detectors, ndmin=1)
        num_det_weights = len(self.weights_det)
        if num_det_angles > 1:
            if num_det_weights == 1:
                self.weights_det = np.tile(self.weights_det, [num_det_angles])
            elif num_det_weights > 1 and not num_det_weights == num_det_angles:
                raise ValueError(
                    "Number of detector weights differs from number of"
                    f" detector angles: {num_det_weights} vs {num_det_angles}"
                )
        if weights_angles is None:
            weights_angles = np.ones((len(self.angles_rot_rad), num_det_angles))
        else:
            weights_angles = np.array(weights_angles)
        self.weights_angles = weights_angles

        device = self.projector_backend.device
        if att_maps is None:
            m = AttenuationVolume(att_in, att_out, self.angles_rot_rad, self.angles_det_rad, maps_dtype=maps_dtype, device=device)
            m.compute_maps(use_multithreading=self.use_multithreading, verbose=self.verbose)
            maps_dev = m.maps_device
            if maps_dev.shape[0] != self._n_slices():
                raise ValueError(
                    f"Attenuation volumes of {maps_dev.shape[0]} slices do not match the volume's {self._n_slices()}"
                )
        else:
            if att_maps.shape[1] != num_det_angles:
                raise ValueError(f"Number of maps ({att_maps.shape[1]}) differs from number of detectors ({num_det_angles})")
            if not np.all(np.equal(att_maps.shape[-2:], self.vol_shape[-2:])):
                raise ValueError(
                    f"Mismatching volume shape of input volume ({att_maps.shape[-2:]})"
                    + f" with vol_shape ({self.vol_shape} in 2D -> {self.vol_shape[-2:]})"
                )
            maps_dev = self._maps_to_device(att_maps)
        self._maps = maps_dev  # (Z, A, D, n, n)
        self._maps_host = None
        self._sync_weights()
        self.executor = None

    # ----------------------------------------------------------------------------- state
    def _sync_weights(self) -> None:
        w = np.asarray(self.weights_det, dtype=np.float64)[None, :] * np.asarray(self.weights_angles, dtype=np.float64)
        self.core.n_det = len(self.angles_det_rad)
        self.core.set_weights(w)  # intensities (set at construction) are folded in by the core

    def _is_3d(self) -> bool:
        return len(self.vol_shape) == 3

    def _n_slices(self) -> int:
        return self.projector_backend.n_slices

    def _maps_to_device(self, maps) -> torch.Tensor:
        """Reference layout ``(A, D, [Z,] n, n)`` -> device layout ``(Z, A, D, n, n)``."""
        tdt = _core.MAPS_DTYPES[self.maps_dtype][0]
        src = maps if isinstance(maps, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(maps))
        src = src.to(device=self.projector_backend.device)
        if self._is_3d():
            if src.dim() != 5 or src.shape[2] != self._n_slices():
                raise ValueError(f"3-D maps must have shape (A, D, {self._n_slices()}, n, n), got {tuple(src.shape)}")
            src = src.permute(2, 0, 1, 3, 4)
        else:
            src = src.reshape(1, *src.shape[-4:])
        return src.to(dtype=tdt).contiguous()

    @property
    def att_vol_angles(self) -> np.ndarray:
        """Host copy of the maps ``(A, D, n, n)``, or ``(A, D, Z, n, n)`` for a 3-D volume (the reference attribute)."""
        if self._maps_host is None:
            m = self._maps.float()
            m = m.permute(1, 2, 0, 3, 4) if self._is_3d() else m[0]
            self._maps_host = m.cpu().numpy()
        return self._maps_host

    @att_vol_angles.setter
    def att_vol_angles(self, maps) -> None:
        self._maps = self._maps_to_device(maps)
        self._maps_host = None

    @property
    def maps_device(self) -> torch.Tensor:
        """Device maps ``(Z, A, D, n, n)`` as consumed by the kernels (Z = 1 for a 2-D volume)."""
        return self._maps

    def __enter__(self):
        return super().__enter__()

    def __exit__(self, *args):
        super().__exit__()

    def collapse_detectors(self) -> None:
        """Convert multi-detector configurations into single-detector (corrct ``projectors.py:492-500``)."""
        weights = np.reshape(self.weights_det, [1, -1, 1, 1]) / np.sum(self.weights_det)
        wt = torch.from_numpy(weights.astype(np.float32)).to(self._maps.device)
        collapsed = torch.sum(self._maps.float() * wt[None], dim=2, keepdim=True)
        self._maps = collapsed.to(self._maps.dtype).contiguous()
        self._maps_host = None
        weights = np.squeeze(weights)
        self.angles_det_rad = np.sum(self.angles_det_rad * weights, keepdims=True)
        self.weights_angles = np.sum(self.weights_angles * weights, axis=1, keepdims=True)
        self.weights_det = np.sum(self.weights_det, keepdims=True)
        self._sync_weights()

    # ------------------------------------------------------------------------ projections
    def _n_det(self) -> int:
        return len(self.angles_det_rad)

    def _from_device_sino(self, sino: torch.Tensor) -> torch.Tensor:
        """Device (Z, D, A', n) -> the reference's (D, [Z,] A', n) with a size-1 D dropped."""
        sino = sino.permute(1, 0, 2, 3) if self._is_3d() else sino[0]
        if sino.shape[0] == 1:
            sino = sino[0]
        return sino

    def _to_device_sino(self, y: torch.Tensor, n_lines: int) -> torch.Tensor:
        """The reference's (D, [Z,] A', n) (a size-1 D may be absent) -> device (Z, D, A', n)."""
        n = int(self.vol_shape[-1])
        z = self._n_slices()
        if self._is_3d():
            return y.reshape(self._n_det(), z, n_lines, n).permute(1, 0, 2, 3).contiguous()
        return y.reshape(1, self._n_det(), n_lines, n).contiguous()

    def fp(self, vol):
        """Attenuated forward projection (corrct ``projectors.py:570-596``).

        (n, n) -> (D, A, n); a 3-D volume (Z, n, n) -> (D, Z, A, n); D = 1 is squeezed, as is a
        leading axis of size 1 after that."""
        dev = self.projector_backend.device
        v, as_np = _to_device(vol, dev)
        n = int(self.vol_shape[-1])
        sino = self._from_device_sino(self.core.fp(v.reshape(self._n_slices(), n, n), self._maps))
        if sino.shape[0] == 1:
            sino = sino[0]
        return _out(sino, as_np, self.data_type)

    def bp(self, sino):
        """Back projection (corrct ``projectors.py:598-622``)."""
        dev = self.projector_backend.device
        y, as_np = _to_device(sino, dev)
        y = self._to_device_sino(y, len(self.angles_rot_rad))
        if self.bp_mode == "adjoint":
            vol = self.core.bp(y, "adjoint", self._maps)
        elif self.is_symmetric:
            vol = self.core.bp(y, "symmetric", self._maps)
        else:
            vol = self.core.bp(y, "reference")
        return _out(vol if self._is_3d() else vol[0], as_np, self.data_type)

    def fp_angle(self, vol, angle_ind: int):
        """Forward-project one angle (corrct ``projectors.py:502-531``): (D, [Z,] n), D = 1 squeezed."""
        dev = self.projector_backend.device
        v, as_np = _to_device(vol, dev)
        a = int(angle_ind)
        n = int(self.vol_shape[-1])
        sino = self.core.fp(v.reshape(self._n_slices(), n, n), self._maps[:, a : a + 1], angles=slice(a, a + 1))
        sino = self._from_device_sino(sino[:, :, :1])
        sino = sino[..., 0, :]
        return _out(sino, as_np, self.data_type)

    def bp_angle(self, sino, angle_ind: int, single_line: bool = False):
        """Back-project one angle (corrct ``projectors.py:533-568``)."""
        dev = self.projector_backend.device
        y, as_np = _to_device(sino, dev)
        a = int(angle_ind)
        if not single_line:
            y = y[..., a, :]
        y = self._to_device_sino(y, 1)
        if self.is_symmetric:
            vol = self.core.bp(y, "symmetric", self._maps[:, a : a + 1], angles=slice(a, a + 1))
        else:
            # weights (w_det * w_angle * intensity) apply per line even without maps
            # (projectors.py:553-557, 296-297): scale, then the plain bp without the line scale
            w = self.core.weights[a] if self.core.weights is not None else None
            if w is not None:
                y = y * w.reshape(1, -1, 1, 1)
            saved = self.core.line_scale
            self.core.line_scale = None
            try:
                vol = self.core.bp(y.contiguous(), "reference", angles=slice(a, a + 1))
            finally:
                self.core.line_scale = saved
        return _out(vol if self._is_3d() else vol[0], as_np, self.data_type)
