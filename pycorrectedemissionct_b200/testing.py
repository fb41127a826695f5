"""Synthetic data generation on the device, with the reference's interface.

Mirrors ``corrct``: ``src/corrct/testing.py`` — ``add_noise`` (``:266-320``) and
``create_sino`` (``:323-409``).  The projection runs on this package's projectors and the noise
(photon scaling, absolute-Gaussian background, Poisson counts, Gaussian read-out noise) in one
kernel (``cct_add_noise``), so a sinogram never leaves HBM between the two.

Random numbers: a counter-based generator keyed by ``seed``; the same seed gives the same data
on any GPU and launch.  ``seed=None`` draws the seed from numpy's global generator, so
``np.random.seed`` makes runs reproducible as it does for the reference.  The draws differ from
numpy's, so the data agree with the reference's in distribution, not value for value.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import numpy as np
import torch

from . import _lib
from . import core as _core


def _seed(seed) -> int:
    if seed is None:
        return int(np.random.randint(0, 2**63 - 1, dtype=np.int64))
    return int(seed) & (2**64 - 1)


def add_noise(
    img_clean,
    num_photons: int | float,
    add_poisson: bool = False,
    readout_noise_std: float | None = None,
    background_avg: float | None = None,
    background_std: float | None = None,
    detection_efficiency: float = 1.0,
    dtype=np.float32,
    seed: int | None = None,
):
    """Add noise to an image (sinogram) (corrct ``testing.py:266-320``).

    Returns ``(img_noise, img_clean, background)``: the noisy and clean images scaled by the
    photons and the efficiency, and the mean background.  numpy in -> numpy out; a CUDA tensor
    stays on its device.
    """
    if np.dtype(dtype) != np.float32:
        raise NotImplementedError("the device noise model computes in float32")
    as_np = not isinstance(img_clean, torch.Tensor)
    if as_np:
        dev = _core.require_cuda()
        src = torch.from_numpy(np.ascontiguousarray(img_clean, dtype=np.float32)).to(dev)
    else:
        dev = _core.require_cuda(img_clean.device)
        src = img_clean.to(dtype=torch.float32).contiguous()
    desc = _lib.NoiseDesc()
    desc.num_photons = float(num_photons)
    desc.detection_efficiency = float(detection_efficiency)
    desc.add_poisson = int(bool(add_poisson))
    desc.has_background = int(background_avg is not None)
    if background_avg is not None:
        desc.background_avg = float(background_avg)
        desc.background_std = float(background_avg * 5e-2 if background_std is None else background_std)
    desc.has_readout = int(readout_noise_std is not None)
    if readout_noise_std is not None:
        desc.readout_std = float(readout_noise_std)
    desc.seed = _seed(seed)

    lib = _lib.load()
    count = ctypes.c_int64(0)
    _lib.check(lib.cct_noise_partials_count(ctypes.byref(count)))
    noisy = torch.empty_like(src)
    clean = torch.empty_like(src)
    partials = torch.empty(count.value, dtype=torch.float64, device=dev)
    background = torch.empty(1, dtype=torch.float64, device=dev)
    flags = torch.zeros(2, dtype=torch.int32, device=dev)
    _lib.check(
        lib.cct_add_noise(
            ctypes.byref(desc), src.data_ptr(), src.numel(), noisy.data_ptr(), clean.data_ptr(), partials.data_ptr(),
            background.data_ptr(), flags.data_ptr(), _core.stream_handle(dev),
        )
    )
    fl = flags.cpu().numpy()
    if fl[0]:
        raise ValueError("lam < 0 or lam is NaN or too large: the Poisson mean must be finite and non-negative")
    if fl[1]:
        raise RuntimeError("a Poisson draw reached its iteration bound")
    bg = float(background.item())
    if as_np:
        return noisy.cpu().numpy(), clean.cpu().numpy(), bg
    return noisy, clean, bg


def create_sino(
    ph,
    num_angles: int,
    start_angle_deg: float = 0.0,
    end_angle_deg: float = 180.0,
    dwell_time_s: float = 1.0,
    photon_flux: float = 1e9,
    detectors_pos_rad: float | Sequence[float] | np.ndarray = (np.pi / 2),
    vol_att_in=None,
    vol_att_out=None,
    psf=None,
    background_avg: float | None = None,
    background_std: float | None = None,
    add_poisson: bool = False,
    readout_noise_std: float | None = None,
    dtype=np.float32,
    seed: int | None = None,
    verbose: bool = True,
):
    """Compute the sinogram of a phantom (corrct ``testing.py:323-409``).

    Returns ``(sino_noise, angles_rad, expected_production, background)`` with the expected
    photon production per voxel ``ph * num_photons * detector_solid_angle``.
    """
    from . import projectors

    if verbose:
        print(f"Creating Sino with {num_angles} angles")
    angles_deg = np.linspace(start_angle_deg, end_angle_deg, num_angles, endpoint=False)
    angles_rad = np.deg2rad(angles_deg)
    if verbose:
        print(angles_deg)

    num_photons = photon_flux * dwell_time_s
    detector_solidangle_sr = (2.4 / 2 / 16 / 2) ** 2

    as_np = not isinstance(ph, torch.Tensor)
    dev = _core.require_cuda(None if as_np else ph.device)
    ph_dev = torch.from_numpy(np.ascontiguousarray(ph, dtype=np.float32)).to(dev) if as_np else ph
    shape = tuple(ph_dev.shape)
    if vol_att_in is None and vol_att_out is None:
        with projectors.ProjectorUncorrected(shape, angles_rad) as p:
            sino = p.fp(ph_dev)
    else:
        with projectors.ProjectorAttenuationXRF(
            shape, angles_rad, att_in=vol_att_in, att_out=vol_att_out, angles_detectors_rad=detectors_pos_rad, psf=psf,
            verbose=verbose,
        ) as p:
            sino = p.fp(ph_dev)

    sino_noise, sino, background = add_noise(
        sino,
        num_photons=num_photons,
        add_poisson=add_poisson,
        readout_noise_std=readout_noise_std,
        background_avg=background_avg,
        background_std=background_std,
        detection_efficiency=detector_solidangle_sr,
        dtype=dtype,
        seed=seed,
    )
    expected = ph * num_photons * detector_solidangle_sr
    if as_np:
        sino_noise = sino_noise.cpu().numpy()
    return sino_noise, angles_rad, expected, background
