"""GPU: 3-D volumes as stacks of independent slices through the reference-facing API.

The reference's own compute_attenuation treats a 3-D attenuation volume slice by slice
(``_projector_backends.py:86-92``); its scikit-image projector is 2-D only.  A 3-D volume here is
Z slices projected with the 2-D discretisation, with the reference's array layouts: maps
``(A, D, Z, n, n)``, projections ``(D, Z, A, n)`` (D = 1 squeezed), and solvers whose stopping
test uses the residual norm of the whole volume.  Checks: every slice of a stacked call equals
the 2-D call on that slice and the oracle port (1e-5 rel-L2); the joint stopping test stops at the
iteration the summed per-slice residual histories predict.
"""

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
Z, N, A = 3, 40, 12
DET = np.array([np.pi / 2, np.pi / 3])
WDET = np.array([1.0, 0.6])


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def volume():
    from pycorrectedemissionct_b200 import phantoms

    xs, mus = [], []
    for z in range(Z):
        rng = phantoms.slice_rng(4242, z)
        xs.append(phantoms.ellipse_phantom(N, rng, 8))
        mus.append(phantoms.disk_attenuation(N, rng, 0.03))
    return np.stack(xs), np.stack(mus), phantoms.angles(A)


def _projector3d(volume, cuda, **kw):
    from pycorrectedemissionct_b200 import backend, projectors

    x, mu, angles = volume
    geom = backend.get_vol_geom_from_volume(x)
    return projectors.ProjectorAttenuationXRF(
        geom, angles, att_in=mu, att_out=0.7 * mu, angles_detectors_rad=DET, weights_detectors=WDET, **kw
    )


def _projector2d(maps_z, angles, **kw):
    from pycorrectedemissionct_b200 import projectors

    return projectors.ProjectorAttenuationXRF(
        (N, N), angles, att_maps=maps_z, angles_detectors_rad=DET, weights_detectors=WDET, **kw
    )


def test_volume_maps_fp_bp_equal_slices(volume, cuda):
    from oracle import port

    x, mu, angles = volume
    p3 = _projector3d(volume, cuda)
    maps = p3.att_vol_angles
    assert maps.shape == (A, len(DET), Z, N, N)
    rad32, deg32 = port.backend_angles(angles)
    sino = p3.fp(x)
    assert sino.shape == (len(DET), Z, A, N)
    y = np.random.default_rng(7).uniform(size=sino.shape).astype(np.float32)
    bp3 = p3.bp(y)
    assert bp3.shape == (Z, N, N)
    for z in range(Z):
        ref_maps = port.compute_maps(mu[z].astype(np.float64), 0.7 * mu[z].astype(np.float64), rad32, DET)
        assert rel_l2(maps[:, :, z], ref_maps) < TOL
        p2 = _projector2d(maps[:, :, z], angles)
        np.testing.assert_allclose(sino[:, z], p2.fp(x[z]), rtol=0, atol=1e-6 * float(np.abs(sino).max()))
        ref = port.fp_xrf(x[z].astype(np.float64), ref_maps, deg32, weights_det=WDET)
        assert rel_l2(sino[:, z], ref) < TOL
        np.testing.assert_allclose(bp3[z], p2.bp(y[:, z]), rtol=0, atol=1e-6 * float(np.abs(bp3).max()))
        assert rel_l2(bp3[z], port.bp_xrf(y[:, z].astype(np.float64), ref_maps, deg32, weights_det=WDET)) < TOL


def test_volume_single_angle_calls(volume, cuda):
    x, _, angles = volume
    p3 = _projector3d(volume, cuda, is_symmetric=True)
    maps = p3.att_vol_angles
    a = 5
    line = p3.fp_angle(x, a)
    assert line.shape == (len(DET), Z, N)
    np.testing.assert_allclose(line, p3.fp(x)[:, :, a], rtol=0, atol=1e-6 * float(np.abs(line).max()))
    y = np.random.default_rng(3).uniform(size=(len(DET), Z, A, N)).astype(np.float32)
    vol = p3.bp_angle(y, a)
    assert vol.shape == (Z, N, N)
    for z in range(Z):
        p2 = _projector2d(maps[:, :, z], angles, is_symmetric=True)
        np.testing.assert_allclose(vol[z], p2.bp_angle(y[:, z], a), rtol=0, atol=1e-6 * float(np.abs(vol).max()))


def test_volume_uncorrected_backend(volume, cuda):
    from oracle import port
    from pycorrectedemissionct_b200 import backend, projectors

    x, _, angles = volume
    _, deg32 = port.backend_angles(angles)
    p = projectors.ProjectorUncorrected(backend.get_vol_geom_from_volume(x), angles)
    sino = p.fp(x)
    assert sino.shape == (Z, A, N)
    assert p.bp(sino).shape == (Z, N, N)
    for z in range(Z):
        assert rel_l2(sino[z], port.fp_uncorrected(x[z].astype(np.float64), deg32)) < TOL
    assert p.fp_angle(x, 3).shape == (Z, N)


def _data(p3, x, seed=11):
    clean = p3.fp(x)
    rng = np.random.default_rng(seed)
    return rng.poisson(clean / clean.max() * 500.0).astype(np.float32)


def test_volume_mlem_equals_slices_and_joint_stop(volume, cuda):
    from pycorrectedemissionct_b200 import solvers

    x, _, angles = volume
    p3 = _projector3d(volume, cuda)
    maps = p3.att_vol_angles
    b = _data(p3, x)
    iters = 24
    x3, info3 = solvers.MLEM()(p3, b, iterations=iters)
    assert x3.shape == (Z, N, N) and info3.iterations == iters
    hist = np.zeros(iters)
    x2s = []
    for z in range(Z):
        p2 = _projector2d(maps[:, :, z], angles)
        x2, info2 = solvers.MLEM()(p2, b[:, z], iterations=iters)
        np.testing.assert_allclose(x3[z], x2, rtol=0, atol=1e-5 * float(np.abs(x2).max()))
        hist += info2.residuals[:iters]
        x2s.append(x2)
    np.testing.assert_allclose(info3.residuals[:iters], hist, rtol=1e-9)
    # joint stop: the first iteration k (0-based) with tol > sum_z residual_z[k]
    k = 15
    tol = 0.5 * (hist[k - 1] + hist[k])
    assert np.all(np.diff(hist[: k + 1]) < 0)
    xt, infot = solvers.MLEM(tolerance=tol)(p3, b, iterations=iters)
    assert infot.iterations == k + 1
    for z in range(Z):
        p2 = _projector2d(maps[:, :, z], angles)
        x2, _ = solvers.MLEM()(p2, b[:, z], iterations=k)
        np.testing.assert_allclose(xt[z], x2, rtol=0, atol=1e-5 * float(np.abs(x2).max()))


def test_volume_sirt_mask_per_slice(volume, cuda):
    from pycorrectedemissionct_b200 import solvers

    x, _, angles = volume
    p3 = _projector3d(volume, cuda)
    maps = p3.att_vol_angles
    b = _data(p3, x, seed=5)
    yy, xx = np.mgrid[:N, :N]
    masks = np.stack([((yy - N / 2) ** 2 + (xx - N / 2) ** 2 < (N / 2 - 2 * z) ** 2) for z in range(Z)]).astype(np.float32)
    x3, _ = solvers.SIRT()(p3, b, iterations=12, x_mask=masks, lower_limit=0.0)
    for z in range(Z):
        p2 = _projector2d(maps[:, :, z], angles)
        x2, _ = solvers.SIRT()(p2, b[:, z], iterations=12, x_mask=masks[z], lower_limit=0.0)
        # the volume's diagonal scaling uses maxima over the whole volume (equal here up to the mask)
        assert rel_l2(x3[z], x2) < 1e-4


def test_volume_sart_equals_slices(volume, cuda):
    from pycorrectedemissionct_b200 import solvers

    x, _, angles = volume
    p3 = _projector3d(volume, cuda)
    p3.collapse_detectors()
    maps = p3.att_vol_angles
    np.random.seed(123)
    x3, _ = solvers.SART()(p3, p3.fp(x), iterations=2)
    assert x3.shape == (Z, N, N)
    for z in range(Z):
        p2 = projectors_2d_collapsed(maps[:, :, z], angles, p3)
        np.random.seed(123)
        x2, _ = solvers.SART()(p2, p2.fp(x[z]), iterations=2)
        assert rel_l2(x3[z], x2) < 1e-4


def projectors_2d_collapsed(maps_z, angles, p3):
    from pycorrectedemissionct_b200 import projectors

    return projectors.ProjectorAttenuationXRF(
        (N, N), angles, att_maps=maps_z, angles_detectors_rad=p3.angles_det_rad, weights_detectors=p3.weights_det,
        weights_angles=p3.weights_angles,
    )
