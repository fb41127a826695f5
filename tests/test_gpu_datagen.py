"""GPU: synthetic data generation (corrct testing.add_noise / create_sino) on the device.

The deterministic parts (photon scaling, the projection) match the oracle port exactly or to
1e-5 rel-L2; the random parts use a different generator than numpy's, so they are checked in
distribution against the model the reference samples from and against the port's own draws:
Poisson means and variances within 5 standard errors, a chi-square goodness of fit of the
counts for small means, the absolute-Gaussian background and Gaussian read-out moments, and
seed reproducibility.
"""

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def test_scaling_is_exact(cuda):
    from oracle import port
    from pycorrectedemissionct_b200 import testing

    clean = np.random.default_rng(1).uniform(0, 3, size=(33, 70)).astype(np.float32)
    noisy, scaled, bg = testing.add_noise(clean, 1e3, detection_efficiency=0.37, seed=5)
    _, ref_scaled, ref_bg = port.add_noise(clean, 1e3, detection_efficiency=0.37)
    np.testing.assert_array_equal(scaled, ref_scaled)
    np.testing.assert_array_equal(noisy, ref_scaled)
    assert bg == 0.0 and ref_bg == 0.0


@pytest.mark.parametrize("lam", [0.3, 3.0, 9.99, 10.0, 37.5, 1e3, 1e5])
def test_poisson_moments(lam, cuda):
    from oracle import port
    from pycorrectedemissionct_b200 import testing

    n = 1 << 20
    img = torch.full((n,), float(lam), device=cuda)
    noisy, _, _ = testing.add_noise(img, 1.0, add_poisson=True, seed=int(lam * 1000) + 1)
    k = noisy.double()
    assert bool(torch.all(k == torch.round(k)).item()) and float(k.min().item()) >= 0
    mean, var = float(k.mean().item()), float(k.var().item())
    assert abs(mean - lam) < 5 * np.sqrt(lam / n)
    assert abs(var / lam - 1) < 5 * np.sqrt((1 / lam + 2) / n)
    # the port's numpy draws estimate the same moments
    np.random.seed(3)
    ref, _, _ = port.add_noise(np.full(n, lam, np.float32), 1.0, add_poisson=True)
    assert abs(mean - ref.mean()) < 5 * np.sqrt(2 * lam / n)


@pytest.mark.parametrize("lam", [0.7, 4.0, 12.0, 30.0])
def test_poisson_counts_fit_pmf(lam, cuda):
    from scipy import stats

    from pycorrectedemissionct_b200 import testing

    n = 1 << 20
    noisy, _, _ = testing.add_noise(torch.full((n,), lam, device=cuda), 1.0, add_poisson=True, seed=99)
    k = noisy.cpu().numpy().astype(np.int64)
    top = int(stats.poisson.ppf(1 - 1e-6, lam))
    obs = np.bincount(np.minimum(k, top), minlength=top + 1)[: top + 1].astype(np.float64)
    exp = stats.poisson.pmf(np.arange(top + 1), lam) * n
    exp[-1] += stats.poisson.sf(top, lam) * n
    keep = exp > 5
    chi2 = float((((obs - exp) ** 2) / exp)[keep].sum())
    dof = int(keep.sum()) - 1
    assert stats.chi2.sf(chi2, dof) > 1e-4


def test_background_and_readout(cuda):
    from scipy import stats

    from pycorrectedemissionct_b200 import testing

    n = 1 << 20
    clean = torch.rand(n, device=cuda, generator=torch.Generator(device=cuda).manual_seed(0))
    photons, eff, avg, std = 800.0, 0.5, 0.02, 0.01
    noisy, scaled, bg = testing.add_noise(clean, photons, background_avg=avg, background_std=std,
                                          detection_efficiency=eff, seed=7)
    d = (noisy.double() - scaled.double())
    assert abs(bg - float(d.mean().item())) < 1e-6 * abs(bg)
    # E|N(avg, std)| (folded normal)
    folded = stats.foldnorm(avg / std, scale=std)
    scale = photons * eff
    assert abs(bg / scale - folded.mean()) < 5 * folded.std() / np.sqrt(n)
    assert abs(float(d.std().item()) / scale - folded.std()) < 0.01 * folded.std()
    # read-out noise only
    noisy2, scaled2, bg2 = testing.add_noise(clean, photons, readout_noise_std=3.0, seed=8)
    r = noisy2.double() - scaled2.double()
    assert bg2 == 0.0
    assert abs(float(r.mean().item())) < 5 * 3.0 / np.sqrt(n)
    assert abs(float(r.std().item()) / 3.0 - 1) < 0.01
    # default background_std = 5 % of the average
    _, _, bg3 = testing.add_noise(clean, photons, background_avg=avg, seed=9)
    assert abs(bg3 / (photons * avg) - 1) < 1e-3


def test_seed_reproducibility_and_errors(cuda):
    from pycorrectedemissionct_b200 import testing

    clean = torch.rand(4096, device=cuda) * 50
    a, _, _ = testing.add_noise(clean, 1.0, add_poisson=True, readout_noise_std=1.0, seed=11)
    b, _, _ = testing.add_noise(clean, 1.0, add_poisson=True, readout_noise_std=1.0, seed=11)
    c, _, _ = testing.add_noise(clean, 1.0, add_poisson=True, readout_noise_std=1.0, seed=12)
    assert torch.equal(a, b) and not torch.equal(a, c)
    np.random.seed(4)
    d, _, _ = testing.add_noise(clean, 1.0, add_poisson=True)
    np.random.seed(4)
    e, _, _ = testing.add_noise(clean, 1.0, add_poisson=True)
    assert torch.equal(d, e)
    with pytest.raises(ValueError):
        testing.add_noise(clean - 100.0, 1.0, add_poisson=True, seed=1)


def test_create_sino_matches_port(cuda):
    from oracle import port
    from pycorrectedemissionct_b200 import phantoms, testing

    n, n_ang = 48, 30
    rng = phantoms.slice_rng(77, 0)
    ph = phantoms.ellipse_phantom(n, rng, 6) * 1e-3
    mu = phantoms.disk_attenuation(n, rng, 0.05)
    sino, angles, expected, bg = testing.create_sino(
        ph, n_ang, vol_att_in=mu, vol_att_out=0.5 * mu, photon_flux=1e9, verbose=False, seed=3,
    )
    assert sino.shape == (n_ang, n) and bg == 0.0
    np.testing.assert_allclose(angles, np.deg2rad(np.linspace(0, 180, n_ang, endpoint=False)))
    rad32, deg32 = port.backend_angles(angles)
    maps = port.compute_maps(mu.astype(np.float64), 0.5 * mu.astype(np.float64), rad32)
    ref = port.fp_xrf(ph.astype(np.float64), maps, deg32)
    sa = (2.4 / 2 / 16 / 2) ** 2
    assert rel_l2(sino, ref * 1e9 * sa) < 1e-5
    np.testing.assert_allclose(expected, ph * 1e9 * sa)
    noisy, _, _, _ = testing.create_sino(ph, n_ang, vol_att_in=mu, vol_att_out=0.5 * mu, add_poisson=True,
                                         verbose=False, seed=4)
    assert np.all(noisy == np.round(noisy)) and abs(noisy.sum() / sino.sum() - 1) < 5 / np.sqrt(sino.sum())
