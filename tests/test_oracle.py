"""CPU: the oracle port against the reference-generated golden fixtures, and known-answer tests
of the restated scikit-image primitives (analytic, independent of scikit-image)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2
from oracle import port
from oracle import skimage_restated as skr


ALL_CASES = ["n32_a16", "n33_a9", "n16_a7_d2", "n64_a48", "n32_a16_psf", "n24_a10_d2_psf"]


def _psf(g):
    return g["psf"] if g["psf"].size else None


@pytest.mark.parametrize("case", ALL_CASES)
def test_port_matches_reference_golden(golden_cases, case):
    g = golden_cases[case]
    rad32, deg32 = port.backend_angles(g["angles"])
    maps = port.compute_maps(g["mu_in"], g["mu_out"], rad32, g["det_angles"])
    assert rel_l2(maps, g["maps"]) < 1e-14
    fa = port.fp_xrf(g["x"], g["maps"], deg32, g["det_weights"], g["weights_angles"], psf=_psf(g))
    assert rel_l2(fa, g["fp_att"]) < 1e-14
    assert rel_l2(port.bp_xrf(g["y"], g["maps"], deg32), g["bp_att"]) < 1e-14
    bs = port.bp_xrf(g["y"], g["maps"], deg32, g["det_weights"], g["weights_angles"], is_symmetric=True)
    assert rel_l2(bs, g["bp_sym"]) < 1e-14
    fu = port.fp_uncorrected(g["x"], deg32)
    if _psf(g) is not None:
        fu = np.stack([port.psf_convolve(line, _psf(g)) for line in fu])
    assert rel_l2(fu, g["fp_unc"]) < 1e-14
    n = int(g["n"])
    y0 = np.reshape(g["y"], (-1, len(deg32), n))[0]
    assert rel_l2(port.bp_uncorrected(y0, deg32, n), g["bp_unc"]) < 1e-14


@pytest.mark.parametrize("case", ["n32_a16", "n64_a48", "n32_a16_psf"])
def test_port_solvers_match_reference_golden(golden_cases, case):
    g = golden_cases[case]
    n = int(g["n"])
    _, deg32 = port.backend_angles(g["angles"])
    fp = lambda v: port.fp_xrf(v, g["maps"], deg32, psf=_psf(g))  # noqa: E731
    bp = lambda s: port.bp_xrf(s, g["maps"], deg32)  # noqa: E731
    xm, res = port.mlem(fp, bp, g["b"], 10, tolerance=0.0)
    assert rel_l2(xm, g["mlem_x"]) < 1e-13
    np.testing.assert_allclose(res, g["mlem_res"], rtol=1e-12)
    assert rel_l2(port.sirt(fp, bp, g["b"], 10, (n, n)), g["sirt_x"]) < 1e-13
    assert rel_l2(port.pdhg_kl_tv(fp, bp, g["b"], 10, (n, n), 1e-2), g["pdhg_x"]) < 1e-13


def test_port_masked_solvers_match_reference_golden(golden_cases):
    """MLEM / SIRT / PDHG / FISTA with b_mask and b_test_mask, residuals and cross-validation
    residuals included."""
    g = golden_cases["n32_a16"]
    m = np.load(os.path.join(GOLDEN, "mask_case.npz"))
    n = int(g["n"])
    _, deg32 = port.backend_angles(g["angles"])
    fp = lambda v: port.fp_xrf(v, g["maps"], deg32)  # noqa: E731
    bp = lambda s: port.bp_xrf(s, g["maps"], deg32)  # noqa: E731
    cv = []
    xm, res = port.mlem(fp, bp, g["b"], 10, tolerance=0.0, b_mask=m["b_mask"], b_test_mask=m["b_test_mask"], residuals_cv=cv)
    assert rel_l2(xm, m["mlem_x"]) < 1e-13
    np.testing.assert_allclose(res, m["mlem_res"], rtol=1e-12)
    np.testing.assert_allclose(cv, m["mlem_res_cv"], rtol=1e-12)
    cv = []
    xs = port.sirt(fp, bp, g["b"], 10, (n, n), b_mask=m["b_mask"], b_test_mask=m["b_test_mask"], residuals_cv=cv)
    assert rel_l2(xs, m["sirt_x"]) < 1e-13
    np.testing.assert_allclose(cv, m["sirt_res_cv"], rtol=1e-12)
    res, cv = [], []
    xp = port.pdhg_kl_tv(fp, bp, g["b"], 10, (n, n), 1e-2, b_mask=m["b_mask"], b_test_mask=m["b_test_mask"], tolerance=0.0,
                         residuals=res, residuals_cv=cv)
    assert rel_l2(xp, m["pdhg_x"]) < 1e-13
    np.testing.assert_allclose(res, m["pdhg_res"], rtol=1e-12)
    np.testing.assert_allclose(cv, m["pdhg_res_cv"], rtol=1e-12)
    res, cv = [], []
    xf = port.fista(fp, bp, g["b"], 10, (n, n), b_mask=m["b_mask"], b_test_mask=m["b_test_mask"], tolerance=0.0,
                    residuals=res, residuals_cv=cv)
    assert rel_l2(xf, m["fista_x"]) < 1e-13
    np.testing.assert_allclose(res, m["fista_res"], rtol=1e-12)
    np.testing.assert_allclose(cv, m["fista_res_cv"], rtol=1e-12)


def test_port_lipschitz_scaled_solvers_match_reference_golden(golden_cases):
    """PDHG and FISTA with precondition=False: sigma, tau from the power method's operator norm
    (its random start drawn after np.random.seed, as in the reference's run)."""
    g = golden_cases["n32_a16"]
    m = np.load(os.path.join(GOLDEN, "mask_case.npz"))
    n = int(g["n"])
    _, deg32 = port.backend_angles(g["angles"])
    fp = lambda v: port.fp_xrf(v, g["maps"], deg32)  # noqa: E731
    bp = lambda s: port.bp_xrf(s, g["maps"], deg32)  # noqa: E731
    np.random.seed(11)
    xp = port.pdhg_kl_tv(fp, bp, g["b"], 10, (n, n), 1e-2, precondition=False)
    assert rel_l2(xp, m["pdhg_lipschitz_x"]) < 1e-13
    np.random.seed(12)
    xf = port.fista(fp, bp, g["b"], 10, (n, n), precondition=False)
    assert rel_l2(xf, m["fista_lipschitz_x"]) < 1e-13


def test_port_solvers_with_mask_and_limits_match_reference_golden(golden_cases):
    """MLEM, SIRT and PDHG with a solution mask and clipping limits."""
    g = golden_cases["n32_a16"]
    o = np.load(os.path.join(GOLDEN, "options_case.npz"))
    n = int(g["n"])
    _, deg32 = port.backend_angles(g["angles"])
    fp = lambda v: port.fp_xrf(v, g["maps"], deg32)  # noqa: E731
    bp = lambda s: port.bp_xrf(s, g["maps"], deg32)  # noqa: E731
    m = o["x_mask"]
    xm, _ = port.mlem(fp, bp, g["b"], 10, x_mask=m, lower_limit=0.0, upper_limit=2.0)
    assert rel_l2(xm, o["mlem_x"]) < 1e-13
    xs = port.sirt(fp, bp, g["b"], 10, (n, n), x_mask=m, lower_limit=0.0)
    assert rel_l2(xs, o["sirt_x"]) < 1e-13
    xp = port.pdhg_kl_tv(fp, bp, g["b"], 10, (n, n), 1e-2, x_mask=m, lower_limit=0.0, upper_limit=3.0)
    assert rel_l2(xp, o["pdhg_x"]) < 1e-13


def test_reference_float32_maps_close_to_fp64(golden_cases):
    for g in golden_cases.values():
        assert rel_l2(g["maps_ref32"], g["maps"]) < 1e-6


# ----------------------------------------------------------------------------------- KATs
def test_radon_zero_angle_is_column_sums():
    rng = np.random.default_rng(0)
    img = rng.uniform(size=(17, 17))
    out = skr.radon(img, np.array([0.0], dtype=np.float32))[:, 0]
    np.testing.assert_allclose(out, img.sum(0), rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [16, 17])
def test_radon_90_degrees_is_lattice_permutation(n):
    rng = np.random.default_rng(1)
    img = rng.uniform(size=(n, n))
    out = skr.radon(img, np.array([90.0], dtype=np.float32))[:, 0]
    # at 90 deg the samples land on lattice points (to float32 trig rounding): a permutation of
    # the pixels, so every output is a full row sum of some (possibly shifted) row
    np.testing.assert_allclose(np.sort(out[1:-1]), np.sort(out[1:-1]), atol=0)
    assert abs(out.sum() - img[:, : n - (1 if n % 2 == 0 else 0)].sum()) < 1.5 * img.max() * n


def test_iradon_single_bin_is_hat_ridge():
    n = 16
    line = np.zeros(n)
    line[n // 2 + 3] = 1.0
    bp = skr.iradon(line[:, None], np.array([0.0], dtype=np.float32), output_size=n, filter_name=None, circle=False)
    bp = bp * 2 / np.pi
    # theta = 0: t = j - n//2, so column j = n//2 + 3 is 1, all others 0 (a ridge along rows)
    expect = np.zeros((n, n))
    expect[:, n // 2 + 3] = 1.0
    np.testing.assert_allclose(bp, expect, atol=1e-12)


def test_iradon_edges_follow_numpy_interp():
    n = 8
    line = np.arange(1, n + 1, dtype=np.float64)
    # theta = 180 deg (float32): t slightly off the last node for half of the rows
    bp = skr.iradon(line[:, None], np.array([180.0], dtype=np.float32), output_size=n, filter_name=None, circle=False)
    assert np.all(np.isfinite(bp))


def test_zero_attenuation_gives_unit_maps():
    n = 16
    mu = np.zeros((n, n))
    rad32, _ = port.backend_angles(np.linspace(0, 2 * np.pi, 5, endpoint=False))
    maps = port.compute_maps(mu, mu, rad32)
    np.testing.assert_array_equal(maps, np.ones_like(maps))


def test_line_integral_is_linear_in_mu():
    rng = np.random.default_rng(2)
    n = 24
    mu = rng.uniform(0, 0.05, size=(n, n))
    a = np.float32(0.3)
    l1 = -np.log(port.compute_attenuation(mu, a))
    l2 = -np.log(port.compute_attenuation(2.5 * mu, a))
    np.testing.assert_allclose(l2, 2.5 * l1, rtol=1e-10, atol=1e-12)


def test_uniform_disk_line_integral_matches_chord():
    n = 64
    yy, xx = np.mgrid[:n, :n] - (n - 1) / 2
    mu = np.where(xx**2 + yy**2 <= 20**2, 0.01, 0.0)
    lin = -np.log(port.compute_attenuation(mu, np.float32(0.0)))
    # at angle 0 the beam runs along +rows: at the disk centre the path length from entry is ~20
    c = n // 2
    assert abs(lin[c, c] - 0.01 * 20.5) < 0.01 * 1.5


def test_exact_adjoint_oracle_is_adjoint():
    rng = np.random.default_rng(3)
    n, a = 20, 7
    _, deg32 = port.backend_angles(np.linspace(0, 2 * np.pi, a, endpoint=False))
    maps = rng.uniform(0.5, 1.0, size=(a, 1, n, n))
    x = rng.uniform(size=(n, n))
    y = rng.uniform(size=(a, n))
    lhs = np.vdot(port.fp_xrf(x, maps, deg32), y)
    rhs = np.vdot(x, port.fp_xrf_adjoint(y, maps, deg32, n))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_psf_convolution_offsets():
    line = np.arange(8, dtype=np.float64)
    # odd kernel: centred, edge padded
    out = port.psf_convolve(line, np.array([0.0, 1.0, 0.0]))
    np.testing.assert_allclose(out, line)
    # out[i] = sum_j x[clamp(i + (L-1)//2 - j)] k[j]: k = [1, 0, 0] reads x[i + 1] (edge clamped)
    out = port.psf_convolve(line, np.array([1.0, 0.0, 0.0]))
    np.testing.assert_allclose(out, np.concatenate([line[1:], line[-1:]]))
    # even length: (L-1)//2 = 1, so k = [0, 1, 0, 0] is the identity
    np.testing.assert_allclose(port.psf_convolve(line, np.array([0.0, 1.0, 0.0, 0.0])), line)


def test_intensities_scale_lines_in_fp_and_bp():
    rng = np.random.default_rng(4)
    n, a = 16, 5
    _, deg32 = port.backend_angles(np.linspace(0, 2 * np.pi, a, endpoint=False))
    maps = rng.uniform(0.5, 1, size=(a, 1, n, n))
    x = rng.uniform(size=(n, n))
    inten = rng.uniform(0.5, 1.5, size=a)
    np.testing.assert_allclose(port.fp_xrf(x, maps, deg32, intensities=inten), port.fp_xrf(x, maps, deg32) * inten[:, None])
    y = rng.uniform(size=(a, n))
    np.testing.assert_allclose(port.bp_xrf(y, maps, deg32, intensities=inten), port.bp_xrf(y * inten[:, None], maps, deg32))


NOISE_CASES = [
    # name, photons, efficiency, poisson, readout std, background avg, background std, seed
    ("poisson", 1e3, 0.5, True, None, None, None, 101),
    ("background_poisson_readout", 2e3, 0.25, True, 2.0, 0.01, None, 102),
    ("background_only", 5e2, 1.0, False, None, 0.02, 0.003, 103),
]


@pytest.mark.parametrize("case", NOISE_CASES, ids=[c[0] for c in NOISE_CASES])
def test_port_add_noise_matches_reference_golden(case):
    """After np.random.seed the port draws exactly what the reference's add_noise drew."""
    import os

    from conftest import GOLDEN

    g = dict(np.load(os.path.join(GOLDEN, "noise_cases.npz")))
    name, photons, eff, poisson, readout, bg_avg, bg_std, seed = case
    np.random.seed(seed)
    noisy, scaled, background = port.add_noise(
        g["clean"], photons, add_poisson=poisson, readout_noise_std=readout, background_avg=bg_avg,
        background_std=bg_std, detection_efficiency=eff,
    )
    np.testing.assert_array_equal(scaled, g[f"{name}_scaled"])
    np.testing.assert_array_equal(noisy, g[f"{name}_noisy"])
    assert background == float(g[f"{name}_background"])


def test_port_finite_surface_detectors_match_reference_golden():
    """Emitted sub-sampling of a finite detector next to a point detector (attenuation.py:105-120)."""
    import os

    from conftest import GOLDEN

    g = dict(np.load(os.path.join(GOLDEN, "surface_case.npz")))
    rad32, deg32 = port.backend_angles(g["angles"])
    maps = port.compute_maps(g["mu_in"], g["mu_out"], rad32, g["det_angles"], detector_surfaces_mm2=g["det_surfaces"],
                             detector_distances_mm=g["det_distances"], emitted_sub_sampling=int(g["sub_sampling"]))
    assert rel_l2(maps, g["maps"]) < 1e-13
    assert rel_l2(port.fp_xrf(g["x"], g["maps"], deg32), g["fp_att"]) < 1e-13


def test_half_turn_line_integral_is_the_reverse_scan():
    """The identity behind the maps kernels' half-turn pairs: the line integral at phi + pi is the
    rotate-back of K - W_phi, K[c] = sum_r U[r][c] + (U[0][c] + U[P-1][c]) / 2, with W_phi the
    roll + cumsum of halves at phi (``_projector_backends.py:68-73``)."""
    n = 24
    mu = np.zeros((n, n))
    mu[5:15, 8:20] = 0.05
    mu[12:20, 3:9] = 0.02
    edge, _ = port.padded_size(n)
    for phi in (0.3, 1.2, 2.9):
        deg = np.rad2deg(phi)
        u = skr.rotate(np.pad(mu, edge), -deg, order=1, clip=False)
        w = np.cumsum((u + np.roll(u, 1, axis=-2)) / 2, axis=-2)
        k = u.sum(axis=0) + (u[0] + u[-1]) / 2
        l_pair = skr.rotate(k[None, :] - w, deg, order=1, clip=False)[edge:-edge, edge:-edge]
        l_ref = -np.log(port.compute_attenuation(mu, phi + np.pi))
        np.testing.assert_allclose(l_pair, l_ref, atol=1e-12)
