"""GPU parity of the CUDA path (called through the C ABI) against the reference-generated golden
fixtures and the FP64 oracle port.

Tolerances (relative L2, FP32 GPU vs FP64 oracle): maps, fp, bp 1e-5; reconstructions after a
fixed iteration count 1e-4; exact-adjoint pair <fp x, y> vs <x, bp y> 1e-6 (FP64 inner products).
BF16-stored maps are reported against FP64 with their own bound (BF16 keeps 8 mantissa bits).
"""

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_RECON = 1e-4
TOL_ADJ = 1e-6

CASES = ["n32_a16", "n33_a9", "n16_a7_d2", "n64_a48", "n32_a16_psf", "n24_a10_d2_psf"]


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _core(g, cuda):
    from pycorrectedemissionct_b200 import core

    n_det = len(g["det_angles"])
    w = np.asarray(g["det_weights"])[None, :] * np.asarray(g["weights_angles"])
    c = core.XrfCore(int(g["n"]), g["angles"], n_det=n_det, weights=w, device=cuda)
    if g["psf"].size:
        c.set_psf(g["psf"])
    return c


def _t(a, cuda, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda, dtype)


@pytest.mark.parametrize("case", CASES)
def test_maps_match_reference(golden_cases, case, cuda):
    from pycorrectedemissionct_b200 import core

    g = golden_cases[case]
    rad32 = np.array(g["angles"], dtype=np.float32)
    maps = core.compute_maps(_t(g["mu_in"], cuda)[None], _t(g["mu_out"], cuda)[None], rad32, g["det_angles"])
    got = maps[0].cpu().numpy()
    assert got.shape == g["maps"].shape
    assert rel_l2(got, g["maps"]) < TOL


@pytest.mark.parametrize("case", CASES)
def test_fp_bp_match_reference(golden_cases, case, cuda):
    g = golden_cases[case]
    c = _core(g, cuda)
    n, n_ang, n_det = int(g["n"]), len(g["angles"]), len(g["det_angles"])
    maps = _t(g["maps"], cuda)[None]
    x = _t(g["x"], cuda)[None]
    fp = c.fp(x, maps)[0].cpu().numpy()
    assert rel_l2(fp.reshape(g["fp_att"].shape), g["fp_att"]) < TOL
    y = _t(np.reshape(g["y"], (1, n_det, n_ang, n)), cuda)
    assert rel_l2(c.bp(y, "reference")[0].cpu().numpy(), g["bp_att"]) < TOL
    assert rel_l2(c.bp(y, "symmetric", maps)[0].cpu().numpy(), g["bp_sym"]) < TOL
    if n_det == 1:
        cu = _core(dict(g, weights_angles=np.ones_like(g["weights_angles"])), cuda)
        assert rel_l2(cu.fp(x)[0, 0].cpu().numpy(), g["fp_unc"]) < TOL
        assert rel_l2(cu.bp(y, "reference")[0].cpu().numpy(), g["bp_unc"]) < TOL


def test_intensities_and_psf_against_port(golden_cases, cuda):
    """Projection intensities (checked against the port: the reference's own intensity path
    raises under numpy >= 2) combined with a PSF, through the public projector."""
    from oracle import port
    from pycorrectedemissionct_b200 import projectors

    g = golden_cases["n24_a10_d2_psf"]
    n, n_ang = int(g["n"]), len(g["angles"])
    rng = np.random.default_rng(21)
    inten = rng.uniform(0.5, 1.5, size=n_ang)
    _, deg32 = port.backend_angles(g["angles"])
    kw = dict(att_maps=g["maps"], angles_detectors_rad=g["det_angles"], weights_detectors=g["det_weights"],
              weights_angles=g["weights_angles"], psf=g["psf"], prj_intensities=inten)
    p = projectors.ProjectorAttenuationXRF((n, n), g["angles"], **kw)
    ref_fp = port.fp_xrf(g["x"], g["maps"], deg32, g["det_weights"], g["weights_angles"], intensities=inten, psf=g["psf"])
    assert rel_l2(p.fp(g["x"]), ref_fp) < TOL
    ref_bp = port.bp_xrf(g["y"], g["maps"], deg32, intensities=inten)
    assert rel_l2(p.bp(g["y"]), ref_bp) < TOL
    ps = projectors.ProjectorAttenuationXRF((n, n), g["angles"], is_symmetric=True, **kw)
    ref_bs = port.bp_xrf(g["y"], g["maps"], deg32, g["det_weights"], g["weights_angles"], True, intensities=inten)
    assert rel_l2(ps.bp(g["y"]), ref_bs) < TOL
    # single-angle paths
    for a in (0, 3):
        line = port.fp_xrf(g["x"], g["maps"][a : a + 1], deg32[a : a + 1], g["det_weights"], g["weights_angles"][a : a + 1],
                           intensities=inten[a : a + 1], psf=g["psf"])
        assert rel_l2(p.fp_angle(g["x"], a), line[:, 0]) < TOL


@pytest.mark.parametrize("case", ["n32_a16", "n33_a9", "n64_a48", "n32_a16_psf"])
def test_solvers_match_reference(golden_cases, case, cuda):
    from pycorrectedemissionct_b200 import projectors, solvers

    g = golden_cases[case]
    n = int(g["n"])
    psf = g["psf"] if g["psf"].size else None
    p = projectors.ProjectorAttenuationXRF((n, n), g["angles"], att_maps=g["maps"], angles_detectors_rad=g["det_angles"], psf=psf)
    xm, info = solvers.MLEM(tolerance=0.0)(p, g["b"], iterations=10)
    assert rel_l2(xm, g["mlem_x"]) < TOL_RECON
    np.testing.assert_allclose(info.residuals[:10], g["mlem_res"], rtol=TOL_RECON)
    assert info.iterations == 10
    xs, _ = solvers.SIRT()(p, g["b"], iterations=10)
    assert rel_l2(xs, g["sirt_x"]) < TOL_RECON
    xp, _ = solvers.PDHG(data_term="kl", regularizer=1e-2)(p, g["b"], iterations=10)
    assert rel_l2(xp, g["pdhg_x"]) < TOL_RECON


@pytest.mark.parametrize("n,maps_dtype", [(72, "float32"), (45, "float32"), (72, "bfloat16"), (72, "fields-float32")])
def test_half_turn_pairs_match_single_angles(n, maps_dtype, cuda):
    """Maps from half-turn pairs (one rotation per direction for angles phi and phi + pi) against
    every angle on its own: the entries' own angles are bit-identical, the partners within the
    float32 rounding of the angles; with a permuted angle order and two detectors, one of them
    finite (3 emitted sub-angles) where the maps dtype allows it."""
    from pycorrectedemissionct_b200 import core, geometry, phantoms

    n_ang = 40
    rad32 = np.array(phantoms.angles(n_ang), dtype=np.float32)[np.random.default_rng(3).permutation(n_ang)]
    fields = maps_dtype == "fields-float32"
    kw = dict(det_angles=[np.pi / 2, np.pi / 3])
    if not fields:
        kw.update(surfaces_mm2=[0.0, 10.0], distances_mm=[1.0, 50.0], sub_sampling=3)
    mus = np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(77, k), 0.04) for k in range(2)])
    mu = torch.from_numpy(mus).to(cuda)
    paired = core.compute_maps(mu, 0.8 * mu, rad32, maps_dtype=maps_dtype, **kw)
    single = core.compute_maps(mu, 0.8 * mu, rad32, maps_dtype=maps_dtype, half_turns=False, **kw)
    pairs = geometry.half_turn_pairs(rad32)
    assert pairs is not None and (pairs[:, 1] >= 0).all()
    own, partner = pairs[:, 0], pairs[:, 1]
    assert torch.equal(paired[:, own], single[:, own])
    tol = 4e-3 if maps_dtype == "bfloat16" else 2e-6
    got, want = paired[:, partner].double().cpu().numpy(), single[:, partner].double().cpu().numpy()
    assert rel_l2(got, want) < tol


@pytest.mark.parametrize("n,n_ang,scale,maps_dtype", [(72, 40, 1.0, "float32"), (45, 48, 0.7, "float32"),
                                                      (72, 40, 0.7, "bfloat16")])
def test_quarter_turn_quads_match_every_direction(n, n_ang, scale, maps_dtype, cuda):
    """Maps from quarter-turn quads (incident fields only; each emitted line integral is
    mu_out / mu_in times the incident one of the angle a quarter turn on) against every direction
    scanned on its own, within the float32 rounding of the angles; with a permuted angle order."""
    from pycorrectedemissionct_b200 import core, geometry, phantoms

    rad32 = np.array(phantoms.angles(n_ang), dtype=np.float32)[np.random.default_rng(5).permutation(n_ang)]
    assert geometry.quarter_turn_quads(rad32, geometry.half_turn_pairs(rad32), np.pi / 2) is not None
    mus = np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(78, k), 0.04) for k in range(2)])
    mu = torch.from_numpy(mus).to(cuda)
    quads = core.compute_maps(mu, scale * mu, rad32, maps_dtype=maps_dtype, emitted_scale=scale)
    every = core.compute_maps(mu, scale * mu, rad32, maps_dtype=maps_dtype)
    tol = 4e-3 if maps_dtype == "bfloat16" else 2e-6
    assert rel_l2(quads.double().cpu().numpy(), every.double().cpu().numpy()) < tol
    # mu_out given as mu_in itself: quads with scale 1
    assert torch.equal(core.compute_maps(mu, mu, rad32, maps_dtype=maps_dtype),
                       core.compute_maps(mu, mu.clone(), rad32, maps_dtype=maps_dtype, emitted_scale=1.0))


@pytest.mark.parametrize("case", ["n32_a16", "n64_a48", "n32_a16_psf"])
def test_quarter_turn_maps_match_reference(golden_cases, case, cuda):
    """The golden cases' emitted attenuation is 0.7 times the incident one: quad maps against the
    reference's own FP64 maps."""
    from pycorrectedemissionct_b200 import core, geometry

    g = golden_cases[case]
    rad32 = np.array(g["angles"], dtype=np.float32)
    assert np.allclose(g["mu_out"], 0.7 * g["mu_in"])
    assert geometry.quarter_turn_quads(rad32, geometry.half_turn_pairs(rad32), float(g["det_angles"][0])) is not None
    mu_in = _t(g["mu_in"], cuda)[None]
    maps = core.compute_maps(mu_in, _t(g["mu_out"], cuda)[None], rad32, g["det_angles"], emitted_scale=0.7)
    assert rel_l2(maps[0].cpu().numpy(), g["maps"]) < TOL


def test_masked_solvers_match_reference(golden_cases, cuda):
    """MLEM, SIRT, PDHG and FISTA with b_mask and b_test_mask, and SART with b_mask, through the
    drop-in solvers: reconstruction, residuals and cross-validation residuals against the
    reference's own run."""
    import os

    from conftest import GOLDEN
    from pycorrectedemissionct_b200 import projectors, solvers

    g = golden_cases["n32_a16"]
    m = dict(np.load(os.path.join(GOLDEN, "mask_case.npz")))
    n = int(g["n"])
    p = projectors.ProjectorAttenuationXRF((n, n), g["angles"], att_maps=g["maps"], angles_detectors_rad=g["det_angles"])
    kw = dict(b_mask=m["b_mask"], b_test_mask=m["b_test_mask"])
    xm, info = solvers.MLEM(tolerance=0.0)(p, g["b"], iterations=10, **kw)
    assert rel_l2(xm, m["mlem_x"]) < TOL_RECON
    np.testing.assert_allclose(info.residuals[:10], m["mlem_res"], rtol=TOL_RECON)
    np.testing.assert_allclose(info.residuals_cv[:10], m["mlem_res_cv"], rtol=TOL_RECON)
    np.testing.assert_allclose([info.residual0, info.residual0_cv], [m["mlem_res0"], m["mlem_res0_cv"]], rtol=TOL_RECON)
    xs, info = solvers.SIRT(tolerance=0.0)(p, g["b"], iterations=10, **kw)
    assert rel_l2(xs, m["sirt_x"]) < TOL_RECON
    np.testing.assert_allclose(info.residuals[:10], m["sirt_res"], rtol=TOL_RECON)
    np.testing.assert_allclose(info.residuals_cv[:10], m["sirt_res_cv"], rtol=TOL_RECON)
    np.testing.assert_allclose([info.residual0, info.residual0_cv], [m["sirt_res0"], m["sirt_res0_cv"]], rtol=TOL_RECON)
    xp, info = solvers.PDHG(data_term="kl", regularizer=1e-2, tolerance=0.0)(p, g["b"], iterations=10, **kw)
    assert rel_l2(xp, m["pdhg_x"]) < TOL_RECON
    np.testing.assert_allclose(info.residuals[:10], m["pdhg_res"], rtol=TOL_RECON)
    np.testing.assert_allclose(info.residuals_cv[:10], m["pdhg_res_cv"], rtol=TOL_RECON)
    np.testing.assert_allclose([info.residual0, info.residual0_cv], [m["pdhg_res0"], m["pdhg_res0_cv"]], rtol=TOL_RECON)
    xf, info = solvers.FISTA(tolerance=0.0)(p, g["b"], iterations=10, **kw)
    assert rel_l2(xf, m["fista_x"]) < TOL_RECON
    np.testing.assert_allclose(info.residuals[:10], m["fista_res"], rtol=TOL_RECON)
    np.testing.assert_allclose(info.residuals_cv[:10], m["fista_res_cv"], rtol=TOL_RECON)
    np.random.seed(5)  # the angle order of SART, as drawn by the reference run
    xa, _ = solvers.SART()(p, g["b"], iterations=3, b_mask=m["b_mask"])
    assert rel_l2(xa, m["sart_x"]) < TOL_RECON
    # a test mask alone holds its pixels out of the reconstruction: equal to b_mask = 1 - test
    xt, _ = solvers.SIRT()(p, g["b"], iterations=10, b_test_mask=m["b_test_mask"])
    xo, _ = solvers.SIRT()(p, g["b"], iterations=10, b_mask=1 - m["b_test_mask"])
    np.testing.assert_array_equal(xt, xo)


def test_solvers_with_mask_and_limits_match_reference(golden_cases, cuda):
    """MLEM, SIRT and PDHG through the drop-in solvers with a solution mask and clipping limits,
    against the reference's own run."""
    import os

    from conftest import GOLDEN
    from pycorrectedemissionct_b200 import projectors, solvers

    g = golden_cases["n32_a16"]
    o = dict(np.load(os.path.join(GOLDEN, "options_case.npz")))
    n = int(g["n"])
    p = projectors.ProjectorAttenuationXRF((n, n), g["angles"], att_maps=g["maps"], angles_detectors_rad=g["det_angles"])
    m = o["x_mask"]
    xm, _ = solvers.MLEM()(p, g["b"], iterations=10, x_mask=m, lower_limit=0.0, upper_limit=2.0)
    assert rel_l2(xm, o["mlem_x"]) < TOL_RECON
    xs, _ = solvers.SIRT()(p, g["b"], iterations=10, x_mask=m, lower_limit=0.0)
    assert rel_l2(xs, o["sirt_x"]) < TOL_RECON
    xp, _ = solvers.PDHG(data_term="kl", regularizer=1e-2)(p, g["b"], iterations=10, x_mask=m, lower_limit=0.0,
                                                          upper_limit=3.0)
    assert rel_l2(xp, o["pdhg_x"]) < TOL_RECON
    # a restart from an unmasked x0 masks it, as the constructor does (solvers.py:750-752)
    from pycorrectedemissionct_b200 import core, engine

    c = core.XrfCore(n, g["angles"], device=cuda)
    b = _t(g["b"], cuda).reshape(1, 1, len(g["angles"]), n)
    sv = engine.BatchedSolver(c, _t(g["maps"], cuda)[None], b, "mlem", x_mask=_t(m, cuda), lower_limit=0.0,
                              upper_limit=2.0)
    sv.run(10, use_graph=False)
    first = sv.x.clone()
    assert rel_l2(first[0].cpu().numpy(), o["mlem_x"]) < TOL_RECON
    sv.reset(torch.ones_like(sv.x))
    sv.run(10, use_graph=False)
    assert torch.equal(sv.x, first)


def test_lipschitz_scaled_solvers_match_reference(golden_cases, cuda):
    """PDHG and FISTA with precondition=False: the power method's random start drawn after the
    same np.random.seed as the reference's run, its iterations on the device."""
    import os

    from conftest import GOLDEN
    from pycorrectedemissionct_b200 import projectors, solvers

    g = golden_cases["n32_a16"]
    m = dict(np.load(os.path.join(GOLDEN, "mask_case.npz")))
    n = int(g["n"])
    p = projectors.ProjectorAttenuationXRF((n, n), g["angles"], att_maps=g["maps"], angles_detectors_rad=g["det_angles"])
    np.random.seed(11)
    xp, _ = solvers.PDHG(data_term="kl", regularizer=1e-2)(p, g["b"], iterations=10, precondition=False)
    assert rel_l2(xp, m["pdhg_lipschitz_x"]) < TOL_RECON
    np.random.seed(12)
    xf, _ = solvers.FISTA()(p, g["b"], iterations=10, precondition=False)
    assert rel_l2(xf, m["fista_lipschitz_x"]) < TOL_RECON


@pytest.mark.parametrize("n,n_ang", [(66, 20), (130, 45), (128, 90), (256, 360)])
def test_against_oracle_port_medium(n, n_ang, cuda):
    from oracle import port
    from pycorrectedemissionct_b200 import core, phantoms

    rng = phantoms.slice_rng(1000 + n, 0)
    x = phantoms.ellipse_phantom(n, rng, 12, dtype=np.float64)
    mu = phantoms.disk_attenuation(n, rng, 0.02, dtype=np.float64)
    angles = phantoms.angles(n_ang)
    rad32, deg32 = port.backend_angles(angles)
    ref_maps = port.compute_maps(mu, 0.7 * mu, rad32, workers=8)
    maps = core.compute_maps(_t(mu, cuda)[None], _t(0.7 * mu, cuda)[None], rad32)
    assert rel_l2(maps[0].cpu().numpy(), ref_maps) < TOL
    c = core.XrfCore(n, angles, device=cuda)
    ref_fp = port.fp_xrf(x, ref_maps, deg32, workers=8)
    fp = c.fp(_t(x, cuda)[None], _t(ref_maps, cuda)[None])[0, 0].cpu().numpy()
    assert rel_l2(fp, ref_fp) < TOL
    y = rng.uniform(size=(n_ang, n))
    ref_bp = port.bp_uncorrected(y, deg32, n, workers=8)
    bp = c.bp(_t(y, cuda)[None, None], "reference")[0].cpu().numpy()
    assert rel_l2(bp, ref_bp) < TOL
    # the sensitivity image A^T 1 exercises np.interp's discontinuous detector edges everywhere
    ones = np.ones((n_ang, n))
    assert rel_l2(c.bp(_t(ones, cuda)[None, None], "reference")[0].cpu().numpy(), port.bp_uncorrected(ones, deg32, n, workers=8)) < TOL


@pytest.mark.parametrize("n,n_ang,n_det", [(64, 16, 1), (96, 31, 2), (128, 180, 1)])
def test_exact_adjoint_pair(n, n_ang, n_det, cuda):
    from pycorrectedemissionct_b200 import core

    rng = np.random.default_rng(n)
    w = rng.uniform(0.5, 1.5, size=(n_ang, n_det))
    c = core.XrfCore(n, np.linspace(0, 2 * np.pi, n_ang, endpoint=False), n_det=n_det, weights=w, device=cuda)
    maps = _t(rng.uniform(0.2, 1.0, size=(1, n_ang, n_det, n, n)), cuda)
    x = _t(rng.uniform(size=(1, n, n)), cuda)
    y = _t(rng.uniform(size=(1, n_det, n_ang, n)), cuda)
    lhs = torch.vdot(c.fp(x, maps).double().flatten(), y.double().flatten()).item()
    rhs = torch.vdot(x.double().flatten(), c.bp(y, "adjoint", maps).double().flatten()).item()
    assert abs(lhs - rhs) / abs(lhs) < TOL_ADJ


def test_exact_adjoint_matches_oracle(golden_cases, cuda):
    from oracle import port

    g = golden_cases["n32_a16"]
    c = _core(g, cuda)
    n, n_ang = int(g["n"]), len(g["angles"])
    _, deg32 = port.backend_angles(g["angles"])
    ref = port.fp_xrf_adjoint(g["y"], g["maps"], deg32, n)
    got = c.bp(_t(g["y"], cuda).reshape(1, 1, n_ang, n), "adjoint", _t(g["maps"], cuda)[None])[0].cpu().numpy()
    assert rel_l2(got, ref) < TOL


def test_batched_equals_single(cuda):
    from pycorrectedemissionct_b200 import core, phantoms

    n, n_ang, s = 96, 45, 3
    angles = phantoms.angles(n_ang)
    mus = np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(7, k), 0.02) for k in range(s)])
    xs = np.stack([phantoms.ellipse_phantom(n, phantoms.slice_rng(8, k)) for k in range(s)])
    rad32 = np.array(angles, dtype=np.float32)
    maps = core.compute_maps(_t(mus, cuda), _t(0.7 * mus, cuda), rad32)
    c = core.XrfCore(n, angles, device=cuda)
    fp_all = c.fp(_t(xs, cuda), maps)
    for k in range(s):
        mk = core.compute_maps(_t(mus[k], cuda)[None], _t(0.7 * mus[k], cuda)[None], rad32)
        assert torch.equal(mk[0], maps[k])
        assert torch.equal(c.fp(_t(xs[k], cuda)[None], mk)[0], fp_all[k])


def test_bf16_maps_error_against_fp64(golden_cases, cuda):
    from pycorrectedemissionct_b200 import core

    g = golden_cases["n64_a48"]
    rad32 = np.array(g["angles"], dtype=np.float32)
    m16 = core.compute_maps(_t(g["mu_in"], cuda)[None], _t(g["mu_out"], cuda)[None], rad32, maps_dtype="bfloat16")
    err = rel_l2(m16[0].float().cpu().numpy(), g["maps"])
    assert err < 4e-3  # bf16: 2^-9 relative rounding
    c = _core(g, cuda)
    fp16 = c.fp(_t(g["x"], cuda)[None], m16)[0, 0].cpu().numpy()
    assert rel_l2(fp16, g["fp_att"]) < 4e-3


def test_full_size_properties(cuda):
    """512 x 512, 720 angles (the benchmark slice): properties that need no oracle run."""
    from pycorrectedemissionct_b200 import core, phantoms

    n, n_ang = 512, 720
    rng = phantoms.slice_rng(42, 0)
    x = _t(phantoms.ellipse_phantom(n, rng), cuda)[None]
    mu = _t(phantoms.disk_attenuation(n, rng, 0.01), cuda)[None]
    angles = phantoms.angles(n_ang)
    maps = core.compute_maps(mu, mu, np.array(angles, dtype=np.float32))
    assert float(maps.max()) <= 1.0 and float(maps.min()) > 0.0
    c = core.XrfCore(n, angles, device=cuda)
    fp1 = c.fp(x, maps)
    fp2 = c.fp(2 * x, maps)
    assert torch.equal(fp2, 2 * fp1)  # exact: scaling by 2 is exact in FP32
    ones = torch.ones_like(maps)
    assert torch.equal(c.fp(x, ones), c.fp(x))  # unit maps == uncorrected projection, bit for bit
    zero = core.compute_maps(torch.zeros_like(mu), torch.zeros_like(mu), np.array(angles, dtype=np.float32))
    assert torch.all(zero == 1.0)
    # uncorrected sinogram mass is conserved up to the image support (phantom inside the circle)
    tot = c.fp(x)[0, 0].double().sum(dim=1)
    assert float((tot / x.double().sum() - 1).abs().max()) < 5e-3
    err = torch.zeros(1, dtype=torch.int32)
    from pycorrectedemissionct_b200 import _lib
    import ctypes

    v = ctypes.c_int32(0)
    _lib.call("cct_device_error", 0, ctypes.byref(v))
    assert v.value == 0


def test_engine_tolerance_and_graph(cuda):
    from pycorrectedemissionct_b200 import core, engine, phantoms

    n, n_ang, s = 64, 60, 4
    angles = phantoms.angles(n_ang)
    rad32 = np.array(angles, dtype=np.float32)
    mus = np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(9, k), 0.02) for k in range(s)])
    xs = np.stack([phantoms.ellipse_phantom(n, phantoms.slice_rng(10, k)) for k in range(s)])
    maps = core.compute_maps(_t(mus, cuda), _t(0.7 * mus, cuda), rad32)
    c = core.XrfCore(n, angles, device=cuda)
    clean = c.fp(_t(xs, cuda), maps)
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * 1e4)
    eager = engine.BatchedSolver(c, maps, b, "mlem", history_len=40)
    eager.run(40, check_every=10, use_graph=False)
    graph = engine.BatchedSolver(c, maps, b, "mlem", history_len=40)
    graph.run(40, check_every=10, use_graph=True)
    assert torch.equal(eager.x, graph.x)
    res = eager.history.cpu().numpy()
    tol = res[:, 25] * (1 + 1e-9)
    # the reference stops at the first iteration whose residual is below the tolerance
    expect = np.array([int(np.argmax(r < t)) + 1 for r, t in zip(res, tol)])
    stop = engine.BatchedSolver(c, maps, b, "mlem", tolerance=tol, history_len=40)
    stop.run(40, check_every=10)
    its = stop.iterations.cpu().numpy()
    np.testing.assert_array_equal(its, expect)
    assert int(stop.active.sum()) == 0
    # stopped slices keep the iterate of their last update
    assert torch.equal(stop.history[:, : int(expect.min())], eager.history[:, : int(expect.min())])


ALL_FP_VARIANTS = ("tma", "slices2")


def _variant(name):
    from pycorrectedemissionct_b200 import _lib

    return {"ldg": 0, "tma": _lib.CCT_VARIANT_FP_TMA, "slices2": _lib.CCT_VARIANT_FP_SLICES2}[name]


@pytest.mark.parametrize("n,n_ang,dtype,s", [(64, 48, "float32", 5), (512, 90, "float32", 5), (512, 90, "bfloat16", 4),
                                             (130, 45, "float32", 3), (1000, 12, "float32", 2), (66, 30, "fields", 6)])
def test_fp_variants_bit_identical(n, n_ang, dtype, s, cuda, tmp_path, monkeypatch):
    """Every fp variant (one slice per CTA with load/store or TMA staging, two slices per CTA)
    gives bit-identical projections, for batches that are not a multiple of the pair, for
    every maps storage type and for an angle range of larger maps; the autotuner picks one of
    them and caches it."""
    from pycorrectedemissionct_b200 import autotune, core, phantoms

    rng = phantoms.slice_rng(77, n)
    x = _t(np.stack([phantoms.ellipse_phantom(n, rng) for _ in range(s)]), cuda)
    c = core.XrfCore(n, phantoms.angles(n_ang), device=cuda)
    if dtype == "fields":
        c.set_channels([0.5, 1.0, 3.0])
        maps = _t(rng.uniform(0.0, 0.3, size=(s // 3, n_ang, 2, n, n)), cuda)
    else:
        maps = _t(rng.uniform(0.3, 1.0, size=(s, n_ang, 1, n, n)), cuda,
                  torch.bfloat16 if dtype == "bfloat16" else torch.float32)
    ref = c.fp(x, maps)
    sub = c.angle_range(slice(n_ang // 3, n_ang // 3 + 7))
    ref_sub = sub.fp(x, maps[:, n_ang // 3: n_ang // 3 + 7])
    for name in ALL_FP_VARIANTS:
        c.variant = sub.variant = _variant(name)
        assert torch.equal(c.fp(x, maps), ref), name
        assert torch.equal(sub.fp(x, maps[:, n_ang // 3: n_ang // 3 + 7]), ref_sub), name
    c.variant = 0
    monkeypatch.setenv("CCT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    v = autotune.tune(c, x, maps)
    assert v in autotune.VARIANTS and (tmp_path / "tune.json").exists()
    assert torch.equal(c.fp(x, maps), ref)


def test_maps_pass_size_tuning(cuda, tmp_path, monkeypatch):
    """The maps autotuner picks the entries per pass of compute_maps for a batch, caches the choice,
    and every pass size gives bit-identical maps."""
    from pycorrectedemissionct_b200 import autotune, core, phantoms

    monkeypatch.setenv("CCT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    n, n_ang, s = 96, 72, 3
    rad32 = np.array(phantoms.angles(n_ang), dtype=np.float32)
    mu = _t(np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(55, k), 0.03) for k in range(s)]), cuda)
    ref = core.compute_maps(mu, 0.7 * mu, rad32)
    assert autotune.maps_entries(cuda, n, n_ang, 1, s) is None
    e = autotune.tune_maps(mu, 0.7 * mu, rad32)
    assert e in autotune.MAPS_ENTRIES and autotune.maps_entries(cuda, n, n_ang, 1, s) == e
    for entries in (1, 5, e):
        ws = torch.empty(entries * core.maps_entry_bytes(n, s), dtype=torch.uint8, device=cuda)
        assert torch.equal(core.compute_maps(mu, 0.7 * mu, rad32, workspace=ws), ref)


@pytest.mark.parametrize("method", ["mlem", "sirt", "pdhg"])
def test_fused_solvers_identical_across_fp_variants(method, cuda):
    """The fused solver epilogues (MLEM ratio and KL residual, SIRT residual, PDHG dual) give the
    same iterates, residuals and stopping decisions with every fp variant, including a slice that
    stops early (its group-mates keep iterating)."""
    from pycorrectedemissionct_b200 import core, engine, phantoms

    n, n_ang, s = 96, 40, 5
    angles = phantoms.angles(n_ang)
    mus = np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(31, k), 0.02) for k in range(s)])
    xs = np.stack([phantoms.ellipse_phantom(n, phantoms.slice_rng(32, k)) for k in range(s)])
    maps = core.compute_maps(_t(mus, cuda), _t(0.7 * mus, cuda), np.array(angles, dtype=np.float32))
    c = core.XrfCore(n, angles, device=cuda)
    clean = c.fp(_t(xs, cuda), maps)
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * 1e4)
    probe = engine.BatchedSolver(c, maps, b, method, history_len=6)
    probe.run(6, check_every=6, use_graph=False)
    res = probe.history.cpu().numpy()
    tol = np.full(s, -1.0)
    if method != "pdhg":
        tol[1] = res[1, 2] * (1 + 1e-9)  # slice 1 stops after its third iteration
    results = {}
    for name in ("ldg",) + ALL_FP_VARIANTS:
        c.variant = _variant(name)
        sv = engine.BatchedSolver(c, maps, b, method, tolerance=tol, history_len=6)
        sv.run(6, check_every=6, use_graph=False)
        results[name] = (sv.x.clone(), sv.history.clone(), sv.iterations.clone())
    for name in ALL_FP_VARIANTS:
        for got, want in zip(results[name], results["ldg"]):
            assert torch.equal(got, want), name
    if method != "pdhg":
        assert int(results["ldg"][2][1]) == 3


def test_finite_surface_detectors_match_reference(cuda):
    """A 10 mm^2 detector (3 emitted sub-angles) next to a point detector, against the reference's
    own AttenuationVolume: through the core and through AttenuationVolume with DetectorXRF."""
    import os

    from conftest import GOLDEN
    from pycorrectedemissionct_b200 import attenuation, core

    g = dict(np.load(os.path.join(GOLDEN, "surface_case.npz")))
    rad32 = np.array(g["angles"], dtype=np.float32)
    maps = core.compute_maps(_t(g["mu_in"], cuda)[None], _t(g["mu_out"], cuda)[None], rad32, g["det_angles"],
                             surfaces_mm2=g["det_surfaces"], distances_mm=g["det_distances"],
                             sub_sampling=int(g["sub_sampling"]))
    assert rel_l2(maps[0].cpu().numpy(), g["maps"]) < TOL
    dets = [attenuation.DetectorXRF(surface_mm2=float(s_), distance_mm=float(d_), angle_rad=float(a_))
            for s_, d_, a_ in zip(g["det_surfaces"], g["det_distances"], g["det_angles"])]
    av = attenuation.AttenuationVolume(g["mu_in"], g["mu_out"], rad32, dets, emitted_sub_sampling=int(g["sub_sampling"]),
                                       device=cuda)
    av.compute_maps(verbose=False)
    assert rel_l2(av.maps, g["maps"]) < TOL
    c = core.XrfCore(int(g["n"]), g["angles"], n_det=2, device=cuda)
    fp = c.fp(_t(g["x"], cuda)[None], maps)[0].cpu().numpy()
    assert rel_l2(fp, g["fp_att"]) < TOL
