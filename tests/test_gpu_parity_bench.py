"""GPU parity at the benchmark shapes against the FP64 oracle port.

The headline workload is 512 x 512 slices over 720 angles (maps mu in [0, 0.01], mu_out = mu_in),
the multi-channel workload 1024 x 1024 over 1440 angles with emitted scales up to 3.  The port
would take minutes per slice for every angle, so each case takes an evenly spaced subset of the
full angle set (the maps, fp and bp of an angle depend only on that angle and n), and the solver
case a reduced angle count.  Bounds (relative L2, FP32 GPU vs FP64 oracle): maps, fp and bp
1e-5; 10 MLEM iterations 1e-4.  Each case prints its error (and appends it to
$CCT_PARITY_REPORT when set).
"""

import numpy as np
import pytest

from conftest import rel_l2, report

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_RECON = 1e-4


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _t(a, cuda, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda, dtype)


@pytest.mark.parametrize("n,n_full,step,mu_max", [(512, 720, 8, 0.01), (1024, 1440, 40, 0.02)])
def test_maps_fp_bp_at_benchmark_shape(n, n_full, step, mu_max, cuda):
    """Maps (with half-turn pairs), attenuated fp (every fp variant) and the reference and
    symmetric back projections of one benchmark slice on every `step`-th angle of the full set."""
    from oracle import port
    from pycorrectedemissionct_b200 import _lib, core, phantoms

    rng = phantoms.slice_rng(20240, 0)
    x = phantoms.ellipse_phantom(n, rng, 12, dtype=np.float64)
    mu = phantoms.disk_attenuation(n, rng, mu_max, dtype=np.float64)
    angles = phantoms.angles(n_full)[::step]
    rad32, deg32 = port.backend_angles(angles)
    ref_maps = port.compute_maps(mu, mu, rad32, workers=16)
    maps = core.compute_maps(_t(mu, cuda)[None], _t(mu, cuda)[None], rad32)
    e = rel_l2(maps[0].cpu().numpy(), ref_maps)
    report(f"maps {n}x{len(angles)}/{n_full}", e, TOL)
    assert e < TOL
    c = core.XrfCore(n, angles, device=cuda)
    ref_fp = port.fp_xrf(x, ref_maps, deg32, workers=16)
    xs = _t(x, cuda)[None].repeat(4, 1, 1)  # four identical slices: the two-slice variant sees full pairs
    m32 = _t(ref_maps, cuda)[None].repeat(4, 1, 1, 1, 1)
    for v in (0, _lib.CCT_VARIANT_FP_TMA, _lib.CCT_VARIANT_FP_SLICES2):
        c.variant = v
        fp = c.fp(xs, m32)[:, 0].cpu().numpy()
        for k in range(4):
            e = rel_l2(fp[k], ref_fp)
            assert e < TOL, (v, k, e)
    report(f"fp {n}x{len(angles)}/{n_full}", e, TOL)
    # the whole chain: GPU maps into the GPU fp, against the FP64 maps into the FP64 fp
    e = rel_l2(c.fp(_t(x, cuda)[None], maps)[0, 0].cpu().numpy(), ref_fp)
    report(f"maps+fp {n}x{len(angles)}/{n_full}", e, TOL)
    assert e < TOL
    y = ref_fp / ref_fp.max()
    ref_bp = port.bp_uncorrected(y, deg32, n, workers=16)
    e = rel_l2(c.bp(_t(y, cuda)[None, None], "reference")[0].cpu().numpy(), ref_bp)
    report(f"bp {n}x{len(angles)}/{n_full}", e, TOL)
    assert e < TOL
    ref_bs = port.bp_xrf(y, ref_maps, deg32, is_symmetric=True, workers=16)
    e = rel_l2(c.bp(_t(y, cuda)[None, None], "symmetric", _t(ref_maps, cuda)[None])[0].cpu().numpy(), ref_bs)
    report(f"bp symmetric {n}x{len(angles)}/{n_full}", e, TOL)
    assert e < TOL


def test_quarter_turn_maps_at_512(cuda):
    """Maps of the benchmark slice from quarter-turn quads (mu_out = mu_in, detector at pi / 2) on
    every 10th of 720 angles (a set closed under the quarter turn) against the FP64 port."""
    from oracle import port
    from pycorrectedemissionct_b200 import core, phantoms

    n = 512
    rng = phantoms.slice_rng(20240, 2)
    phantoms.ellipse_phantom(n, rng, 12)
    mu = phantoms.disk_attenuation(n, rng, 0.01, dtype=np.float64)
    rad32, _ = port.backend_angles(phantoms.angles(720)[::10])
    ref = port.compute_maps(mu, mu, rad32, workers=16)
    m = _t(mu, cuda)[None]
    e = rel_l2(core.compute_maps(m, m, rad32)[0].cpu().numpy(), ref)
    report(f"maps from quarter-turn quads 512x{len(rad32)}/720", e, TOL)
    assert e < TOL


def test_channel_fields_at_1024(cuda):
    """Multi-channel workload: line-integral fields of one 1024 x 1024 slice, channels with emitted
    scales 1 and 3 (mu_out,c = s_c mu_in), on every 60th of 1440 angles: the channel maps
    exp(-(L_in + s_c L_out)) and the fp read from the fields against the FP64 port run with
    mu_out = s_c mu_in."""
    from oracle import port
    from pycorrectedemissionct_b200 import core, phantoms

    n = 1024
    rng = phantoms.slice_rng(777, 3)
    x = phantoms.ellipse_phantom(n, rng, 12, dtype=np.float64)
    mu = phantoms.disk_attenuation(n, rng, 0.01, dtype=np.float64)
    angles = phantoms.angles(1440)[::60]
    rad32, deg32 = port.backend_angles(angles)
    fields = core.compute_maps(_t(mu, cuda)[None], _t(mu, cuda)[None], rad32, maps_dtype="fields-float32")
    f = fields[0].double().cpu().numpy()  # (A, 2, n, n): L_in, L_out
    c = core.XrfCore(n, angles, device=cuda)
    scales = [1.0, 3.0]
    c.set_channels(scales)
    fp = c.fp(_t(x, cuda)[None].repeat(2, 1, 1), fields)[:, 0].cpu().numpy()
    for k, sc in enumerate(scales):
        ref_maps = port.compute_maps(mu, sc * mu, rad32, workers=16)
        got = np.exp(-(f[:, 0] + np.float32(sc) * f[:, 1]))[:, None]
        e = rel_l2(got, ref_maps)
        report(f"channel maps s_c={sc} 1024x{len(angles)}/1440", e, TOL)
        assert e < TOL
        e = rel_l2(fp[k], port.fp_xrf(x, ref_maps, deg32, workers=16))
        report(f"channel fp s_c={sc} 1024x{len(angles)}/1440", e, TOL)
        assert e < TOL


def test_mlem_at_512(cuda):
    """Ten fused MLEM iterations on one 512 x 512 benchmark slice over 90 angles (the drop-in
    projector and solver) against the FP64 port's MLEM with the FP64 maps."""
    from oracle import port
    from pycorrectedemissionct_b200 import projectors, phantoms, solvers

    n = 512
    rng = phantoms.slice_rng(20240, 1)
    x = phantoms.ellipse_phantom(n, rng, 12, dtype=np.float64)
    mu = phantoms.disk_attenuation(n, rng, 0.01, dtype=np.float64)
    angles = phantoms.angles(720)[::8]
    rad32, deg32 = port.backend_angles(angles)
    ref_maps = port.compute_maps(mu, mu, rad32, workers=16)
    clean = port.fp_xrf(x, ref_maps, deg32, workers=16)
    b = np.random.default_rng(5).poisson(clean / clean.max() * 1e5).astype(np.float64)
    fp = lambda v: port.fp_xrf(v, ref_maps, deg32, workers=16)  # noqa: E731
    bp = lambda s: port.bp_xrf(s, ref_maps, deg32, workers=16)  # noqa: E731
    x_ref, _ = port.mlem(fp, bp, b, 10)
    p = projectors.ProjectorAttenuationXRF((n, n), angles, att_maps=ref_maps.astype(np.float32))
    x_gpu, info = solvers.MLEM(tolerance=0.0)(p, b.astype(np.float32), iterations=10)
    e = rel_l2(x_gpu, x_ref)
    report("mlem(10) 512x90/720", e, TOL_RECON)
    assert e < TOL_RECON
    assert info.iterations == 10
