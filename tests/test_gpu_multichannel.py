"""GPU: multi-channel XRF (several fluorescence lines per slice) as batched channel-slices.

Each channel has its own emission phantom and emitted attenuation mu_out,c = s_c * mu_in with
s_c in {0.5, 0.75, 1, 1.25, 1.5, 2, 2.5, 3}, sharing the incident attenuation of its slice; the
channels of all slices are one batch of the fused kernels.  Checks against the oracle port per
channel: maps and fp (1e-5 rel-L2) and 10 PDHG iterations with the KL data term and isotropic TV,
lambda = 1e-2 (1e-4), plus the line-integral linearity the channel maps obey:
-log(map_c) = L_in + s_c L_out(mu_in).
"""

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SCALES = [0.5, 0.75, 1.0, 1.25, 1.5, 2.0, 2.5, 3.0]
N, A, SLICES = 48, 40, 2


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def batch(cuda):
    from pycorrectedemissionct_b200 import core, phantoms

    mus, xs, mu_in, mu_out = [], [], [], []
    for s in range(SLICES):
        rng = phantoms.slice_rng(9090, s)
        mu = phantoms.disk_attenuation(N, rng, 0.02)
        mus.append(mu)
        for c, sc in enumerate(SCALES):
            xs.append(phantoms.ellipse_phantom(N, phantoms.slice_rng(9191 + s, c), 8))
            mu_in.append(mu)
            mu_out.append(sc * mu)
    angles = phantoms.angles(A)
    cr = core.XrfCore(N, angles, device=cuda)
    t = lambda v: torch.from_numpy(np.stack(v).astype(np.float32)).to(cuda)  # noqa: E731
    maps = core.compute_maps(t(mu_in), t(mu_out), cr.angles_rad32)
    x = t(xs)
    clean = cr.fp(x, maps)
    rngp = np.random.default_rng(1)
    b = torch.from_numpy(rngp.poisson(clean.cpu().numpy() / float(clean.max()) * 1e4).astype(np.float32)).to(cuda)
    return cr, maps, x, b, mus, xs, angles


def test_channel_maps_and_fp(batch):
    from oracle import port

    cr, maps, x, b, mus, xs, angles = batch
    rad32, deg32 = port.backend_angles(angles)
    fp = cr.fp(x, maps).cpu().numpy()
    for idx in (0, 5, 8 + 7):
        s, c = divmod(idx, len(SCALES))
        mu = mus[s].astype(np.float64)
        ref_maps = port.compute_maps(mu, SCALES[c] * mu, rad32)
        assert rel_l2(maps[idx].cpu().numpy(), ref_maps) < 1e-5
        assert rel_l2(fp[idx, 0], port.fp_xrf(xs[idx].astype(np.float64), ref_maps, deg32)) < 1e-5


def test_channel_maps_are_linear_in_the_emitted_scale(batch):
    from pycorrectedemissionct_b200 import core

    cr, maps, *_ = batch
    mus = batch[4]
    # L_in from a map without emitted attenuation, L_out(mu_in) from one without incident
    mu = torch.from_numpy(mus[0]).to(maps.device)[None]
    l_in = -torch.log(core.compute_maps(mu, None, cr.angles_rad32).double())
    l_out = -torch.log(core.compute_maps(None, mu, cr.angles_rad32).double())
    for c, sc in enumerate(SCALES):
        got = -torch.log(maps[c].double())
        want = l_in[0] + sc * l_out[0]
        assert rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-5


def test_channel_pdhg_tv(batch):
    from oracle import port
    from pycorrectedemissionct_b200 import engine

    cr, maps, x, b, mus, xs, angles = batch
    solver = engine.BatchedSolver(cr, maps, b, "pdhg", tv_lambda=1e-2)
    for _ in range(10):
        solver.step()
    got = solver.x.cpu().numpy()
    _, deg32 = port.backend_angles(angles)
    for idx in (1, 8 + 3):
        m = maps[idx].double().cpu().numpy()
        fp = lambda v: port.fp_xrf(v, m, deg32)  # noqa: E731
        bp = lambda y: port.bp_xrf(y, m, deg32)  # noqa: E731
        ref = port.pdhg_kl_tv(fp, bp, b[idx, 0].double().cpu().numpy(), 10, (N, N), 1e-2)
        assert rel_l2(got[idx], ref) < 1e-4


@pytest.fixture(scope="module")
def fields_core(batch):
    from pycorrectedemissionct_b200 import core

    cr, maps, x, b, mus, xs, angles = batch
    cf = core.XrfCore(N, angles, device=maps.device)
    cf.set_channels(SCALES)
    mu = torch.from_numpy(np.stack(mus).astype(np.float32)).to(maps.device)
    fields = core.compute_maps(mu, mu, cf.angles_rad32, maps_dtype="fields-float32")
    return cf, fields


def test_fields_hold_the_line_integrals(batch, fields_core):
    from pycorrectedemissionct_b200 import core

    cf, fields = fields_core
    assert tuple(fields.shape) == (SLICES, A, 2, N, N)
    mu = torch.from_numpy(batch[4][1].astype(np.float32)).to(fields.device)[None]
    l_in = -torch.log(core.compute_maps(mu, None, cf.angles_rad32).double())[0, :, 0]
    l_out = -torch.log(core.compute_maps(None, mu, cf.angles_rad32).double())[0, :, 0]
    assert rel_l2(fields[1, :, 0].double().cpu().numpy(), l_in.cpu().numpy()) < 1e-5
    assert rel_l2(fields[1, :, 1].double().cpu().numpy(), l_out.cpu().numpy()) < 1e-5


def test_fields_projections_equal_channel_maps(batch, fields_core):
    """fp, symmetric / adjoint bp and MLEM with 2 fields per slice equal those with 8 channel maps."""
    from pycorrectedemissionct_b200 import engine

    cr, maps, x, b, *_ = batch
    cf, fields = fields_core
    assert rel_l2(cf.fp(x, fields).cpu().numpy(), cr.fp(x, maps).cpu().numpy()) < 1e-6
    y = cr.fp(x, maps)
    for mode in ("symmetric", "adjoint"):
        assert rel_l2(cf.bp(y, mode, fields).cpu().numpy(), cr.bp(y, mode, maps).cpu().numpy()) < 1e-6
    a = engine.BatchedSolver(cr, maps, b, "mlem")
    f = engine.BatchedSolver(cf, fields, b, "mlem")
    for _ in range(10):
        a.step()
        f.step()
    assert rel_l2(f.x.cpu().numpy(), a.x.cpu().numpy()) < 1e-5
    # angle ranges of fields (a view with a slice stride) as for maps
    sub = cf.angle_range(slice(5, 17))
    sub_ref = cr.angle_range(slice(5, 17))
    got = sub.fp(x, fields[:, 5:17], angles=None)
    assert rel_l2(got.cpu().numpy(), sub_ref.fp(x, maps[:, 5:17]).cpu().numpy()) < 1e-6
