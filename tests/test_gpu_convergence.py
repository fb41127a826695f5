"""GPU: the solvers converge on consistent data — the reference's own solver test adapted to this
path (corrct ``tests/test_solvers.py:124-170``: a flat object, ``processing.circular_mask(shape, -2)``,
noise-free data, every solution within 1e-2 of the object).  The reference builds a random dense
``ProjectorMatrix``; here the operator is the attenuated XRF projector of a 16x16 slice over 64
angles of a full turn, and the comparison covers the inscribed circle.  That operator is far less
well conditioned near the circle's edge: unconstrained SIRT (2500 iterations) stays 0.10 away at
the object's rim and unconstrained KL-PDHG (500) oscillates by up to 3, in the oracle port as on
the GPU, so those two cases are checked against the port over long runs instead, and the
constrained cases (limits [0, 1]) against the object."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N, N_ANG = 16, 64
TOLERANCE = 1e-2


@pytest.fixture(scope="module")
def flat_case():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pycorrectedemissionct_b200 import phantoms, projectors

    c = (N - 1) / 2
    yy, xx = np.mgrid[:N, :N]
    r = np.hypot(yy - c, xx - c)
    vol = (r <= N / 2 - 2).astype(np.float32)  # circular_mask(shape, -2)
    mu = phantoms.disk_attenuation(N, phantoms.slice_rng(606, 0), 0.05)
    p = projectors.ProjectorAttenuationXRF((N, N), phantoms.angles(N_ANG), att_in=mu, att_out=0.7 * mu)
    data = p.fp(vol)
    inside = r <= N / 2 - 1
    return p, vol, data, inside


CASES = [
    ("PDHG", 500, dict(data_term="kl", regularizer=1e-4), dict(lower_limit=0, upper_limit=1)),
    ("FISTA", 1_000, {}, dict(lower_limit=0, upper_limit=1)),
    ("MLEM", 10_000, {}, dict(lower_limit=0, upper_limit=1)),
]


@pytest.mark.parametrize("name,iterations,init,call", CASES)
def test_flat_object(flat_case, name, iterations, init, call):
    from pycorrectedemissionct_b200 import solvers

    p, vol, data, inside = flat_case
    sol, info = getattr(solvers, name)(**init)(p, data, iterations=iterations, **call)
    dev = np.abs(sol - vol)[inside]
    assert np.all(np.isfinite(sol))
    assert dev.max() < TOLERANCE, (name, float(dev.max()))


def test_unconstrained_long_runs_match_the_port(flat_case):
    from oracle import port
    from pycorrectedemissionct_b200 import phantoms, solvers

    p, vol, data, inside = flat_case
    rad32, deg32 = port.backend_angles(phantoms.angles(N_ANG))
    mu = phantoms.disk_attenuation(N, phantoms.slice_rng(606, 0), 0.05)
    maps = port.compute_maps(mu, 0.7 * mu, rad32)
    fp = lambda v: port.fp_xrf(v, maps, deg32)  # noqa: E731
    bp = lambda s: port.bp_xrf(s, maps, deg32)  # noqa: E731
    b = fp(vol.astype(np.float64))
    xs, _ = solvers.SIRT()(p, data, iterations=500)
    ref = port.sirt(fp, bp, b, 500, (N, N))
    assert np.linalg.norm(xs - ref) / np.linalg.norm(ref) < 1e-4
    xp, _ = solvers.PDHG(data_term="kl", regularizer=1e-4)(p, data, iterations=200)
    ref = port.pdhg_kl_tv(fp, bp, b, 200, (N, N), 1e-4)
    assert np.linalg.norm(xp - ref) / np.linalg.norm(ref) < 1e-3
