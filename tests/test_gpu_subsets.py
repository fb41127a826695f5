"""GPU: ordered-subsets EM passes (the non-learned warm start) against the oracle port.

One subset is plain MLEM (bit-identical iterates); k subsets apply the MLEM update of every
subset of angles in turn, which the port computes with its own fp / bp restricted to the
subset (1e-4 rel-L2 after the passes, the reconstruction bar); MLEM started from the passes
reaches a plain-MLEM residual in fewer full-data passes than from a cold start.
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


def _problem(n, n_ang, seed, cuda, perm=None):
    from pycorrectedemissionct_b200 import core, phantoms

    rng = phantoms.slice_rng(seed, 0)
    x = phantoms.ellipse_phantom(n, rng, 8)
    mu = phantoms.disk_attenuation(n, rng, 0.02)
    angles = phantoms.angles(n_ang)
    if perm is not None:
        angles = angles[perm]
    c = core.XrfCore(n, angles, device=cuda)
    mu_t = torch.from_numpy(mu).to(cuda)[None]
    maps = core.compute_maps(mu_t, 0.7 * mu_t, c.angles_rad32)
    clean = c.fp(torch.from_numpy(x).to(cuda)[None], maps)
    b = torch.from_numpy(np.random.default_rng(seed).poisson(clean.cpu().numpy() / float(clean.max()) * 1e4)
                         .astype(np.float32)).to(cuda)
    return c, maps, b


def test_one_subset_is_mlem(cuda):
    from pycorrectedemissionct_b200 import engine

    c, maps, b = _problem(48, 20, 5, cuda)
    os_ = engine.OrderedSubsets(c, maps, b, [(1, 6)])
    x_os = os_.run().clone()
    ml = engine.BatchedSolver(c, maps, b, "mlem")
    for _ in range(6):
        ml.step()
    assert torch.equal(x_os, ml.x)


def test_subset_passes_match_port(cuda):
    from oracle import port
    from pycorrectedemissionct_b200 import engine

    n, n_ang, levels = 40, 24, [(6, 2), (3, 1), (1, 1)]
    perm = engine.subset_permutation(n_ang, [k for k, _ in levels])
    c, maps, b = _problem(n, n_ang, 9, cuda, perm)
    x = engine.OrderedSubsets(c, maps, b, levels).run(use_graph=False).cpu().numpy()[0]
    maps_np = maps[0].double().cpu().numpy()
    b_np = b[0, 0].double().cpu().numpy()
    _, deg32 = port.backend_angles(c.angles_rad32)
    ref = np.ones((n, n))
    for k, passes in levels:
        per = n_ang // k
        for _ in range(passes):
            for m in range(k):
                rng = slice(m * per, (m + 1) * per)
                fp = lambda v, rng=rng: port.fp_xrf(v, maps_np[rng], deg32[rng])  # noqa: E731
                bp = lambda s, rng=rng: port.bp_xrf(s, maps_np[rng], deg32[rng])  # noqa: E731
                ref, _ = port.mlem(fp, bp, b_np[rng], 1, x0=ref)
    assert rel_l2(x, ref) < 1e-4


def test_subsets_then_mlem_reach_the_residual_sooner(cuda):
    from pycorrectedemissionct_b200 import engine

    n, n_ang = 64, 60
    c0, maps0, b0 = _problem(n, n_ang, 21, cuda)
    plain = engine.BatchedSolver(c0, maps0, b0, "mlem")
    plain.run(100, check_every=100, use_graph=False)
    tol = plain.residuals.cpu().numpy() * (1 + 1e-9)
    levels = [(10, 4), (5, 4)]
    perm = engine.subset_permutation(n_ang, [k for k, _ in levels])
    c, maps, _ = _problem(n, n_ang, 21, cuda, perm)
    b = b0[:, :, torch.from_numpy(perm).to(cuda)].contiguous()
    os_ = engine.OrderedSubsets(c, maps, b, levels)
    x0 = os_.run()
    judge = engine.BatchedSolver(c, maps, b, "mlem", tolerance=tol, x0=x0)
    judge.run(100, check_every=1, use_graph=False)
    its = int(judge.iterations[0].item())
    assert int(judge.active[0].item()) == 0
    assert os_.passes + its < 100 / 2
