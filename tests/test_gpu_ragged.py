"""GPU: ragged batches — one launch per operator over groups of slices with different sizes,
angle counts and detectors (``cct_ragged_step``) — against stepping every group on its own.

The ragged kernels run the same per-CTA code as the uniform ones, so iterates, residual
histories, iteration counts and stopping flags must be bit-identical, also when some slices meet
their tolerance part-way and stop while others go on.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# (n, angles, slices, detectors)
GROUPS = [(64, 30, 2, 1), (96, 45, 1, 1), (40, 17, 3, 2), (128, 90, 1, 1), (33, 12, 2, 1)]


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _group(n, n_ang, s, d, seed, cuda, maps_dtype="float32"):
    from pycorrectedemissionct_b200 import core, phantoms

    det = [np.pi / 2, np.pi / 3][:d]
    w = np.random.default_rng(seed).uniform(0.5, 1.5, size=(n_ang, d)) if d > 1 else None
    c = core.XrfCore(n, phantoms.angles(n_ang), n_det=d, weights=w, device=cuda)
    xs, mus = [], []
    for k in range(s):
        rng = phantoms.slice_rng(seed, k)
        xs.append(phantoms.ellipse_phantom(n, rng, 6))
        mus.append(phantoms.disk_attenuation(n, rng, 0.03))
    mu = torch.from_numpy(np.stack(mus)).to(cuda)
    maps = core.compute_maps(mu, 0.7 * mu, c.angles_rad32, det, maps_dtype=maps_dtype)
    clean = c.fp(torch.from_numpy(np.stack(xs)).to(cuda), maps)
    gen = torch.Generator(device=cuda)
    gen.manual_seed(seed)
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * 2e3, generator=gen)
    return c, maps, b


def _pairs(method, cuda, maps_dtype="float32", iterations=14):
    from pycorrectedemissionct_b200 import engine

    singles, raggeds = [], []
    for gi, (n, n_ang, s, d) in enumerate(GROUPS):
        c, maps, b = _group(n, n_ang, s, d, 300 + gi, cuda, maps_dtype)
        # tolerances between the residuals of two iterations so some slices stop early
        probe = engine.BatchedSolver(c, maps, b, method, history_len=iterations)
        for _ in range(iterations):
            probe.step()
        h = probe.history.cpu().numpy()
        stop = [min(iterations - 1, 3 + (gi + k) % 8) for k in range(s)]
        tol = np.array([0.5 * (h[k, i - 1] + h[k, i]) for k, i in enumerate(stop)])
        if gi % 2 == 1:
            tol = None  # some groups run without a tolerance
        kw = dict(tolerance=tol, history_len=iterations)
        singles.append(engine.BatchedSolver(c, maps, b, method, **kw))
        raggeds.append(engine.BatchedSolver(c, maps, b, method, **kw))
    rag = engine.RaggedSolvers(raggeds)
    for _ in range(iterations):
        for sv in singles:
            sv.step()
        rag.step()
    torch.cuda.synchronize(cuda)
    return singles, raggeds


@pytest.mark.parametrize("method", ["mlem", "sirt"])
def test_ragged_equals_separate_steps(method, cuda):
    singles, raggeds = _pairs(method, cuda)
    stopped = 0
    for a, b in zip(singles, raggeds):
        assert torch.equal(a.x, b.x)
        assert torch.equal(a.history, b.history)
        assert torch.equal(a.iterations, b.iterations)
        assert torch.equal(a.active, b.active)
        stopped += int((a.active == 0).sum().item())
    assert stopped > 0  # the case exercises early stops


def test_ragged_bf16_maps(cuda):
    singles, raggeds = _pairs("mlem", cuda, maps_dtype="bfloat16", iterations=6)
    for a, b in zip(singles, raggeds):
        assert torch.equal(a.x, b.x)


def test_ragged_rejects_mixed_groups(cuda):
    from pycorrectedemissionct_b200 import engine

    c1, m1, b1 = _group(48, 10, 1, 1, 1, cuda)
    c2, m2, b2 = _group(48, 10, 1, 1, 2, cuda, maps_dtype="bfloat16")
    with pytest.raises(NotImplementedError):
        engine.RaggedSolvers([engine.BatchedSolver(c1, m1, b1, "mlem"), engine.BatchedSolver(c2, m2, b2, "mlem")])
    with pytest.raises(ValueError):
        engine.RaggedSolvers([engine.BatchedSolver(c1, m1, b1, "mlem"), engine.BatchedSolver(c1, m1, b1, "sirt")])
