"""GPU: the ragged stream — jobs of different sizes, angle counts and methods packed in waves,
each operator one ragged launch per wave — against solving every job on its own.

SIRT jobs and cold-started MLEM jobs must equal their single-job solves bit for bit; with the
ordered-subsets warm start every MLEM job must reach its tolerance (the residual of 60 plain
MLEM iterations) in fewer passes.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(48, 30, "mlem"), (64, 37, "sirt"), (48, 45, "mlem"), (64, 30, "mlem"), (40, 45, "sirt"),
          (48, 30, "mlem"), (64, 37, "mlem"), (40, 33, "sirt")]


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _jobs(cuda):
    from pycorrectedemissionct_b200 import core, engine, phantoms, stream

    jobs, singles = [], []
    for k, (n, n_ang, method) in enumerate(SHAPES):
        r = phantoms.slice_rng(5150, k)
        x = phantoms.ellipse_phantom(n, r, 6)
        mu = phantoms.disk_attenuation(n, r, 0.03)
        angles = np.linspace(0, 2 * np.pi, n_ang, endpoint=False)
        c = core.XrfCore(n, angles, device=cuda)
        mu_t = torch.from_numpy(mu).to(cuda)[None]
        maps = core.compute_maps(mu_t, 0.7 * mu_t, c.angles_rad32)
        clean = c.fp(torch.from_numpy(x).to(cuda)[None], maps)
        b = np.random.default_rng(k).poisson(clean[0, 0].cpu().numpy() / float(clean.max()) * 3e3).astype(np.float32)
        bt = torch.from_numpy(b).to(cuda)[None, None]
        job = stream.Job(n, angles, mu, 0.7 * mu, b, method=method, iterations=20)
        if method == "mlem":
            probe = engine.BatchedSolver(c, maps, bt, "mlem")
            probe.run(60, check_every=60, use_graph=False)
            job.tolerance = float(probe.residuals[0].item()) * (1 + 1e-9)
            single = engine.BatchedSolver(c, maps, bt, "mlem", tolerance=[job.tolerance])
            single.run(200, check_every=1, use_graph=False)
        else:
            single = engine.BatchedSolver(c, maps, bt, "sirt")
            for _ in range(20):
                single.step()
        torch.cuda.synchronize(cuda)
        jobs.append(job)
        singles.append(single)
    return jobs, singles


def test_cold_stream_equals_single_solves(cuda):
    from pycorrectedemissionct_b200 import stream

    jobs, singles = _jobs(cuda)
    # a small memory budget forces several waves
    st = stream.RaggedStream(cuda, memory_budget=2 << 20, warm_start=False, check_every=1)
    res = st.solve(jobs, max_iterations=200)
    assert res["slices"] == len(jobs) and res["p50_s"] <= res["p99_s"]
    assert len(st.waves(jobs)) > 1
    for job, single in zip(jobs, singles):
        np.testing.assert_array_equal(job.x, single.x[0].cpu().numpy())
        if job.method == "mlem":
            assert job.iterations_done == int(single.iterations[0].item())
        assert job.finished_s > 0


def test_warm_stream_reaches_tolerances_sooner(cuda):
    from pycorrectedemissionct_b200 import stream

    jobs, singles = _jobs(cuda)
    st = stream.RaggedStream(cuda, schedule=((10, 3), (5, 2)), check_every=1)
    st.solve(jobs, max_iterations=200)
    for job, single in zip(jobs, singles):
        if job.method != "mlem":
            continue
        assert job.extra["residual"] <= job.tolerance
        assert job.iterations_done < int(single.iterations[0].item())


def test_learned_stream_reaches_tolerances(cuda):
    """The learned start inside the stream (one network evaluation per MLEM group): every MLEM job
    still reaches its tolerance, and its pass count includes the start's three passes."""
    import os

    from pycorrectedemissionct_b200 import stream
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    weights = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pycorrectedemissionct_b200",
                           "weights", "warmstart.pt")
    if not os.path.exists(weights):
        pytest.skip("no committed warm-start weights")
    net = WarmStartNet(device=cuda)
    net.load(weights)
    jobs, singles = _jobs(cuda)
    st = stream.RaggedStream(cuda, warm_start="learned", net=net, check_every=1)
    st.solve(jobs, max_iterations=200)
    learned, cold = [], []
    for job, single in zip(jobs, singles):
        if job.method != "mlem":
            continue
        assert job.extra["residual"] <= job.tolerance
        assert job.iterations_done >= 3
        learned.append(job.iterations_done)
        cold.append(int(single.iterations[0].item()))
    print(f"learned start in the stream: passes {learned}, cold {cold}")
    with pytest.raises(ValueError):
        stream.RaggedStream(cuda, warm_start="learned")
