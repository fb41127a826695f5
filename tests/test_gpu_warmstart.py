"""GPU: the learned warm start.

1. The training path end to end at a small size: pairs from the GPU MLEM, a few hundred steps with
   the project's tensor-core kernels, and the learned start + MLEM reaching the plain solver's
   final KL residual on held-out seeds (the plain solver judges every slice).
2. What the committed network gains: on held-out textured slices (textured phantoms, mu up to 0.02,
   1e4 peak counts, 256 x 256 over 360 angles), the learned start (a snapshot ordered-subsets pass,
   the network, one pass per ordered-subsets level) followed by MLEM needs at most half the
   full-data passes of plain MLEM to reach plain MLEM's 200-iteration KL residual, and fewer than
   the same ordered-subsets passes without the network.
3. The learned start as PDHG's x0: PDHG-KL-TV reaches plain PDHG's 200-iteration data residual in
   at most half the passes.
"""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pycorrectedemissionct_b200",
                       "weights", "warmstart.pt")


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def test_training_path_and_learned_start(cuda):
    from pycorrectedemissionct_b200 import train_warmstart as tw
    from pycorrectedemissionct_b200.engine import BatchedSolver
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    n, n_ang, plain_its = 64, 80, 100
    net = WarmStartNet(seed=1, device=cuda)
    net.multiplicative = True
    net.pass_angles = 8
    levels = net.os_levels(n_ang)
    assert levels == [10, 2]
    inputs, targets = tw.generate_pairs(96, n, n_ang, seed=5000, batch=48, target_iterations=plain_its, device=cuda,
                                        net=net)
    losses = tw.train(net, inputs, targets, steps=300, batch=16, lr=2e-3, verbose=False, log_every=50)
    assert losses[-1] < 0.9 * losses[0]

    seeds = [90000 + k for k in range(8)]
    c, maps, b, _ = tw.synth_batch(n, n_ang, seeds, 0.02, 1e4, cuda, subsets=levels)
    plain = BatchedSolver(c, maps, b, "mlem")
    plain.run(plain_its, check_every=plain_its, use_graph=False)
    tol = plain.residuals.cpu().numpy() * (1 + 1e-9)
    solver, total = tw.warm_started_solve(net, c, maps, b, tol, max_iterations=2 * plain_its)
    assert int(solver.active.sum()) == 0  # every slice reached the plain solver's final residual
    assert np.all(solver.residuals.cpu().numpy() <= tol)
    assert np.all(total >= 3)  # the three ordered-subsets passes are counted


def test_committed_network_gains_over_the_method_without_it(cuda):
    if not os.path.exists(WEIGHTS):
        pytest.skip("no committed warm-start weights")
    from pycorrectedemissionct_b200 import train_warmstart as tw
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    net = WarmStartNet(device=cuda)
    net.load(WEIGHTS)
    assert net.os_levels(360) == [45, 9]
    r = tw.evaluate(net, 256, 360, 16, seed=970_000, batch=16, device=cuda)
    print(f"learned start: {r['learned_mean']:.1f} passes (max {r['learned_max']}), without the network "
          f"{r['without_network_mean']:.1f} (max {r['without_network_max']}), plain {r['plain_passes']}")
    assert r["reached_residual"] == 16
    assert r["learned_mean"] <= 0.5 * r["plain_passes"]
    assert r["learned_mean"] < r["without_network_mean"]


def test_committed_network_warm_starts_pdhg(cuda):
    """The learned start as PDHG's x0 (corrct's hook): on held-out textured slices (256 x 256, 360
    angles), PDHG-KL-TV from the learned start reaches the data residual that plain PDHG (zero
    start) reaches after 200 iterations in at most half the full-data passes."""
    if not os.path.exists(WEIGHTS):
        pytest.skip("no committed warm-start weights")
    from pycorrectedemissionct_b200 import train_warmstart as tw
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    net = WarmStartNet(device=cuda)
    net.load(WEIGHTS)
    r = tw.evaluate_pdhg(net, 256, 360, 8, seed=975_000, batch=8, device=cuda)
    print(f"PDHG from the learned start: {r['learned_mean']:.1f} passes (max {r['learned_max']}), without the "
          f"network {r['without_network_mean']:.1f}, plain {r['plain_iterations']}")
    assert r["reached_residual"] == 8
    assert r["learned_mean"] <= 0.5 * r["plain_iterations"]
