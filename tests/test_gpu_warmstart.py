"""GPU: the learned warm start end to end at a small size — pairs from the GPU MLEM, training with
the project's tensor-core kernels, and what the trained network gains: warm-started MLEM reaches
the plain solver's final KL residual in fewer total iterations (including the 10 iterations the
network consumes) on held-out seeds, and the plain solver remains the judge of that residual."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pass_angles", [0, 6])
def test_warm_start_gains_over_plain_mlem(pass_angles):
    """pass_angles 0: inputs are the first 10 MLEM iterates; 6: 10 snapshots of one
    ordered-subsets pass over 10 subsets of 6 angles (the data in that pass's angle order)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pycorrectedemissionct_b200 import train_warmstart as tw
    from pycorrectedemissionct_b200.engine import BatchedSolver
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    dev = torch.device("cuda", 0)
    n, n_ang, plain_its = 64, 60, 100
    net = WarmStartNet(seed=1, device=dev)
    net.multiplicative = True
    net.pass_angles = pass_angles
    inputs, targets = tw.generate_pairs(96, n, n_ang, seed=5000, batch=48, target_iterations=plain_its, device=dev, net=net)
    losses = tw.train(net, inputs, targets, steps=300, batch=16, lr=2e-3, verbose=False, log_every=50)
    assert losses[-1] < 0.9 * losses[0]

    seeds = [90000 + k for k in range(8)]
    c, maps, b, _ = tw.synth_batch(n, n_ang, seeds, 0.02, 1e4, dev, subsets=net.pass_subsets(n_ang))
    plain = BatchedSolver(c, maps, b, "mlem", history_len=plain_its)
    plain.run(plain_its, check_every=plain_its, use_graph=False)
    tol = plain.residuals.cpu().numpy() * (1 + 1e-9)
    solver, total = tw.warm_started_solve(net, c, maps, b, tol, max_iterations=2 * plain_its)
    assert int(solver.active.sum()) == 0  # every slice reached the plain solver's final residual
    assert np.all(solver.residuals.cpu().numpy() <= tol)
    # the small network trained for seconds must at least not cost more than the plain solve
    assert total.mean() <= plain_its + 10, total
