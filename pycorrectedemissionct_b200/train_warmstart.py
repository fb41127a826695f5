"""Training pairs, training loop and warm-started solves for the MLEM warm-start network.

Pairs come from this package's own batched GPU MLEM on seeded synthetic slices (no dataset is
public on this path): textured phantoms (5-20 ellipses with a smooth Gaussian-random-field
texture, values in [0, 1]), disk attenuation (mu in [0, 0.02], emitted mu = 0.7 incident mu),
Poisson data.  Input = 10 snapshots of the iterate during one ordered-subsets pass over subsets of
``net.pass_angles`` angles (in the subset order of ``net.os_levels``) plus the normalised
back-projection A^T b / A^T 1, each slice divided by the mean of its last snapshot (with
``pass_angles`` 0: the first 10 MLEM iterates); target = the iterate after ``target_iterations``
MLEM iterations, as a correction to the last snapshot in the same units.

The learned start (``learned_start``): the snapshot pass, the network, then one more pass at each
of the two ordered-subsets levels; plain MLEM then finishes to the data-residual tolerance and
judges every slice.

The learned start also serves as PDHG's ``x0`` (``evaluate_pdhg``: passes until PDHG-KL-TV reaches
the data residual of plain PDHG after 200 iterations, from the learned start and without the
network).

Usage (GPU):  python -m pycorrectedemissionct_b200.train_warmstart --slices 20000 --steps 12000 --out w.pt
              python -m pycorrectedemissionct_b200.train_warmstart --weights w.pt --eval-slices 256 \
                  --eval-pdhg-slices 64
"""

from __future__ import annotations

import argparse
import ctypes
import time

import numpy as np
import torch

from . import _lib, core, phantoms
from .engine import BatchedSolver, OrderedSubsets, subset_permutation
from .warmstart import N_ITERATES, WarmStartNet


def textured_phantom(n: int, rng: np.random.Generator) -> np.ndarray:
    """5-20 ellipses modulated by a smooth Gaussian random field, clipped to [0, 1]."""
    base = phantoms.ellipse_phantom(n, rng, num_ellipses=int(rng.integers(5, 21)), dtype=np.float64)
    noise = rng.standard_normal((n, n))
    f = np.fft.fftfreq(n)
    k2 = f[:, None] ** 2 + f[None, :] ** 2
    sigma = 4.0 / n  # correlation length ~ n / 25 pixels
    grf = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-k2 / (2 * sigma**2))))
    grf /= max(grf.std(), 1e-12)
    img = np.where(base > 0, base * (1.0 + 0.25 * grf), 0.0)
    return np.clip(img, 0.0, 1.0).astype(np.float32)


def slice_means(x: torch.Tensor) -> torch.Tensor:
    """Per-slice mean of a (S, n, n) FP32 tensor with the FP64 norm kernel (x >= 0)."""
    return (core.reduce_norm(x.contiguous(), ord=1) / (x.shape[1] * x.shape[2])).float().clamp_min(1e-12)


def normalized_backprojection(c: core.XrfCore, b: torch.Tensor, tau: torch.Tensor) -> torch.Tensor:
    """A^T b / A^T 1 (reference back projection), (S, n, n)."""
    bp = c.bp(b, "reference")
    out = torch.empty_like(bp)
    _lib.check(_lib.load().cct_net_ratio(bp.data_ptr(), tau.data_ptr(), out.data_ptr(), bp.numel(), tau.numel(),
                                         core.stream_handle(c.device)))
    return out


def first_iterates(solver: BatchedSolver, count: int = N_ITERATES) -> list[torch.Tensor]:
    """Run `count` MLEM iterations, keeping a copy of every iterate."""
    its = []
    for _ in range(count):
        solver.step()
        its.append(solver.x.clone())
    return its


def pass_snapshots(os_: OrderedSubsets, count: int = N_ITERATES) -> list[torch.Tensor]:
    """One pass of a one-level ordered-subsets schedule of k subsets, keeping a copy of the
    iterate after every (k // count)-th subset step (the last one after the whole pass)."""
    subsets = os_.levels[0]
    k = len(subsets)
    stride = max(1, k // count)
    its = []
    for t, sm in enumerate(subsets):
        sm.step()
        if t + 1 == k or ((t + 1) % stride == 0 and len(its) < count - 1):
            its.append(os_.x.clone())
    while len(its) < count:
        its.append(os_.x.clone())
    return its


def synth_batch(n: int, n_angles: int, seeds: list[int], mu_max: float, peak: float, device, textured: bool = True,
                subsets=0, emitted_ratio: float = 0.7, return_mu: bool = False):
    """Phantoms, attenuation, maps and Poisson data for one batch of slices (angles in the
    ``subset_permutation`` order of ``subsets``, one count or a list of levels, when given).
    Returns (core, maps, b, x), and the incident mu as a fifth item with ``return_mu``."""
    xs, mus = [], []
    for sd in seeds:
        rng = phantoms.slice_rng(sd, 0)
        xs.append(textured_phantom(n, rng) if textured else phantoms.ellipse_phantom(n, rng, 12))
        mus.append(phantoms.disk_attenuation(n, rng, mu_max))
    angles = phantoms.angles(n_angles)
    levels = [subsets] if isinstance(subsets, int) else list(subsets)
    levels = [k for k in levels if k > 0]
    if levels:
        angles = angles[subset_permutation(n_angles, levels)]
    c = core.XrfCore(n, angles, device=device)
    mu = torch.from_numpy(np.stack(mus)).to(device)
    maps = core.compute_maps(mu, emitted_ratio * mu, c.angles_rad32)
    x = torch.from_numpy(np.stack(xs)).to(device)
    clean = c.fp(x, maps)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seeds[0]))
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * peak, generator=gen)
    if return_mu:
        return c, maps, b, x, mu
    return c, maps, b, x


def generate_pairs(n_slices: int, n: int = 256, n_angles: int = 360, seed: int = 100_000, batch: int = 64,
                   peak: float = 1e4, mu_max: float = 0.02, target_iterations: int = 500, device=None, net=None):
    """(inputs NHWC bf16 (N, n, n, 16), targets FP32 (N, n, n)) on the device."""
    device = core.require_cuda(device)
    helper = net if net is not None else WarmStartNet(device=device)
    inputs, targets = [], []
    levels = helper.os_levels(n_angles)
    for s0 in range(0, n_slices, batch):
        seeds = [seed + k for k in range(s0, min(n_slices, s0 + batch))]
        c, maps, b, _ = synth_batch(n, n_angles, seeds, mu_max, peak, device, subsets=levels)
        solver = BatchedSolver(c, maps, b, "mlem")
        if levels:
            its = pass_snapshots(OrderedSubsets(c, maps, b, [(levels[0], 1), (levels[1], 1)]))
            bpn = normalized_backprojection(c, b, solver.tau)
            solver.run(target_iterations, check_every=target_iterations, use_graph=False)
        else:
            its = first_iterates(solver)
            bpn = normalized_backprojection(c, b, solver.tau)
            solver.run(target_iterations - N_ITERATES, check_every=target_iterations, use_graph=False)
        scale = slice_means(its[-1])
        inputs.append(helper.pack(its + [bpn], scale))
        sc = scale[:, None, None]
        if helper.multiplicative:
            off = helper.log_floor * sc
            targets.append(torch.log((solver.x + off) / (its[-1] + off)).contiguous())
        else:
            targets.append(((solver.x - its[-1]) / sc).contiguous())
        del maps, solver
    return torch.cat(inputs), torch.cat(targets)


def train(net: WarmStartNet, inputs: torch.Tensor, targets: torch.Tensor, steps: int, batch: int = 16,
          lr: float = 1e-3, seed: int = 0, log_every: int = 100, verbose: bool = True) -> list[float]:
    """Adam on random mini-batches with random 90-degree rotations / flips; returns the logged losses."""
    rng = np.random.default_rng(seed)
    losses = []
    n = inputs.shape[0]
    for step in range(steps):
        idx = torch.from_numpy(rng.choice(n, size=min(batch, n), replace=False)).to(inputs.device)
        x = inputs.index_select(0, idx)
        t = targets.index_select(0, idx)
        k = int(rng.integers(4))
        if k:
            x = torch.rot90(x, k, dims=(1, 2)).contiguous()
            t = torch.rot90(t, k, dims=(1, 2)).contiguous()
        lr_t = lr * 0.5 * (1 + np.cos(np.pi * step / max(steps, 1)))  # cosine decay
        out = net.forward(x)
        net.zero_grad()
        loss, g = net.mse(out, t)
        net.backward(g)
        net.adam_step(lr=float(lr_t))
        if step % log_every == 0 or step == steps - 1:
            losses.append(float(loss.item()))
            if verbose:
                print(f"step {step:5d} loss {losses[-1]:.5f}", flush=True)
    return losses


def learned_start(net: WarmStartNet, os_: OrderedSubsets, c: core.XrfCore, b: torch.Tensor,
                  tau: torch.Tensor) -> torch.Tensor:
    """The learned start on an ordered-subsets solver whose levels are ``net.os_levels(A)`` (data in
    that order): one pass over the first level keeping 10 snapshots, the network on the snapshots
    and the normalised back projection (A^T b / tau), then one pass over each level from the
    network's prediction.  Three full-data passes and one network evaluation; returns the shared
    iterate."""
    its = pass_snapshots(os_)
    bpn = normalized_backprojection(c, b, tau)
    x0 = net.predict(its + [bpn], base=its[-1], slice_scale=slice_means(its[-1]))
    os_.x.copy_(x0)
    os_.run_level(0)
    os_.run_level(1)
    return os_.x


def warm_started_solve(net: WarmStartNet, c: core.XrfCore, maps: torch.Tensor, b: torch.Tensor, tolerance,
                       max_iterations: int = 400, check_every: int = 1, history_len: int = 0, use_net: bool = True):
    """The learned start (``learned_start``), then MLEM from it until `tolerance`; ``c``, ``maps`` and
    ``b`` in ``subset_permutation(A, net.os_levels(A))`` angle order.  With ``use_net`` False the
    network is skipped (the same three passes from the snapshot pass's end): the method without
    the network.  Networks fed the first 10 MLEM iterates (``pass_angles`` 0) run them instead.

    Returns (solver, total full-data passes per slice as a numpy array)."""
    first = BatchedSolver(c, maps, b, "mlem")
    levels = net.os_levels(c.n_angles)
    if levels:
        os_ = OrderedSubsets(c, maps, b, [(levels[0], 1), (levels[1], 1)])
        if use_net:
            x0 = learned_start(net, os_, c, b, first.tau)
        else:
            os_.run_level(0)
            os_.run_level(0)
            x0 = os_.run_level(1)
        passes = 3
    else:
        its = first_iterates(first)
        bpn = normalized_backprojection(c, b, first.tau)
        x0 = net.predict(its + [bpn], base=its[-1], slice_scale=slice_means(its[-1])) if use_net else its[-1]
        passes = N_ITERATES
    solver = BatchedSolver(c, maps, b, "mlem", tolerance=tolerance, x0=x0, history_len=history_len)
    solver.run(max_iterations, check_every=check_every, use_graph=False)
    return solver, solver.iterations.cpu().numpy() + passes


def evaluate(net: WarmStartNet, n: int, n_angles: int, n_slices: int, seed: int, batch: int = 32, device=None,
             plain_iterations: int = 200) -> dict:
    """Held-out evaluation on textured slices (mu up to 0.02, 1e4 peak counts): per slice, the full-data passes that plain
    MLEM (cold start), the learned start + MLEM, and the same passes without the network need to
    reach the KL residual plain MLEM reaches after ``plain_iterations`` iterations."""
    device = core.require_cuda(device)
    levels = net.os_levels(n_angles)
    learned, without, ok = [], [], 0
    for s0 in range(0, n_slices, batch):
        seeds = [seed + k for k in range(s0, min(n_slices, s0 + batch))]
        c, maps, b, _ = synth_batch(n, n_angles, seeds, 0.02, 1e4, device, subsets=levels)
        plain = BatchedSolver(c, maps, b, "mlem")
        plain.run(plain_iterations, check_every=plain_iterations, use_graph=False)
        tol = plain.residuals.cpu().numpy() * (1 + 1e-9)
        sv, total = warm_started_solve(net, c, maps, b, tol, max_iterations=2 * plain_iterations)
        ok += int((sv.residuals.cpu().numpy() <= tol).sum())
        learned.append(total)
        _, total0 = warm_started_solve(net, c, maps, b, tol, max_iterations=2 * plain_iterations, use_net=False)
        without.append(total0)
        del maps, plain, sv
    learned, without = np.concatenate(learned), np.concatenate(without)
    return {"n": n, "angles": n_angles, "slices": int(learned.size), "plain_passes": plain_iterations,
            "learned_mean": float(learned.mean()), "learned_max": int(learned.max()),
            "without_network_mean": float(without.mean()), "without_network_max": int(without.max()),
            "reached_residual": ok}


def evaluate_pdhg(net: WarmStartNet, n: int, n_angles: int, n_slices: int, seed: int, batch: int = 16, device=None,
                  plain_iterations: int = 200, tv_lambda: float = 1e-2) -> dict:
    """Held-out evaluation of the learned start as PDHG's ``x0`` (corrct's hook,
    ``solvers.py:1133-1137``): per slice, the full-data passes that PDHG-KL-TV needs to reach the
    data residual plain PDHG (zero start) reaches after ``plain_iterations`` iterations, from the
    learned start (its three ordered-subsets passes counted) and from the same passes without the
    network; PDHG stops on the reference's rule, ``tolerance > residual``."""
    device = core.require_cuda(device)
    levels = net.os_levels(n_angles)
    learned, without, ok = [], [], 0
    for s0 in range(0, n_slices, batch):
        seeds = [seed + k for k in range(s0, min(n_slices, s0 + batch))]
        c, maps, b, _ = synth_batch(n, n_angles, seeds, 0.02, 1e4, device, subsets=levels)
        plain = BatchedSolver(c, maps, b, "pdhg", tv_lambda=tv_lambda, tolerance=np.zeros(b.shape[0]))
        plain.run(plain_iterations, check_every=plain_iterations, use_graph=False)
        tol = plain.residuals.cpu().numpy() * (1 + 1e-9)
        del plain
        tau = BatchedSolver(c, maps, b, "mlem").tau
        for use_net, out in ((True, learned), (False, without)):
            os_ = OrderedSubsets(c, maps, b, [(levels[0], 1), (levels[1], 1)])
            if use_net:
                x0 = learned_start(net, os_, c, b, tau).clone()
            else:
                os_.run_level(0)
                os_.run_level(0)
                x0 = os_.run_level(1).clone()
            sv = BatchedSolver(c, maps, b, "pdhg", tv_lambda=tv_lambda, tolerance=tol, x0=x0)
            sv.run(2 * plain_iterations, check_every=1, use_graph=False)
            if use_net:
                ok += int((sv.residuals.cpu().numpy() <= tol).sum())
            out.append(sv.iterations.cpu().numpy() + 3)
        del maps
    learned, without = np.concatenate(learned), np.concatenate(without)
    return {"n": n, "angles": n_angles, "slices": int(learned.size), "plain_iterations": plain_iterations,
            "tv_lambda": tv_lambda, "learned_mean": float(learned.mean()), "learned_max": int(learned.max()),
            "without_network_mean": float(without.mean()), "without_network_max": int(without.max()),
            "reached_residual": ok}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--slices", type=int, default=20000)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--angles", type=int, default=360)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--target-iterations", type=int, default=500)
    ap.add_argument("--additive", action="store_true", help="additive instead of log-ratio (multiplicative) targets")
    ap.add_argument("--log-floor", type=float, default=1e-3, help="floor of the log-ratio target, in slice means")
    ap.add_argument("--pass-angles", type=int, default=8,
                    help="inputs: 10 snapshots of one ordered-subsets pass over subsets of this many angles "
                         "(0: the first 10 MLEM iterates)")
    ap.add_argument("--finish-factor", type=int, default=5)
    ap.add_argument("--eval-slices", type=int, default=0, help="held-out slices per evaluation shape")
    ap.add_argument("--eval-pdhg-slices", type=int, default=0,
                    help="held-out slices for the PDHG-KL-TV warm-start evaluation (at --n x --angles)")
    ap.add_argument("--weights", default=None, help="evaluate these weights instead of training")
    ap.add_argument("--out", default="warmstart.pt")
    a = ap.parse_args()
    dev = core.require_cuda()
    t0 = time.time()
    net = WarmStartNet(seed=0, device=dev)
    net.multiplicative = not a.additive
    net.log_floor = a.log_floor
    net.pass_angles = a.pass_angles
    net.finish_factor = a.finish_factor
    if a.weights is not None:
        net.load(a.weights)
        evaluate_all(net, a, dev)
        return
    inputs, targets = generate_pairs(a.slices, a.n, a.angles, target_iterations=a.target_iterations, device=dev,
                                     net=net, batch=128)
    torch.cuda.synchronize()
    t1 = time.time()
    print(f"pairs: {inputs.shape[0]} in {t1 - t0:.1f} s; params {net.n_params()}", flush=True)
    losses = train(net, inputs, targets, a.steps, a.batch, a.lr, log_every=1000)
    torch.cuda.synchronize()
    print(f"trained {a.steps} steps in {time.time() - t1:.1f} s; loss {losses[0]:.4f} -> {losses[-1]:.4f}", flush=True)
    v = ctypes.c_int32(0)
    _lib.check(_lib.load().cct_net_timeout(0, ctypes.byref(v)))
    if v.value:
        raise RuntimeError("a tensor-core wait timed out during training")
    net.save(a.out)
    del inputs, targets
    torch.cuda.empty_cache()
    evaluate_all(net, a, dev)


def evaluate_all(net: WarmStartNet, a, dev) -> None:
    import json

    if a.eval_slices > 0:
        for n, n_ang in ((a.n, a.angles), (2 * a.n, 2 * a.angles)):
            r = evaluate(net, n, n_ang, a.eval_slices, seed=900_000 + n, device=dev)
            print("eval", json.dumps(r), flush=True)
    if a.eval_pdhg_slices > 0:
        r = evaluate_pdhg(net, a.n, a.angles, a.eval_pdhg_slices, seed=950_000, device=dev)
        print("eval_pdhg", json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
