"""Training pairs, training loop and warm-started solves for the MLEM warm-start network.

Pairs come from this package's own batched GPU MLEM on seeded synthetic slices (no dataset is
public on this path): textured phantoms (5-20 ellipses with a smooth Gaussian-random-field
texture, values in [0, 1]), disk attenuation (mu in [0, 0.02], emitted mu = 0.7 incident mu),
Poisson data.  Input = the first 10 MLEM iterates plus the normalised back-projection
A^T b / A^T 1, each slice divided by the mean of its 10th iterate; target = the iterate after
``target_iterations`` MLEM iterations, as a correction to the 10th iterate in the same units.

Usage (GPU):  python -m pycorrectedemissionct_b200.train_warmstart --slices 1024 --steps 1500 --out w.pt
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
                subsets: int = 0):
    """Phantoms, attenuation, maps and Poisson data for one batch of slices (angles in the
    ``subset_permutation`` order of ``subsets`` subsets when ``subsets`` > 0)."""
    xs, mus = [], []
    for sd in seeds:
        rng = phantoms.slice_rng(sd, 0)
        xs.append(textured_phantom(n, rng) if textured else phantoms.ellipse_phantom(n, rng, 12))
        mus.append(phantoms.disk_attenuation(n, rng, mu_max))
    angles = phantoms.angles(n_angles)
    if subsets > 0:
        angles = angles[subset_permutation(n_angles, [subsets])]
    c = core.XrfCore(n, angles, device=device)
    mu = torch.from_numpy(np.stack(mus)).to(device)
    maps = core.compute_maps(mu, 0.7 * mu, c.angles_rad32)
    x = torch.from_numpy(np.stack(xs)).to(device)
    clean = c.fp(x, maps)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seeds[0]))
    b = torch.poisson(clean / clean.amax(dim=(1, 2, 3), keepdim=True) * peak, generator=gen)
    return c, maps, b, x


def generate_pairs(n_slices: int, n: int = 256, n_angles: int = 360, seed: int = 100_000, batch: int = 64,
                   peak: float = 1e4, mu_max: float = 0.02, target_iterations: int = 500, device=None, net=None):
    """(inputs NHWC bf16 (N, n, n, 16), targets FP32 (N, n, n)) on the device."""
    device = core.require_cuda(device)
    helper = net if net is not None else WarmStartNet(device=device)
    inputs, targets = [], []
    n_sub = helper.pass_subsets(n_angles)
    for s0 in range(0, n_slices, batch):
        seeds = [seed + k for k in range(s0, min(n_slices, s0 + batch))]
        c, maps, b, _ = synth_batch(n, n_angles, seeds, mu_max, peak, device, subsets=n_sub)
        solver = BatchedSolver(c, maps, b, "mlem")
        if n_sub > 0:
            its = pass_snapshots(OrderedSubsets(c, maps, b, [(n_sub, 1)]))
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


def warm_started_solve(net: WarmStartNet, c: core.XrfCore, maps: torch.Tensor, b: torch.Tensor, tolerance,
                       max_iterations: int = 400, check_every: int = 5, history_len: int = 0):
    """10 plain MLEM iterations (or 10 snapshots of one ordered-subsets pass, by the network's
    inputs) -> network -> MLEM from the prediction until `tolerance`.  With ordered-subsets inputs,
    ``c``, ``maps`` and ``b`` must be in ``subset_permutation(A, [net.pass_subsets(A)])`` angle
    order.

    Returns (solver, total full-data passes per slice as a numpy array)."""
    first = BatchedSolver(c, maps, b, "mlem")
    n_sub = net.pass_subsets(c.n_angles)
    if n_sub > 0:
        its = pass_snapshots(OrderedSubsets(c, maps, b, [(n_sub, 1)]))
    else:
        its = first_iterates(first)
    bpn = normalized_backprojection(c, b, first.tau)
    scale = slice_means(its[-1])
    x0 = net.predict(its + [bpn], base=its[-1], slice_scale=scale)
    solver = BatchedSolver(c, maps, b, "mlem", tolerance=tolerance, x0=x0, history_len=history_len)
    solver.run(max_iterations, check_every=check_every)
    return solver, solver.iterations.cpu().numpy() + (1 if n_sub > 0 else N_ITERATES)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--slices", type=int, default=1024)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--angles", type=int, default=360)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--target-iterations", type=int, default=500)
    ap.add_argument("--additive", action="store_true", help="additive instead of log-ratio (multiplicative) targets")
    ap.add_argument("--log-floor", type=float, default=1e-3, help="floor of the log-ratio target, in slice means")
    ap.add_argument("--pass-angles", type=int, default=0,
                    help="inputs: 10 snapshots of one ordered-subsets pass over subsets of this many angles "
                         "(0: the first 10 MLEM iterates)")
    ap.add_argument("--out", default="warmstart.pt")
    a = ap.parse_args()
    dev = core.require_cuda()
    t0 = time.time()
    net = WarmStartNet(seed=0, device=dev)
    net.multiplicative = not a.additive
    net.log_floor = a.log_floor
    net.pass_angles = a.pass_angles
    inputs, targets = generate_pairs(a.slices, a.n, a.angles, target_iterations=a.target_iterations, device=dev, net=net)
    torch.cuda.synchronize()
    t1 = time.time()
    print(f"pairs: {inputs.shape[0]} in {t1 - t0:.1f} s; params {net.n_params()}", flush=True)
    losses = train(net, inputs, targets, a.steps, a.batch, a.lr)
    torch.cuda.synchronize()
    print(f"trained {a.steps} steps in {time.time() - t1:.1f} s; loss {losses[0]:.4f} -> {losses[-1]:.4f}", flush=True)
    v = ctypes.c_int32(0)
    _lib.check(_lib.load().cct_net_timeout(0, ctypes.byref(v)))
    if v.value:
        raise RuntimeError("a tensor-core wait timed out during training")
    net.save(a.out)


if __name__ == "__main__":
    main()
