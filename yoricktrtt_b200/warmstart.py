"""Learned warm start of the TV-regularised cone-beam reconstruction.

Pipeline (all on the GPU):

1. ``Problem.sample(seed)``: a random-ellipsoid phantom, its cone-beam
   transmission data with Poisson noise (I0 photons per ray), log data
   ``y = log(I0 / counts) / kappa`` in phantom units and statistical weights
   ``w = counts / I0``.
2. ``Problem.backprojection(y, w)``: the normalised backprojection
   ``H'(w y) / H'(w H 1)``, the network input.
3. ``Problem.reconstruct``: VMLM-B + TV (``recon.vmlmb_native``, the cost
   of ``recon.Objective``), the plain method; run from zero it produces the
   training targets, and it is the arbiter of every warm start.
4. ``train``: the U-Net of ``unet.py`` fitted to (backprojection, converged
   reconstruction) pairs by Adam on the tensor-core kernels.
5. ``evaluate``: held-out seeds reconstructed from a zero start, from the
   backprojection and from the network output, each run to the same
   relative-objective stopping rule; wall time includes the network.

The reference reconstructs from zero with the same cost
(``Tomography_3D/Ytrtt3D_optim.i:128-234,663``); steps 1-2 and 4-5 have no
reference counterpart.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import geometry as G, phantoms as P
from .projectors import Projector3D
from .recon import Objective, vmlmb_native

KAPPA = 0.02  # attenuation of one phantom unit over one voxel (mm^-1)


def _torch():
    import torch
    return torch


class Problem:
    """Cone-beam circular orbit (SID 1000 mm, SDD 1500 mm, 1 mm voxels and
    cells) of an n^3 volume onto an nd^2 detector, `views` views."""

    def __init__(self, n=128, nd=256, views=90, i0=1e4, mu=5.0, eps=1e-2, kappa=KAPPA,
                 n_ellipsoids=20):
        self.n, self.nd, self.views = n, nd, views
        self.i0, self.mu, self.eps, self.kappa = float(i0), float(mu), float(eps), float(kappa)
        self.n_ellipsoids = n_ellipsoids
        self.scan = G.circular_scan_3d(n, n, n, 1.0, 3, nd, nd, 1.0, 1.0, views)
        self.pr = Projector3D(self.scan)

    def phantom(self, seed):
        torch = _torch()
        n = self.n
        return torch.tensor(P.ellipsoids_3d(n, n, n, n=self.n_ellipsoids, seed=seed), device="cuda")

    def counts(self, seed):
        """(truth, Poisson counts) for one seed."""
        torch = _torch()
        truth = self.phantom(seed)
        p = self.pr.forward(truth) * self.kappa
        gen = torch.Generator(device="cuda").manual_seed(int(seed) * 7919 + 17)
        return truth, torch.poisson(self.i0 * torch.exp(-p), generator=gen).clamp_(min=1.0)

    def data(self, counts):
        """(y, w) from Poisson counts: log data in phantom units, weights."""
        torch = _torch()
        c = counts.float()
        return torch.log(self.i0 / c) / self.kappa, c / self.i0

    def sample(self, seed):
        """(truth, y, w) for one seed."""
        truth, counts = self.counts(seed)
        y, w = self.data(counts)
        return truth, y, w

    def backprojection(self, y, w):
        torch = _torch()
        num = self.pr.backward(w * y)
        h1 = self.pr.forward(torch.ones(self.pr.volume_shape(), device="cuda"))
        den = self.pr.backward(w * h1)
        return num / den.clamp(min=1e-6 * float(den.max()))

    def objective(self, y, w):
        return Objective(self.pr, y, w, mu=self.mu, eps=self.eps)

    def reconstruct(self, y, w, x0=None, frtol=1e-6, maxiter=500):
        """VMLM-B + TV (native solver) from x0 (zero if None), x >= 0."""
        return vmlmb_native(self.pr, y, w, x0, mu=self.mu, eps=self.eps, lower=0.0,
                            maxiter=maxiter, frtol=frtol)


class Pairs:
    """Training set: inputs (N, n, n, n) = normalised backprojections,
    targets = VMLM-B + TV from zero, the Poisson counts of every sample
    (int16, to rebuild y and w) and the targets' objective values."""

    def __init__(self, inputs, targets, counts, f_target):
        self.inputs, self.targets, self.counts, self.f_target = inputs, targets, counts, f_target

    def __len__(self):
        return self.inputs.shape[0]


def generate_pairs(problem: Problem, seeds, frtol=1e-6, maxiter=150, log=None, keep_counts=True):
    """Training pairs made by the plain method (see Pairs)."""
    torch = _torch()
    n = problem.n
    N = len(seeds)
    inputs = torch.empty(N, n, n, n, device="cuda")
    targets = torch.empty(N, n, n, n, device="cuda")
    counts = (torch.empty((N,) + problem.pr.detector_shape(), dtype=torch.int16, device="cuda")
              if keep_counts else None)
    f_target = np.zeros(N)
    t0 = time.perf_counter()
    its = []
    for i, s in enumerate(seeds):
        _, c = problem.counts(s)
        y, w = problem.data(c)
        if counts is not None:
            counts[i] = c.to(torch.int16)
        inputs[i] = problem.backprojection(y, w)
        x, info = problem.reconstruct(y, w, frtol=frtol, maxiter=maxiter)
        targets[i] = x
        f_target[i] = info.f[-1]
        its.append(info.iterations)
        if log and (i + 1) % max(1, N // 10) == 0:
            log(f"pairs {i + 1}/{N}  {time.perf_counter() - t0:.1f} s  iterations {info.iterations}")
    problem.pr.status()
    return Pairs(inputs, targets, counts, f_target), {
        "seconds": time.perf_counter() - t0, "iterations_mean": float(np.mean(its)),
        "iterations_max": int(np.max(its))}


def train(net, pairs, epochs=10, batch=2, lr=1e-3, lr_final=1e-4, seed=0, log=None,
          problem: Problem | None = None, obj_weight=0.0):
    """Adam with a cosine learning-rate schedule and random flips; returns
    the per-epoch mean losses and the training time.

    obj_weight > 0 adds the term obj_weight log(f(max(out, 0)) / f_target)
    to the MSE loss, f the sample's own TV objective (the cost the
    warm-started iteration will minimise; f_target, the objective of the
    target, is its minimum up to the target's convergence): its gradient
    grad f / f at the network output reaches the network through
    ``extra_grad``.  Low-frequency errors, which dominate the data term and
    which the mean squared error weighs no more than any other, are then
    penalised by what they cost the iteration; dividing by f (the log)
    keeps the term bounded while f is still far above its minimum."""
    torch = _torch()
    inputs, targets = pairs.inputs, pairs.targets
    N = inputs.shape[0]
    obj = None
    if obj_weight > 0:
        if problem is None or pairs.counts is None:
            raise ValueError("the objective term needs the problem and the counts of every pair")
        y0, w0 = problem.data(pairs.counts[0])
        obj = problem.objective(y0, w0)
    steps_per_epoch = max(1, N // batch)
    total = epochs * steps_per_epoch
    rng = np.random.default_rng(seed)
    losses = []
    t0 = time.perf_counter()
    step = 0
    for ep in range(epochs):
        perm = rng.permutation(N)
        acc = 0.0
        for b in range(steps_per_epoch):
            idx = perm[b * batch:(b + 1) * batch]
            xb, tb = inputs[idx], targets[idx]
            dims = [d + 1 for d in range(3) if rng.uniform() < 0.5]
            if dims:
                xb, tb = torch.flip(xb, dims), torch.flip(tb, dims)
            net.lr = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * step / total))
            xb, tb = xb.contiguous(), tb.contiguous()
            extra = None
            if obj is not None:
                out = net.forward(xb)
                extra = torch.empty_like(out)
                back = [d - 1 for d in dims]
                for j, i in enumerate(idx):
                    xh = torch.flip(out[j], back) if back else out[j]
                    obj.y, obj.w = problem.data(pairs.counts[int(i)])
                    fv, g = obj(xh.clamp(min=0.0).contiguous())
                    g = g * (xh > 0) * (obj_weight / fv)
                    extra[j] = torch.flip(g, back) if back else g
            acc += float(net.train_step(xb, tb, extra_grad=extra))
            step += 1
        losses.append(acc / steps_per_epoch)
        if log:
            log(f"epoch {ep + 1}/{epochs}  loss {losses[-1]:.4e}  {time.perf_counter() - t0:.1f} s")
    net.status()
    return losses, time.perf_counter() - t0


def _hit(info, f_ref, rtol):
    """(iteration, wall time) of the first iterate with f <= f_ref (1 + rtol)."""
    lim = f_ref + rtol * abs(f_ref)
    for k, (f, t) in enumerate(zip(info.f, info.times)):
        if f <= lim:
            return k, t
    return None, None


TOLS = (1e-4, 1e-5, 1e-6)


def evaluate(problem: Problem, nets, seeds, frtol=1e-6, maxiter=500, ref_maxiter=600, log=None):
    """Per held-out seed: the plain method from zero, from the normalised
    backprojection and from each network's output (``nets``: a network or
    {name: network}), each to the stopping rule |f_k - f_k+1| <= frtol
    max(|f_k|, |f_k+1|).  f_ref is the lowest objective reached by these
    runs and, if ref_maxiter > 0, by a reference run from zero without the
    stopping rule (ref_maxiter iterations);
    for every start the iterations and wall time to f <= f_ref (1 + tol) are
    reported for tol in TOLS.  Times are wall clock (the iteration reads FP64
    scalars back every step) and include building the start
    (backprojection, network inference)."""
    torch = _torch()
    if not isinstance(nets, dict):
        nets = {"learned": nets}
    rows = []
    for s in seeds:
        _, y, w = problem.sample(s)
        res = {"seed": int(s)}
        runs = {}
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x0, info0 = problem.reconstruct(y, w, frtol=frtol, maxiter=maxiter)
        torch.cuda.synchronize()
        runs["zero"] = (time.perf_counter() - t0, 0.0, x0, info0)
        for name in ["backprojection"] + list(nets):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            bp = problem.backprojection(y, w)
            start = bp if name == "backprojection" else nets[name].forward(bp.unsqueeze(0))[0]
            start = start.clamp(min=0.0)
            torch.cuda.synchronize()
            t_start = time.perf_counter() - t0
            x, info = problem.reconstruct(y, w, x0=start, frtol=frtol, maxiter=maxiter)
            torch.cuda.synchronize()
            runs[name] = (time.perf_counter() - t0, t_start, x, info)
        f_ref = min(r[3].f[-1] for r in runs.values())
        if ref_maxiter > 0:
            _, info_ref = problem.reconstruct(y, w, frtol=0.0, maxiter=ref_maxiter)
            f_ref = min(f_ref, info_ref.f[-1])
        res["f_ref"] = f_ref
        for name, (sec, t_start, x, info) in runs.items():
            d = {"seconds": sec, "start_seconds": t_start, "iterations": info.iterations,
                 "evaluations": info.evaluations, "f": info.f[-1], "f_start": info.f[0],
                 "converged": info.converged,
                 "rel_diff_vs_zero": float(torch.linalg.norm(x - x0) / torch.linalg.norm(x0))}
            for tol in TOLS:
                k, t = _hit(info, f_ref, tol)
                d[f"to_{tol:g}"] = None if k is None else {"iterations": k, "seconds": t_start + t}
            res[name] = d
        rows.append(res)
        if log:
            log(f"seed {s}: " + ", ".join(
                f"{k} {res[k]['iterations']} it / {res[k]['seconds']:.2f} s"
                f" (1e-5: {res[k]['to_1e-05']['iterations'] if res[k]['to_1e-05'] else '-'} it)"
                for k in runs))
    problem.pr.status()
    return rows


def summarize(rows):
    out = {}
    names = [k for k in rows[0] if k not in ("seed", "f_ref")]
    for name in names:
        sec = [r[name]["seconds"] for r in rows]
        it = [r[name]["iterations"] for r in rows]
        o = {"stop_rule": {"seconds_mean": float(np.mean(sec)), "seconds_median": float(np.median(sec)),
                           "iterations_mean": float(np.mean(it)),
                           "converged": int(sum(bool(r[name]["converged"]) for r in rows)),
                           "final_f_rel_excess_mean": float(np.mean(
                               [(r[name]["f"] - r["f_ref"]) / abs(r["f_ref"]) for r in rows]))}}
        for tol in TOLS:
            hits = [r[name][f"to_{tol:g}"] for r in rows]
            ok = [h for h in hits if h is not None]
            o[f"to_{tol:g}"] = {"reached": len(ok),
                                "iterations_median": float(np.median([h["iterations"] for h in ok])) if ok else None,
                                "seconds_median": float(np.median([h["seconds"] for h in ok])) if ok else None}
        out[name] = o
    z = out["zero"]
    for name in names:
        if name == "zero":
            continue
        o = out[name]
        o["speedup_vs_zero"] = {"stop_rule_seconds_mean": z["stop_rule"]["seconds_mean"] /
                                o["stop_rule"]["seconds_mean"]}
        for tol in TOLS:
            k = f"to_{tol:g}"
            if z[k]["iterations_median"] and o[k]["iterations_median"]:
                o["speedup_vs_zero"][k + "_iterations_median"] = z[k]["iterations_median"] / max(
                    1.0, o[k]["iterations_median"])
    return out
