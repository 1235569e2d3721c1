"""Learned warm start: what the trained network (weights shipped in
yoricktrtt_b200/weights/) gains over the plain method's own starts on a
held-out seed, with the plain method as the arbiter of the result."""
import os

import numpy as np
import pytest

WEIGHTS = os.path.join(os.path.dirname(__file__), "..", "yoricktrtt_b200", "weights", "unet_warmstart_128.npz")


@pytest.mark.gpu
def test_learned_start_against_zero_and_backprojection():
    import torch
    from yoricktrtt_b200.unet import UNet3D
    from yoricktrtt_b200.warmstart import Problem
    assert os.path.exists(WEIGHTS), "trained weights missing"
    net = UNet3D.load(WEIGHTS)
    pb = Problem()
    _, y, w = pb.sample(20000)  # held out: training seeds are 10000..
    bp = pb.backprojection(y, w)
    start = net.forward(bp.unsqueeze(0))[0].clamp(min=0.0)
    net.status()
    obj = pb.objective(y, w)
    f_zero = obj(torch.zeros_like(bp))[0]
    f_bp = obj(bp.clamp(min=0.0).contiguous())[0]
    f_learned = obj(start.contiguous())[0]
    # the network's start is far closer to the optimum than both plain starts
    assert f_learned < 0.2 * f_bp and f_learned < 0.01 * f_zero
    x0, i0 = pb.reconstruct(y, w, frtol=1e-6, maxiter=500)
    xl, il = pb.reconstruct(y, w, x0=start, frtol=1e-6, maxiter=500)
    pb.pr.status()
    assert i0.converged and il.converged
    # both runs end at the same optimum (the plain method decides the result);
    # the relative-change stopping rule leaves the final objectives of
    # different starts (and of repeated runs: the summation order of the
    # atomics varies) scattered by a few 1e-4
    assert abs(il.f[-1] - i0.f[-1]) <= 1e-3 * i0.f[-1]
    assert float(torch.linalg.norm(xl - x0) / torch.linalg.norm(x0)) <= 0.05
    # the warm-started run starts below the zero start's objective after
    # its first iterations: the first iterate of the plain run that gets as
    # low as the learned start
    k = int(np.argmax(np.array(i0.f) <= f_learned))
    assert k >= 3
