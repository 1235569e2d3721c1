"""Measured workloads for the benchmark configurations other than the
cone-beam projector pair (which bench.py times by default).

Each function builds the configuration with seeded synthetic data, runs it on
the current CUDA device and returns a dict of measured quantities (CUDA-event
or wall-clock times, errors against the FP64 oracle where one applies).

* ``parallel2d_recon``: 2D parallel beam, 256^2 image of 10 ellipses, cubic
  B-spline, 180 views over [0, pi), 367 bins, 1% Gaussian noise; one
  projector pair plus 50 VMLM-B iterations with TV (mu = 1e-2).
* ``fan2d``: 2D fan beam, 512^2 image, 720 views over 2 pi, 1024-bin flat
  detector, SID 1000 mm, SDD 1500 mm, 0.5 mm pixels: B-spline (closed-form
  and table footprints) and Long-Fessler pair throughput, parity against the
  FP64 oracle on sample views, FP64 adjoint test.
* ``cone3d_recon``: 3D cone beam 256^3 -> 360 x 512^2, VMLM-B + TV until the
  relative objective change falls below 1e-6 (at most 100 iterations).
* ``gates4d``: 10 respiratory gates of 128x128x64, ellipsoid phantom
  translated along z by up to 10 mm, views per gate drawn from U{20..60},
  256^2 detector; all gates projected (direct and transpose) by one launch
  each, tiles autotuned, the pair captured in a CUDA graph and replayed.
* ``learned_warmstart``: 128^3 random-ellipsoid phantoms, 90 cone-beam views
  on a 256^2 detector, Poisson noise I0 = 1e4; training pairs (normalised
  backprojection -> VMLM-B + TV reconstruction) generated by the plain
  method, the 3D U-Net trained on them with the tensor-core kernels, then
  held-out seeds reconstructed to 1e-6 relative objective change from zero,
  from the backprojection and from the network output.
* ``learned_eval``: the evaluation half of ``learned_warmstart`` with saved
  network weights.
"""
from __future__ import annotations

import math
import time

import numpy as np


def _torch():
    import torch
    return torch


def _events():
    torch = _torch()
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time(fn, reps=3):
    torch = _torch()
    fn()
    torch.cuda.synchronize()
    best = math.inf
    for _ in range(reps):
        a, b = _events()
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def parallel2d_recon(iterations=50, seed=0):
    torch = _torch()
    from . import geometry as G, phantoms as P
    from .recon import Objective, Projector2D, vmlmb
    sc = G.circular_scan_2d(256, 256, 1.0, 3, 367, 1.0, 180, mode=G.TRTT_PARALLEL_BEAM)
    truth = P.ellipses_2d(256, 256, n=10, seed=seed)
    pr = Projector2D(sc)
    xt = torch.tensor(truth, dtype=torch.float32, device="cuda")
    y = pr.forward(xt)
    rng = np.random.default_rng(seed + 1)
    noise = torch.tensor(rng.standard_normal(tuple(y.shape)), dtype=torch.float32, device="cuda")
    y = y + 0.01 * float(y.max()) * noise
    out_f = torch.zeros_like(y)
    out_b = torch.zeros_like(xt)
    t_pair = _time(lambda: (pr.forward(xt, out=out_f.zero_()), pr.backward(y, out=out_b.zero_())))
    obj = Objective(pr, y, mu=1e-2, eps=1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x, info = vmlmb(obj, torch.zeros_like(xt), lower=0.0, maxiter=iterations, frtol=0.0)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    pr.status()
    err = float(torch.linalg.norm(x - xt) / torch.linalg.norm(xt))
    return {"config": "2D parallel 256^2, 180 views, 367 bins, cubic, VMLM-B + TV mu=1e-2",
            "pair_ms": t_pair, "iterations": info.iterations, "evaluations": info.evaluations,
            "recon_s": wall, "f_first": info.f[0], "f_last": info.f[-1],
            "rel_err_vs_phantom": err}


def fan2d(sample_views=4, seed=0, reference=None):
    """2D fan-beam throughput of the B-spline (closed-form and table) and
    Long-Fessler pairs.  ``reference(kind, view, img, scan, table, lf)``, when
    given, returns the FP64 reference projection of one view (the caller
    supplies the checker; this package does not import one), and the result
    then carries the largest relative L2 error over ``sample_views`` views."""
    torch = _torch()
    from . import dropin, footprint as F, geometry as G, phantoms as P
    from .recon import Projector2D, dot
    sc = G.circular_scan_2d(512, 512, 0.5, 3, 1024, 0.5, 720, mode=G.TRTT_FAN_BEAM,
                            rsc=1000.0, rsd=1500.0)
    img = P.ellipses_2d(512, 512, n=10, seed=seed)
    xt = torch.tensor(img, dtype=torch.float32, device="cuda")
    res = {"config": "2D fan 512^2, 720 views / 2 pi, 1024 bins, SID 1000, SDD 1500, 0.5 mm"}
    tab = F.make_footprint(3, 10001)
    views = np.linspace(0, 719, sample_views).astype(int)
    # Long-Fessler with the same geometry (Ytrtt_2D_projectors_Long_Fessler.i:216-233)
    lf = dict(pixelSize=0.5, pixelStep=0.5, voxelSize=0.5, sourceDistance=1000.0,
              detectorDistance=500.0, objectOffset1=0.0, objectOffset2=0.0,
              objectDimension1=512, objectDimension2=512, detectorDimension=1024)
    beta = sc.theta - math.pi / 2
    cases = [("bspline_cubic", Projector2D(sc), None, sc.nv),
             ("bspline_table", Projector2D(sc, tab), tab, sc.nv),
             ("long_fessler", Projector2D(lf_params=dropin.LF2DParams(**lf), beta=beta,
                                          offset=np.zeros(sc.nviews)), None, 1024)]
    for name, pr, table, nbins in cases:
        y = torch.zeros(sc.nviews, nbins, device="cuda")
        b = torch.zeros_like(xt)
        tf = _time(lambda: pr.forward(xt, out=y.zero_()))
        yy = torch.rand_like(y)
        tb = _time(lambda: pr.backward(yy, out=b.zero_()))
        pr.forward(xt, out=y.zero_())
        pr.backward(yy, out=b.zero_())
        adj = abs(dot(y, yy) - dot(xt, b)) / (math.sqrt(dot(y, y)) * math.sqrt(dot(yy, yy)))
        r = {"fwd_ms": tf, "back_ms": tb, "projections_per_s": 2 * sc.nviews / ((tf + tb) / 1e3),
             "adjoint_rel": adj}
        if reference is not None:
            yh = y.double().cpu().numpy()
            errs = []
            for v in views:
                ref = reference("lf" if name == "long_fessler" else "fb2d", int(v), img, sc, table,
                                dict(lf, beta=float(beta[v])))
                errs.append(float(np.linalg.norm(yh[v] - ref) / np.linalg.norm(ref)))
            r["max_rel_l2_vs_fp64"] = max(errs)
            r["sample_views"] = [int(v) for v in views]
        res[name] = r
    return res


def cone3d_recon(maxiter=100, frtol=1e-6, seed=0, n=256, nd=512, views=360):
    torch = _torch()
    from . import geometry as G, phantoms as P
    from .projectors import Projector3D
    from .recon import vmlmb_native
    sc = G.circular_scan_3d(n, n, n, 1.0, 3, nd, nd, 1.0, 1.0, views)
    truth = torch.tensor(P.ellipsoids_3d(n, n, n, n=20, seed=seed), device="cuda")
    pr = Projector3D(sc)
    y = pr.forward(truth)
    rng = np.random.default_rng(seed + 1)
    y = y + 0.01 * float(y.max()) * torch.tensor(rng.standard_normal(tuple(y.shape)),
                                                 dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x, info = vmlmb_native(pr, y, None, None, mu=1e-2, eps=1e-3, lower=0.0, maxiter=maxiter, frtol=frtol)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    pr.status()
    err = float(torch.linalg.norm(x - truth) / torch.linalg.norm(truth))
    f = np.asarray(info.f)
    rel = np.abs(np.diff(f)) / np.maximum(np.abs(f[:-1]), np.abs(f[1:]))
    first_below = {f"{t:g}": (int(np.argmax(rel <= t)) + 1 if np.any(rel <= t) else None)
                   for t in (1e-2, 1e-3, 1e-4, 1e-5, 1e-6)}
    return {"config": f"3D cone {n}^3 -> {views} x {nd}^2, VMLM-B + TV (native solver) to {frtol:g} "
                      f"relative objective change, at most {maxiter} iterations",
            "iterations": info.iterations, "evaluations": info.evaluations,
            "converged": info.converged, "reason": info.reason, "seconds": wall,
            "ms_per_iteration": 1e3 * wall / max(1, info.iterations),
            "f_first": info.f[0], "f_last": info.f[-1], "rel_err_vs_phantom": err,
            "first_iteration_with_relative_change_below": first_below,
            "f_every_10": f[::10].tolist()}


def gates4d(nt=10, seed=0, replays=5):
    """10 gates of 128x128x64 (breathing phantom), views per gate from
    U{20..60}, 256^2 detector.  Two forms of one data-term evaluation:
    the direct and transpose grid kernels (tiles autotuned) captured in a
    CUDA graph, and the persistent launch resid = H x - y, grad = H^T resid
    (trtt_b200_plan3d_wls_grad, tile shape autotuned), which also computes
    the residual and the FP64 cost."""
    torch = _torch()
    from . import geometry as G, phantoms as P
    from .projectors import Projector3D
    rng = np.random.default_rng(seed)
    counts = rng.integers(20, 61, nt)
    # each gate's views sit at fractional gate indices inside [g, g+1)
    t_index = np.concatenate([g + rng.uniform(0.0, 1.0, c) for g, c in enumerate(counts)])
    nviews = int(counts.sum())
    # acquisition order: angles over the orbit as the dates advance
    theta = np.sort(rng.uniform(0, 2 * math.pi, nviews))
    sc = G.circular_scan_3d(128, 128, 64, 1.0, 3, 256, 256, 1.0, 1.0, nviews, theta=theta)
    gates = torch.tensor(P.breathing_gates(128, 128, 64, nt, 1.0, amplitude_mm=10.0, seed=seed),
                         device="cuda")
    pr = Projector3D(sc)
    pr.set_gates(nt, t_index)
    from .projectors import columns_from_xyz
    xc = columns_from_xyz(gates)
    times, choice = pr.autotune(xc, layout="columns", nview=nviews, reps=2)
    y = torch.zeros(pr.detector_shape(), device="cuda")
    back = torch.zeros_like(xc)

    def pair():
        y.zero_()
        back.zero_()
        pr.forward(xc, out=y, layout="columns")
        pr.backward(y, out=back, layout="columns")

    graph = pr.capture(pair)
    torch.cuda.synchronize()
    best = math.inf
    for _ in range(replays):
        a, b = _events()
        a.record()
        graph.replay()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    pr.status()
    # persistent launch on measurements of the projections' size
    meas = (y * 0.9).contiguous()
    wtimes, wchoice = pr.autotune_wls(xc, meas, reps=2)
    grad = torch.zeros_like(xc)
    wbest = math.inf
    for _ in range(replays):
        grad.zero_()
        a, b = _events()
        a.record()
        cost = pr.wls_grad(xc, meas, grad)
        b.record()
        torch.cuda.synchronize()
        wbest = min(wbest, a.elapsed_time(b))
    pr.status()
    return {"config": f"4D: {nt} gates of 128x128x64, views per gate U{{20..60}} (total {nviews}), 256^2",
            "views_per_gate": counts.tolist(), "tiles": list(choice),
            "autotune_ms": {str(k): v for k, v in times.items()},
            "pair_graph_ms": best, "projections_per_s": 2 * nviews / (best / 1e3),
            "persistent": {"tiles_band_rows_ctas_per_sm": list(wchoice),
                           "autotune_ms": {str(k): v for k, v in wtimes.items()},
                           "ms": wbest, "projections_per_s": 2 * nviews / (wbest / 1e3),
                           "cost": float(cost.item()),
                           "what": "resid = H x - y, 1/2 |resid|^2 (FP64), grad = H^T resid, "
                                   "one cooperative launch"}}


def _log(msg):
    import sys
    print(msg, file=sys.stderr, flush=True)


def learned_warmstart(n_train=400, n_test=20, epochs=8, batch=2, lr=1e-3, target_maxiter=150,
                      eval_maxiter=500, ref_maxiter=600, obj_weight=0.0, compare=False, weights=None,
                      seed=0):
    """compare=True trains two networks from the same initialisation, with
    the mean squared error alone and with the objective term of
    warmstart.train (obj_weight), and evaluates both."""
    from .unet import UNet3D
    from .warmstart import Problem, evaluate, generate_pairs, summarize, train
    torch = _torch()
    pb = Problem()
    train_seeds = list(range(seed + 10000, seed + 10000 + n_train))
    test_seeds = list(range(seed + 20000, seed + 20000 + n_test))
    pairs, gen = generate_pairs(pb, train_seeds, maxiter=target_maxiter, log=_log,
                                keep_counts=obj_weight > 0)
    variants = {"learned_mse": 0.0, "learned_obj": obj_weight} if compare else \
        {"learned": obj_weight}
    nets, train_info = {}, {}
    for name, lam in variants.items():
        net = UNet3D(seed=seed, lr=lr)
        losses, t_train = train(net, pairs, epochs=epochs, batch=batch, lr=lr, seed=seed, log=_log,
                                problem=pb, obj_weight=lam)
        nets[name] = net
        train_info[name] = {"obj_weight": lam, "seconds": t_train, "epoch_losses": losses}
        if weights:
            net.save(weights if len(variants) == 1 else weights.replace(".npz", f"_{name}.npz"))
    del pairs
    torch.cuda.empty_cache()
    rows = evaluate(pb, nets, test_seeds, maxiter=eval_maxiter, ref_maxiter=ref_maxiter, log=_log)
    return {"config": f"learned warm start: 128^3 ellipsoid phantoms, 90 cone-beam views on 256^2, "
                      f"Poisson I0=1e4, VMLM-B + TV (mu={pb.mu:g}, eps={pb.eps:g}); {n_train} training "
                      f"pairs (targets: VMLM-B from zero, at most {target_maxiter} iterations or 1e-6), "
                      f"{n_test} held-out seeds to 1e-6 relative objective change",
            "train_seeds": [train_seeds[0], train_seeds[-1]], "test_seeds": [test_seeds[0], test_seeds[-1]],
            "pair_generation": gen, "training": train_info,
            "summary": summarize(rows), "per_seed": rows}


def learned_eval(weights=None, n_test=20, eval_maxiter=500, ref_maxiter=600, seed=0):
    import os
    from .unet import UNet3D
    from .warmstart import Problem, evaluate, summarize
    if weights is None:
        weights = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet_warmstart_128.npz")
    net = UNet3D.load(weights)
    pb = Problem()
    test_seeds = list(range(seed + 20000, seed + 20000 + n_test))
    rows = evaluate(pb, net, test_seeds, maxiter=eval_maxiter, ref_maxiter=ref_maxiter, log=_log)
    return {"config": f"learned warm start evaluation ({os.path.basename(weights)}): {n_test} held-out "
                      f"seeds, 128^3, 90 views, 256^2, Poisson I0=1e4, VMLM-B + TV to 1e-6",
            "summary": summarize(rows), "per_seed": rows}


def projector_case(n=128, nd=256, views=90, nz=None, direct=1, transpose=1, reps=1, dense=0,
                   tiles=None, sym=2, gshape=None, table=0, seed=0):
    """One cone-beam projector case for profiling: an n x n x nz volume of 20
    ellipsoids (``dense=1`` adds a positive floor so that every voxel is
    non-zero), ``views`` views on an nd x nd detector, SID 1000 mm, SDD
    1500 mm, closed-form cubic footprint, columns layout.  Runs ``reps``
    direct and/or transpose launches, checks the status flag and returns the
    CUDA-event time of the last launch of each direction.  ``tiles`` is a
    set_tiles() argument list; ``sym=0`` bypasses the group kernels, ``sym=1``
    selects per-member profiles; ``gshape`` is a set_group_shape() list;
    ``table > 0`` uses the tabulated cubic footprint with that many samples
    (the table model runs the per-view kernels)."""
    torch = _torch()
    from . import footprint as F, geometry as G, phantoms as P
    from .projectors import Projector3D, columns_from_xyz
    nz = nz or n
    sc = G.circular_scan_3d(n, n, nz, 1.0, 3, nd, nd, 1.0, 1.0, views, rsc=1000.0, rsd=1500.0)
    vol = P.ellipsoids_3d(n, n, nz, n=20, seed=seed, dtype=np.float32)
    if dense:
        vol = vol + np.float32(0.05)
    pr = Projector3D(sc, F.make_footprint(3, int(table)) if table else None)
    if tiles:
        pr.set_tiles(*tiles)
    pr.set_symmetry(int(sym))
    if gshape:
        pr.set_group_shape(*gshape)
    x = columns_from_xyz(torch.tensor(vol, device="cuda"))
    y = torch.zeros(pr.detector_shape(), device="cuda")
    b = torch.zeros_like(x)
    model = f"cubic table of {int(table)} samples" if table else "cubic"
    res = {"config": f"cone {n}x{n}x{nz} -> {views} x {nd}^2, {model}, {'dense' if dense else 'phantom'}",
           "groups": pr.groups(), "symmetry": int(sym), "gshape": gshape}
    for _ in range(reps):
        if direct:
            a, e = _events()
            a.record()
            pr.forward(x, out=y.zero_(), layout="columns")
            e.record()
            torch.cuda.synchronize()
            res["direct_ms"] = a.elapsed_time(e)
        if transpose:
            a, e = _events()
            a.record()
            pr.backward(y if direct else torch.ones_like(y), out=b.zero_(), layout="columns")
            e.record()
            torch.cuda.synchronize()
            res["transpose_ms"] = a.elapsed_time(e)
    pr.status()
    res["voxel_views"] = n * n * nz * views
    return res


def unet_case(size=128, batch=1, reps=1, train=1, tma=-1, seed=0):
    """One U-Net case for profiling the tensor-core convolutions: ``reps``
    forward passes (and training steps when ``train``) on a batch of
    size^3 inputs; returns the CUDA-event time of the last of each.
    ``tma`` selects the staging of the forward / input-gradient
    convolutions (trtt_b200_conv3_set_tma): 0 cp.async, 1 TMA one tile per
    CTA, 2 TMA in persistent CTAs, -1 the default."""
    torch = _torch()
    from . import _lib
    from .unet import UNet3D
    _lib.check(_lib.load().trtt_b200_conv3_set_tma(int(tma)), "trtt_b200_conv3_set_tma")
    net = UNet3D(seed=seed)
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.rand(batch, size, size, size, device="cuda", generator=g)
    t = torch.rand(batch, size, size, size, device="cuda", generator=g)
    res = {"config": f"U-Net 3 levels 16/32/64, batch {batch} x {size}^3, "
                     f"staging {({0: 'cp.async', 1: 'TMA per tile', 2: 'TMA persistent'}).get(int(tma), 'default')}"}
    for _ in range(reps):
        a, e = _events()
        a.record()
        net.forward(x)
        e.record()
        torch.cuda.synchronize()
        res["forward_ms"] = a.elapsed_time(e)
        if train:
            a, e = _events()
            a.record()
            net.train_step(x, t)
            e.record()
            torch.cuda.synchronize()
            res["train_step_ms"] = a.elapsed_time(e)
    net.status()
    return res
