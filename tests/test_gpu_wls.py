"""The weighted least-squares data term of a (4D) scan in one persistent
launch (trtt_b200_plan3d_wls_grad): resid = W (H x - y), cost =
1/2 sum W (H x - y)^2 and grad += H^T resid per gate, the cost evaluation of
the reference's 4D reconstruction (Tomography_4D/Ytrtt4D_optim.i:87-223).

Checked against the FP64 oracle (per view: the gate-interpolated volume
projected by the reference's cone-beam projector, the residual, its
transpose scattered into the two gates), at a small gated scan and at the
4D configuration (10 gates of 128x128x64, 20-60 views per gate, 256^2
detector) with the tile shape the autotuner picks; against the grid kernels
of the same plan; and the bounded device wait: with a test hook that makes
the column items wait for band items that do not exist, the wait runs out
within its short limit, the status reports it and the plan stays usable."""
import concurrent.futures as cf
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import geometry as G, phantoms as P

pytestmark = pytest.mark.gpu

TOL = 1e-5
THREADS = max(1, min(16, os.cpu_count() or 1))


def _gated_scan(nt, counts, n=(128, 128, 64), nd=256, seed=0, **kw):
    rng = np.random.default_rng(seed)
    t_index = np.concatenate([g + rng.uniform(0.0, 1.0, c) for g, c in enumerate(counts)])
    nviews = int(sum(counts))
    theta = np.sort(rng.uniform(0, 2 * math.pi, nviews))
    sc = G.circular_scan_3d(n[0], n[1], n[2], 1.0, 3, nd, nd, 1.0, 1.0, nviews, theta=theta, **kw)
    return sc, t_index


def _oracle_wls(orc, sc, t_index, nt, gates, y, w):
    """FP64 cost and per-gate gradient (inputs are the FP32 values)."""
    g64 = gates.astype(np.float64)

    def chunk(ks):
        grad = np.zeros_like(g64)
        cost = 0.0
        bt = np.zeros(g64.shape[1:])
        for k in ks:
            (g0, g1), (w0, w1) = G.gate_weights(float(t_index[k]), nt)
            x = np.ascontiguousarray(w0 * g64[g0] + w1 * g64[g1])
            hx = np.zeros((sc.nv, sc.nu))
            assert orc.cb3d(hx, x, sc, k, 0) == 0
            r = hx - y[k]
            wr = np.ascontiguousarray(w[k] * r if w is not None else r)
            cost += 0.5 * float((wr * r).sum())
            bt.fill(0.0)
            assert orc.cb3d(bt, wr, sc, k, 1) == 0
            if g0 != g1:
                grad[g0] += w0 * bt
                grad[g1] += w1 * bt
            else:
                grad[g0] += w1 * bt  # repeated index: the second write wins
        return cost, grad

    parts = [list(range(t, sc.nviews, THREADS)) for t in range(THREADS)]
    with cf.ThreadPoolExecutor(THREADS) as ex:
        res = list(ex.map(chunk, parts))
    return sum(r[0] for r in res), sum(r[1] for r in res)


def _run(sc, t_index, nt, gates, weighted, seed=3, autotune=False):
    import torch
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz, xyz_from_columns
    pr = Projector3D(sc)
    pr.set_gates(nt, t_index)
    xc = columns_from_xyz(torch.tensor(gates, device="cuda"))
    # measurements of the size of the projections, not close to them
    hx = pr.forward(xc, layout="columns")
    g = torch.Generator(device="cuda").manual_seed(seed)
    y = torch.rand(hx.shape, device="cuda", generator=g) * float(hx.mean()) * 2.0
    w = (0.5 + torch.rand(hx.shape, device="cuda", generator=g)) if weighted else None
    choice = None
    if autotune:
        _, choice = pr.autotune_wls(xc, y, w, reps=1)
    grad = torch.zeros_like(xc)
    cost = pr.wls_grad(xc, y, grad, w)
    pr.status()
    out = (float(cost.item()), xyz_from_columns(grad).double().cpu().numpy(),
           y.double().cpu().numpy(), None if w is None else w.double().cpu().numpy())
    # the grid kernels of the same plan
    r = hx - y
    wr = r * w if w is not None else r
    grad2 = xyz_from_columns(pr.backward(wr.contiguous(), layout="columns")).double().cpu().numpy()
    cost2 = 0.5 * float((wr.double() * r.double()).sum())
    return out, (cost2, grad2), pr, choice


@pytest.mark.parametrize("weighted", [False, True])
def test_wls_small_gated(oracle_port, weighted):
    nt = 3
    sc, t_index = _gated_scan(nt, [5, 2, 6], n=(24, 20, 16), nd=40, rsc=60.0, rsd=90.0, seed=1)
    gates = P.breathing_gates(24, 20, 16, nt, 1.0, amplitude_mm=3.0, seed=2)
    (cost, grad, y, w), (cost2, grad2), _, _ = _run(sc, t_index, nt, gates, weighted)
    ref_cost, ref_grad = _oracle_wls(oracle_port, sc, t_index, nt, gates, y, w)
    assert abs(cost - ref_cost) <= TOL * abs(ref_cost)
    assert rel_l2(grad, ref_grad) <= TOL
    assert abs(cost - cost2) <= 1e-6 * abs(cost2) and rel_l2(grad, grad2) <= 1e-6


def test_wls_long_columns(oracle_port):
    """Columns of 128 voxels: the band items spread under row locks."""
    nt = 2
    sc, t_index = _gated_scan(nt, [4, 3], n=(16, 12, 128), nd=200, rsc=150.0, rsd=225.0, seed=4)
    gates = P.breathing_gates(16, 12, 128, nt, 1.0, amplitude_mm=4.0, seed=5)
    (cost, grad, y, w), (cost2, grad2), _, _ = _run(sc, t_index, nt, gates, True)
    ref_cost, ref_grad = _oracle_wls(oracle_port, sc, t_index, nt, gates, y, w)
    assert abs(cost - ref_cost) <= TOL * abs(ref_cost)
    assert rel_l2(grad, ref_grad) <= TOL
    assert abs(cost - cost2) <= 1e-6 * abs(cost2) and rel_l2(grad, grad2) <= 1e-6


def test_wls_config4_autotuned(oracle_port):
    """10 gates of 128x128x64, views per gate drawn from U{20..60}, 256^2."""
    nt = 10
    counts = np.random.default_rng(0).integers(20, 61, nt)
    sc, t_index = _gated_scan(nt, counts, seed=0)
    gates = P.breathing_gates(128, 128, 64, nt, 1.0, amplitude_mm=10.0, seed=0)
    (cost, grad, y, w), (cost2, grad2), _, choice = _run(sc, t_index, nt, gates, True, autotune=True)
    ref_cost, ref_grad = _oracle_wls(oracle_port, sc, t_index, nt, gates, y, w)
    print(f"C4 persistent WLS: tiles {choice}, cost rel {abs(cost - ref_cost) / ref_cost:.2e}, "
          f"grad rel-L2 {rel_l2(grad, ref_grad):.2e}")
    assert abs(cost - ref_cost) <= TOL * abs(ref_cost)
    assert rel_l2(grad, ref_grad) <= TOL


def test_wls_bounded_wait_runs_out():
    import torch
    from yoricktrtt_b200 import _lib
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz
    nt = 2
    sc, t_index = _gated_scan(nt, [3, 4], n=(16, 16, 12), nd=32, rsc=60.0, rsd=90.0, seed=4)
    gates = P.breathing_gates(16, 16, 12, nt, 1.0, amplitude_mm=2.0, seed=5)
    pr = Projector3D(sc)
    pr.set_gates(nt, t_index)
    xc = columns_from_xyz(torch.tensor(gates, device="cuda"))
    y = torch.rand(pr.detector_shape(), device="cuda")
    grad = torch.zeros_like(xc)
    pr.set_persistent(wait_seconds=0.05, extra_wait=1)  # a band item that never finishes
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    pr.wls_grad(xc, y, grad)
    b.record()
    torch.cuda.synchronize()
    assert a.elapsed_time(b) < 5000.0  # returned after its limit, well before any watchdog
    with pytest.raises(_lib.TrttError, match="bounded device wait"):
        pr.status()
    # the plan and the context stay usable
    pr.set_persistent(wait_seconds=2.0, extra_wait=0)
    grad.zero_()
    c1 = pr.wls_grad(xc, y, grad)
    pr.status()
    grad2 = torch.zeros_like(xc)
    c2 = pr.wls_grad(xc, y, grad2)
    pr.status()
    # the band sums are shared-memory atomics: equal to FP32 summation order
    assert abs(float(c1.item()) - float(c2.item())) <= 1e-6 * abs(float(c2.item()))
    assert rel_l2(grad.cpu().numpy(), grad2.cpu().numpy()) <= 1e-6
