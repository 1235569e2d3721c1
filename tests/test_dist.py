"""View-parallel evaluation on CPU ranks (gloo, world size 2 and 3): the
sharded data-fidelity value and gradient equal the single-process ones, and
a rank that fails before the collective makes the others fail (no hang).

The per-rank projector here is the FP64 oracle on a tiny 2D fan-beam scan;
what is under test is the sharding and the reduction, not the projector."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_views_partition():
    from yoricktrtt_b200.dist import shard_views
    for nviews in (1, 7, 360, 361):
        for world in (1, 2, 3, 8):
            blocks = [shard_views(nviews, world, r) for r in range(world)]
            covered = []
            for first, count in blocks:
                covered.extend(range(first, first + count))
            assert covered == list(range(nviews))
            assert max(c for _, c in blocks) - min(c for _, c in blocks) <= 1
    with pytest.raises(ValueError):
        shard_views(10, 2, 2)


def _problem():
    sys.path.insert(0, ROOT)
    from yoricktrtt_b200 import geometry as G, phantoms as P
    sc = G.circular_scan_2d(20, 18, 1.0, 3, 40, 1.0, 7, mode=G.TRTT_FAN_BEAM, rsc=80.0, rsd=120.0)
    x = np.ascontiguousarray(P.ellipses_2d(20, 18, n=4, seed=3))
    rng = np.random.default_rng(0)
    y = rng.random((sc.nviews, sc.nv))
    w = rng.uniform(0.5, 1.5, (sc.nviews, sc.nv))
    return sc, x, y, w


def _ops(sc, views):
    import torch
    from oracle import oracle
    orc = oracle.get("port")

    def project(x):
        xn = np.ascontiguousarray(x.numpy())
        out = np.zeros((len(views), sc.nv))
        for n, v in enumerate(views):
            orc.p2d("FB2D", out[n], xn, sc, v, 0, None)
        return torch.from_numpy(out)

    def backproject(r):
        rn = r.numpy()
        out = np.zeros((sc.ny, sc.nx))
        for n, v in enumerate(views):
            orc.p2d("FB2D", out, np.ascontiguousarray(rn[n]), sc, v, 1, None)
        return torch.from_numpy(out)
    return project, backproject


def _rank_main(rank, world, port, q, fail_rank=-1):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from yoricktrtt_b200.dist import ShardedPair, shard_views
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected rank failure")
        sc, x, y, w = _problem()
        first, count = shard_views(sc.nviews, world, rank)
        views = list(range(first, first + count))
        project, backproject = _ops(sc, views)
        term = ShardedPair(project, backproject, torch.from_numpy(y[first:first + count]),
                           torch.from_numpy(w[first:first + count]))
        f, g = term.cost_grad(torch.from_numpy(x))
        q.put((rank, "ok", f, g.numpy()))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _spawn(world, fail_rank=-1):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, status, a, b = q.get(timeout=120)
        out[r] = (status, a, b)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_cost_grad_matches_single(world):
    import torch
    from yoricktrtt_b200.dist import ShardedPair
    sc, x, y, w = _problem()
    project, backproject = _ops(sc, list(range(sc.nviews)))
    f1, g1 = ShardedPair(project, backproject, torch.from_numpy(y), torch.from_numpy(w)).cost_grad(
        torch.from_numpy(x))
    out = _spawn(world)
    for r in range(world):
        status, f, g = out[r]
        assert status == "ok", f
        assert abs(f - f1) <= 1e-12 * abs(f1)
        assert np.allclose(g, g1.numpy(), rtol=1e-12, atol=1e-14)


def test_rank_failure_surfaces():
    out = _spawn(2, fail_rank=1)
    assert out[1][0] == "error" and "injected" in out[1][1]
    # the surviving rank's collective ends with an error instead of hanging
    assert out[0][0] == "error"


# ---------------------------------------------------------------------------
# View-sharded reconstruction
# ---------------------------------------------------------------------------
def _recon_rank(rank, world, port, q, maxiter, mu):
    """One rank of a sharded VMLM-B + TV solve with the FP64 oracle as the
    projector of its views (sharded_fg: data terms summed by all-reduce,
    TV from rank 0)."""
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from oracle import recon_oracle as RO
    from yoricktrtt_b200.dist import shard_views, sharded_fg
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        sc, _, y, w = _problem()
        first, count = shard_views(sc.nviews, world, rank)
        project, backproject = _ops(sc, list(range(first, first + count)))
        data = RO.objective(lambda x: project(_t(x)).numpy(), lambda r: backproject(_t(r)).numpy(),
                            y[first:first + count], w[first:first + count])
        fg = sharded_fg(data, lambda x: _tv_term(RO, x, mu), rank=rank)
        x, fs, _ = RO.vmlmb(fg, np.zeros((sc.ny, sc.nx)), maxiter=maxiter, frtol=0.0)
        q.put((rank, "ok", fs, x))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a))


def _tv_term(RO, x, mu, eps=1e-3):
    """mu TV(S x) and its gradient (the regulariser of the objective)."""
    ft, gz = RO.tv(RO.spline_sample(x), eps)
    return mu * ft, mu * RO.spline_sample(gz)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_reconstruction_matches_single_iterate_by_iterate(world):
    """VMLM-B + TV with the data term sharded over views on gloo ranks gives
    the single-process iterates: the same objective at every iteration and
    the same final image (FP64 oracle projectors on each rank)."""
    import multiprocessing as mp
    sys.path.insert(0, ROOT)
    from oracle import recon_oracle as RO
    maxiter, mu = 8, 0.05
    sc, _, y, w = _problem()
    project, backproject = _ops(sc, list(range(sc.nviews)))
    fg1 = RO.objective(lambda x: project(_t(x)).numpy(), lambda r: backproject(_t(r)).numpy(),
                       y, w, mu=mu)
    x1, f1, _ = RO.vmlmb(fg1, np.zeros((sc.ny, sc.nx)), maxiter=maxiter, frtol=0.0)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_recon_rank, args=(r, world, port, q, maxiter, mu))
             for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, status, fs, x = q.get(timeout=300)
        out[r] = (status, fs, x)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    for r in range(world):
        status, fs, x = out[r]
        assert status == "ok", fs
        assert len(fs) == len(f1)
        assert np.allclose(fs, f1, rtol=1e-10, atol=0.0), (r, fs, f1)
        assert np.allclose(x, x1, rtol=1e-8, atol=1e-12)


def _native_rank(rank, world, port, q, maxiter):
    """One rank of the native sharded solver (trtt_b200_recon3d_sharded) on
    the shared GPU; reductions through gloo on host copies, so no kernel of
    one rank waits for another rank's kernel."""
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from yoricktrtt_b200 import geometry as G
    from yoricktrtt_b200.dist import shard_views, vmlmb_native_sharded
    from yoricktrtt_b200.projectors import Projector3D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        sc, y, truth = _native_problem()
        first, count = shard_views(sc.nviews, world, rank)
        sub = G.Scan3D(sc.nx, sc.ny, sc.nz, sc.s_scl, sc.s_deg, sc.nu, sc.nv, sc.u_scl, sc.v_scl,
                       sc.mode, sc.xos[first:first + count].copy(), sc.xsd[first:first + count].copy())
        pr = Projector3D(sub)
        yt = torch.tensor(y[first:first + count], device="cuda")
        x, info = vmlmb_native_sharded(pr, yt, mu=0.05, maxiter=maxiter, frtol=0.0)
        q.put((rank, "ok", info.f, x.cpu().numpy()))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _native_problem():
    from yoricktrtt_b200 import geometry as G, phantoms as P
    sc = G.circular_scan_3d(28, 28, 20, 1.0, 3, 48, 44, 1.0, 1.0, 10, rsc=90.0, rsd=140.0)
    truth = P.ellipsoids_3d(28, 28, 20, n=6, seed=7)
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    y = Projector3D(sc).forward(torch.tensor(truth, device="cuda")).cpu().numpy()
    return sc, y, truth


@pytest.mark.gpu
def test_native_sharded_solver_two_ranks_one_gpu():
    """trtt_b200_recon3d_sharded on two ranks (one GPU shared, gloo
    reductions) follows the single-rank native solver iterate by iterate
    (FP32 projections: relative 1e-4 on the objective, 1e-3 on the image),
    and both ranks end with the same image."""
    import multiprocessing as mp

    import torch
    from yoricktrtt_b200.projectors import Projector3D
    from yoricktrtt_b200.recon import vmlmb_native
    maxiter = 6
    sc, y, _ = _native_problem()
    x1, info1 = vmlmb_native(Projector3D(sc), torch.tensor(y, device="cuda"), mu=0.05,
                             maxiter=maxiter, frtol=0.0)
    x1 = x1.cpu().numpy()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_native_rank, args=(r, 2, port, q, maxiter)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, status, fs, x = q.get(timeout=300)
        out[r] = (status, fs, x)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    for r in range(2):
        status, fs, x = out[r]
        assert status == "ok", fs
        assert len(fs) == len(info1.f)
        assert np.allclose(fs, info1.f, rtol=1e-4), (fs, info1.f)
        assert np.linalg.norm(x - x1) <= 1e-3 * np.linalg.norm(x1)
    assert np.array_equal(out[0][2], out[1][2]) or \
        np.linalg.norm(out[0][2] - out[1][2]) <= 1e-6 * np.linalg.norm(x1)
