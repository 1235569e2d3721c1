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
