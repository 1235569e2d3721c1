"""Reconstruction layer: TV / spline / WLS kernels against FP64 numpy, the
FP64 restatement's gradient against finite differences (CPU), and the GPU
VMLM-B iteration against the FP64 CPU restatement on a small 2D scan."""
import numpy as np
import pytest

from conftest import rel_l2


def test_oracle_tv_gradient_fd():
    from oracle import recon_oracle as R
    rng = np.random.default_rng(0)
    for shape in [(7, 9), (4, 5, 6)]:
        x = rng.random(shape)
        f0, g = R.tv(R.spline_sample(x), 1e-2)
        # gradient of TV(S x) is S^T g, S symmetric
        gx = R.spline_sample(g)
        d = rng.standard_normal(shape)
        h = 1e-6
        fp, _ = R.tv(R.spline_sample(x + h * d), 1e-2)
        fm, _ = R.tv(R.spline_sample(x - h * d), 1e-2)
        assert abs((fp - fm) / (2 * h) - np.sum(gx * d)) <= 1e-6 * max(1.0, abs(np.sum(gx * d)))


def test_oracle_spline_is_symmetric():
    from oracle import recon_oracle as R
    rng = np.random.default_rng(1)
    a, b = rng.random((5, 6, 7)), rng.random((5, 6, 7))
    assert abs(np.sum(R.spline_sample(a) * b) - np.sum(a * R.spline_sample(b))) < 1e-12


@pytest.mark.gpu
def test_tv_spline_wls_kernels():
    import ctypes as C

    import torch
    from oracle import recon_oracle as R
    from yoricktrtt_b200 import _lib
    from yoricktrtt_b200.recon import _Scalar, _ptr, dot
    lib = _lib.load()
    rng = np.random.default_rng(2)
    for shape in [(33, 47), (12, 20, 18)]:
        x = rng.random(shape)
        xt = torch.tensor(x, dtype=torch.float32, device="cuda")
        nz, ny, nx = (1,) + shape if len(shape) == 2 else shape
        z = torch.empty_like(xt)
        tmp = torch.empty_like(xt)
        _lib.check(lib.trtt_b200_spline_sample(_ptr(xt), _ptr(z), _ptr(tmp), nx, ny, nz, None), "s")
        torch.cuda.synchronize()
        zr = R.spline_sample(x)
        assert rel_l2(z.double().cpu().numpy(), zr) <= 1e-6
        acc = _Scalar(xt.device)
        g = torch.zeros_like(xt)
        _lib.check(lib.trtt_b200_tv(_ptr(z), nx, ny, nz, 1e-2, 0.5, _ptr(g), acc.reset(), None), "tv")
        f = acc.value()
        fr, gr = R.tv(z.double().cpu().numpy(), 1e-2)
        assert abs(f - 0.5 * fr) <= 1e-6 * abs(fr)
        assert rel_l2(g.double().cpu().numpy(), 0.5 * gr) <= 1e-5
        assert abs(dot(xt, z) - float(np.sum(x.astype(np.float32).astype(np.float64) *
                                              z.double().cpu().numpy()))) <= 1e-9 * abs(dot(xt, z))
    # weighted residual
    hx = torch.rand(1000, device="cuda")
    y = torch.rand(1000, device="cuda")
    w = torch.rand(1000, device="cuda")
    wr = torch.empty_like(hx)
    acc = _Scalar(hx.device)
    _lib.check(lib.trtt_b200_wls_residual(_ptr(hx), _ptr(y), _ptr(w), _ptr(wr), 1000, acc.reset(), None),
               "wls")
    r = (hx - y).double()
    ref = 0.5 * float((w.double() * r * r).sum())
    assert abs(acc.value() - ref) <= 1e-6 * ref  # w*r is formed in FP32
    assert rel_l2(wr.double().cpu().numpy(), (w.double() * r).cpu().numpy()) <= 1e-7


@pytest.mark.gpu
def test_vmlmb_matches_fp64_restatement():
    """Same scan, data, weights and iteration rules: the GPU iterate follows
    the FP64 CPU restatement (differences come only from FP32 projections)."""
    import torch
    from oracle import oracle, recon_oracle as R
    from yoricktrtt_b200 import geometry as G, phantoms as P
    from yoricktrtt_b200.recon import Objective, Projector2D, vmlmb
    sc = G.circular_scan_2d(48, 48, 1.0, 3, 70, 1.0, 30, mode=G.TRTT_PARALLEL_BEAM)
    truth = P.ellipses_2d(48, 48, n=6, seed=7)
    orc = oracle.get("port")

    def project(x):
        out = np.zeros((sc.nviews, sc.nv))
        xc = np.ascontiguousarray(x)
        for v in range(sc.nviews):
            orc.p2d("PB2D", out[v], xc, sc, v, 0, None)
        return out

    def backproject(r):
        out = np.zeros((sc.ny, sc.nx))
        for v in range(sc.nviews):
            orc.p2d("PB2D", out, np.ascontiguousarray(r[v]), sc, v, 1, None)
        return out

    rng = np.random.default_rng(3)
    y = project(truth)
    y = y + 0.01 * y.max() * rng.standard_normal(y.shape)
    fg_cpu = R.objective(project, backproject, y, mu=1e-2, eps=1e-2)
    x_cpu, f_cpu, it_cpu = R.vmlmb(fg_cpu, np.zeros_like(truth), lower=0.0, maxiter=8, frtol=0.0)

    pr = Projector2D(sc)
    obj = Objective(pr, torch.tensor(y, dtype=torch.float32, device="cuda"), mu=1e-2, eps=1e-2)
    x_gpu, info = vmlmb(obj, torch.zeros(48, 48, device="cuda"), lower=0.0, maxiter=8, frtol=0.0)
    pr.status()
    assert info.iterations == it_cpu == 8
    assert abs(info.f[-1] - f_cpu[-1]) <= 1e-4 * abs(f_cpu[-1])
    assert rel_l2(x_gpu.double().cpu().numpy(), x_cpu) <= 2e-3
    # the iteration decreases the objective and approaches the phantom
    assert info.f[-1] < 0.2 * info.f[0]


@pytest.mark.gpu
def test_native_vmlmb_matches_python_driver():
    """trtt_b200_recon3d (C++ driver, fused kernels) against recon.vmlmb on
    recon.Objective: same cost, same rules, on a small 3D cone-beam scan
    with weights, bounds and TV."""
    import torch
    from yoricktrtt_b200 import geometry as G, phantoms as P
    from yoricktrtt_b200.projectors import Projector3D
    from yoricktrtt_b200.recon import Objective, vmlmb, vmlmb_native
    sc = G.circular_scan_3d(32, 32, 24, 1.0, 3, 56, 40, 1.0, 1.0, 30)
    pr = Projector3D(sc)
    truth = torch.tensor(P.ellipsoids_3d(32, 32, 24, n=8, seed=4), device="cuda")
    y = pr.forward(truth)
    g = torch.Generator(device="cuda").manual_seed(9)
    y = y + 0.02 * float(y.max()) * torch.randn(y.shape, device="cuda", generator=g)
    w = torch.rand(y.shape, device="cuda", generator=g) + 0.5
    obj = Objective(pr, y, w, mu=0.5, eps=1e-2)
    x_py, info_py = vmlmb(obj, torch.zeros_like(truth), lower=0.0, upper=2.0, maxiter=25, frtol=0.0)
    x_c, info_c = vmlmb_native(pr, y, w, None, mu=0.5, eps=1e-2, lower=0.0, upper=2.0, maxiter=25,
                               frtol=0.0)
    pr.status()
    assert info_c.iterations == info_py.iterations == 25
    f_py, f_c = np.array(info_py.f), np.array(info_c.f)
    assert np.max(np.abs(f_c - f_py) / np.abs(f_py)) <= 1e-4
    assert rel_l2(x_c.double().cpu().numpy(), x_py.double().cpu().numpy()) <= 1e-3
    assert float(x_c.min()) >= 0.0 and float(x_c.max()) <= 2.0
    # columns layout gives the same result (up to the atomics' summation order,
    # which differs from run to run and grows over the iterations)
    from yoricktrtt_b200.projectors import xyz_from_columns
    x_col, info_col = vmlmb_native(pr, y, w, None, mu=0.5, eps=1e-2, lower=0.0, upper=2.0, maxiter=25,
                                   frtol=0.0, layout="columns")
    assert rel_l2(xyz_from_columns(x_col).double().cpu().numpy(), x_c.double().cpu().numpy()) <= 1e-3
    # stopping rule
    _, info_s = vmlmb_native(pr, y, w, None, mu=0.5, eps=1e-2, lower=0.0, maxiter=500, frtol=1e-6)
    assert info_s.converged and info_s.iterations < 500
