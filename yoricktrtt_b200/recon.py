"""Regularised reconstruction on the GPU: weighted least squares + total
variation, minimised by VMLM-B (limited-memory variable metric with bound
constraints).

Mirrors the cost function of the reference
(``Tomography_3D/Ytrtt3D_optim.i:128-234``):

    f(x) = 1/2 sum_k (H_k x - y_k)' W_k (H_k x - y_k) + mu * TV(S x)

with x the B-spline coefficients, S the sampling of the spline at the voxel
centres and TV the smoothed isotropic total variation, minimised under the
bounds ``lower <= x <= upper`` by ``op_mnb`` (OptimPack's VMLM-B, called at
``Tomography_3D/Ytrtt3D_optim.i:663``).  OptimPack and YTotVar are external
packages absent from the reference repository, so the optimiser and the
regulariser here are restated from their published definitions
(Thiebaut 2002, "Optimization issues in blind deconvolution algorithms";
smoothed TV sqrt(|grad z|^2 + eps^2)); ``oracle/recon_oracle.py`` is the FP64
CPU restatement of the same iteration used to check this one.

All vectors stay on the device in FP32; inner products, the objective and
the line-search scalars are FP64.
"""
from __future__ import annotations

import ctypes as C
import math
import time
import warnings
from dataclasses import dataclass, field

import numpy as np

from . import _lib


def _torch():
    import torch
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class _Scalar:
    """A device FP64 accumulator read back after each kernel sequence."""

    def __init__(self, device):
        torch = _torch()
        self.t = torch.zeros(1, dtype=torch.float64, device=device)

    def reset(self):
        self.t.zero_()
        return _ptr(self.t)

    def value(self) -> float:
        return float(self.t.item())


def dot(a, b, acc: _Scalar | None = None) -> float:
    """FP64-accumulated inner product of two FP32 device tensors."""
    acc = acc or _Scalar(a.device)
    _lib.check(_lib.load().trtt_b200_dot(_ptr(a), _ptr(b), a.numel(), acc.reset(), _stream()),
               "trtt_b200_dot")
    return acc.value()


class Projector2D:
    """All views of a 2D B-spline (trtt_PB2D/FB2D) or Long-Fessler scan on
    one GPU.  Images are (ny, nx) float32, sinograms (nviews, nv)."""

    def __init__(self, scan=None, table=None, lf_params=None, beta=None, offset=None,
                 line_integ=False):
        torch = _torch()
        if not torch.cuda.is_available():
            raise _lib.TrttError("Projector2D needs a CUDA device (no CPU fallback)")
        lib = _lib.load()
        h = C.c_void_p()
        if lf_params is not None:
            beta = np.ascontiguousarray(beta, dtype=np.float64)
            offset = np.ascontiguousarray(offset, dtype=np.float64)
            rc = lib.trtt_b200_plan2d_create_lf(C.byref(h), C.addressof(lf_params),
                                                1 if line_integ else 0, len(beta),
                                                _lib.dptr(beta), _lib.dptr(offset))
            self.nx, self.ny = lf_params.objectDimension1, lf_params.objectDimension2
            self.nv, self.nviews = lf_params.detectorDimension, len(beta)
        else:
            from .geometry import TRTT_PARALLEL_BEAM
            geom = 3 if scan.mode == TRTT_PARALLEL_BEAM else 5
            xos = np.ascontiguousarray(scan.xos)
            xsd = np.ascontiguousarray(scan.xsd)
            if table is None:
                rc = lib.trtt_b200_plan2d_create(C.byref(h), geom, scan.nx, scan.ny, scan.s_scl,
                                                 scan.s_deg, None, 0, 1.0, None, scan.nv,
                                                 scan.v_scl, scan.nviews, _lib.dptr(xos),
                                                 _lib.dptr(xsd))
            else:
                rc = lib.trtt_b200_plan2d_create(C.byref(h), geom, scan.nx, scan.ny, scan.s_scl,
                                                 scan.s_deg, _lib.dptr(table.cum), table.size,
                                                 table.step, _lib.dptr(table.coord), scan.nv,
                                                 scan.v_scl, scan.nviews, _lib.dptr(xos),
                                                 _lib.dptr(xsd))
            self.nx, self.ny, self.nv, self.nviews = scan.nx, scan.ny, scan.nv, scan.nviews
        _lib.check(rc, "trtt_b200_plan2d_create")
        self._h = h

    def forward(self, x, out=None):
        torch = _torch()
        if out is None:
            out = torch.zeros(self.nviews, self.nv, dtype=torch.float32, device=x.device)
        _lib.check(_lib.load().trtt_b200_plan2d_forward(self._h, _ptr(x), _ptr(out), _stream()),
                   "trtt_b200_plan2d_forward")
        return out

    def backward(self, y, out=None):
        torch = _torch()
        if out is None:
            out = torch.zeros(self.ny, self.nx, dtype=torch.float32, device=y.device)
        _lib.check(_lib.load().trtt_b200_plan2d_backward(self._h, _ptr(y), _ptr(out), _stream()),
                   "trtt_b200_plan2d_backward")
        return out

    def status(self):
        _lib.check(_lib.load().trtt_b200_plan2d_status(self._h, _stream()), "projector")

    def sparse_system(self, max_cells: int = 64) -> "SparseSystem2D":
        """The plan's system matrix H, assembled once, for sparse products
        (B-spline plans only)."""
        return SparseSystem2D(self, max_cells)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().trtt_b200_plan2d_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class SparseSystem2D:
    """Precomputed-matrix mode of a 2D B-spline plan (the reference's sparse
    system, Ytrtt_2D_projectors.i:212-369, applied with trtt_mvmult in
    Tomography_2D/Ytrtt2D_optim.i:320-387).  H (nviews*nv x ny*nx) is
    assembled on the GPU by trtt_b200_plan2d_assemble, sorted once into
    compressed rows for H and for H^T (torch's sparse conversion, done
    once), and every product is one trtt_b200_csr_spmv launch in FP64.
    Images are (ny, nx), sinograms (nviews, nv), float64 CUDA tensors."""

    def __init__(self, plan: Projector2D, max_cells: int = 64):
        torch = _torch()
        lib = _lib.load()
        self.nx, self.ny, self.nv, self.nviews = plan.nx, plan.ny, plan.nv, plan.nviews
        npix = self.nx * self.ny
        n = self.nviews * npix * max_cells
        a = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = torch.zeros(n, dtype=torch.int64, device="cuda")
        c = torch.zeros(n, dtype=torch.int64, device="cuda")
        _lib.check(lib.trtt_b200_plan2d_assemble(plan._h, max_cells, _ptr(a), _ptr(r), _ptr(c),
                                                 _stream()), "trtt_b200_plan2d_assemble")
        plan.status()  # a footprint wider than max_cells or a source-plane pixel raises here
        view = torch.arange(n, device="cuda") // (npix * max_cells)
        keep = r > 0
        rows = view[keep] * self.nv + (r[keep] - 1)
        cols = c[keep] - 1
        vals = a[keep]
        shape = (self.nviews * self.nv, npix)
        with warnings.catch_warnings():  # torch flags its CSR layout as beta; only the sort is used
            warnings.simplefilter("ignore", UserWarning)
            h = torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, shape).coalesce().to_sparse_csr()
            ht = torch.sparse_coo_tensor(torch.stack([cols, rows]), vals,
                                         shape[::-1]).coalesce().to_sparse_csr()
        self._h = (h.crow_indices().contiguous(), h.col_indices().contiguous(), h.values().contiguous())
        self._ht = (ht.crow_indices().contiguous(), ht.col_indices().contiguous(), ht.values().contiguous())
        self.nnz = int(vals.numel())

    def _apply(self, m, nrows, ncols, x, out, accumulate):
        _lib.check(_lib.load().trtt_b200_csr_spmv(_ptr(m[0]), _ptr(m[1]), _ptr(m[2]), nrows, ncols,
                                                  _ptr(x), _ptr(out), 1 if accumulate else 0,
                                                  _stream()), "trtt_b200_csr_spmv")
        return out

    def forward(self, x, out=None, accumulate=False):
        """H x: image (ny, nx) -> sinogram (nviews, nv)."""
        torch = _torch()
        if out is None:
            out = torch.empty(self.nviews, self.nv, dtype=torch.float64, device=x.device)
        return self._apply(self._h, self.nviews * self.nv, self.nx * self.ny, x.contiguous(), out, accumulate)

    def backward(self, y, out=None, accumulate=False):
        """H^T y: sinogram (nviews, nv) -> image (ny, nx)."""
        torch = _torch()
        if out is None:
            out = torch.empty(self.ny, self.nx, dtype=torch.float64, device=y.device)
        return self._apply(self._ht, self.nx * self.ny, self.nviews * self.nv, y.contiguous(), out, accumulate)

    def status(self):
        _lib.check(_lib.load().trtt_b200_csr_status(_stream()), "sparse product")


class Objective:
    """f(x) = 1/2 ||Hx - y||^2_W + mu TV(S x) and its gradient.

    ``proj`` has forward(x, out) / backward(r, out) (Projector2D, or
    Projector3D on (nz, ny, nx) volumes); ``y`` and ``w`` have the detector
    shape (``w`` None: unit weights).  ``spline=True`` applies TV to the
    spline samples S x, as the reference does; False to x itself."""

    def __init__(self, proj, y, w=None, mu=0.0, eps=1e-3, spline=True):
        torch = _torch()
        self.proj, self.y, self.w = proj, y, w
        self.mu, self.eps, self.spline = float(mu), float(eps), spline
        self.hx = torch.empty_like(y)
        self.wr = torch.empty_like(y)
        self._acc = _Scalar(y.device)
        self.nevals = 0

    def _dims(self, x):
        if x.dim() == 2:
            return x.shape[1], x.shape[0], 1
        return x.shape[2], x.shape[1], x.shape[0]

    def __call__(self, x):
        torch = _torch()
        lib = _lib.load()
        st = _stream()
        self.hx.zero_()
        self.proj.forward(x, out=self.hx)
        facc = self._acc.reset()
        _lib.check(lib.trtt_b200_wls_residual(_ptr(self.hx), _ptr(self.y),
                                              _ptr(self.w) if self.w is not None else None,
                                              _ptr(self.wr), self.y.numel(), facc, st),
                   "trtt_b200_wls_residual")
        g = torch.zeros_like(x)
        self.proj.backward(self.wr, out=g)
        if self.mu > 0:
            nx, ny, nz = self._dims(x)
            if self.spline:
                z = torch.empty_like(x)
                tmp = torch.empty_like(x)
                _lib.check(lib.trtt_b200_spline_sample(_ptr(x), _ptr(z), _ptr(tmp), nx, ny, nz, st),
                           "spline_sample")
                gz = torch.zeros_like(x)
                _lib.check(lib.trtt_b200_tv(_ptr(z), nx, ny, nz, self.eps, self.mu, _ptr(gz),
                                            facc, st), "trtt_b200_tv")
                sg = torch.empty_like(x)
                _lib.check(lib.trtt_b200_spline_sample(_ptr(gz), _ptr(sg), _ptr(tmp), nx, ny, nz, st),
                           "spline_sample")
                g += sg
            else:
                _lib.check(lib.trtt_b200_tv(_ptr(x), nx, ny, nz, self.eps, self.mu, _ptr(g), facc, st),
                           "trtt_b200_tv")
        self.nevals += 1
        return self._acc.value(), g


@dataclass
class VMLMBInfo:
    iterations: int = 0
    evaluations: int = 0
    f: list = field(default_factory=list)
    times: list = field(default_factory=list)
    converged: bool = False
    reason: str = ""


_REASONS = {1: "relative objective change below frtol", 2: "projected gradient is zero",
            0: "", -1: "line search failed"}


def vmlmb_native(proj, y, w=None, x0=None, mu=0.0, eps=1e-3, lower=0.0, upper=None, mem=5,
                 maxiter=100, frtol=1e-6, layout="xyz", stream=None):
    """VMLM-B + TV on a Projector3D with the native solver
    (trtt_b200_recon3d): the cost of ``Objective`` (spline=True) and the
    rules of ``vmlmb``, driven from C++ with fused vector kernels.
    Returns (x, VMLMBInfo) like ``vmlmb``."""
    torch = _torch()
    from .projectors import LAYOUTS
    if proj.nt != 1:
        raise ValueError("vmlmb_native: gated (4D) projectors are not supported")
    shape = proj.volume_shape(layout)
    x = (torch.zeros(shape, device=y.device) if x0 is None else x0).clone().contiguous()
    if tuple(x.shape) != tuple(shape) or x.dtype != torch.float32:
        raise ValueError(f"x0 must be float32 with shape {tuple(shape)}")
    y = y.contiguous()
    w = None if w is None else w.contiguous()
    fh = np.zeros(maxiter + 1)
    th = np.zeros(maxiter + 1)
    info_c = _lib.VMLMBInfoC()
    st = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
    rc = _lib.load().trtt_b200_recon3d(
        proj._h, _ptr(y), _ptr(w) if w is not None else None, _ptr(x), LAYOUTS[layout], float(mu),
        float(eps), -math.inf if lower is None else float(lower), math.inf if upper is None else float(upper),
        int(mem), int(maxiter), float(frtol), fh.ctypes.data_as(C.POINTER(C.c_double)),
        th.ctypes.data_as(C.POINTER(C.c_double)), C.byref(info_c), st)
    _lib.check(rc, "trtt_b200_recon3d")
    k = info_c.iterations
    info = VMLMBInfo(iterations=k, evaluations=info_c.evaluations, f=fh[:k + 1].tolist(),
                     times=th[:k + 1].tolist(), converged=info_c.converged > 0,
                     reason=_REASONS.get(info_c.converged, ""))
    return x, info


def dot_dev(a, b):
    """FP64-accumulated inner product left on the device (0-dim float64
    tensor), so that several can be read back with one synchronisation."""
    torch = _torch()
    out = torch.zeros((), dtype=torch.float64, device=a.device)
    _lib.check(_lib.load().trtt_b200_dot(_ptr(a), _ptr(b), a.numel(), _ptr(out), _stream()),
               "trtt_b200_dot")
    return out


def _fetch(*vals):
    """Read several device scalars with one synchronisation."""
    torch = _torch()
    return torch.stack([v.reshape(()) for v in vals]).tolist()


def vmlmb(fg, x0, lower=0.0, upper=None, mem=5, maxiter=100, frtol=1e-6, armijo=1e-4,
          max_backtrack=30, callback=None):
    """VMLM-B: L-BFGS restricted to the free variables of the box
    lower <= x <= upper, projected Armijo backtracking with safeguarded
    quadratic steps, stop when |f_k - f_{k+1}| <= frtol max(|f_k|,|f_{k+1}|).

    Inner products are FP64 (trtt_b200_dot) and stay on the device: the
    two-loop recursion applies its coefficients as device scalars, and the
    host reads back only the values it branches on (a few synchronisations
    per iteration).  The same rules are restated in FP64 on the CPU by
    oracle/recon_oracle.py.  Returns (x, VMLMBInfo)."""
    torch = _torch()
    lo = -math.inf if lower is None else float(lower)
    hi = math.inf if upper is None else float(upper)

    def clip(v):
        return v.clamp(min=None if lo == -math.inf else lo, max=None if hi == math.inf else hi)

    t0 = time.perf_counter()
    x = clip(x0.clone())
    f, g = fg(x)
    info = VMLMBInfo(evaluations=1, f=[f], times=[0.0])
    S, Y = [], []
    cand = None  # (s, y) of the last step, kept if s'y > 0
    for it in range(1, maxiter + 1):
        blocked = None
        if lo > -math.inf:
            blocked = (x <= lo) & (g > 0)
        if hi < math.inf:
            b2 = (x >= hi) & (g < 0)
            blocked = b2 if blocked is None else blocked | b2
        free = torch.ones_like(x) if blocked is None else (~blocked).to(x.dtype)
        pg = g * free
        # one read-back: |pg|^2, |x|^2, s'y of the candidate pair and the
        # free-restricted s'y of every stored pair and of the candidate
        pend = list(zip(S, Y)) + ([cand] if cand is not None else [])
        sfs = [(s * free, y * free) for s, y in pend]
        vals = [dot_dev(pg, pg), dot_dev(x, x)]
        if cand is not None:
            vals.append(dot_dev(cand[0], cand[1]))
        vals += [dot_dev(sf, yf) for sf, yf in sfs]
        got = _fetch(*vals)
        pgn, xn = math.sqrt(got[0]), math.sqrt(got[1])
        sys_free = got[3:] if cand is not None else got[2:]
        if cand is not None:
            if got[2] > 0.0:
                S.append(cand[0])
                Y.append(cand[1])
            else:
                sfs.pop()
                sys_free.pop()
            cand = None
            if len(S) > mem:
                S.pop(0)
                Y.pop(0)
                sfs.pop(0)
                sys_free.pop(0)
        if pgn == 0.0:
            info.converged, info.reason = True, "projected gradient is zero"
            break
        # two-loop recursion on the free subspace
        q = pg.clone()
        used = []
        for (sf, yf), sy in reversed(list(zip(sfs, sys_free))):
            if sy <= 0.0:
                continue
            a = dot_dev(sf, q) / sy
            q -= a * yf
            used.append((sf, yf, sy, a))
        if used:
            sf, yf, sy, _ = used[0]
            q *= sy / dot_dev(yf, yf)
            for sf, yf, sy, a in reversed(used):
                b = dot_dev(yf, q) / sy
                q += (a - b) * sf
            d = -(q * free)
            alpha = 1.0
        else:
            d = -pg
            alpha = (0.1 * xn if xn > 0 else 1.0) / pgn
        gd = _fetch(dot_dev(g, d))[0]
        if gd >= 0.0:  # not a descent direction: restart with the gradient
            S.clear()
            Y.clear()
            d = -pg
            alpha = (0.1 * xn if xn > 0 else 1.0) / pgn
            gd = _fetch(dot_dev(g, d))[0]
        for _ in range(max_backtrack):
            xt = clip(x + alpha * d)
            step = xt - x
            gs = dot_dev(g, step)
            ft, gt = fg(xt)
            info.evaluations += 1
            if ft <= f + armijo * _fetch(gs)[0]:
                break
            # safeguarded quadratic interpolation of phi(alpha)
            denom = 2.0 * (ft - f - gd * alpha)
            aq = -gd * alpha * alpha / denom if denom > 0 else 0.5 * alpha
            alpha = min(max(aq, 0.1 * alpha), 0.5 * alpha)
        else:
            info.reason = "line search failed"
            break
        cand = (step, gt - g)
        fprev = f
        x, f, g = xt, ft, gt
        info.iterations = it
        info.f.append(f)
        info.times.append(time.perf_counter() - t0)
        if callback:
            callback(it, x, f)
        if abs(fprev - f) <= frtol * max(abs(fprev), abs(f)):
            info.converged, info.reason = True, "relative objective change below frtol"
            break
    return x, info
