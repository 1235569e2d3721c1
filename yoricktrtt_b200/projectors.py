"""Operator layer: multi-view B200 projectors on device-resident tensors.

Mirrors the Yorick operator layer of TRTT (``Ytrtt_3D_projectors.i:56-187``):
a projector is built from a tomographic object and a set of views and is
applied as ``C(x, job)`` with ``job`` 0 = direct and 1 = transpose.  Here one
``Projector3D`` holds all views of a scan on the GPU (a ``trtt_b200_plan3d``)
and applies them in a single launch per direction; ``single_view`` returns
the per-view closure of the reference (``A_single_3D``).

Tensors are torch CUDA float32.  Volumes are (nz, ny, nx) in the reference
order (``layout="xyz"``) or (ny, nx, nz) columns (``layout="columns"``, the
kernels' native order, no conversion); 4D volumes carry a leading gate
axis.  Detector stacks are (nviews, nv, nu).  Results are accumulated into
``out`` when it is given, as in the reference (the caller zeroes it).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .footprint import FootprintTable
from .geometry import Scan3D, TRTT_CONE_BEAM, TRTT_FAN_BEAM, TRTT_PARALLEL_BEAM

LAYOUTS = {"xyz": 0, "columns": 1}


def _torch():
    import torch
    return torch


def _stream_ptr(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Projector3D:
    """All views of a 3D parallel / cone beam scan on one GPU.

    ``table`` selects the tabulated footprint (``trtt_PB3D``/``trtt_CB3D``);
    ``None`` the closed-form cubic one (``trtt_PB3D_cubic``/``trtt_CB3D_cubic``).
    """

    def __init__(self, scan: Scan3D, table: FootprintTable | None = None,
                 device=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise _lib.TrttError("Projector3D needs a CUDA device (no CPU fallback)")
        self.scan = scan
        self.table = table
        self.device = torch.device("cuda", torch.cuda.current_device()
                                   if device is None else torch.device(device).index or 0)
        self.nt = 1
        lib = _lib.load()
        xos = np.ascontiguousarray(scan.xos, dtype=np.float64)
        xsd = np.ascontiguousarray(scan.xsd, dtype=np.float64)
        handle = C.c_void_p()
        geom = {TRTT_PARALLEL_BEAM: 3, TRTT_CONE_BEAM: 4, TRTT_FAN_BEAM: 5}[scan.mode]
        with torch.cuda.device(self.device):
            if table is None:
                rc = lib.trtt_b200_plan3d_create(
                    C.byref(handle), geom, scan.nx, scan.ny, scan.nz, scan.s_scl,
                    scan.s_deg, None, 0, 1.0, None, scan.nu, scan.nv, scan.u_scl,
                    scan.v_scl, scan.nviews, _lib.dptr(xos), _lib.dptr(xsd))
            else:
                rc = lib.trtt_b200_plan3d_create(
                    C.byref(handle), geom, scan.nx, scan.ny, scan.nz, scan.s_scl,
                    scan.s_deg, _lib.dptr(table.cum), table.size, table.step,
                    _lib.dptr(table.coord), scan.nu, scan.nv, scan.u_scl, scan.v_scl,
                    scan.nviews, _lib.dptr(xos), _lib.dptr(xsd))
        _lib.check(rc, "trtt_b200_plan3d_create")
        self._h = handle

    # -- configuration -------------------------------------------------------
    def set_gates(self, nt: int, t_index) -> None:
        """4D: view k projects the linear interpolation of gates floor/ceil of
        t_index[k] (Ytrtt_3D_projectors.i:301-311)."""
        t = np.ascontiguousarray(t_index, dtype=np.float64)
        if t.shape != (self.scan.nviews,):
            raise ValueError("t_index must have one entry per view")
        _lib.check(_lib.load().trtt_b200_plan3d_set_gates(self._h, nt, _lib.dptr(t)),
                   "trtt_b200_plan3d_set_gates")
        self.nt = int(nt)

    def set_tiles(self, band_rows: int = 0, warps: int = 0, cols: int = 1) -> None:
        """Direct-projector kernel shape: (band rows, warps) of the band kernel
        ((0, 0): automatic; (-2, 0): atomic-free variant; (-3, 0): band
        accumulated on the tensor cores) and the number of neighbouring
        columns spread together (1 or 2)."""
        lib = _lib.load()
        _lib.check(lib.trtt_b200_plan3d_set_columns(self._h, 1), "trtt_b200_plan3d_set_columns")
        _lib.check(lib.trtt_b200_plan3d_set_tiles(self._h, band_rows, warps),
                   "trtt_b200_plan3d_set_tiles")
        _lib.check(lib.trtt_b200_plan3d_set_columns(self._h, cols), "trtt_b200_plan3d_set_columns")

    def set_symmetry(self, on=True) -> None:
        """Use (default) or bypass the group kernels that share footprints
        between views related by turns of the volume grid: True or 2 (the
        default: interleaved member profiles in the direct group kernel), 1
        (one profile per member, shared-memory atomics), False or 0."""
        mode = int(on) if not isinstance(on, bool) else (2 if on else 0)
        _lib.check(_lib.load().trtt_b200_plan3d_set_symmetry(self._h, mode),
                   "trtt_b200_plan3d_set_symmetry")

    def groups(self):
        """(singles, pairs, quads) of views the group kernels use."""
        c = (C.c_long * 3)()
        _lib.check(_lib.load().trtt_b200_plan3d_groups(self._h, c), "trtt_b200_plan3d_groups")
        return tuple(int(x) for x in c)

    def set_group_shape(self, band_rows4=0, utile4=0, ctas_per_sm4=0):
        """Direct kernel shape for groups of 4 views (see
        trtt_b200_plan3d_set_group_shape)."""
        _lib.check(_lib.load().trtt_b200_plan3d_set_group_shape(self._h, band_rows4, utile4, ctas_per_sm4),
                   "trtt_b200_plan3d_set_group_shape")

    def set_group_tiles(self, band_rows4=0, band_rows2=0, band_rows1=0, back_chunk_bytes=0):
        _lib.check(_lib.load().trtt_b200_plan3d_set_group_tiles(
            self._h, band_rows4, band_rows2, band_rows1, back_chunk_bytes),
            "trtt_b200_plan3d_set_group_tiles")

    def wls_grad(self, vol, y, grad, w=None, cost=None):
        """One persistent launch: grad += H^T W (H vol - y), returns the
        device FP64 cost 1/2 sum W (H vol - y)^2 (columns layout, gates
        stacked; y, w: (nviews, nv, nu) float32)."""
        torch = _torch()
        if cost is None:
            cost = torch.zeros(1, dtype=torch.float64, device=vol.device)
        self._check(vol, self.volume_shape("columns"), "vol")
        self._check(grad, self.volume_shape("columns"), "grad")
        self._check(y, self.detector_shape(), "y")
        if w is not None:
            self._check(w, self.detector_shape(), "w")
        lib = _lib.load()
        _lib.check(lib.trtt_b200_plan3d_wls_grad(
            self._h, C.c_void_p(vol.data_ptr()), C.c_void_p(y.data_ptr()),
            C.c_void_p(w.data_ptr()) if w is not None else None, C.c_void_p(grad.data_ptr()),
            C.c_void_p(cost.data_ptr()), _stream_ptr(torch.cuda.current_stream())),
            "trtt_b200_plan3d_wls_grad")
        return cost

    def set_persistent(self, band_rows=0, ctas_per_sm=0, wait_seconds=0.0, extra_wait=0):
        _lib.check(_lib.load().trtt_b200_plan3d_set_persistent(
            self._h, band_rows, ctas_per_sm, float(wait_seconds), extra_wait),
            "trtt_b200_plan3d_set_persistent")

    WLS_CANDIDATES = [(16, 1), (32, 1), (16, 2), (32, 2), (8, 2)]

    def autotune_wls(self, vol, y, w=None, candidates=None, reps=2):
        """Time the persistent launch with each (band rows, CTAs per SM)
        candidate on the given data and keep the fastest; returns
        ({candidate: ms}, choice)."""
        torch = _torch()
        grad = torch.zeros_like(vol)
        times = {}
        for cand in candidates or self.WLS_CANDIDATES:
            try:
                self.set_persistent(*cand)
            except _lib.TrttError:
                continue
            self.wls_grad(vol, y, grad, w)
            torch.cuda.synchronize()
            best = math.inf
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                self.wls_grad(vol, y, grad, w)
                b.record()
                torch.cuda.synchronize()
                best = min(best, a.elapsed_time(b))
            times[cand] = best
        self.status()
        choice = min(times, key=times.get)
        self.set_persistent(*choice)
        self.wls_tiles = choice
        return times, choice

    @property
    def factorized(self) -> bool:
        return bool(_lib.load().trtt_b200_plan3d_factorized(self._h))

    # -- shapes ---------------------------------------------------------------
    def volume_shape(self, layout="xyz"):
        s = self.scan
        base = (s.nz, s.ny, s.nx) if layout == "xyz" else (s.ny, s.nx, s.nz)
        return ((self.nt,) + base) if self.nt > 1 else base

    def detector_shape(self, nviews=None):
        s = self.scan
        return (s.nviews if nviews is None else nviews, s.nv, s.nu)

    def _check(self, t, shape, name):
        torch = _torch()
        if not isinstance(t, torch.Tensor) or t.device.type != "cuda" or t.dtype != torch.float32:
            raise TypeError(f"{name} must be a float32 CUDA tensor")
        if tuple(t.shape) != tuple(shape) or not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous with shape {tuple(shape)}, got {tuple(t.shape)}")

    # -- application ------------------------------------------------------------
    def forward(self, vol, out=None, view0: int = 0, nview: int | None = None,
                layout: str = "xyz", stream=None):
        """out[v] += H_v vol for views [view0, view0+nview)."""
        torch = _torch()
        nview = self.scan.nviews - view0 if nview is None else nview
        self._check(vol, self.volume_shape(layout), "vol")
        if out is None:
            out = torch.zeros(self.detector_shape(nview), dtype=torch.float32, device=vol.device)
        self._check(out, self.detector_shape(nview), "out")
        rc = _lib.load().trtt_b200_plan3d_forward(
            self._h, C.c_void_p(vol.data_ptr()), C.c_void_p(out.data_ptr()), view0, nview,
            LAYOUTS[layout], _stream_ptr(stream))
        _lib.check(rc, "trtt_b200_plan3d_forward")
        return out

    def backward(self, sino, out=None, view0: int = 0, nview: int | None = None,
                 layout: str = "xyz", stream=None):
        """out += sum_v H_v^T sino[v] over views [view0, view0+nview)."""
        torch = _torch()
        nview = self.scan.nviews - view0 if nview is None else nview
        self._check(sino, self.detector_shape(nview), "sino")
        if out is None:
            out = torch.zeros(self.volume_shape(layout), dtype=torch.float32, device=sino.device)
        self._check(out, self.volume_shape(layout), "out")
        rc = _lib.load().trtt_b200_plan3d_backward(
            self._h, C.c_void_p(sino.data_ptr()), C.c_void_p(out.data_ptr()), view0, nview,
            LAYOUTS[layout], _stream_ptr(stream))
        _lib.check(rc, "trtt_b200_plan3d_backward")
        return out

    def __call__(self, x, job: int = 0, **kw):
        """Yorick-style evaluator C(x, job): job 0 direct, 1 transpose."""
        if job == 0:
            return self.forward(x, **kw)
        if job == 1:
            return self.backward(x, **kw)
        raise ValueError("unsupported job (0 = direct, 1 = transpose)")

    # -- tuning and graph capture ----------------------------------------------
    # (-3, 0), the tensor-core band kernel, is not a candidate: its FP32
    # accumulation in tensor memory rounds toward zero, which at 256^3 ->
    # 512^2 leaves 1.5-1.8e-5 relative error against FP64 (the CUDA-core
    # kernels: 4.6e-7)
    TILE_CANDIDATES = [(0, 0), (16, 16), (24, 16), (32, 8), (32, 12), (48, 8), (-2, 0),
                       (0, 0, 2), (32, 16, 2), (32, 8, 2), (24, 8, 2), (16, 16, 2)]

    def autotune(self, vol=None, layout="columns", candidates=None, reps=2, nview=None):
        """Time the direct projector with each candidate (band_rows, warps[,
        cols]) setting (see set_tiles; (-2, 0) is the atomic-free band
        kernel, cols = 2 the column-pair kernel) on `vol` (random data of the
        plan's volume shape if None) and keep the fastest.  Returns
        {candidate: ms} and the choice."""
        torch = _torch()
        if vol is None:
            vol = torch.rand(self.volume_shape(layout), device=self.device)
        nview = min(self.scan.nviews, nview or 32)
        out = torch.zeros(self.detector_shape(nview), device=vol.device)
        times = {}
        for cand in candidates or self.TILE_CANDIDATES:
            try:
                self.set_tiles(*cand)
            except _lib.TrttError:
                continue
            self.forward(vol, out=out, nview=nview, layout=layout)
            torch.cuda.synchronize()
            best = math.inf
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                self.forward(vol, out=out, nview=nview, layout=layout)
                b.record()
                torch.cuda.synchronize()
                best = min(best, a.elapsed_time(b))
            times[cand] = best
        choice = min(times, key=times.get)
        self.set_tiles(*choice)
        self.tiles = choice
        return times, choice

    def capture(self, fn):
        """Capture `fn()` (a sequence of forward/backward calls on fixed
        tensors) into a CUDA graph after one warm-up run; returns the graph
        (replay with graph.replay())."""
        torch = _torch()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fn()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        torch.cuda.synchronize()
        return g

    def status(self, stream=None) -> None:
        """Raise if a kernel flagged an error (a voxel in the source plane)."""
        _lib.check(_lib.load().trtt_b200_plan3d_status(self._h, _stream_ptr(stream)),
                   "projector")

    def single_view(self, k: int):
        """Per-view closure ``A_single_3D`` (Ytrtt_3D_projectors.i:56-138)."""
        def op(x, job=0, **kw):
            return self(x, job, view0=k, nview=1, **kw)
        return op

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().trtt_b200_plan3d_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass


def columns_from_xyz(vol):
    """(…, nz, ny, nx) -> (…, ny, nx, nz) (reference order to kernel order)."""
    return vol.movedim(-3, -1).contiguous()


def xyz_from_columns(vol):
    """(…, ny, nx, nz) -> (…, nz, ny, nx)."""
    return vol.movedim(-1, -3).contiguous()
