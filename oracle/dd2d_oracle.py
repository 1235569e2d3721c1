"""FP64 CPU restatement of the reference's 2D distance-driven projector.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
distance-driven kernels, never by the product path.

The reference implements the distance-driven model (De Man & Basu) in
Yorick, not in its C plugin: ``_trtt_single_distance_driven_PB2D_projector``
and ``_trtt_single_distance_driven_FB2D_projector``
(Ytrtt_2D_projectors.i:943-1245), with the helpers
``_trtt_2D_projection_O_to_D`` (:132-170), ``_trtt_2D_distorsion_O_to_D``
(:173-190) and ``_trtt_2D_magnification_O_to_D`` (:192-210).  This module
follows those functions step by step: per slice of pixels along the passive
axis it projects the pixel boundaries of the active axis onto the detector,
merges them with the detector-cell boundaries, and distributes the lengths of
the merged intervals with Yorick's ``digitize`` / ``histogram`` index
arithmetic (translated from 1-based indices).

Pinning: Yorick is not available here, so the restatement cannot be run
against the Yorick code itself.  In parallel beam it is pinned to the
reference's compiled C: the distance-driven 3D projector trtt_DD_PB3D
(plugin/trtt_3D_projectors.c:1077-1173) on a one-slice scan with a detector
row one voxel high gives this projection times the voxel size, cell by
cell, to ~1e-14 (except the detector's last cell, which that C projector
leaves empty).  Fan beam is unpinned (the reference's cone-beam DD,
plugin/trtt_3D_projectors.c:1340-1434, is commented out); it is
cross-checked against an independent overlap formulation (``dd2d_overlap``)
and, at model level, against analytic line integrals of ellipses.

Images are numpy [j][i] (x fastest, the reference's x(i, j)); xos / xsd are
the 12 coefficients of the view's (xos . xotilt) and xsd transforms
(geometry.dd_coefs_2d).
"""
from __future__ import annotations

import numpy as np

PARALLEL, FAN = 3, 5  # TRTT_PARALLEL_BEAM, TRTT_FAN_BEAM


def _grids(nx, ny, s, nv, v):
    xn = (np.arange(nx) - 0.5 * (nx - 1)) * s
    yn = (np.arange(ny) - 0.5 * (ny - 1)) * s
    xb = (np.arange(nx + 1) - 0.5 * nx) * s
    yb = (np.arange(ny + 1) - 0.5 * ny) * s
    vb = (np.arange(nv + 1) - 0.5 * nv) * v
    return xn, yn, xb, yb, vb


def projection_o_to_d(xn, yn, xos, xsd, mode):
    """Detector coordinate of the points (xn[a], yn[b]), shape (len(xn),
    len(yn)) (Ytrtt_2D_projectors.i:132-170)."""
    xs = xos[0] * xn[:, None] + xos[1] * yn[None, :] + xos[3]
    ys = xos[4] * xn[:, None] + xos[5] * yn[None, :] + xos[7]
    a1inv = 1.0 / xsd[0]
    a2, a4, a5, a6, a8 = xsd[1], xsd[3], xsd[4], xsd[5], xsd[7]
    b1 = a6 + a1inv * a5 * a2
    b3 = a8 + a1inv * a5 * a4
    if mode == PARALLEL:
        return b1 * ys + b3
    tan_gamma = ys / xs
    xeq = -(1.0 / (xsd[0] + a2 * tan_gamma)) * a4
    return b1 * tan_gamma * xeq + b3


def magnification_o_to_d(xn, yn, xos, xsd):
    xs = xos[0] * xn[:, None] + xos[1] * yn[None, :] + xos[3]
    return np.abs(xsd[3] / xs)


def distorsion_o_to_d(xn, yn, xos, xsd):
    xs = xos[0] * xn[:, None] + xos[1] * yn[None, :] + xos[3]
    ys = xos[4] * xn[:, None] + xos[5] * yn[None, :] + xos[7]
    return np.sqrt(1 + (ys / xs) ** 2.0)


def _digitize(x, bins):
    """Yorick digitize (1-based): i with bins(i-1) <= x < bins(i)."""
    return np.digitize(x, bins) + 1


def _histogram(ids, w, top):
    """Yorick histogram(ids, w, top=top) for 1-based ids in [1, top]."""
    return np.bincount(np.asarray(ids, dtype=np.int64) - 1, weights=w, minlength=top)[:top]


def dd2d(out, x, nx, ny, s_scl, nv, v_scl, xos, xsd, mode, job):
    """out += H x (job 0: x image [ny][nx], out detector [nv]) or
    out += H^T x (job 1: x detector [nv], out image [ny][nx]) for one view."""
    xos = np.asarray(xos, dtype=np.float64)
    xsd = np.asarray(xsd, dtype=np.float64)
    xn, yn, xb, yb, vb = _grids(nx, ny, s_scl, nv, v_scl)
    border_down, border_up = vb[0], vb[-1]
    img = np.asarray(x, dtype=np.float64)
    if abs(xos[4]) < abs(xos[5]):
        axis, n_active, n_passive = 1, ny, nx
        proj_var = projection_o_to_d(xn, yb, xos, xsd, mode).T      # [ny+1][nx]
        get_vals = (lambda q: img[:, q]) if job == 0 else None
        if mode == FAN:
            magnification = magnification_o_to_d(xn, yn, xos, xsd).T   # [ny][nx]
            distorsion = distorsion_o_to_d(xn, yn, xos, xsd).T
    else:
        axis, n_active, n_passive = 2, nx, ny
        proj_var = projection_o_to_d(xb, yn, xos, xsd, mode)        # [nx+1][ny]
        get_vals = (lambda q: img[q, :]) if job == 0 else None
        if mode == FAN:
            magnification = magnification_o_to_d(xn, yn, xos, xsd)      # [nx][ny]
            distorsion = distorsion_o_to_d(xn, yn, xos, xsd)
    if mode == PARALLEL:
        h_par = (s_scl ** 2.0) / np.mean(np.abs(np.diff(proj_var, axis=0)))
    for q in range(n_passive):
        vals = get_vals(q).copy() if job == 0 else None
        p = proj_var[:, q].copy()
        if mode == FAN:
            magn = magnification[:, q].copy()
            delta = distorsion[:, q].copy()
        test_order = bool(np.any(np.diff(p) < 0.0))
        if test_order:
            io = np.argsort(p, kind="stable")
            p = p[io]
            perm = io[1:]
            if mode == FAN:
                magn, delta = magn[perm], delta[perm]
            if job == 0:
                vals = vals[perm]
        voxpos_up = p.max()
        if mode == FAN:
            h_norm = delta * magn * (s_scl ** 2.0) * (1.0 / np.diff(p))
        idproj = np.nonzero((p > border_down) & (p < border_up))[0]
        iddet_out = np.nonzero(vb >= voxpos_up)[0]
        ids_tmp = _digitize(vb, p) - 1
        ids_tmp[iddet_out] = n_active + 1
        id_neigh_vox = np.sort(np.concatenate([ids_tmp, idproj + 1]))
        proj_in = p[idproj]
        id_neigh_det = np.sort(np.concatenate([np.arange(1, nv + 2), _digitize(proj_in, vb) - 1]))
        merged = np.sort(np.concatenate([proj_in, vb]))
        coefs = np.diff(merged)
        if mode == PARALLEL:
            coefs = h_par * coefs
        nco = len(coefs)
        idvox = np.nonzero((id_neigh_vox > 0) & (id_neigh_vox < n_active + 1))[0]
        if len(idvox) == 0:
            continue
        if idvox[-1] + 1 > nco:
            idvox = idvox[:-1]
        ivox = id_neigh_vox[idvox] - 1
        if job == 0:
            voxels = np.zeros(len(id_neigh_vox) - 1)
            voxels[idvox] = (h_norm * vals)[ivox] if mode == FAN else vals[ivox]
            out += _histogram(id_neigh_det[:-1], coefs * voxels, nv)
        else:
            sino = np.asarray(x, dtype=np.float64)[id_neigh_det[:-1] - 1]
            w = (coefs * sino)[idvox]
            if mode == FAN:
                w = h_norm[ivox] * w
            out_q = _histogram(id_neigh_vox[idvox], w, n_active)
            if test_order:
                out_q = out_q[perm]
            if axis == 1:
                out[:, q] += out_q
            else:
                out[q, :] += out_q
    return 0


def dd2d_overlap(out, x, nx, ny, s_scl, nv, v_scl, xos, xsd, mode, job):
    """The same operator written as overlaps: pixel i of a slice covers
    [min(p_i, p_i+1), max(p_i, p_i+1)] and meets detector cell d over
    max(0, min(hi, v_d+1) - max(lo, v_d)), weighted by h (parallel: s^2 /
    mean |dp|; fan: distortion * magnification * s^2 / |dp_i| at the pixel
    centre).  Independent of the merged-index arithmetic above."""
    xos = np.asarray(xos, dtype=np.float64)
    xsd = np.asarray(xsd, dtype=np.float64)
    xn, yn, xb, yb, vb = _grids(nx, ny, s_scl, nv, v_scl)
    y_active = abs(xos[4]) < abs(xos[5])
    if y_active:
        P = projection_o_to_d(xn, yb, xos, xsd, mode).T          # [ny+1][nx]: slices are x columns
    else:
        P = projection_o_to_d(xb, yn, xos, xsd, mode)            # [nx+1][ny]: slices are y rows
    lo = np.minimum(P[:-1], P[1:])                                # [active][passive]
    hi = np.maximum(P[:-1], P[1:])
    if mode == PARALLEL:
        H = np.full(lo.shape, (s_scl ** 2.0) / np.mean(np.abs(np.diff(P, axis=0))))
    else:
        md = distorsion_o_to_d(xn, yn, xos, xsd) * magnification_o_to_d(xn, yn, xos, xsd)  # [nx][ny]
        H = (md.T if y_active else md) * (s_scl ** 2.0) / (hi - lo)
    ov = np.maximum(0.0, np.minimum(hi[..., None], vb[1:]) - np.maximum(lo[..., None], vb[:-1]))
    W = H[..., None] * ov                                         # [active][passive][nv]
    if job == 0:
        img = np.asarray(x, dtype=np.float64)
        A = img if y_active else img.T                            # [active][passive]
        out += np.einsum("apd,ap->d", W, A)
    else:
        A = np.einsum("apd,d->ap", W, np.asarray(x, dtype=np.float64))
        out += A if y_active else A.T
    return 0
