"""Flattened source measures for structured Q1 meshes.

Replaces the deal.II part of source setup that the accelerated path needs:
``FE_Q(1)`` + ``MappingQ1`` + ``QGauss(order)`` on an axis-aligned
[lo, hi]^dim mesh (include/SemiDiscreteOT/utils/utils.h:776-850), with the
density given at the mesh vertices, Q1-interpolated to the quadrature points
and normalised by sum_q |rho_q| JxW_q like
``SemiDiscreteOT::normalize_density`` (src/core/SemiDiscreteOT.cc:422-449).
The output layout is that of ``save_discrete_measures``
(SemiDiscreteOT.cc:2489-2558) plus per-cell offsets and centres.
"""
from __future__ import annotations

import numpy as np


def gauss_legendre01(order: int):
    """Gauss-Legendre nodes/weights on [0, 1] (QGauss<1>(order))."""
    xi, wi = np.polynomial.legendre.leggauss(order)
    return 0.5 * (xi + 1.0), 0.5 * wi


def structured_source(dim: int, n: int, order: int, lo: float = 0.0, hi: float = 1.0,
                      nodal_density=None, normalize: bool = True) -> dict:
    """Quadrature data of an n^dim Q1 mesh on [lo, hi]^dim.

    nodal_density: (n+1)^dim vertex values (x fastest) or a callable f(points)
    evaluated at the vertices, or None for a uniform density.
    Returns dict(x, jxw, density, cell_offsets, cell_centers)."""
    if dim not in (2, 3):
        raise ValueError("dim must be 2 or 3")
    h = (hi - lo) / n
    g, w = gauss_legendre01(order)
    # vertex coordinates and nodal values
    ax = lo + np.arange(n + 1) * h
    if dim == 2:
        VX, VY = np.meshgrid(ax, ax, indexing="xy")
        verts = np.stack([VX.ravel(), VY.ravel()], axis=1)
    else:
        VZ, VY, VX = np.meshgrid(ax, ax, ax, indexing="ij")
        verts = np.stack([VX.ravel(), VY.ravel(), VZ.ravel()], axis=1)
    if nodal_density is None:
        nodal = np.ones(verts.shape[0])
    elif callable(nodal_density):
        nodal = np.asarray(nodal_density(verts), dtype=np.float64)
    else:
        nodal = np.asarray(nodal_density, dtype=np.float64).ravel()
    # reference-cell quadrature (x fastest) and Q1 shape values
    if dim == 2:
        QX, QY = np.meshgrid(g, g, indexing="xy")
        xi = np.stack([QX.ravel(), QY.ravel()], axis=1)
        wq = np.outer(w, w).ravel()
    else:
        QZ, QY, QX = np.meshgrid(g, g, g, indexing="ij")
        xi = np.stack([QX.ravel(), QY.ravel(), QZ.ravel()], axis=1)
        wq = np.einsum("i,j,k->ijk", w, w, w).ravel()
    nv = 1 << dim
    phi = np.ones((xi.shape[0], nv))
    for v in range(nv):
        for d in range(dim):
            phi[:, v] *= xi[:, d] if (v >> d) & 1 else (1.0 - xi[:, d])
    # cells (x fastest) and their vertex indices
    idx = np.arange(n)
    if dim == 2:
        CJ, CI = np.meshgrid(idx, idx, indexing="ij")
        ci = np.stack([CI.ravel(), CJ.ravel()], axis=1)
    else:
        CK, CJ, CI = np.meshgrid(idx, idx, idx, indexing="ij")
        ci = np.stack([CI.ravel(), CJ.ravel(), CK.ravel()], axis=1)
    ncell = ci.shape[0]
    vid = np.zeros((ncell, nv), dtype=np.int64)
    for v in range(nv):
        off = [(v >> d) & 1 for d in range(dim)]
        lin = ci[:, 0] + off[0]
        stride = n + 1
        for d in range(1, dim):
            lin = lin + (ci[:, d] + off[d]) * stride
            stride *= n + 1
        vid[:, v] = lin
    X0 = lo + ci * h                                     # lower corner of each cell
    centers = X0 + 0.5 * h
    x = (X0[:, None, :] + xi[None, :, :] * h).reshape(-1, dim)
    jxw = np.tile(wq * h ** dim, ncell)
    vals = nodal[vid]                                    # (ncell, nv)
    rho = (vals @ phi.T).ravel()                         # Q1 interpolation at the q points
    if normalize:
        l1 = np.sum(np.abs(rho) * jxw)
        if l1 > 0:
            nodal = nodal / l1
            rho = (nodal[vid] @ phi.T).ravel()
    qpc = xi.shape[0]
    offsets = np.arange(ncell + 1, dtype=np.int64) * qpc
    return {"x": np.ascontiguousarray(x), "jxw": jxw, "density": rho, "cell_offsets": offsets,
            "cell_centers": np.ascontiguousarray(centers), "nodal": nodal, "dim": dim, "n": n, "order": order}


def sphere_source(n_theta: int, n_phi: int, order: int, theta_max: float = np.pi, density=None,
                  normalize: bool = True) -> dict:
    """Quadrature data of the spherical cap {polar angle <= theta_max} of the
    unit sphere (the whole sphere at pi), for the spherical distance.

    Cells are the (polar angle, azimuth) rectangles of an n_theta x n_phi
    grid; each holds order^2 Gauss points of the rectangle mapped to the
    sphere, with JxW = Gauss weight x cell extents x sin(polar angle) (the
    area element), and the cell centre is the image of the rectangle's centre.
    density: a callable f(points) at the quadrature points, or None for a
    uniform density; normalised by sum_q |rho_q| JxW_q like the structured
    sources.  Returns the layout of structured_source (points in 3D)."""
    g, w = gauss_legendre01(order)
    ht, hp = theta_max / n_theta, 2.0 * np.pi / n_phi
    T0, P0 = np.meshgrid(np.arange(n_theta) * ht, np.arange(n_phi) * hp, indexing="ij")
    T0, P0 = T0.ravel(), P0.ravel()
    gt, gp = np.meshgrid(g, g, indexing="ij")
    wt = np.outer(w, w).ravel()
    th = T0[:, None] + gt.ravel()[None, :] * ht          # (ncell, order^2)
    ph = P0[:, None] + gp.ravel()[None, :] * hp

    def to_xyz(t, p):
        return np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], axis=-1)

    x = to_xyz(th, ph).reshape(-1, 3)
    jxw = (wt[None, :] * ht * hp * np.sin(th)).ravel()
    centers = to_xyz(T0 + 0.5 * ht, P0 + 0.5 * hp)
    rho = np.ones(x.shape[0]) if density is None else np.asarray(density(x), dtype=np.float64)
    if normalize:
        l1 = np.sum(np.abs(rho) * jxw)
        if l1 > 0:
            rho = rho / l1
    qpc = order * order
    ncell = T0.size
    return {"x": np.ascontiguousarray(x), "jxw": jxw, "density": rho,
            "cell_offsets": np.arange(ncell + 1, dtype=np.int64) * qpc,
            "cell_centers": np.ascontiguousarray(centers), "dim": 3, "order": order}
