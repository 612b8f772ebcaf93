"""Simplex sources: P1 densities on triangle / tetrahedron meshes, flattened
into the per-cell quadrature layout that ``SotSolver.setup_source`` takes.

The reference switches to FE_SimplexP(1), MappingFE and QGaussSimplex(order)
when the source mesh has simplices (include/SemiDiscreteOT/utils/utils.h
:776-809, used at src/solvers/SotSolver.cc:244-251, :686-693, :893-900).  The
device path is independent of the rule: any rule with the same number of
points in every cell runs through it.  QGaussSimplex's tables belong to
deal.II (not in the reference tree), so the rules here are published or
derived ones with deal.II's point counts, each tested for exactness:

- triangle (weights sum to 1/2): n=1 centroid (degree 1); n=2 the 3-point
  rule at (1/6, 1/6) and permutations (degree 2); n=3 Radon's 7-point rule
  (centroid + two 3-point orbits at (6 -+ sqrt 15)/21, degree 5).
- tetrahedron (weights sum to 1/6): n=1 centroid; n=2 the 4-point rule at
  barycentric (a, a, a, 1-3a), a = (5 - sqrt 5)/20 (degree 2); n=3 a
  10-point rule with an S31 orbit (a, a, a, 1-3a) and an S22 orbit
  (b, b, 1/2-b, 1/2-b): the symmetric moment equations up to degree 3 leave
  one free parameter, fixed here at the positive-weight member with the
  smallest degree-4 moment residual (constants below, degree 3).

Cells: the density at a point is the P1 interpolant of the nodal values, JxW
the rule weight times |det J| of the affine map, the cell centre the vertex
average (deal.II's cell->center() on an affine simplex).
"""
from __future__ import annotations

import itertools
import math
from typing import Dict, Tuple

import numpy as np

_T3_A = 0.07354529547071434
_T3_B = 0.09373097910985062
_T3_WA = 0.007899830989354817
_T3_WB = 0.022511223784874565


def simplex_rule(dim: int, n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Barycentric points (k x dim+1) and weights (sum = reference volume)."""
    if dim == 2:
        if n == 1:
            return np.array([[1 / 3, 1 / 3, 1 / 3]]), np.array([0.5])
        if n == 2:
            a = 1.0 / 6.0
            P = np.array([[a, a, 1 - 2 * a], [1 - 2 * a, a, a], [a, 1 - 2 * a, a]])
            return P, np.full(3, 1.0 / 6.0)
        if n == 3:
            s = math.sqrt(15.0)
            pts, w = [[1 / 3, 1 / 3, 1 / 3]], [9.0 / 80.0]
            for a, wa in (((6 - s) / 21, (155 - s) / 2400), ((6 + s) / 21, (155 + s) / 2400)):
                for k in range(3):
                    p = [a, a, a]
                    p[k] = 1 - 2 * a
                    pts.append(p)
                    w.append(wa)
            return np.array(pts), np.array(w)
    elif dim == 3:
        if n == 1:
            return np.full((1, 4), 0.25), np.array([1.0 / 6.0])
        if n == 2:
            a = (5 - math.sqrt(5.0)) / 20
            P = np.full((4, 4), a)
            np.fill_diagonal(P, 1 - 3 * a)
            return P, np.full(4, 1.0 / 24.0)
        if n == 3:
            P = np.full((4, 4), _T3_A)
            np.fill_diagonal(P, 1 - 3 * _T3_A)
            Q = []
            for i, j in itertools.combinations(range(4), 2):
                q = [0.5 - _T3_B] * 4
                q[i] = q[j] = _T3_B
                Q.append(q)
            return np.vstack([P, np.array(Q)]), np.concatenate([np.full(4, _T3_WA), np.full(6, _T3_WB)])
    raise ValueError(f"no simplex rule for dim={dim}, n={n} (n = 1, 2, 3)")


def simplex_source(vertices, cells, nodal_density=None, order: int = 3, normalize: bool = True) -> Dict[str, np.ndarray]:
    """Flattened source of a triangle (dim 2) or tetrahedron (dim 3) mesh.

    vertices (V x dim), cells (C x dim+1 vertex indices), nodal_density (V,)
    or a callable of the vertex coordinates (default 1).  normalize divides
    the density by sum_q |rho_q| JxW_q like SemiDiscreteOT::normalize_density
    (src/core/SemiDiscreteOT.cc:422-449)."""
    Vx = np.asarray(vertices, dtype=np.float64)
    T = np.asarray(cells, dtype=np.int64)
    dim = Vx.shape[1]
    if T.shape[1] != dim + 1:
        raise ValueError("cells must list dim+1 vertices")
    if nodal_density is None:
        rho_v = np.ones(Vx.shape[0])
    elif callable(nodal_density):
        rho_v = np.asarray(nodal_density(Vx), dtype=np.float64)
    else:
        rho_v = np.asarray(nodal_density, dtype=np.float64)
    B, w = simplex_rule(dim, order)
    corners = Vx[T]                                     # C x (dim+1) x dim
    J = corners[:, :dim, :] - corners[:, dim:dim + 1, :]  # rows: v_i - v_last
    det = np.abs(np.linalg.det(J))
    x = np.einsum("qk,ckd->cqd", B, corners)            # C x Q x dim
    rho = np.einsum("qk,ck->cq", B, rho_v[T])
    jxw = det[:, None] * w[None, :]
    nq = B.shape[0]
    out = {"x": x.reshape(-1, dim), "jxw": jxw.reshape(-1), "density": rho.reshape(-1),
           "cell_offsets": np.arange(T.shape[0] + 1, dtype=np.int64) * nq,
           "cell_centers": corners.mean(axis=1)}
    if normalize:
        s = float(np.sum(np.abs(out["density"]) * out["jxw"]))
        if s > 0:
            out["density"] = out["density"] / s
    return out


def triangle_square_mesh(n: int, lo: float = 0.0, hi: float = 1.0) -> Tuple[np.ndarray, np.ndarray]:
    """n x n squares, each cut into two triangles along alternating diagonals."""
    t = np.linspace(lo, hi, n + 1)
    X, Y = np.meshgrid(t, t, indexing="xy")
    V = np.stack([X.ravel(), Y.ravel()], axis=1)
    cells = []
    for j in range(n):
        for i in range(n):
            v0, v1, v2, v3 = j * (n + 1) + i, j * (n + 1) + i + 1, (j + 1) * (n + 1) + i, (j + 1) * (n + 1) + i + 1
            if (i + j) % 2 == 0:
                cells += [[v0, v1, v3], [v0, v3, v2]]
            else:
                cells += [[v0, v1, v2], [v1, v3, v2]]
    return V, np.array(cells, dtype=np.int64)


def tetra_cube_mesh(n: int, lo: float = -1.0, hi: float = 1.0) -> Tuple[np.ndarray, np.ndarray]:
    """n^3 cubes of [lo, hi]^3, each cut into 24 tetrahedra over its corners
    and face centres (no interior vertex): 8 corner tets (a corner and the
    centres of its 3 faces), 12 edge tets (an edge and the centres of its 2
    faces) and the face-centre octahedron cut into 4 around its x axis."""
    h = (hi - lo) / n
    idx: Dict[Tuple[int, int, int], int] = {}
    pts = []

    def vid(key):  # key in half-steps from lo
        k = idx.get(key)
        if k is None:
            k = idx[key] = len(pts)
            pts.append([lo + 0.5 * h * key[0], lo + 0.5 * h * key[1], lo + 0.5 * h * key[2]])
        return k

    cells = []
    for k, j, i in itertools.product(range(n), repeat=3):
        b = (2 * i, 2 * j, 2 * k)

        def corner(cx, cy, cz):
            return vid((b[0] + 2 * cx, b[1] + 2 * cy, b[2] + 2 * cz))

        def face(ax, side):
            key = [b[0] + 1, b[1] + 1, b[2] + 1]
            key[ax] = b[ax] + 2 * side
            return vid(tuple(key))

        for cx, cy, cz in itertools.product((0, 1), repeat=3):
            cells.append([corner(cx, cy, cz), face(0, cx), face(1, cy), face(2, cz)])
        for ax in range(3):
            o = [d for d in range(3) if d != ax]
            for s0, s1 in itertools.product((0, 1), repeat=2):
                e0, e1 = [0, 0, 0], [0, 0, 0]
                e0[o[0]] = e1[o[0]] = s0
                e0[o[1]] = e1[o[1]] = s1
                e1[ax] = 1
                cells.append([corner(*e0), corner(*e1), face(o[0], s0), face(o[1], s1)])
        ring = [face(1, 0), face(2, 0), face(1, 1), face(2, 1)]
        for r in range(4):
            cells.append([face(0, 0), face(0, 1), ring[r], ring[(r + 1) % 4]])
    return np.array(pts, dtype=np.float64), np.array(cells, dtype=np.int64)


def read_msh_source(path: str, nodal_density=None, order: int = 3, normalize: bool = True) -> Dict[str, np.ndarray]:
    """Simplex source from a gmsh 2.2 ASCII mesh (the highest-dimensional elements)."""
    from .io import read_msh
    m = read_msh(path)
    return simplex_source(m["nodes"][:, :m["dim"]], m["cells"], nodal_density, order, normalize)
