"""On-disk formats of the reference, so runs can exchange data with it.

- ``write_vector`` / ``read_vector``: Utils::write_vector / read_vector
  (include/SemiDiscreteOT/utils/utils.h:55-174).  Text: one value (or one
  point, coordinates separated by a space) per line, 17 significant digits
  (``std::numeric_limits<double>::max_digits10``); binary: the raw doubles.
  ``read_vector`` infers the mode from the extension like the reference.
- ``save_discrete_measures`` / ``load_discrete_measures``:
  SemiDiscreteOT::save_discrete_measures (src/core/SemiDiscreteOT.cc:2489-2558):
  quadrature_points, quadrature_weights (JxW), density_values, target_points,
  target_density and metadata.txt.  The cells are consecutive groups of
  "Number of quadrature points per cell"; their centres are not saved, so the
  loader takes the mean of each cell's points (the vertex average for Gauss
  rules on affine cells, up to rounding).
- ``write_hierarchy`` / ``load_hierarchy``: the files of
  PointCloudHierarchyManager (src/core/PointCloudHierarchy.cc:236-294):
  level_<L>_points.txt, level_<L>_density.txt (default stream precision, 6
  significant digits), level_<L>_parents.txt for L < last and
  level_<L>_children.txt for L > 0 (each line: count, then the indices; the
  children of a level-L point are level L-1 indices).
- ``write_potentials`` / ``read_potentials``: potentials as written by
  save_results (write_vector of the potential vector).
- ``read_msh`` / ``write_msh``: gmsh 2.2 ASCII meshes as deal.II's
  GridIn::read_msh takes them for the simplex source meshes (tutorial_0 reads
  its source.msh, examples/tutorial_0/src/tutorial_0.cc:37-47): nodes, and the
  elements of the highest dimension present (triangles, type 2, or
  tetrahedra, type 4) as cells; lower-dimensional elements are boundary data.
- ``write_ply`` / ``read_ply``: the ASCII point files of
  Lloyd::run_centroid_iteration (src/core/Lloyd.cc:139-171): a PLY header with
  one float property per coordinate, then each point's coordinates at the
  default stream precision, each followed by a space.
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


def _fmt17(v: float) -> str:
    return format(float(v), ".17g")


def _fmt6(v: float) -> str:
    return format(float(v), ".6g")


def write_vector(values, filepath: str, mode: str = "txt") -> str:
    """Utils::write_vector: `filepath` without extension; returns the file written."""
    a = np.asarray(values, dtype=np.float64)
    d = os.path.dirname(filepath)
    if d:
        os.makedirs(d, exist_ok=True)
    if mode == "bin":
        path = filepath + ".bin"
        with open(path, "wb") as f:
            f.write(np.ascontiguousarray(a).tobytes())
        return path
    if mode != "txt":
        raise ValueError("Invalid file mode specified.")
    path = filepath + ".txt"
    with open(path, "w") as f:
        if a.ndim == 1:
            f.writelines(_fmt17(v) + "\n" for v in a)
        else:
            f.writelines(" ".join(_fmt17(v) for v in row) + "\n" for row in a)
    return path


def read_vector(filepath: str, mode: Optional[str] = None, dim: Optional[int] = None) -> np.ndarray:
    """Utils::read_vector.  Points come back as (n, dim) when `dim` is given."""
    path, m = filepath, mode
    if not m:
        ext = os.path.splitext(filepath)[1].lstrip(".")
        if ext in ("txt", "bin"):
            m = ext
        else:
            m, path = "txt", filepath + ".txt"
    elif not filepath.endswith("." + m):
        path = filepath + "." + m
    if m == "bin":
        a = np.fromfile(path, dtype=np.float64)
    elif m == "txt":
        with open(path) as f:
            a = np.array([float(t) for t in f.read().split()], dtype=np.float64)
    else:
        raise ValueError(f"Invalid file mode specified: {m}")
    if dim is not None:
        a = a.reshape(-1, dim)
    return a


def write_potentials(psi, filepath: str, mode: str = "txt") -> str:
    return write_vector(psi, filepath, mode)


def read_potentials(filepath: str, mode: Optional[str] = None) -> np.ndarray:
    return read_vector(filepath, mode)


def save_discrete_measures(directory: str, x, jxw, density, y, nu, dim: int, n_q_per_cell: int,
                           quadrature_order: int, spacedim: Optional[int] = None, io_coding: str = "txt",
                           tetrahedral: bool = False) -> None:
    x = np.asarray(x, dtype=np.float64)
    sd = spacedim or dim
    x = x.reshape(-1, sd)
    y = np.asarray(y, dtype=np.float64).reshape(-1, sd)
    os.makedirs(directory, exist_ok=True)
    write_vector(x, os.path.join(directory, "quadrature_points"), io_coding)
    write_vector(jxw, os.path.join(directory, "quadrature_weights"), io_coding)
    write_vector(density, os.path.join(directory, "density_values"), io_coding)
    write_vector(y, os.path.join(directory, "target_points"), io_coding)
    write_vector(nu, os.path.join(directory, "target_density"), io_coding)
    with open(os.path.join(directory, "metadata.txt"), "w") as f:
        f.write(f"Dimension: {dim}\n")
        f.write(f"Space dimension: {sd}\n")
        f.write(f"Number of quadrature points per cell: {n_q_per_cell}\n")
        f.write(f"Total number of quadrature points: {x.shape[0]}\n")
        f.write(f"Number of target points: {y.shape[0]}\n")
        f.write(f"Quadrature order: {quadrature_order}\n")
        f.write(f"Using tetrahedral mesh: {int(bool(tetrahedral))}\n")


def load_discrete_measures(directory: str, io_coding: Optional[str] = None) -> Dict[str, object]:
    """Returns a source dict in the layout of SotSolver.setup_source plus the targets."""
    meta = {}
    with open(os.path.join(directory, "metadata.txt")) as f:
        for line in f:
            if ":" in line:
                k, v = line.split(":", 1)
                meta[k.strip()] = v.strip()
    sd = int(meta["Space dimension"])
    qpc = int(meta["Number of quadrature points per cell"])
    ext = io_coding or ("bin" if os.path.exists(os.path.join(directory, "quadrature_points.bin")) else "txt")

    def rd(name, dim=None):
        return read_vector(os.path.join(directory, name), ext, dim)

    x = rd("quadrature_points", sd)
    jxw = rd("quadrature_weights")
    dens = rd("density_values")
    if x.shape[0] % qpc:
        raise ValueError("the point count is not a multiple of the points per cell")
    ncell = x.shape[0] // qpc
    centres = x.reshape(ncell, qpc, sd).mean(axis=1)
    src = {"x": x, "jxw": jxw, "density": dens, "cell_offsets": np.arange(ncell + 1, dtype=np.int64) * qpc,
           "cell_centers": centres}
    return {"source": src, "y": rd("target_points", sd), "nu": rd("target_density"), "metadata": meta,
            "dim": int(meta["Dimension"]), "spacedim": sd}


def write_hierarchy(directory: str, points: Sequence[np.ndarray], densities: Sequence[np.ndarray],
                    children: Sequence[Sequence[Sequence[int]]], parents: Optional[Sequence] = None) -> None:
    """points[L], densities[L] per level (0 = finest); children[L - 1][i] = the
    level L-1 children of point i of level L; parents[L][i] = the level L+1
    parents of point i of level L (derived from children when not given)."""
    os.makedirs(directory, exist_ok=True)
    nl = len(points)
    if parents is None:
        parents = []
        for L in range(nl - 1):
            par: List[List[int]] = [[] for _ in range(len(points[L]))]
            for i, ch in enumerate(children[L]):
                for k in ch:
                    par[k].append(i)
            parents.append(par)
    for L in range(nl):
        P = np.asarray(points[L], dtype=np.float64)
        with open(os.path.join(directory, f"level_{L}_points.txt"), "w") as f:
            f.writelines(" ".join(_fmt6(v) for v in row) + "\n" for row in P)
        with open(os.path.join(directory, f"level_{L}_density.txt"), "w") as f:
            f.writelines(_fmt6(v) + "\n" for v in np.asarray(densities[L], dtype=np.float64))
        if L < nl - 1:
            with open(os.path.join(directory, f"level_{L}_parents.txt"), "w") as f:
                f.writelines(" ".join([str(len(p))] + [str(int(i)) for i in p]) + "\n" for p in parents[L])
        if L > 0:
            with open(os.path.join(directory, f"level_{L}_children.txt"), "w") as f:
                f.writelines(" ".join([str(len(c))] + [str(int(i)) for i in c]) + "\n" for c in children[L - 1])


def _read_lists(path: str) -> List[List[int]]:
    out = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            n = int(t[0])
            if len(t) != n + 1:
                raise ValueError(f"{path}: a line lists {len(t) - 1} indices but declares {n}")
            out.append([int(v) for v in t[1:]])
    return out


def load_hierarchy(directory: str, dim: Optional[int] = None) -> Dict[str, list]:
    """Levels found in `directory`: points, densities, children (as CSR offsets
    and indices: children of level-L point i are level L-1 indices) and parents."""
    pts, dens, ch, par = [], [], [], []
    L = 0
    while os.path.exists(os.path.join(directory, f"level_{L}_points.txt")):
        P = read_vector(os.path.join(directory, f"level_{L}_points.txt"))
        d = dim
        if d is None:
            with open(os.path.join(directory, f"level_{L}_points.txt")) as f:
                d = len(f.readline().split())
        pts.append(P.reshape(-1, d))
        dens.append(read_vector(os.path.join(directory, f"level_{L}_density.txt")))
        L += 1
    for L in range(1, len(pts)):
        lists = _read_lists(os.path.join(directory, f"level_{L}_children.txt"))
        off = np.zeros(len(lists) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(c) for c in lists])
        idx = np.array([k for c in lists for k in c], dtype=np.int64)
        ch.append((off, idx))
    for L in range(len(pts) - 1):
        p = os.path.join(directory, f"level_{L}_parents.txt")
        par.append(_read_lists(p) if os.path.exists(p) else None)
    return {"points": pts, "densities": dens, "children": ch, "parents": par}


def child_csr_from_parents(parent: np.ndarray, n_coarse: int) -> Tuple[np.ndarray, np.ndarray]:
    """CSR children (offsets, indices, ascending fine index) from a parent index per fine point."""
    parent = np.asarray(parent, dtype=np.int64)
    order = np.argsort(parent, kind="stable")
    counts = np.bincount(parent, minlength=n_coarse)
    off = np.zeros(n_coarse + 1, dtype=np.int64)
    off[1:] = np.cumsum(counts)
    return off, order.astype(np.int64)


def write_ply(points, path: str) -> str:
    P = np.asarray(points, dtype=np.float64)
    P = P.reshape(P.shape[0], -1)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\n")
        f.write(f"element vertex {P.shape[0]}\n")
        for k in range(P.shape[1]):
            f.write(f"property float {'xyz'[k]}\n")
        f.write("end_header\n")
        f.writelines("".join(_fmt6(v) + " " for v in row) + "\n" for row in P)
    return path


def read_ply(path: str) -> np.ndarray:
    with open(path) as f:
        lines = f.read().splitlines()
    n, dim, k = 0, 0, 0
    while lines[k] != "end_header":
        t = lines[k].split()
        if t[:2] == ["element", "vertex"]:
            n = int(t[2])
        elif t[:1] == ["property"]:
            dim += 1
        k += 1
    rows = [[float(v) for v in line.split()] for line in lines[k + 1:k + 1 + n]]
    return np.array(rows, dtype=np.float64).reshape(n, dim)


_MSH_NODES = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 15: 1}
_MSH_DIM = {1: 1, 2: 2, 3: 2, 4: 3, 5: 3, 15: 0}


def read_msh(path: str) -> Dict[str, np.ndarray]:
    """gmsh 2.2 ASCII: {"nodes": (V, 3), "cells": (C, dim+1) vertex indices,
    "dim": 2 or 3, "cell_tags": (C, ntags) physical/elementary tags}.  Only
    simplex cells (triangles, tetrahedra) are accepted as the top dimension."""
    with open(path) as f:
        lines = f.read().split("\n")
    k = 0
    nodes = None
    ids: Dict[int, int] = {}
    elems: Dict[int, list] = {}
    tags: Dict[int, list] = {}
    while k < len(lines):
        t = lines[k].strip()
        if t == "$MeshFormat":
            ver = lines[k + 1].split()
            if not ver or not ver[0].startswith("2") or ver[1] != "0":
                raise ValueError("only gmsh 2.x ASCII meshes are read")
            k += 2
        elif t == "$Nodes":
            n = int(lines[k + 1])
            nodes = np.empty((n, 3))
            for i in range(n):
                v = lines[k + 2 + i].split()
                ids[int(v[0])] = i
                nodes[i] = [float(v[1]), float(v[2]), float(v[3])]
            k += n + 2
        elif t == "$Elements":
            n = int(lines[k + 1])
            for i in range(n):
                v = [int(a) for a in lines[k + 2 + i].split()]
                et, nt = v[1], v[2]
                if et not in _MSH_NODES:
                    raise ValueError(f"unsupported gmsh element type {et}")
                elems.setdefault(et, []).append(v[3 + nt:3 + nt + _MSH_NODES[et]])
                tags.setdefault(et, []).append(v[3:3 + nt])
            k += n + 2
        else:
            k += 1
    if nodes is None or not elems:
        raise ValueError(f"{path}: no nodes or elements")
    top = max(_MSH_DIM[et] for et in elems)
    if top == 3 and 5 in elems or top == 2 and 3 in elems:
        raise ValueError("hexahedra / quadrilaterals: use a structured Q1 source")
    et = 4 if top == 3 else 2
    cells = np.array([[ids[a] for a in c] for c in elems[et]], dtype=np.int64)
    return {"nodes": nodes, "cells": cells, "dim": top, "cell_tags": np.array(tags[et], dtype=np.int64)}


def write_msh(path: str, nodes, cells) -> str:
    """gmsh 2.2 ASCII with one element block (triangles or tetrahedra)."""
    P = np.asarray(nodes, dtype=np.float64)
    T = np.asarray(cells, dtype=np.int64)
    et = {3: 2, 4: 4}[T.shape[1]]
    if P.shape[1] == 2:
        P = np.hstack([P, np.zeros((P.shape[0], 1))])
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
        f.write(f"{P.shape[0]}\n")
        f.writelines(f"{i + 1} {_fmt17(p[0])} {_fmt17(p[1])} {_fmt17(p[2])}\n" for i, p in enumerate(P))
        f.write("$EndNodes\n$Elements\n")
        f.write(f"{T.shape[0]}\n")
        f.writelines(f"{i + 1} {et} 2 0 0 " + " ".join(str(int(a) + 1) for a in c) + "\n" for i, c in enumerate(T))
        f.write("$EndElements\n")
    return path
