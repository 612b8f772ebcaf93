"""Source measures for the tensor-grid cell tests: cells whose Gauss points form a tensor grid symmetric about the
cell centre, with one spacing per dimension for every cell (structured_source) or a spacing per cell column
(graded_source)."""
import numpy as np

from semidiscreteot_b200 import structured_source


def graded_source(rng, dim, n, order):
    """structured_source with the cell columns along x given random widths (each cell mapped affinely, so
    its points stay a tensor grid symmetric about its centre, with a spacing of its own)."""
    src = structured_source(dim, n, order)
    h = 1.0 / n
    wid = rng.uniform(0.5, 1.5, n)
    wid /= wid.sum()
    left = np.concatenate([[0.0], np.cumsum(wid)[:-1]])
    qpc = order ** dim
    ncell = src["cell_centers"].shape[0]
    col = np.arange(ncell) % n                    # cells are x fastest
    x = src["x"].copy().reshape(ncell, qpc, dim)
    x0 = col * h
    x[:, :, 0] = left[col][:, None] + (x[:, :, 0] - x0[:, None]) * (wid[col] / h)[:, None]
    c = src["cell_centers"].copy()
    c[:, 0] = left[col] + 0.5 * wid[col]
    jxw = (src["jxw"].reshape(ncell, qpc) * (wid[col] / h)[:, None]).ravel()
    return dict(x=x.reshape(-1, dim), jxw=jxw, density=src["density"], cell_offsets=src["cell_offsets"],
                cell_centers=c)
