"""File formats of the reference (write_vector / read_vector, save_discrete_measures,
point-cloud hierarchy files, potentials): exact round trips and the reference's line layout."""
import os

import numpy as np

from semidiscreteot_b200 import structured_source
from semidiscreteot_b200 import io as sio


def test_vector_text_layout_and_round_trip(tmp_path):
    v = np.array([0.1, -2.5e-300, 1.0 / 3.0, 123456789.125])
    p = sio.write_vector(v, str(tmp_path / "pot"), "txt")
    assert p.endswith("pot.txt")
    lines = open(p).read().splitlines()
    assert lines[0] == "0.10000000000000001"          # std::setprecision(max_digits10)
    assert np.array_equal(sio.read_vector(p), v)       # mode from the extension
    assert np.array_equal(sio.read_vector(str(tmp_path / "pot")), v)   # no extension: txt
    pts = np.array([[0.5, 0.25, 1e-3], [1.0, 2.0, 3.0]])
    q = sio.write_vector(pts, str(tmp_path / "sub" / "points"), "txt")
    assert open(q).read().splitlines()[1] == "1 2 3"   # Point<3>: coordinates separated by a space
    assert np.array_equal(sio.read_vector(q, dim=3), pts)


def test_vector_binary_is_raw_doubles(tmp_path):
    v = np.random.default_rng(0).standard_normal(37)
    p = sio.write_vector(v, str(tmp_path / "b"), "bin")
    assert os.path.getsize(p) == 37 * 8
    assert np.array_equal(np.fromfile(p, dtype=np.float64), v)
    assert np.array_equal(sio.read_vector(str(tmp_path / "b"), "bin"), v)


def test_discrete_measures_round_trip(tmp_path):
    src = structured_source(2, 5, 3, nodal_density=lambda p: 1.0 + p[:, 0])
    rng = np.random.default_rng(1)
    y, nu = rng.random((17, 2)), rng.dirichlet(np.ones(17))
    for coding in ("txt", "bin"):
        d = str(tmp_path / coding)
        sio.save_discrete_measures(d, src["x"], src["jxw"], src["density"], y, nu, dim=2, n_q_per_cell=9,
                                   quadrature_order=3, io_coding=coding)
        meta = open(os.path.join(d, "metadata.txt")).read()
        assert "Number of quadrature points per cell: 9" in meta and "Total number of quadrature points: 225" in meta
        got = sio.load_discrete_measures(d)
        s = got["source"]
        assert np.array_equal(s["x"], src["x"].reshape(-1, 2)) and np.array_equal(s["jxw"], src["jxw"])
        assert np.array_equal(s["density"], src["density"]) and np.array_equal(got["y"], y)
        assert np.array_equal(s["cell_offsets"], src["cell_offsets"])
        assert np.max(np.abs(s["cell_centers"] - np.asarray(src["cell_centers"]).reshape(-1, 2))) < 1e-15


def test_hierarchy_files(tmp_path):
    rng = np.random.default_rng(2)
    fine = rng.random((12, 3))
    parent = np.array([0, 1, 2, 0, 1, 2, 0, 1, 2, 2, 1, 0])
    coarse = np.stack([fine[parent == i].mean(axis=0) for i in range(3)])
    children = [[list(np.nonzero(parent == i)[0]) for i in range(3)]]
    sio.write_hierarchy(str(tmp_path), [fine, coarse], [np.full(12, 1 / 12), np.full(3, 1 / 3)], children)
    assert open(tmp_path / "level_1_children.txt").read().splitlines()[0] == "4 0 3 6 11"
    assert open(tmp_path / "level_0_parents.txt").read().splitlines()[0] == "1 0"
    assert open(tmp_path / "level_1_density.txt").read().splitlines()[0] == "0.333333"   # default precision
    h = sio.load_hierarchy(str(tmp_path))
    assert len(h["points"]) == 2 and h["points"][0].shape == (12, 3)
    off, idx = h["children"][0]
    assert list(off) == [0, 4, 8, 12]
    assert list(idx[:4]) == [0, 3, 6, 11]
    off2, idx2 = sio.child_csr_from_parents(parent, 3)
    assert np.array_equal(off, off2) and np.array_equal(idx, idx2)
    assert np.max(np.abs(h["points"][0] - fine)) < 1e-5   # 6 significant digits


def test_ply_round_trip(tmp_path):
    from semidiscreteot_b200.io import read_ply, write_ply
    P = np.array([[0.125, 0.5, 1.0 / 3.0], [2.0, -1e-7, 123456.789]])
    path = write_ply(P, str(tmp_path / "barycenters_0.ply"))
    text = open(path).read().splitlines()
    assert text[:7] == ["ply", "format ascii 1.0", "element vertex 2", "property float x", "property float y",
                        "property float z", "end_header"]
    assert text[7] == "0.125 0.5 0.333333 "
    np.testing.assert_allclose(read_ply(path), P, rtol=1e-5)


def test_lloyd_step_norm():
    from semidiscreteot_b200.lloyd import step_norm
    a = np.zeros((4, 2))
    b = np.array([[3.0, 4.0], [0, 0], [0, 0], [0, 0]])
    assert step_norm(b, a) == np.sqrt(25.0 / 4)


def test_combined_level_schedule():
    from semidiscreteot_b200.multilevel import combined_level_indices
    assert combined_level_indices(3, 5) == [(0, 0), (0, 1), (0, 2), (1, 3), (2, 4)]
    assert combined_level_indices(4, 2) == [(0, 0), (1, 0), (2, 0), (3, 1)]
    for s, t in ((1, 1), (2, 7), (6, 3)):
        idx = combined_level_indices(s, t)
        assert len(idx) == max(s, t) and idx[-1] == (s - 1, t - 1)
        assert all(b[0] - a[0] in (0, 1) and b[1] - a[1] in (0, 1) for a, b in zip(idx, idx[1:]))
