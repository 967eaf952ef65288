"""Synthetic workload generators: shapes, orientation and sizes of the configs."""
import numpy as np

from bielcc_b200 import workloads as W


def test_uv_sphere_shapes_and_outward_normals():
    c = W.uv_sphere(16, 32)
    assert c.shape == (512, 4, 3)
    n = W.normals(c)
    assert np.all(np.einsum("ij,ij->i", n, W.centres(c)) > 0)
    # pole rows are degenerate quads with two identical vertices
    assert np.array_equal(c[0, 0], c[0, 3]) and np.array_equal(c[-1, 1], c[-1, 2])
    assert W.uv_sphere(64, 128).shape == (8192, 4, 3)


def test_icosphere_level5_and_perturbation():
    c = W.perturbed_icosphere(level=5, seed=2)
    assert c.shape == (20480, 3, 3)
    r = np.linalg.norm(c.reshape(-1, 3), axis=1)
    assert 0.8 < r.min() and r.max() < 1.2
    n = W.normals(c)
    assert np.mean(np.einsum("ij,ij->i", n, W.centres(c)) > 0) > 0.99


def test_po_currents_lit_shadow():
    c = W.uv_sphere(16, 32)
    J = W.po_currents(c, 2 * np.pi)
    lit = W.normals(c) @ np.array([0, 0, 1.0]) < 0
    assert J.shape == (1, 512, 3)
    assert np.all(J[0, ~lit] == 0) and np.all(np.abs(J[0, lit]).sum(1) > 0)


def test_config_points():
    c1 = W.config1()
    assert c1["pts"].shape == (1000, 3)
    assert np.allclose(np.linalg.norm(c1["pts"], axis=1), 3.0)
    c2 = W.config2()
    assert c2["pts"].shape == (20000, 3)
    r = np.linalg.norm(c2["pts"][:18000], axis=1)
    assert r.min() >= 2.0 and r.max() <= 5.0


def test_batch_meshes_mix_quads_and_triangles():
    """The batched workload draws quads and triangles (config 4: "quad or
    triangle cells"), 200-20,000 cells, no degenerate triangles."""
    js = W.batch_meshes(n_meshes=24, seed=3)
    nv = {j["cells"].shape[1] for j in js}
    assert nv == {3, 4}
    for j in js:
        c = j["cells"]
        assert 150 <= len(c) <= 21000
        assert np.isfinite(W.normals(c)).all()
    q = W.uv_sphere(8, 16)
    t = W.triangulate(q)
    # the pole quads lose their collapsed halves; every other quad gives two triangles
    assert len(t) == 2 * len(q) - 2 * 16
    area = lambda c: 0.5 * np.linalg.norm(np.cross(c[:, 1] - c[:, 0], c[:, 2] - c[:, 0]), axis=1).sum()
    assert abs(area(t) - sum(area(q[:, [0, 1, 2]]) + area(q[:, [2, 3, 0]]) for _ in [0])) < 1e-9
