"""Host readers of the reference's mesh and current files (no GPU): files
written here in the reference's formats read back bit for bit, the
reference's own example meshes parse to the cell counts their headers state,
and malformed files are errors, as the reference's readers throw."""
import os

import numpy as np
import pytest

from bielcc_b200 import abi, gpu
from bielcc_b200 import workloads as W

REF_DATA = os.path.join(os.environ.get("BIELCC_REF_SRC", "/root/reference"), "examples", "data", "surface_mesh")


def _write_dat(path, objects):
    """objects: list of modules lists, each module an array [nfm][n_vert][3]."""
    with open(path, "w") as f:
        f.write(f"{len(objects)}\n")
        for mods in objects:
            f.write(f"{len(mods)}\n")
            for cells in mods:
                f.write(f"1 {len(cells)} 0 0\n")
                for c in cells:
                    f.write(" ".join(f"{v:.17g}" for v in c.ravel()) + "\n")
        f.write("0\n")


def _write_vtk(path, cells, polydata=True, extra_poly=None):
    pts = cells.reshape(-1, 3)
    nv = cells.shape[1]
    polys = [list(range(i * nv, (i + 1) * nv)) for i in range(len(cells))]
    if extra_poly is not None:
        polys.insert(1, extra_poly)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 2.0\ntest\nASCII\n")
        f.write("DATASET POLYDATA\n" if polydata else "DATASET UNSTRUCTURED_GRID\n")
        f.write(f"POINTS {len(pts)} double\n")
        for p in pts:
            f.write(" ".join(f"{v:.17g}" for v in p) + "\n")
        kw = "POLYGONS" if polydata else "CELLS"
        f.write(f"{kw} {len(polys)} {sum(len(p) + 1 for p in polys)}\n")
        for p in polys:
            f.write(f"{len(p)} " + " ".join(map(str, p)) + "\n")
        if not polydata:
            f.write(f"CELL_TYPES {len(polys)}\n" + "9\n" * len(polys))


def test_dat_round_trip(tmp_path):
    q = W.uv_sphere(6, 12)
    t = W.perturbed_icosphere(1, seed=3)
    p = tmp_path / "q.dat"
    _write_dat(p, [[q[:30], q[30:]], [q[:5]]])
    got = gpu.read_mesh_dat(str(p), 4)
    assert np.array_equal(got, np.concatenate([q, q[:5]]))
    p2 = tmp_path / "t.dat"
    _write_dat(p2, [[t]])
    assert np.array_equal(gpu.read_mesh_dat(str(p2), 3), t)


@pytest.mark.parametrize("polydata", [True, False])
def test_vtk_round_trip_skips_other_polygons(tmp_path, polydata):
    q = W.torus(9, 4)
    p = tmp_path / "q.vtk"
    _write_vtk(p, q, polydata, extra_poly=[0, 1, 2])  # a triangle among quads is skipped
    cells, skipped = gpu.read_mesh_vtk(str(p), 4)
    assert skipped == 1 and np.array_equal(cells, q)


def test_currents_round_trip(tmp_path):
    J = W.po_currents(W.uv_sphere(4, 8), 3.0)[0]
    for name, part in (("re", J.real), ("im", J.imag)):
        with open(tmp_path / name, "w") as f:
            f.write(f"{len(J)} 1\n")
            for row in part:
                f.write(" ".join(f"{v:.17g}" for v in row) + "\n")
    assert np.array_equal(gpu.read_currents(str(tmp_path / "re"), str(tmp_path / "im")), J)


def test_errors(tmp_path):
    with pytest.raises(gpu.BielccError) as e:
        gpu.read_mesh_dat(str(tmp_path / "missing.dat"), 4)
    assert e.value.code == abi.ERR_IO
    p = tmp_path / "short.dat"
    p.write_text("1\n1\n1 2 0 0\n0 0 0 1 0 0 1 1 0 0 1 0\n")  # second cell missing
    with pytest.raises(gpu.BielccError) as e:
        gpu.read_mesh_dat(str(p), 4)
    assert e.value.code == abi.ERR_IO
    v = tmp_path / "bad.vtk"
    v.write_text("# vtk\nx\nASCII\nDATASET POLYDATA\nPOINTS 3 float\n0 0 0\n1 0 0\n0 1 0\nPOLYGONS 1 4\n3 0 1 7\n")
    with pytest.raises(gpu.BielccError) as e:
        gpu.read_mesh_vtk(str(v), 3)
    assert e.value.code == abi.ERR_IO


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="the reference's example data are not present")
def test_reference_example_meshes():
    q = gpu.read_mesh_dat(os.path.join(REF_DATA, "sphere_quad.dat"), 4)
    assert q.shape == (450, 4, 3) and np.allclose(np.linalg.norm(q.reshape(-1, 3), axis=1), 1.0, atol=1e-5)
    t = gpu.read_mesh_dat(os.path.join(REF_DATA, "sphere_triangle.dat"), 3)
    assert t.shape[1:] == (3, 3) and len(t) > 0
    v, skipped = gpu.read_mesh_vtk(os.path.join(REF_DATA, "sphere_quad.vtk"), 4)
    assert len(v) + skipped == 1020 and len(v) > 0
    p, _ = gpu.read_mesh_vtk(os.path.join(REF_DATA, "plate_oxy.vtk"), 4)
    assert p.shape == (900, 4, 3)


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="the reference's example data are not present")
def test_readers_match_the_reference_readers_cell_by_cell():
    """Every example mesh of the reference read by its own SurfMesh reader
    (ReadFromFile -> ReadFromDatFile / ReadFromVtkFile, mesh/surf_mesh.cpp:18-175,
    surf_mesh.h:388-555) and by ours gives the same cells, bit for bit, for
    both cell types; where the reference throws (no polygon of that vertex
    count), ours reports BIELCC_ERR_IO. The example currents
    (examples/data/currents/E_{real,image}.gv) read by SurfaceCurrentsC_fromFiles
    (electrodynamics/currents.cpp:74-109) and by ours are identical."""
    import oracle

    if not oracle.available("ref"):
        pytest.skip("reference build absent")
    seen = 0
    for name in sorted(os.listdir(REF_DATA)):
        path = os.path.join(REF_DATA, name)
        fmt = name.rsplit(".", 1)[-1]
        for nv in (3, 4):
            if fmt == "dat" and f"_{'quad' if nv == 4 else 'triangle'}." not in name:
                continue  # a .dat file holds one cell kind, named in the file name
            try:
                ref = oracle.ref_read_mesh(path, nv, fmt)
            except RuntimeError:
                with pytest.raises(gpu.BielccError) as e:
                    gpu.read_mesh_vtk(path, nv) if fmt == "vtk" else gpu.read_mesh_dat(path, nv)
                assert e.value.code == abi.ERR_IO
                continue
            ours = gpu.read_mesh_vtk(path, nv)[0] if fmt == "vtk" else gpu.read_mesh_dat(path, nv)
            assert np.array_equal(ours, ref), (name, nv)
            seen += 1
    assert seen >= 4
    cur = os.path.join(os.path.dirname(REF_DATA), "currents")
    Jr = oracle.ref_read_currents(os.path.join(cur, "E_real.gv"), os.path.join(cur, "E_image.gv"))
    Jo = gpu.read_currents(os.path.join(cur, "E_real.gv"), os.path.join(cur, "E_image.gv"))
    assert len(Jr) > 0 and np.array_equal(Jo, Jr)
