"""The oracle against the reference compiled here (oracle/_ref), on fresh
seeded inputs beyond the golden fixtures. Skipped where the reference could
not be built (its sources are absent on the GPU box)."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from bielcc_b200 import workloads as W
from conftest import rel_l2

_needs_ref = pytest.mark.skipif(not oracle.available("ref"), reason="reference build absent")


@_needs_ref
@pytest.mark.parametrize("seed", [1, 2])
def test_field_random(seed):
    rng = np.random.default_rng(seed)
    cells = W.uv_sphere(8, 16) if seed == 1 else W.perturbed_icosphere(1, seed=seed)
    J = W.po_currents(cells, 3.0, directions=2, seed=seed)
    pts = np.concatenate([W.sphere_points(16, 2.0, seed), W.near_points(cells, 8, 0.01, 0.2, rng)])
    npm = abi.NumParam.default(p_max=2, p_max_seg=2, n_start=4, n_start_seg=5)
    for k in (3.0, complex(3.0, 0.2)):
        Eo, Ho = oracle.field_EH(cells, J, k, pts, npm, mult=complex(1, 2))
        Er, Hr = oracle.field_EH(cells, J, k, pts, npm, mult=complex(1, 2), which="ref")
        assert rel_l2(Eo, Er) < 1e-13
        assert rel_l2(Ho, Hr) < 1e-13


@_needs_ref
def test_k0_variants():
    rng = np.random.default_rng(3)
    cells = W.uv_sphere(8, 16)
    idx = rng.integers(0, len(cells), 32)
    cc = cells[idx]
    x = W.centres(cc) + rng.normal(size=(32, 3)) * 0.2
    j = rng.normal(size=(32, 3)) + 1j * rng.normal(size=(32, 3))
    for fid in (abi.F_GRADSIMPLEPOT_H, abi.F_NU_SIMPLEPOT_H, abi.F_GRADSIMPLEPOT_HM1):
        for common in (0, 1):
            for pm in (1, 3):
                # the records are in/out: each call gets its own copy
                kpa = abi.kernelparam_array(32, smoothR=0.05, smoothRMin=1e-6, k=2.0)
                kpb = abi.kernelparam_array(32, smoothR=0.05, smoothRMin=1e-6, k=2.0)
                a = oracle.k0(fid, common, cc, x, j, kpa, 10, pm, 1e-6)
                b = oracle.k0(fid, common, cc, x, j, kpb, 10, pm, 1e-6, which="ref")
                assert rel_l2(a, b) < 1e-13, (fid, common, pm)
                # smoothR left as the reference leaves it (shared across the edges, halved per pass)
                assert [r.smoothR for r in kpa] == [r.smoothR for r in kpb]
                assert kpa[0].smoothR < 0.05 or common == 1


@_needs_ref
def test_cell_geometry_matches_cellfill():
    for cells in (W.uv_sphere(16, 32), W.perturbed_icosphere(2)):
        assert np.abs(oracle.cell_geometry(cells) - oracle.cell_geometry(cells, which="ref")).max() < 1e-15


def test_tangent_basis_is_orthonormal():
    """tau1, tau2, normal of every cell form an orthonormal frame (CellFill, mesh/cell.cpp)."""
    for cells in (W.uv_sphere(16, 32), W.perturbed_icosphere(2)):
        g = oracle.cell_geometry(cells)
        n, t1, t2 = g[:, 4:7], g[:, 7:10], g[:, 10:13]
        for v in (n, t1, t2):
            assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-12)
        assert np.abs(np.einsum("ij,ij->i", t1, t2)).max() < 1e-12
        assert np.abs(np.einsum("ij,ij->i", n, t1)).max() < 1e-12
