"""The step after assembly: the dense LU solve and the perfect-conductor
collocation system (bielcc_solve_dense, bielcc_solve_pec) against numpy's
solve of the oracle's matrix, and the physics the solution must show (the
total field vanishes inside the conductor)."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from bielcc_b200 import workloads as W
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c64,tol", [(False, 1e-12), (True, 2e-5)])
def test_solve_dense_matches_numpy(gctx, c64, tol):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    n, nrhs = 300, 2
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 30 * np.eye(n)
    B = rng.standard_normal((nrhs, n)) + 1j * rng.standard_normal((nrhs, n))
    X = np.linalg.solve(A, B.T).T
    dt = torch.complex64 if c64 else torch.complex128
    tA = torch.from_numpy(A).to(dt).cuda()
    tB = torch.from_numpy(B).to(dt).cuda()
    info = gctx.solve_dense(n, nrhs, c64, tA.data_ptr(), tB.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert info == 0
    assert rel_l2(tB.cpu().numpy().astype(np.complex128), X) < tol


def _pec_case(cells, k):
    kv, e0, hs = W.planewave(k, direction=(0.3, 0.2, 0.93))
    e0 = np.cross(kv / np.linalg.norm(kv), np.array([0.0, 1.0, 0.0]))
    e0 /= np.linalg.norm(e0)
    return abi.PlaneWave.make(kv, e0, hs, True, True), kv, e0, hs


def test_solve_pec_matches_cpu_solve(gctx):
    cells = W.perturbed_icosphere(level=2, seed=2)
    k = 2.0
    inc, kv, e0, _ = _pec_case(cells, k)
    mult = 1j / k
    m = gctx.mesh(cells)
    geo = m.geometry()  # centre(3), diam, normal(3), tau1(3), tau2(3), area
    c, t1, t2 = geo[:, 0:3], geo[:, 7:10], geo[:, 10:13]
    A = oracle.assemble_K(cells, k, layout=abi.LAYOUT_TAU2)
    ph = np.exp(1j * (c @ kv))
    b = np.empty(2 * len(cells), np.complex128)
    b[0::2] = -(t1 @ e0) * ph / mult
    b[1::2] = -(t2 @ e0) * ph / mult
    x = np.linalg.solve(A, b)
    J_ref = x[0::2, None] * t1 + x[1::2, None] * t2
    J = gctx.solve_pec(m, k, inc, mult, precision="fp64")
    assert rel_l2(J, J_ref) < 1e-9
    Jm = gctx.solve_pec(m, k, inc, mult, precision="mixed")
    assert rel_l2(Jm, J_ref) < 1e-3


def test_solve_pec_null_field_inside(gctx):
    """Scattered + incident field inside a perfectly conducting sphere is zero
    (ka = 2, below the first interior resonance): a check of the whole chain
    assembly -> solve -> currents -> field that needs no reference."""
    cells = W.uv_sphere(24, 48)
    k = 2.0
    inc, kv, e0, hs = _pec_case(cells, k)
    mult = 1j / k
    m = gctx.mesh(cells)
    J = gctx.solve_pec(m, k, inc, mult, precision="fp64")
    pts = W.shell_points(100, 0.0, 0.6, np.random.default_rng(1))
    E, H, _ = gctx.field_EH(m, J, k, pts, mult=mult, precision="fp64")
    Einc = e0[None, :] * np.exp(1j * (pts @ kv))[:, None]
    assert rel_l2(E[0], -Einc) < 0.05  # |E_scat + E_inc| / |E_inc|
