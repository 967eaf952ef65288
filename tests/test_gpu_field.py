"""GPU field path (GetFieldE_Ideal + H) through the C ABI against the
reference's golden outputs and the oracle: FP64 within 1e-12 relative L2,
mixed within 1e-6."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, TOL_MIXED, golden, rel_l2

pytestmark = pytest.mark.gpu


def _inc(g):
    return abi.PlaneWave.make(g["kvec"], g["e0"], float(g["h_scale"]), True, True)


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_golden_quad512(gctx, precision, tol):
    g = golden("field_quad512.npz")
    m = gctx.mesh(g["cells"])
    E, H, rep = gctx.field_EH(m, g["J"], float(g["k"]), g["pts"], inc=_inc(g), precision=precision)
    assert rel_l2(E, g["E"]) < tol
    assert rel_l2(H, g["H"]) < tol
    assert rep.n_near_pairs > 0 and rep.n_nonfinite == 0
    if precision == "mixed":
        assert 0 < rep.est_rel_l2 < tol
    m.close()


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_golden_tri80_complex_k_two_rhs(gctx, precision, tol):
    g = golden("field_tri80.npz")
    m = gctx.mesh(g["cells"])
    E, H, _ = gctx.field_EH(m, g["J"], complex(g["k"]), g["pts"], mult=complex(g["mult"]), precision=precision)
    assert E.shape == g["E"].shape
    assert rel_l2(E, g["E"]) < tol
    assert rel_l2(H, g["H"]) < tol


def test_sphere512_1000_points_fp64(gctx):
    c = W.config1()
    kv, e0, hs = c["inc"]
    inc = abi.PlaneWave.make(kv, e0, hs, True, True)
    m = gctx.mesh(c["cells"])
    E, H, rep = gctx.field_EH(m, c["J"], c["k"], c["pts"], inc=inc)
    Eo, Ho = oracle.field_EH(c["cells"], c["J"], c["k"], c["pts"], inc=inc)
    assert rel_l2(E, Eo) < TOL_FP64 and rel_l2(H, Ho) < TOL_FP64
    assert rep.n_pairs == 512 * 1000 and rep.n_near_pairs == 0
    Em, Hm, repm = gctx.field_EH(m, c["J"], c["k"], c["pts"], inc=inc, precision="mixed")
    assert rel_l2(Em, Eo) < TOL_MIXED and rel_l2(Hm, Ho) < TOL_MIXED


def test_sphere8192_near_and_far_subset(gctx):
    c = W.config2()
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(18000, 96, replace=False), 18000 + rng.choice(2000, 32, replace=False)])
    pts = c["pts"][idx]
    m = gctx.mesh(c["cells"])
    E, H, rep = gctx.field_EH(m, c["J"], c["k"], pts)
    Eo, Ho = oracle.field_EH(c["cells"], c["J"], c["k"], pts)
    assert rep.n_near_pairs > 0
    assert rel_l2(E, Eo) < TOL_FP64 and rel_l2(H, Ho) < TOL_FP64
    Em, Hm, _ = gctx.field_EH(m, c["J"], c["k"], pts, precision="mixed")
    assert rel_l2(Em, Eo) < TOL_MIXED and rel_l2(Hm, Ho) < TOL_MIXED


@pytest.mark.parametrize("n_start,n_seg,p_max", [(4, 5, 1), (10, 12, 1), (20, 10, 1), (4, 6, 2), (8, 10, 2),
                                                  (3, 4, 3), (8, 10, 3), (4, 5, 4)])
def test_quadrature_splits_and_adaptive(gctx, n_start, n_seg, p_max):
    """Node tiles that fill one stage partially (n=4), several cells per stage
    (n=10), chunked cells (n=20: 400 nodes > one stage) and adaptive refinement:
    p_max = 2 runs the far pairs through the table-driven kernels at 2 n_start;
    p_max >= 3 tests convergence between the passes at n_start and 2 n_start
    for every far pair and runs the failing ones through the whole loop. FP64
    and mixed, against the oracle's full refinement loop."""
    cells = W.uv_sphere(8, 16)
    J = W.po_currents(cells, 4.0, directions=3, seed=5)
    rng = np.random.default_rng(n_start)
    pts = np.concatenate([W.sphere_points(40, 2.0, n_start), W.near_points(cells, 12, 0.02, 0.3, rng)])
    npm = abi.NumParam.default(n_start=n_start, n_start_seg=n_seg, p_max=p_max, p_max_seg=p_max)
    m = gctx.mesh(cells)
    E, H, _ = gctx.field_EH(m, J, 4.0, pts, numparam=npm)
    Eo, Ho = oracle.field_EH(cells, J, 4.0, pts, npm)
    assert rel_l2(E, Eo) < TOL_FP64 and rel_l2(H, Ho) < TOL_FP64
    Em, Hm, _ = gctx.field_EH(m, J, 4.0, pts, numparam=npm, precision="mixed")
    assert rel_l2(Em, Eo) < TOL_MIXED and rel_l2(Hm, Ho) < TOL_MIXED


@pytest.mark.parametrize("p_max", [3, 4])
@pytest.mark.parametrize("eps", [1e-14, 1e3])
def test_adaptive_far_refinement_paths(gctx, eps, p_max):
    """Every far pair failing the convergence test at the second pass (eps =
    1e-14: with p_max = 3 all take the third pass from the 4 n_start tables,
    with p_max = 4 the whole loop in the refinement kernel) and none failing
    (eps = 1e3: all take the pass at 2 n_start); triangles and quads, complex
    k, 3 RHS; FP64 against the oracle's loop."""
    rng = np.random.default_rng(8)
    for cells, k in ((W.uv_sphere(6, 12), 3.0), (W.perturbed_icosphere(1, seed=3), complex(2.5, 0.4))):
        J = W.po_currents(cells, abs(k), directions=3, seed=2)
        pts = np.concatenate([W.sphere_points(20, 2.0, 7), W.near_points(cells, 6, 0.02, 0.4, rng)])
        npm = abi.NumParam.default(n_start=3, n_start_seg=4, p_max=p_max, p_max_seg=2)
        npm.eps = eps
        m = gctx.mesh(cells)
        E, H, _ = gctx.field_EH(m, J, k, pts, numparam=npm)
        Eo, Ho = oracle.field_EH(cells, J, k, pts, npm)
        assert rel_l2(E, Eo) < TOL_FP64 and rel_l2(H, Ho) < TOL_FP64
        m.close()


def test_multi_rhs_chunks_and_large_k(gctx):
    """7 RHS (chunks of 4 + 2 + 1) and a large k (mixed-form phase beyond 4 rad per cell)."""
    cells = W.uv_sphere(12, 24)
    J = W.po_currents(cells, 40.0, directions=7, seed=9)
    pts = W.sphere_points(64, 2.5, 3)
    m = gctx.mesh(cells)
    for k in (2.0, 40.0, complex(6.0, 0.7)):
        E, H, _ = gctx.field_EH(m, J, k, pts, mult=complex(0.5, 2.0))
        Eo, Ho = oracle.field_EH(cells, J, k, pts, mult=complex(0.5, 2.0))
        assert rel_l2(E, Eo) < TOL_FP64 and rel_l2(H, Ho) < TOL_FP64
        Em, Hm, _ = gctx.field_EH(m, J, k, pts, mult=complex(0.5, 2.0), precision="mixed")
        assert rel_l2(Em, Eo) < TOL_MIXED and rel_l2(Hm, Ho) < TOL_MIXED


def test_edge_cases(gctx):
    cells = W.uv_sphere(4, 8)
    J = W.po_currents(cells, 1.0)
    m = gctx.mesh(cells)
    # no points
    E, H, rep = gctx.field_EH(m, J, 1.0, np.zeros((0, 3)))
    assert E.shape == (1, 0, 3)
    # one point, one cell mesh
    one = gctx.mesh(cells[5:6])
    p = np.array([[3.0, 0.1, -0.2]])
    E1, H1, _ = gctx.field_EH(one, J[:, 5:6], 1.0, p)
    Eo, Ho = oracle.field_EH(cells[5:6], J[:, 5:6], 1.0, p)
    assert rel_l2(E1, Eo) < TOL_FP64 and rel_l2(H1, Ho) < TOL_FP64
    # a point at a cell centre: R_Rot_Colloc is 0 there, K near path smooths
    pc = W.centres(cells)[[3]] + 0.0
    E2, H2, _ = gctx.field_EH(m, J, 1.0, pc * 1.0000001)
    Eo2, Ho2 = oracle.field_EH(cells, J, 1.0, pc * 1.0000001)
    assert rel_l2(E2, Eo2) < TOL_FP64 and rel_l2(H2, Ho2) < TOL_FP64
    # bad arguments fail with a status, not a crash
    from bielcc_b200.gpu import BielccError

    with pytest.raises((ValueError, BielccError)):
        gctx.field_EH(m, J[:, :3], 1.0, p)
    with pytest.raises(BielccError):
        gctx.field_EH(m, J, 1.0, p, numparam=abi.NumParam.default(n_start=0))


def test_device_buffers_through_torch(gctx):
    """The device-pointer entry point on a torch stream matches the host one."""
    torch = pytest.importorskip("torch")
    c = W.config1()
    m = gctx.mesh(c["cells"])
    pts = c["pts"][:256]
    E, H, _ = gctx.field_EH(m, c["J"], c["k"], pts)
    dev = torch.device("cuda:0")
    Jd = torch.from_numpy(np.ascontiguousarray(c["J"])).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    Ed = torch.zeros((1, 256, 3), dtype=torch.complex128, device=dev)
    Hd = torch.zeros_like(Ed)
    st = torch.cuda.current_stream()
    gctx.field_EH_device(m, Jd.data_ptr(), c["k"], Pd.data_ptr(), Ed.data_ptr(), Hd.data_ptr(), 1, 256,
                         stream=st.cuda_stream)
    torch.cuda.synchronize()
    assert rel_l2(Ed.cpu().numpy(), E) == 0.0
    assert rel_l2(Hd.cpu().numpy(), H) == 0.0


def test_mesh_geometry_rows(gctx):
    """Centres, diameters, normals and the CellFill tangent basis computed on the device."""
    for cells in (W.uv_sphere(16, 32), W.perturbed_icosphere(level=2, seed=2)):
        m = gctx.mesh(cells)
        g = m.geometry()
        o = oracle.cell_geometry(cells)
        assert np.abs(g[:, :13] - o[:, :13]).max() < 1e-14
        assert np.abs(g[:, 13] - o[:, 13]).max() < 1e-14
        m.close()


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
@pytest.mark.parametrize("S", [3, 16])
def test_many_rhs_single_job_routes_through_batched_kernel(gctx, precision, tol, S):
    """3 and 16 right-hand sides on 4000 points: the single-job call takes the
    batched kernel (moments once, contracted with every RHS) and agrees with
    one-RHS single-job launches and, on a point subset, with the oracle."""
    cells = W.uv_sphere(16, 32)
    k = 2 * np.pi
    J = W.po_currents(cells, k, directions=S, seed=8)
    rng = np.random.default_rng(8)
    pts = np.concatenate([W.shell_points(3800, 2.0, 4.0, rng), W.near_points(cells, 200, 0.02, 0.1, rng)])
    m = gctx.mesh(cells)
    E, H, rep = gctx.field_EH(m, J, k, pts, mult=complex(0.3, 0.7), precision=precision)
    for g in range(S):
        Eg, Hg, _ = gctx.field_EH(m, J[g:g + 1], k, pts, mult=complex(0.3, 0.7), precision=precision)
        assert rel_l2(E[g:g + 1], Eg) < tol and rel_l2(H[g:g + 1], Hg) < tol
    sub = np.r_[0:60, 3800:3840]
    Eo, Ho = oracle.field_EH(cells, J, k, pts[sub], mult=complex(0.3, 0.7))
    assert rel_l2(E[:, sub], Eo) < tol and rel_l2(H[:, sub], Ho) < tol
    assert rep.n_near_pairs > 0


def test_mixed_error_estimate_is_the_sample_error(gctx):
    """The mixed form's est_rel_l2 is its relative L2 error against the FP64
    form over min(P, 256) points spread over the set (evaluated beside the
    main evaluation): equal to the error measured against a full FP64 run at
    those points."""
    c = W.config1()
    m = gctx.mesh(c["cells"])
    for P in (1000, 100):
        pts = c["pts"][:P]
        Em, Hm, rep = gctx.field_EH(m, c["J"], c["k"], pts, precision="mixed")
        E6, H6, _ = gctx.field_EH(m, c["J"], c["k"], pts, precision="fp64")
        Q = min(P, 256)
        idx = np.arange(Q) * P // Q
        num = np.sum(np.abs(Em[:, idx] - E6[:, idx]) ** 2) + np.sum(np.abs(Hm[:, idx] - H6[:, idx]) ** 2)
        den = np.sum(np.abs(E6[:, idx]) ** 2) + np.sum(np.abs(H6[:, idx]) ** 2)
        assert rep.est_sample == Q
        assert rep.est_rel_l2 == pytest.approx(np.sqrt(num / den), rel=1e-6)


def test_context_created_again_after_destroy():
    """Destroying a context leaves no CUDA error behind: a context created
    after it uploads a mesh and evaluates as the first did."""
    from bielcc_b200 import gpu

    c = W.config1()
    pts = c["pts"][:64]
    out = []
    for _ in range(2):
        ctx = gpu.Context(0)
        m = ctx.mesh(c["cells"])
        E, H, _ = ctx.field_EH(m, c["J"], c["k"], pts, precision="mixed")
        out.append((E, H))
        m.close()
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_zero_wavenumber_static_limit(gctx):
    """k = 0 (the static limit): the real-k far node folds k into its phase
    denominator and the FP64 split takes its shortest Taylor level; both forms
    match the oracle, single-job and batched."""
    cells = W.uv_sphere(8, 16)
    J = W.po_currents(cells, 2.0, directions=2, seed=11)
    rng = np.random.default_rng(11)
    pts = np.concatenate([W.shell_points(150, 2.0, 4.0, rng), W.near_points(cells, 20, 0.02, 0.2, rng)])
    m = gctx.mesh(cells)
    Eo, Ho = oracle.field_EH(cells, J, 0.0, pts)
    assert np.all(np.isfinite(Eo)) and np.linalg.norm(Eo) > 0
    for precision, tol in (("fp64", TOL_FP64), ("mixed", TOL_MIXED)):
        E, H, _ = gctx.field_EH(m, J, 0.0, pts, precision=precision)
        assert rel_l2(E, Eo) < tol and rel_l2(H, Ho) < tol
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    Ed = torch.zeros((2, len(pts), 3), dtype=torch.complex128, device=dev)
    Hd = torch.zeros_like(Ed)
    jobs = gctx.make_jobs([dict(mesh=m, n_rhs=2, n_pts=len(pts), J=Jd.data_ptr(), pts=Pd.data_ptr(), E=Ed.data_ptr(),
                                H=Hd.data_ptr(), k=0.0)])
    gctx.field_EH_batch(jobs, precision="mixed", stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel_l2(Ed.cpu().numpy(), Eo) < TOL_MIXED and rel_l2(Hd.cpu().numpy(), Ho) < TOL_MIXED
