"""Batched field evaluation (many meshes, uneven sizes, several RHS, one
persistent launch) against the single-job path and the oracle; a job's
result is the same alone and inside a mixed batch."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, TOL_MIXED, rel_l2

pytestmark = pytest.mark.gpu


def _batch(torch, gctx, specs_np, precision, numparam=None):
    dev = torch.device("cuda:0")
    keep, specs = [], []
    for sp in specs_np:
        Jd = torch.from_numpy(np.ascontiguousarray(sp["J"])).to(dev)
        Pd = torch.from_numpy(np.ascontiguousarray(sp["pts"])).to(dev)
        S, P = sp["J"].shape[0], len(sp["pts"])
        Ed = torch.zeros((S, P, 3), dtype=torch.complex128, device=dev)
        Hd = torch.zeros_like(Ed)
        keep += [Jd, Pd, Ed, Hd]
        specs.append(dict(mesh=sp["mesh"], n_rhs=S, n_pts=P, J=Jd.data_ptr(), pts=Pd.data_ptr(), E=Ed.data_ptr(),
                          H=Hd.data_ptr(), k=sp["k"], mult=sp.get("mult", 1.0), inc=sp.get("inc"), out=(Ed, Hd)))
    jobs = gctx.make_jobs(specs)
    rep = gctx.field_EH_batch(jobs, numparam=numparam, precision=precision,
                              stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    outs = [(sp["out"][0].cpu().numpy(), sp["out"][1].cpu().numpy()) for sp in specs]
    return outs, rep


def _jobs(gctx, seed=0):
    rng = np.random.default_rng(seed)
    meshes = [W.uv_sphere(6, 12), W.perturbed_icosphere(1, seed=4), W.torus(18, 6), W.spheroid(5, 10, 1.0, 2.5)]
    specs = []
    for i, cells in enumerate(meshes):
        k = [2.0, 5.0, complex(3.0, 0.2), 9.0][i]
        S = [1, 5, 3, 7][i]
        ext = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        pts = np.concatenate([W.shell_points(40 + 13 * i, 1.6 * ext, 3 * ext, rng),
                              W.near_points(cells, 6, 0.02, 0.2, rng)])
        specs.append(dict(mesh=gctx.mesh(cells), cells=cells, J=W.po_currents(cells, abs(k), directions=S, seed=i),
                          pts=pts, k=k, mult=complex(1.0, 0.5 * i)))
    return specs


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_batch_matches_oracle(gctx, precision, tol):
    torch = pytest.importorskip("torch")
    specs = _jobs(gctx)
    outs, rep = _batch(torch, gctx, specs, precision)
    assert rep.n_near_pairs > 0
    for sp, (E, H) in zip(specs, outs):
        Eo, Ho = oracle.field_EH(sp["cells"], sp["J"], sp["k"], sp["pts"], mult=sp["mult"])
        assert rel_l2(E, Eo) < tol and rel_l2(H, Ho) < tol


def test_batch_job_alone_equals_in_mix(gctx):
    torch = pytest.importorskip("torch")
    specs = _jobs(gctx, seed=3)
    mix, _ = _batch(torch, gctx, specs, "mixed")
    for i in (0, 3):
        alone, _ = _batch(torch, gctx, [specs[i]], "mixed")
        assert np.array_equal(alone[0][0], mix[i][0]) and np.array_equal(alone[0][1], mix[i][1])


def test_batch_fallback_adaptive_and_autotune(gctx):
    torch = pytest.importorskip("torch")
    specs = _jobs(gctx, seed=5)[:2]
    # p_max = 2 runs the batched kernel's far pass at 2 n_start; p_max = 3 one call per job
    for pm in (2, 3):
        npm = abi.NumParam.default(n_start=4, n_start_seg=5, p_max=pm, p_max_seg=2)
        for precision, tol in (("fp64", TOL_FP64), ("mixed", TOL_MIXED)):
            outs, _ = _batch(torch, gctx, specs, precision, numparam=npm)
            for sp, (E, H) in zip(specs, outs):
                Eo, Ho = oracle.field_EH(sp["cells"], sp["J"], sp["k"], sp["pts"], npm, mult=sp["mult"])
                assert rel_l2(E, Eo) < tol and rel_l2(H, Ho) < tol
    dev = torch.device("cuda:0")
    keep = []
    s2 = []
    for sp in specs:
        Jd = torch.from_numpy(np.ascontiguousarray(sp["J"])).to(dev)
        Pd = torch.from_numpy(np.ascontiguousarray(sp["pts"])).to(dev)
        Ed = torch.zeros((sp["J"].shape[0], len(sp["pts"]), 3), dtype=torch.complex128, device=dev)
        keep += [Jd, Pd, Ed]
        s2.append(dict(mesh=sp["mesh"], n_rhs=sp["J"].shape[0], n_pts=len(sp["pts"]), J=Jd.data_ptr(),
                       pts=Pd.data_ptr(), E=Ed.data_ptr(), k=sp["k"]))
    c = gctx.batch_autotune(gctx.make_jobs(s2), precision="mixed")
    assert c > 0


SPLIT_DEFAULT = 16 << 30


@pytest.mark.parametrize("mode", ["split, one wave", "split, many waves", "fused", "tensor cores",
                                  "split, tensor cores", "fused, p_max 2"])
def test_batch_plan_graph_replay_with_new_currents(gctx, mode):
    """A planned batch replayed from its CUDA graph after the currents changed
    in place gives the same result as a fresh batched call with those
    currents, and matches the oracle: the split pipeline (a plan of one wave,
    the default, keeps its moments and replays only the contraction, and the
    fresh call runs the fused kernel; a plan of many waves with every batch
    split), the fused kernel, the tensor-core forms."""
    torch = pytest.importorskip("torch")
    gctx.set_batch_tensor_cores("tensor cores" in mode)
    cap, every = {"split, one wave": (SPLIT_DEFAULT, False), "split, many waves": (100_000, True),
                  "split, tensor cores": (SPLIT_DEFAULT, True)}.get(mode, (0, False))
    gctx.set_batch_split(cap, all_batches=every)
    npm = abi.NumParam.default(n_start=4, n_start_seg=5, p_max=2, p_max_seg=2) if "p_max 2" in mode else None
    try:
        _plan_replay(torch, gctx, npm)
    finally:
        gctx.set_batch_tensor_cores(False)
        gctx.set_batch_split(SPLIT_DEFAULT)


def _plan_replay(torch, gctx, npm=None):
    dev = torch.device("cuda:0")
    specs = _jobs(gctx, seed=7)
    tens, jspecs = [], []
    for sp in specs:
        Jd = torch.from_numpy(np.ascontiguousarray(sp["J"])).to(dev)
        Pd = torch.from_numpy(np.ascontiguousarray(sp["pts"])).to(dev)
        S, P = sp["J"].shape[0], len(sp["pts"])
        Ed = torch.zeros((S, P, 3), dtype=torch.complex128, device=dev)
        Hd = torch.zeros_like(Ed)
        tens.append((Jd, Pd, Ed, Hd))
        jspecs.append(dict(mesh=sp["mesh"], n_rhs=S, n_pts=P, J=Jd.data_ptr(), pts=Pd.data_ptr(), E=Ed.data_ptr(),
                           H=Hd.data_ptr(), k=sp["k"], mult=sp["mult"]))
    jobs = gctx.make_jobs(jspecs)
    sc = torch.cuda.current_stream().cuda_stream
    plan = gctx.batch_plan(jobs, numparam=npm, precision="mixed", stream=sc)
    torch.cuda.synchronize()
    first = [(E.clone(), H.clone()) for _, _, E, H in tens]
    fresh, _ = _batch(torch, gctx, specs, "mixed", numparam=npm)
    for (E, H), (Ef, Hf) in zip(first, fresh):
        assert np.array_equal(E.cpu().numpy(), Ef) and np.array_equal(H.cpu().numpy(), Hf)
    # new currents in place, then replay the graph (twice: replays are repeatable)
    for sp, (Jd, _, _, _) in zip(specs, tens):
        sp["J"] = W.po_currents(sp["cells"], abs(sp["k"]), directions=sp["J"].shape[0], seed=99)
        Jd.copy_(torch.from_numpy(sp["J"]))
    for _ in range(2):
        plan.launch(stream=sc)
    torch.cuda.synchronize()
    fresh, _ = _batch(torch, gctx, specs, "mixed", numparam=npm)
    for sp, (_, _, E, H), (Ef, Hf) in zip(specs, tens, fresh):
        E, H = E.cpu().numpy(), H.cpu().numpy()
        assert np.array_equal(E, Ef) and np.array_equal(H, Hf)
        Eo, Ho = oracle.field_EH(sp["cells"], sp["J"], sp["k"], sp["pts"], npm, mult=sp["mult"])
        assert rel_l2(E, Eo) < TOL_MIXED and rel_l2(H, Ho) < TOL_MIXED
    assert plan.report.n_near_pairs > 0
    plan.close()


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_batch_edge_cases(gctx, precision, tol):
    """An empty batch; a job without points; a one-cell mesh; 70 right-hand
    sides (more than one staged pass of 64); all in one launch, against the
    oracle; and the largest staged split, n_start = 22."""
    torch = pytest.importorskip("torch")
    assert gctx.field_EH_batch(gctx.make_jobs([]), precision=precision).n_pairs == 0
    rng = np.random.default_rng(9)
    sph = W.uv_sphere(4, 8)
    specs = [
        dict(mesh=gctx.mesh(sph[7:8]), cells=sph[7:8], J=W.po_currents(sph, 2.0)[:, 7:8], pts=np.array([[2.5, 0.3, 0.1]]),
             k=2.0, mult=1.0),
        dict(mesh=gctx.mesh(sph), cells=sph, J=W.po_currents(sph, 3.0, directions=70, seed=4),
             pts=np.concatenate([W.shell_points(20, 2.0, 3.0, rng), W.near_points(sph, 4, 0.02, 0.1, rng)]), k=3.0,
             mult=complex(0.0, 1.0)),
        dict(mesh=gctx.mesh(sph), cells=sph, J=W.po_currents(sph, 1.0), pts=np.zeros((0, 3)), k=1.0, mult=1.0),
    ]
    outs, _ = _batch(torch, gctx, specs, precision)
    for sp, (E, H) in zip(specs, outs):
        if len(sp["pts"]) == 0:
            assert E.shape[1] == 0
            continue
        Eo, Ho = oracle.field_EH(sp["cells"], sp["J"], sp["k"], sp["pts"], mult=sp["mult"])
        assert rel_l2(E, Eo) < tol and rel_l2(H, Ho) < tol
    npm = abi.NumParam.default(n_start=22)
    sp = specs[1]
    sp22 = dict(sp, J=sp["J"][:3])
    outs, _ = _batch(torch, gctx, [sp22], precision, numparam=npm)
    Eo, Ho = oracle.field_EH(sp22["cells"], sp22["J"], sp22["k"], sp22["pts"], npm, mult=sp22["mult"])
    assert rel_l2(outs[0][0], Eo) < tol and rel_l2(outs[0][1], Ho) < tol


def test_batch_tensor_core_contraction_matches_cuda_cores(gctx):
    """Mixed batches contract the far moments with the currents on the tensor
    cores (TF32 hi + lo, FP32 over 16 cells, FP64 across): the result agrees
    with the CUDA-core contraction and the oracle within the mixed tolerance,
    for 1, 5, 16, 17, 33 and 64 right-hand sides (one, two, three and four
    staged current groups), quads and triangles, real and complex k; a job
    with more than 64 right-hand sides takes the CUDA-core contraction."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    meshes = [W.uv_sphere(8, 16), W.perturbed_icosphere(2, seed=5), W.torus(24, 8), W.rounded_cube(6, 0.1, 1.0),
              W.spheroid(6, 12, 1.0, 3.0), W.triangulate(W.uv_sphere(6, 12))]
    specs = []
    for i, cells in enumerate(meshes):
        k = [2.0, 6.0, complex(3.0, 0.3), 9.0, 1.5, 4.0][i]
        S = [1, 5, 16, 17, 33, 64][i]
        ext = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        pts = np.concatenate([W.shell_points(45 + 7 * i, 1.6 * ext, 3 * ext, rng),
                              W.near_points(cells, 5, 0.02, 0.2, rng)])
        specs.append(dict(mesh=gctx.mesh(cells), cells=cells, J=W.po_currents(cells, abs(k), directions=S, seed=i),
                          pts=pts, k=k, mult=complex(0.5, 1.0)))
    try:
        gctx.set_batch_tensor_cores(True)
        tc, rep = _batch(torch, gctx, specs, "mixed")
        gctx.set_batch_tensor_cores(False)
        cc, _ = _batch(torch, gctx, specs, "mixed")
    finally:
        gctx.set_batch_tensor_cores(False)
    assert rep.n_near_pairs > 0
    for sp, (E, H), (Ec, Hc) in zip(specs, tc, cc):
        assert rel_l2(E, Ec) < TOL_MIXED and rel_l2(H, Hc) < TOL_MIXED
        s2 = min(3, sp["J"].shape[0])
        Eo, Ho = oracle.field_EH(sp["cells"], sp["J"][:s2], sp["k"], sp["pts"], mult=sp["mult"])
        assert rel_l2(E[:s2], Eo) < TOL_MIXED and rel_l2(H[:s2], Ho) < TOL_MIXED
    # more than 64 right-hand sides: the CUDA-core contraction, same results as per-job calls
    big = dict(specs[0], J=W.po_currents(meshes[0], 2.0, directions=70, seed=3))
    out, _ = _batch(torch, gctx, [big], "mixed")
    Eo, Ho = oracle.field_EH(big["cells"], big["J"][::23], big["k"], big["pts"], mult=big["mult"])
    assert rel_l2(out[0][0][::23], Eo) < TOL_MIXED and rel_l2(out[0][1][::23], Ho) < TOL_MIXED


@pytest.mark.parametrize("tensor_cores", [False, True])
@pytest.mark.parametrize("cap", [SPLIT_DEFAULT, 200_000])
def test_batch_split_pipeline_equals_fused_kernel(gctx, cap, tensor_cores):
    """The split pipeline (moments to a device buffer, then the contraction on
    the CUDA or the tensor cores; one wave, or many waves of a small buffer)
    against the fused kernel of the same contraction: 1 to 70 right-hand sides
    (the tensor cores: up to 64), quads and triangles, real and complex k,
    near points. With the CUDA-core contraction the results are bit-identical.
    The fused tensor-core kernel evaluates one cell per warp with that cell's
    own phase polynomial, while the moments kernel pairs cells c and c + 4 of
    each block under the polynomial of the larger phase range, so the
    tensor-core forms agree within the mixed tolerance, not bit for bit."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(21)
    meshes = [W.uv_sphere(8, 16), W.perturbed_icosphere(2, seed=5), W.torus(24, 8), W.rounded_cube(6, 0.1, 1.0),
              W.triangulate(W.uv_sphere(6, 12))]
    specs = []
    for i, cells in enumerate(meshes):
        k = [2.0, 6.0, complex(3.0, 0.3), 9.0, 4.0][i]
        S = [1, 5, 17, 33, 64 if tensor_cores else 70][i]
        ext = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        pts = np.concatenate([W.shell_points(45 + 7 * i, 1.6 * ext, 3 * ext, rng),
                              W.near_points(cells, 5, 0.02, 0.2, rng)])
        specs.append(dict(mesh=gctx.mesh(cells), cells=cells, J=W.po_currents(cells, abs(k), directions=S, seed=i),
                          pts=pts, k=k, mult=complex(0.5, 1.0)))
    try:
        gctx.set_batch_tensor_cores(tensor_cores)
        gctx.set_batch_split(0)
        fused, _ = _batch(torch, gctx, specs, "mixed")
        gctx.set_batch_split(cap, all_batches=True)
        split, rep = _batch(torch, gctx, specs, "mixed")
    finally:
        gctx.set_batch_split(SPLIT_DEFAULT)
        gctx.set_batch_tensor_cores(False)
    assert rep.n_near_pairs > 0
    for (E, H), (Ef, Hf) in zip(split, fused):
        if tensor_cores:
            assert rel_l2(E, Ef) < TOL_MIXED and rel_l2(H, Hf) < TOL_MIXED
        else:
            assert np.array_equal(E, Ef) and np.array_equal(H, Hf)
    sp = specs[2]
    Eo, Ho = oracle.field_EH(sp["cells"], sp["J"][:2], sp["k"], sp["pts"], mult=sp["mult"])
    assert rel_l2(split[2][0][:2], Eo) < TOL_MIXED and rel_l2(split[2][1][:2], Ho) < TOL_MIXED
