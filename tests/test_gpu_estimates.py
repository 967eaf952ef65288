"""Every mixed-precision result reports its error against the FP64 form: the
single-job device-buffer call, the full Stratton-Chu field, every job of a
batch (its est_dev and the batch's report), every served field request and
the mixed collocation matrix. Each estimate must equal the relative L2
difference, measured here against a separate FP64 run, over the sample the
library states (points q * P / Q, the first RHS; rows r * N / R)."""
import numpy as np
import pytest

from bielcc_b200 import abi, gpu
from bielcc_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))


def _sample_err(Em, Hm, E6, H6, Q, S):
    P = Em.shape[1]
    idx = np.arange(Q) * P // Q
    num = np.sum(np.abs(Em[:S, idx] - E6[:S, idx]) ** 2) + np.sum(np.abs(Hm[:S, idx] - H6[:S, idx]) ** 2)
    den = np.sum(np.abs(E6[:S, idx]) ** 2) + np.sum(np.abs(H6[:S, idx]) ** 2)
    return float(np.sqrt(num / den))


def test_device_call_reports_its_error(gctx):
    torch = pytest.importorskip("torch")
    c = W.config1()
    cells, J, k = c["cells"], c["J"], c["k"]
    rng = np.random.default_rng(2)
    pts = np.concatenate([c["pts"][:600], W.near_points(cells, 40, 0.02, 0.1, rng)])
    m = gctx.mesh(cells)
    dev = torch.device("cuda:0")
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    out = {}
    for prec in ("mixed", "fp64"):
        E = torch.zeros((1, len(pts), 3), dtype=torch.complex128, device=dev)
        H = torch.zeros_like(E)
        rep = gctx.field_EH_device(m, Jd.data_ptr(), k, Pd.data_ptr(), E.data_ptr(), H.data_ptr(), 1, len(pts),
                                   precision=prec, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        out[prec] = (E.cpu().numpy(), H.cpu().numpy(), rep)
    Em, Hm, rep = out["mixed"]
    E6, H6, rep6 = out["fp64"]
    assert rep6.est_rel_l2 == 0.0 and rep.est_sample == 256
    want = _sample_err(Em, Hm, E6, H6, 256, 1)
    assert 0 < want < 1e-6
    assert rep.est_rel_l2 == pytest.approx(want, rel=1e-5)


def test_full_field_reports_its_error(gctx):
    c = W.config1()
    cells, k = c["cells"], c["k"]
    JE = W.po_currents(cells, k, directions=2, seed=1)
    JM = 0.3 * W.po_currents(cells, k, directions=2, seed=5)
    pts = c["pts"][:300]
    m = gctx.mesh(cells)
    mE, mH = complex(0.2, 1.1), complex(-0.4, 0.7)
    Em, Hm, rep = gctx.field_EH_full(m, JE, JM, k, pts, multE=mE, multH=mH, precision="mixed")
    E6, H6, _ = gctx.field_EH_full(m, JE, JM, k, pts, multE=mE, multH=mH, precision="fp64")
    assert rep.est_sample == 256
    assert rep.est_rel_l2 == pytest.approx(_sample_err(Em, Hm, E6, H6, 256, 2), rel=1e-5)


def test_batch_reports_every_jobs_error(gctx):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(4)
    meshes = [W.uv_sphere(6, 12), W.perturbed_icosphere(2, seed=3), W.torus(18, 6)]
    specs, keep = [], []
    est = torch.full((len(meshes),), -1.0, dtype=torch.float64, device=dev)
    for i, cells in enumerate(meshes):
        S = [1, 6, 3][i]
        k = [2.0, 5.0, complex(3.0, 0.2)][i]
        ext = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        pts = np.concatenate([W.shell_points(70 + 20 * i, 1.6 * ext, 3 * ext, rng),
                              W.near_points(cells, 6, 0.02, 0.2, rng)])
        J = W.po_currents(cells, abs(k), directions=S, seed=i)
        Jd = torch.from_numpy(J).to(dev)
        Pd = torch.from_numpy(pts).to(dev)
        outs = {p: (torch.zeros((S, len(pts), 3), dtype=torch.complex128, device=dev),
                    torch.zeros((S, len(pts), 3), dtype=torch.complex128, device=dev)) for p in ("mixed", "fp64")}
        keep.append((Jd, Pd, outs))
        specs.append(dict(mesh=gctx.mesh(cells), n_rhs=S, n_pts=len(pts), J=Jd.data_ptr(), pts=Pd.data_ptr(), k=k))
    res = {}
    for prec in ("mixed", "fp64"):
        sp = [dict(s, E=keep[i][2][prec][0].data_ptr(), H=keep[i][2][prec][1].data_ptr(),
                   est=est[i:].data_ptr() if prec == "mixed" else None) for i, s in enumerate(specs)]
        res[prec] = gctx.field_EH_batch(gctx.make_jobs(sp), precision=prec,
                                        stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
    num = den = 0.0
    est_h = est.cpu().numpy()
    for i, (_, _, outs) in enumerate(keep):
        Em, Hm = (t.cpu().numpy() for t in outs["mixed"])
        E6, H6 = (t.cpu().numpy() for t in outs["fp64"])
        P, S = Em.shape[1], Em.shape[0]
        Q, Ss = min(P, 32), min(S, 4)
        e = _sample_err(Em, Hm, E6, H6, Q, Ss)
        assert est_h[i] == pytest.approx(e, rel=1e-5), i
        idx = np.arange(Q) * P // Q
        num += np.sum(np.abs(Em[:Ss, idx] - E6[:Ss, idx]) ** 2) + np.sum(np.abs(Hm[:Ss, idx] - H6[:Ss, idx]) ** 2)
        den += np.sum(np.abs(E6[:Ss, idx]) ** 2) + np.sum(np.abs(H6[:Ss, idx]) ** 2)
    assert res["mixed"].est_sample == 3 * 32
    assert res["mixed"].est_rel_l2 == pytest.approx(np.sqrt(num / den), rel=1e-5)
    assert res["fp64"].est_rel_l2 == 0.0


def test_served_requests_report_their_error(gctx):
    rng = np.random.default_rng(6)
    cells = W.rounded_cube(6, 0.1, 1.0)
    k = 4.0
    J = W.po_currents(cells, k, directions=3, seed=2)
    m = gctx.mesh(cells)
    sv = gpu.Server(gctx, n_slots=2, precision="mixed")
    try:
        reqs = []
        for P in (50, 400):
            pts = W.shell_points(P, 2.5, 4.0, rng)
            reqs.append((pts, sv.submit_field(m, J, pts, k, out_c64=False)))
        for pts, t in reqs:
            st, _, out = sv.wait(t, timeout=120.0)
            assert st == 0
            E6, H6, _ = gctx.field_EH(m, J, k, pts, precision="fp64")
            e = _sample_err(out["E"], out["H"], E6, H6, min(len(pts), 32), 3)
            assert out["est"] == pytest.approx(e, rel=1e-5)
    finally:
        sv.close()


def test_assembly_reports_its_error(gctx):
    cells = W.perturbed_icosphere(level=3, seed=2)
    m = gctx.mesh(cells)
    k = 4 * np.pi
    Am, rep = gctx.assemble_K(m, k, c64=True, precision="mixed")
    A6, rep6 = gctx.assemble_K(m, k, precision="fp64")
    N = len(cells)
    R = min(N, 16)
    rows = (np.arange(R) * N // R)
    sel = np.concatenate([2 * rows[:, None] + np.arange(2)[None, :]], axis=0).ravel()
    assert rep.est_sample == R and rep6.est_rel_l2 == 0.0
    assert rep.est_rel_l2 == pytest.approx(_rel(Am[sel].astype(np.complex128), A6[sel]), rel=1e-4)
    assert 0 < rep.est_rel_l2 < 1e-6
