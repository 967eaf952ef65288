"""Per-pair operators, universal quadratures and analytic integrals on the GPU
against the reference's golden outputs (and the oracle)."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi, gpu
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, golden, rel_l2

pytestmark = pytest.mark.gpu


def test_pair_ops_golden(gctx):
    g = golden("pair_ops.npz")
    keys = sorted({k[: -len("_res")] for k in g.files if k.endswith("_res")})
    for key in keys:
        pm = int(key.split("_p")[-1])
        op = int(key.split("_op")[1].split("_")[0])
        npm = abi.NumParam.default(p_max=pm, p_max_seg=pm)
        r = gctx.pair_op(op, g[key + "_cells"], g[key + "_x"], g[key + "_j"], complex(g[key + "_k"]), npm)
        ref = g[key + "_res"]
        fin = np.isfinite(ref).all(axis=1)
        assert np.array_equal(fin, np.isfinite(r).all(axis=1)), key
        assert rel_l2(r[fin], ref[fin]) < TOL_FP64, key


def test_integrals_golden(gctx):
    g = golden("integrals.npz")
    for name in ("quad", "tri"):
        for fid in abi.PAIR_INTEGRANDS:
            for pm in (1, 2):
                key = f"{name}_f{fid}_p{pm}"
                n = len(g[key + "_x"])
                kp = abi.kernelparam_array(n, smoothR=g[key + "_sR"], smoothRMin=g[key + "_sRm"], k=g[key + "_k"],
                                           current=g[key + "_cur"], vec_dbl=g[key + "_vec"], normal=g[key + "_vec"])
                r = gctx.integral_pnt(fid, g[key + "_cells"], g[key + "_x"], kp, 8, pm, 1e-6)
                assert rel_l2(r, g[key + "_res"]) < TOL_FP64, key
    for fid in abi.PAIR_INTEGRANDS:
        for pm in (1, 3):
            key = f"seg_f{fid}_p{pm}"
            a, b = g[key + "_a"], g[key + "_b"]
            kp = abi.kernelparam_array(len(a), smoothR=g[key + "_sR"], smoothRMin=1e-3, k=g[key + "_k"],
                                       current=a + 1j * b, vec_dbl=b - a, normal=b - a)
            r = gctx.integral_seg_pnt(fid, a, b, g[key + "_x"], kp, 10, pm, 1e-6)
            assert rel_l2(r, g[key + "_res"]) < TOL_FP64, key


def test_integrals_one_point_form_golden(gctx):
    """IntegralUniversal (F(x) form) and the segment F(x) overload on the GPU
    against the reference's outputs, incl. the mutated smoothR; the pair and
    one-point entry points refuse each other's integrands."""
    g = golden("integrals_fx.npz")

    def kp_for(key, n):
        return abi.kernelparam_array(n, smoothR=0.1, smoothRMin=0.01, k=2 * np.pi, vec_dbl=g[key + "_kv"],
                                     e0=g[key + "_e0"])

    for fid in abi.FX_INTEGRANDS:
        for pm in (1, 3):
            for name in ("quad", "tri"):
                key = f"{name}_f{fid}_p{pm}"
                kp = kp_for(key, len(g[key + "_cells"]))
                r = gctx.integral(fid, g[key + "_cells"], kp, 8, pm, 1e-6)
                assert rel_l2(r, g[key + "_res"]) < TOL_FP64, key
                assert np.array_equal([kp[i].smoothR for i in range(len(kp))], g[key + "_sR"]), key
            key = f"seg_f{fid}_p{pm}"
            kp = kp_for(key, len(g[key + "_a"]))
            r = gctx.integral_seg(fid, g[key + "_a"], g[key + "_b"], kp, 10, pm, 1e-6)
            assert rel_l2(r, g[key + "_res"]) < TOL_FP64, key
    cells = g["quad_f12_p1_cells"][:2]
    kp = abi.kernelparam_array(2)
    with pytest.raises(gpu.BielccError):
        gctx.integral(abi.F_SIMPLEPOT_H, cells, kp, 8, 1, 1e-6)
    with pytest.raises(gpu.BielccError):
        gctx.integral_pnt(abi.F_PLANEWAVE_E, cells, W.centres(cells), kp, 8, 1, 1e-6)


def test_k0_against_oracle(gctx):
    rng = np.random.default_rng(3)
    cells = W.perturbed_icosphere(1)
    idx = rng.integers(0, len(cells), 40)
    cc = cells[idx]
    x = W.centres(cc) + rng.normal(size=(40, 3)) * 0.2
    j = rng.normal(size=(40, 3)) + 1j * rng.normal(size=(40, 3))
    for fid in (abi.F_GRADSIMPLEPOT_H, abi.F_NU_SIMPLEPOT_H, abi.F_ROTROTSIMPLEPOT_H):
        for common in (0, 1):
            for pm in (1, 2):
                kpa = abi.kernelparam_array(40, smoothR=0.05, smoothRMin=1e-6, k=complex(2.0, 0.1))
                kpb = abi.kernelparam_array(40, smoothR=0.05, smoothRMin=1e-6, k=complex(2.0, 0.1))
                a = gctx.k0(fid, common, cc, x, j, kpa, 10, pm, 1e-6)
                b = oracle.k0(fid, common, cc, x, j, kpb, 10, pm, 1e-6)
                assert rel_l2(a, b) < TOL_FP64
                assert [r.smoothR for r in kpa] == [r.smoothR for r in kpb]  # KernelParam left as the reference does


def test_analytic_golden(gctx):
    g = golden("analytic.npz")
    quad = W.uv_sphere(16, 32)
    tri = W.perturbed_icosphere(level=1, seed=2)
    for name, cells in (("quad", quad), ("tri", tri)):
        for tag in ("centre", "off"):
            x = g[f"{name}_{tag}_x"]
            assert rel_l2(gctx.integral_1divr(cells, x), g[f"{name}_{tag}_1divr"]) < TOL_FP64
            hs = gctx.integral_surf_simplepot_h_hs(cells, x, 3.0, 8, 1, 1e-6, 2 * np.pi)
            assert rel_l2(hs, g[f"{name}_{tag}_hs"]) < TOL_FP64
    a, b, x = g["seg_a"], g["seg_b"], g["seg_x"]
    assert rel_l2(gctx.integral_grad1divr_seg(a, b, x), g["seg_grad1divr"]) < TOL_FP64
    assert rel_l2(gctx.integral_seg_gradsimplepot_h_hs(a, b, x, 3.0, 10, 1, 1e-6, 2 * np.pi), g["seg_hs"]) < TOL_FP64


def test_known_answers_on_gpu(gctx):
    ka = golden("known_answers.npz")
    rut1 = np.array([[0., 0., 0.], [2., 0., 0.], [3., 2., 0.], [0., 2., 0.]])
    x = np.array([[2., 1.5, 0.]])
    kp = abi.kernelparam_array(1, k=0.0)
    area = gctx.integral_pnt(abi.F_ONE, rut1[None], x, kp, 8, 1, 1e-6)[0, 0]
    assert area == pytest.approx(5.0, abs=1e-13)
    npk = abi.NumParam(1e-6, 2.0, 2.0, 3.0, 80, 100, 6, 6)
    k = gctx.pair_op(abi.OP_K_HS, rut1[None], x, np.array([[1, 0, 0]], complex), 1.0, npk)[0]
    assert rel_l2(k, ka["k_hs_rut1"]) < TOL_FP64
    npc = abi.NumParam(1e-6, 2.2e-16, 2.2e-16, 3.0, 80, 100, 4, 4)
    z = gctx.pair_op(abi.OP_R_COLLOC, rut1[None], np.array([[1.25, 1.0, 0.0]]), np.array([[1, 1, 1]], complex), 1.0,
                     npc)[0]
    assert np.all(z == 0)
