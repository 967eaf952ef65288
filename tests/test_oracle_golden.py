"""The oracle (oracle/bielcc_oracle.cpp) against golden vectors produced by
the reference itself (tests/golden/make_golden.py) and against the values the
reference's example programs print."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from conftest import golden, rel_l2

TOL = 1e-13  # oracle vs reference, both FP64 on the CPU


def test_field_quad512():
    g = golden("field_quad512.npz")
    inc = abi.PlaneWave.make(g["kvec"], g["e0"], float(g["h_scale"]), True, True)
    E, H = oracle.field_EH(g["cells"], g["J"], float(g["k"]), g["pts"], inc=inc)
    assert rel_l2(E, g["E"]) < TOL
    assert rel_l2(H, g["H"]) < TOL


def test_field_tri80_complex_k_multi_rhs():
    g = golden("field_tri80.npz")
    E, H = oracle.field_EH(g["cells"], g["J"], complex(g["k"]), g["pts"], mult=complex(g["mult"]))
    assert E.shape[0] == 2
    assert rel_l2(E, g["E"]) < TOL
    assert rel_l2(H, g["H"]) < TOL


def _pair_cases():
    g = golden("pair_ops.npz")
    keys = sorted({k[: -len("_res")] for k in g.files if k.endswith("_res")})
    return g, keys


def test_pair_ops():
    g, keys = _pair_cases()
    assert len(keys) == 2 * 8 * 2 * 2
    for key in keys:
        pm = int(key.split("_p")[-1])
        op = int(key.split("_op")[1].split("_")[0])
        npm = abi.NumParam.default(p_max=pm, p_max_seg=pm)
        r = oracle.pair_op(op, g[key + "_cells"], g[key + "_x"], g[key + "_j"], complex(g[key + "_k"]), npm)
        ref = g[key + "_res"]
        fin = np.isfinite(ref).all(axis=1)
        assert np.array_equal(fin, np.isfinite(r).all(axis=1)), key
        assert rel_l2(r[fin], ref[fin]) < TOL, key


def test_integrals():
    g = golden("integrals.npz")
    for name in ("quad", "tri"):
        for fid in abi.PAIR_INTEGRANDS:
            for pm in (1, 2):
                key = f"{name}_f{fid}_p{pm}"
                n = len(g[key + "_x"])
                kp = abi.kernelparam_array(n, smoothR=g[key + "_sR"], smoothRMin=g[key + "_sRm"], k=g[key + "_k"],
                                           current=g[key + "_cur"], vec_dbl=g[key + "_vec"], normal=g[key + "_vec"])
                r = oracle.integral_pnt(fid, g[key + "_cells"], g[key + "_x"], kp, 8, pm, 1e-6)
                assert rel_l2(r, g[key + "_res"]) < TOL, key
    for fid in abi.PAIR_INTEGRANDS:
        for pm in (1, 3):
            key = f"seg_f{fid}_p{pm}"
            a, b = g[key + "_a"], g[key + "_b"]
            kp = abi.kernelparam_array(len(a), smoothR=g[key + "_sR"], smoothRMin=1e-3, k=g[key + "_k"],
                                       current=a + 1j * b, vec_dbl=b - a, normal=b - a)
            r = oracle.integral_seg_pnt(fid, a, b, g[key + "_x"], kp, 10, pm, 1e-6)
            assert rel_l2(r, g[key + "_res"]) < TOL, key


def _fx_kp(g, key, n):
    return abi.kernelparam_array(n, smoothR=0.1, smoothRMin=0.01, k=2 * np.pi, vec_dbl=g[key + "_kv"],
                                 e0=g[key + "_e0"])


def test_integrals_one_point_form():
    """IntegralUniversal and the segment F(x) overload (F = 1, PlaneWaveFieldE)
    against the reference's outputs, with the smoothR it leaves behind."""
    g = golden("integrals_fx.npz")
    for fid in abi.FX_INTEGRANDS:
        for pm in (1, 3):
            for name in ("quad", "tri"):
                key = f"{name}_f{fid}_p{pm}"
                kp = _fx_kp(g, key, len(g[key + "_cells"]))
                r = oracle.integral(fid, g[key + "_cells"], kp, 8, pm, 1e-6)
                assert rel_l2(r, g[key + "_res"]) < TOL, key
                assert np.array_equal([kp[i].smoothR for i in range(len(kp))], g[key + "_sR"]), key
            key = f"seg_f{fid}_p{pm}"
            kp = _fx_kp(g, key, len(g[key + "_a"]))
            r = oracle.integral_seg(fid, g[key + "_a"], g[key + "_b"], kp, 10, pm, 1e-6)
            assert rel_l2(r, g[key + "_res"]) < TOL, key
            assert np.array_equal([kp[i].smoothR for i in range(len(kp))], g[key + "_sR"]), key
    # F = 1 over the trapezoid of the reference's Test0 is its area, 5
    kp = abi.kernelparam_array(1)
    rut1 = np.array([[[0., 0., 0.], [2., 0., 0.], [3., 2., 0.], [0., 2., 0.]]])
    assert abs(oracle.integral(abi.F_ONE, rut1, kp, 8, 1, 1e-6)[0, 0] - 5.0) < 1e-12


def test_analytic():
    g = golden("analytic.npz")
    from bielcc_b200 import workloads as W

    quad = W.uv_sphere(16, 32)
    tri = W.perturbed_icosphere(level=1, seed=2)
    for name, cells in (("quad", quad), ("tri", tri)):
        for tag in ("centre", "off"):
            x = g[f"{name}_{tag}_x"]
            assert rel_l2(oracle.integral_1divr(cells, x), g[f"{name}_{tag}_1divr"]) < 1e-12
            hs = oracle.integral_surf_simplepot_h_hs(cells, x, 3.0, 8, 1, 1e-6, 2 * np.pi)
            assert rel_l2(hs, g[f"{name}_{tag}_hs"]) < 1e-12
    a, b, x = g["seg_a"], g["seg_b"], g["seg_x"]
    assert rel_l2(oracle.integral_grad1divr_seg(a, b, x), g["seg_grad1divr"]) < TOL
    assert rel_l2(oracle.integral_seg_gradsimplepot_h_hs(a, b, x, 3.0, 10, 1, 1e-6, 2 * np.pi), g["seg_hs"]) < TOL


RUT1 = np.array([[0., 0., 0.], [2., 0., 0.], [3., 2., 0.], [0., 2., 0.]])
RUT2 = np.array([[0., 2., 0.], [0., 0., 0.], [2., 0., 0.]])
RUT3 = np.array([[3., 2., 0.], [2., 0., 0.], [0., 2., 0.]])
X_EX = np.array([2., 1.5, 0.])


def test_known_answers_printed_by_reference_examples():
    """Values printed by examples/integrators/main0_integrals.cpp, ED_Operators/main0_K.cpp and
    main0_R.cpp (6 significant digits), and the golden full-precision values."""
    ka = golden("known_answers.npz")
    # Test0: area of the trapezoid rut1 is 5 (main0_integrals.cpp:24-27)
    assert oracle.area_by_quadrature(RUT1) == pytest.approx(5.0, abs=1e-14)
    kp = abi.kernelparam_array(1, smoothR=2.0 * 3.605551275463989 / 64, smoothRMin=1e-6, k=1.0)
    t1 = oracle.integral_pnt(abi.F_SIMPLEPOT_H, RUT1[None], X_EX[None], kp, 64, 8, 1e-6)[0, 0]
    assert t1 == pytest.approx(complex(4.64269, 3.82485), abs=6e-6)
    assert abs(t1 - ka["t1_quad"]) < 1e-12
    hs = oracle.integral_surf_simplepot_h_hs(RUT1[None], X_EX[None], 3.0, 64, 8, 1e-6, 1.0)[0]
    assert hs == pytest.approx(complex(4.64545, 3.82485), abs=6e-6)
    assert abs(hs - ka["t1_hs"]) < 1e-12
    npk = abi.NumParam(1e-6, 2.0, 2.0, 3.0, 80, 100, 6, 6)
    k = oracle.pair_op(abi.OP_K_HS, RUT1[None], X_EX[None], np.array([[1, 0, 0]], complex), 1.0, npk)[0]
    assert np.allclose(k, [complex(0.133183, 0.214862), complex(0.116903, 0.00838917), 0], atol=6e-7)
    assert rel_l2(k, ka["k_hs_rut1"]) < 1e-12
    npr = abi.NumParam(1e-6, 3.0, 3.0, 3.0, 160, 400, 4, 4)
    r = oracle.pair_op(abi.OP_R_SMOOTH, RUT1[None], X_EX[None], np.array([[1, 1, 1]], complex), 1.0, npr)[0]
    assert np.allclose(r, [complex(-0.139686, -0.0448552), complex(0.152198, 0.073226),
                           complex(-0.012512, -0.0283708)], atol=6e-7)
    assert rel_l2(r, ka["r_smooth_rut1"]) < 1e-12
    npc = abi.NumParam(1e-6, 2.2e-16, 2.2e-16, 3.0, 80, 100, 4, 4)
    z = oracle.pair_op(abi.OP_R_COLLOC, RUT1[None], np.array([[1.25, 1.0, 0.0]]), np.array([[1, 1, 1]], complex),
                       1.0, npc)[0]
    assert np.all(z == 0)  # R.h:95-97
