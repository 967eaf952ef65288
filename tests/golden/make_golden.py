"""Generates tests/golden/*.npz by running the REFERENCE implementation
(AlenaSetukha/BIELcc compiled from its own sources into
oracle/_ref/libbielcc_ref.so by oracle/Makefile) on small seeded cases.

Run in a container where the reference sources exist:
    make -C oracle ref && python tests/golden/make_golden.py [part ...]
with parts "main" (field, pair operators, pair integrands, analytic, known
answers) and "fx" (the one-point F(x) forms); no argument runs both.
The fixtures pin the oracle (tests/test_oracle_golden.py) and the GPU path
(tests/test_gpu_*.py) where the reference itself cannot travel.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from bielcc_b200 import abi  # noqa: E402
from bielcc_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF = "ref"

# cells of the reference's example programs (examples/integrators/main0_integrals.cpp:91-104)
RUT1 = np.array([[0., 0., 0.], [2., 0., 0.], [3., 2., 0.], [0., 2., 0.]])
RUT2 = np.array([[0., 2., 0.], [0., 0., 0.], [2., 0., 0.]])
RUT3 = np.array([[3., 2., 0.], [2., 0., 0.], [0., 2., 0.]])
X_EX = np.array([2., 1.5, 0.])


def random_pairs(cells, n, rng, spread):
    idx = rng.integers(0, len(cells), n)
    cc = cells[idx]
    x = W.centres(cc) + rng.normal(size=(n, 3)) * spread
    j = rng.normal(size=(n, 3)) + 1j * rng.normal(size=(n, 3))
    return cc, x, j


def main():
    rng = np.random.default_rng(20261203)
    quad = W.uv_sphere(16, 32)
    tri = W.perturbed_icosphere(level=1, seed=2)

    # ---- field driver: 512-quad sphere, far + near points, real k
    c1 = W.config1()
    pts = np.concatenate([c1["pts"][:48], W.near_points(quad, 16, 0.02, 0.1, rng)])
    kv, e0, hs = c1["inc"]
    inc = abi.PlaneWave.make(kv, e0, hs, True, True)
    E, H = oracle.field_EH(quad, c1["J"], c1["k"], pts, inc=inc, which=REF)
    np.savez_compressed(os.path.join(OUT, "field_quad512.npz"), cells=quad, J=c1["J"], k=c1["k"], pts=pts,
                        kvec=kv, e0=e0, h_scale=hs, E=E, H=H)

    # ---- field driver: 80-triangle perturbed icosphere, complex k, 2 RHS
    kt = complex(4 * np.pi, 0.5)
    Jt = W.po_currents(tri, 4 * np.pi, directions=2, seed=7)
    ptst = np.concatenate([W.sphere_points(24, 2.5, 11), W.near_points(tri, 8, 0.05, 0.2, rng)])
    np_t = abi.NumParam.default()
    Et, Ht = oracle.field_EH(tri, Jt, kt, ptst, numparam=np_t, mult=complex(0.3, -1.2), which=REF)
    np.savez_compressed(os.path.join(OUT, "field_tri80.npz"), cells=tri, J=Jt, k=kt, pts=ptst, mult=complex(0.3, -1.2),
                        E=Et, H=Ht)

    # ---- per-pair operators on quads and triangles, real and complex k, default and p_max = 3
    ops = {}
    for name, cells, spread in (("quad", quad, 0.15), ("tri", tri, 0.3)):
        for op in range(abi.OP_R_NEAR + 1):
            for kk, tag in ((2 * np.pi, "k"), (complex(2 * np.pi, 0.4), "kc")):
                for pm in (1, 3):
                    npm = abi.NumParam.default(p_max=pm, p_max_seg=pm)
                    cc, x, j = random_pairs(cells, 24, rng, spread)
                    r = oracle.pair_op(op, cc, x, j, kk, npm, which=REF)
                    key = f"{name}_op{op}_{tag}_p{pm}"
                    ops[key + "_cells"] = cc
                    ops[key + "_x"] = x
                    ops[key + "_j"] = j
                    ops[key + "_k"] = np.complex128(kk)
                    ops[key + "_res"] = r
    np.savez_compressed(os.path.join(OUT, "pair_ops.npz"), **ops)

    # ---- universal quadratures of every integrand
    ints = {}
    for name, cells in (("quad", quad), ("tri", tri)):
        for fid in abi.PAIR_INTEGRANDS:
            cc, x, j = random_pairs(cells, 16, rng, 0.2)
            dm = W.diameters(cc)
            kk = np.where(rng.random(16) < 0.5, 2 * np.pi, 2 * np.pi + 0.3j)
            sR = 2.0 * dm / 8.0
            nrm = rng.normal(size=(16, 3))
            for pm in (1, 2):
                # fresh records per call: the call leaves smoothR mutated, as the reference does
                kp = abi.kernelparam_array(16, smoothR=sR, smoothRMin=dm / 100, k=kk, current=j, vec_dbl=nrm,
                                           normal=nrm)
                r = oracle.integral_pnt(fid, cc, x, kp, 8, pm, 1e-6, which=REF)
                key = f"{name}_f{fid}_p{pm}"
                ints[key + "_cells"] = cc
                ints[key + "_x"] = x
                ints[key + "_sR"] = sR
                ints[key + "_sRm"] = dm / 100
                ints[key + "_k"] = kk
                ints[key + "_cur"] = j
                ints[key + "_vec"] = nrm
                ints[key + "_res"] = r
    for fid in abi.PAIR_INTEGRANDS:
        a = rng.normal(size=(16, 3))
        b = a + rng.normal(size=(16, 3)) * 0.3
        x = (a + b) / 2 + rng.normal(size=(16, 3)) * 0.2
        kk = np.where(rng.random(16) < 0.5, 2 * np.pi, 2 * np.pi + 0.3j)
        sR = np.full(16, 0.05)
        for pm in (1, 3):
            kp = abi.kernelparam_array(16, smoothR=sR, smoothRMin=1e-3, k=kk, current=a + 1j * b, vec_dbl=b - a,
                                       normal=b - a)
            r = oracle.integral_seg_pnt(fid, a, b, x, kp, 10, pm, 1e-6, which=REF)
            key = f"seg_f{fid}_p{pm}"
            ints.update({key + "_a": a, key + "_b": b, key + "_x": x, key + "_sR": sR, key + "_k": kk,
                         key + "_res": r})
    np.savez_compressed(os.path.join(OUT, "integrals.npz"), **ints)

    # ---- analytic integrals
    an = {}
    for name, cells in (("quad", quad), ("tri", tri)):
        x_on = W.centres(cells)
        x_off = x_on + rng.normal(size=x_on.shape) * 0.05
        for tag, x in (("centre", x_on), ("off", x_off)):
            an[f"{name}_{tag}_x"] = x
            an[f"{name}_{tag}_1divr"] = oracle.integral_1divr(cells, x, which=REF)
            an[f"{name}_{tag}_hs"] = oracle.integral_surf_simplepot_h_hs(cells, x, 3.0, 8, 1, 1e-6, 2 * np.pi,
                                                                         which=REF)
    a = rng.normal(size=(32, 3))
    b = a + rng.normal(size=(32, 3)) * 0.3
    x = (a + b) / 2 + rng.normal(size=(32, 3)) * 0.2
    an.update(seg_a=a, seg_b=b, seg_x=x, seg_grad1divr=oracle.integral_grad1divr_seg(a, b, x, which=REF),
              seg_hs=oracle.integral_seg_gradsimplepot_h_hs(a, b, x, 3.0, 10, 1, 1e-6, 2 * np.pi, which=REF))
    np.savez_compressed(os.path.join(OUT, "analytic.npz"), **an)

    # ---- known answers of the reference's example programs
    ka = {}
    ka["area_rut1"] = oracle.area_by_quadrature(RUT1, 8, 1, 1e-6, which=REF)
    # main0_integrals Test1 (n_start 64, p_max 8, k = 1)
    kp = abi.kernelparam_array(1, smoothR=2.0 * W.diameters(RUT1[None])[0] / 64, smoothRMin=1e-6, k=1.0)
    ka["t1_quad"] = oracle.integral_pnt(abi.F_SIMPLEPOT_H, RUT1[None], X_EX[None], kp, 64, 8, 1e-6, which=REF)[0, 0]
    ka["t1_hs"] = oracle.integral_surf_simplepot_h_hs(RUT1[None], X_EX[None], 3.0, 64, 8, 1e-6, 1.0, which=REF)[0]
    kp2 = abi.kernelparam_array(1, smoothR=np.finfo(float).eps, smoothRMin=np.finfo(float).eps, k=1.0)
    kp3 = abi.kernelparam_array(1, smoothR=2.0 * W.diameters(RUT3[None])[0] / 64, smoothRMin=1e-6, k=1.0)
    ka["t1_tri"] = (oracle.integral_pnt(abi.F_SIMPLEPOT_H, RUT2[None], X_EX[None], kp2, 64, 8, 1e-6, which=REF)[0, 0] +
                    oracle.integral_pnt(abi.F_SIMPLEPOT_H, RUT3[None], X_EX[None], kp3, 64, 8, 1e-6, which=REF)[0, 0])
    # main0_K Test2: K_RotRot_HS on rut1, num_param(1e-6, 2, 2, 3, 80, 100, 6, 6), k = 1, j = x-hat
    npk = abi.NumParam(1e-6, 2.0, 2.0, 3.0, 80, 100, 6, 6)
    ka["k_hs_rut1"] = oracle.pair_op(abi.OP_K_HS, RUT1[None], X_EX[None], np.array([[1, 0, 0]], complex), 1.0, npk,
                                     which=REF)[0]
    # main0_R Test1: R_Rot_Smooth on rut1, num_param(1e-6, 3, 3, 3, 160, 400, 4, 4), j = (1, 1, 1)
    npr = abi.NumParam(1e-6, 3.0, 3.0, 3.0, 160, 400, 4, 4)
    ka["r_smooth_rut1"] = oracle.pair_op(abi.OP_R_SMOOTH, RUT1[None], X_EX[None], np.array([[1, 1, 1]], complex), 1.0,
                                         npr, which=REF)[0]
    # main0_R Test2: R_Rot_Colloc at the centre of rut1 is exactly 0
    npc = abi.NumParam(1e-6, np.finfo(float).eps, np.finfo(float).eps, 3.0, 80, 100, 4, 4)
    ka["r_colloc_centre"] = oracle.pair_op(abi.OP_R_COLLOC, RUT1[None], np.array([[1.25, 1.0, 0.0]]),
                                           np.array([[1, 1, 1]], complex), 1.0, npc, which=REF)[0]
    np.savez_compressed(os.path.join(OUT, "known_answers.npz"), **ka)
    for k_, v in ka.items():
        print(k_, v)


def fx():
    """IntegralUniversal (integral_universal.h:252-431) and the segment F(x)
    overload (integral_universal_seg.h:120-179) with F = 1 and PlaneWaveFieldE
    (incident_field.h:20-29), at p_max 1 and 3, on quads (incl. degenerate
    pole quads), triangles and segments."""
    rng = np.random.default_rng(20261204)
    quad = W.uv_sphere(16, 32)
    tri = W.perturbed_icosphere(level=1, seed=2)
    out = {}
    for name, cells in (("quad", quad), ("tri", tri)):
        idx = np.concatenate([np.arange(4), rng.integers(0, len(cells), 20)])  # quads 0..3: a pole row
        cc = cells[idx]
        n = len(cc)
        kv = rng.normal(size=(n, 3)) * 6.0
        e0 = rng.normal(size=(n, 3))
        for fid in abi.FX_INTEGRANDS:
            for pm in (1, 3):
                kp = abi.kernelparam_array(n, smoothR=0.1, smoothRMin=0.01, k=2 * np.pi, vec_dbl=kv, e0=e0)
                r = oracle.integral(fid, cc, kp, 8, pm, 1e-6, which=REF)
                key = f"{name}_f{fid}_p{pm}"
                out.update({key + "_cells": cc, key + "_kv": kv, key + "_e0": e0, key + "_res": r,
                            key + "_sR": np.array([kp[i].smoothR for i in range(n)])})
    a = rng.normal(size=(16, 3))
    b = a + rng.normal(size=(16, 3)) * 0.5
    kv = rng.normal(size=(16, 3)) * 6.0
    e0 = rng.normal(size=(16, 3))
    for fid in abi.FX_INTEGRANDS:
        for pm in (1, 3):
            kp = abi.kernelparam_array(16, smoothR=0.1, smoothRMin=0.01, k=2 * np.pi, vec_dbl=kv, e0=e0)
            r = oracle.integral_seg(fid, a, b, kp, 10, pm, 1e-6, which=REF)
            key = f"seg_f{fid}_p{pm}"
            out.update({key + "_a": a, key + "_b": b, key + "_kv": kv, key + "_e0": e0, key + "_res": r,
                        key + "_sR": np.array([kp[i].smoothR for i in range(16)])})
    np.savez_compressed(os.path.join(OUT, "integrals_fx.npz"), **out)


if __name__ == "__main__":
    parts = sys.argv[1:] or ["main", "fx"]
    if "main" in parts:
        main()
    if "fx" in parts:
        fx()
