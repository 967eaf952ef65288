"""CPU ORACLE — test infrastructure only.

Loads the two CPU checkers built by oracle/Makefile and wraps them with numpy:
  * ``port``: oracle/liboracle.so, the C++ restatement (bielcc_oracle.cpp);
  * ``ref``:  oracle/_ref/libbielcc_ref.so, the reference (AlenaSetukha/BIELcc)
    compiled from its own sources plus ref_glue.cpp (only where it was built).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs may import this module, and only as the checker or the timed CPU
baseline. The product package (bielcc_b200) never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from bielcc_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbielcc_ref.so")

_libs = {}


def build(ref=True):
    """Builds liboracle.so, and where the reference sources are present the
    reference library and the drop-in checker (which links the GPU library)."""
    targets = ["oracle"]
    if ref and os.path.isdir(os.environ.get("BIELCC_REF_SRC", "/root/reference")):
        targets.append("ref")
        if os.path.exists(os.path.join(HERE, "..", "bielcc_b200", "libbielcc_gpu.so")):
            targets.append("dropin")
    env = dict(os.environ)
    if "BIELCC_REF_SRC" in env:
        targets.append("REF=" + env["BIELCC_REF_SRC"])
    subprocess.run(["make", "-s", "-C", HERE, "-j8"] + targets, check=True, env=env)


def available(which):
    return os.path.exists(PORT_SO if which == "port" else REF_SO)


def lib(which="port"):
    if which in _libs:
        return _libs[which]
    path = PORT_SO if which == "port" else REF_SO
    if not os.path.exists(path):
        if which == "port":
            build(ref=False)
        else:
            raise FileNotFoundError(path + " (reference build needs its sources; see oracle/Makefile)")
    L = C.CDLL(path)
    prefix = "oracle_" if which == "port" else "ref_"
    abi.declare_common(L, prefix)
    dp = C.POINTER(C.c_double)
    f = getattr(L, prefix + "field_EH")
    f.argtypes = [C.c_int, C.c_int, dp, C.c_int, dp, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.POINTER(abi.PlaneWave), C.POINTER(abi.NumParam), C.c_int, dp, dp, dp, C.c_int]
    f.restype = C.c_int
    f = getattr(L, prefix + "area_by_quadrature")
    f.argtypes = [C.c_int, dp, C.c_int, C.c_int, C.c_double, dp]
    f.restype = C.c_int
    f = getattr(L, prefix + "cell_geometry")
    f.argtypes = [C.c_int, C.c_int, dp, dp]
    f.restype = C.c_int
    if which == "ref":
        f = L.ref_read_mesh
        f.argtypes = [C.c_int, C.c_int, C.c_char_p, C.POINTER(C.c_int), dp]
        f.restype = C.c_int
        f = L.ref_read_currents
        f.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), dp]
        f.restype = C.c_int
        f = L.ref_material
        f.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, dp, C.c_double, dp]
        f.restype = C.c_int
    if which == "port":
        f = L.oracle_assemble_K
        f.argtypes = [C.c_int, C.c_int, dp, C.c_double, C.c_double, C.POINTER(abi.NumParam), C.c_int,
                      C.c_int, C.c_int, dp]
        f.restype = C.c_int
    _libs[which] = (L, prefix)
    return _libs[which]


def _f(which, name):
    L, prefix = lib(which)
    return getattr(L, prefix + name)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def field_EH(cells, J, k, pts, numparam=None, mult=1.0, inc=None, with_H=True, n_threads=0, which="port"):
    """E, H of GetFieldE_Ideal + the R loop; J [S][N][3] complex, pts [M][3]."""
    cells = _c(cells)
    J = _c(J, np.complex128)
    if J.ndim == 2:
        J = J[None]
    pts = _c(pts)
    S, N = J.shape[0], cells.shape[0]
    M = pts.shape[0]
    E = np.zeros((S, M, 3), np.complex128)
    H = np.zeros((S, M, 3), np.complex128) if with_H else None
    np_ = numparam if numparam is not None else abi.NumParam.default()
    k = complex(k)
    mult = complex(mult)
    rc = _f(which, "field_EH")(cells.shape[1], N, abi.dptr(cells), S, abi.dptr(J), k.real, k.imag, mult.real,
                               mult.imag, C.byref(inc) if inc is not None else None, C.byref(np_), M,
                               abi.dptr(pts), abi.dptr(E), abi.dptr(H), int(n_threads))
    if rc != 0:
        raise RuntimeError(f"{which} field_EH failed: {rc}")
    return E, H


def pair_op(op, cells, x, j, k, numparam=None, which="port"):
    cells = _c(cells)
    x = _c(x)
    j = _c(j, np.complex128)
    n = cells.shape[0]
    res = np.zeros((n, 3), np.complex128)
    np_ = numparam if numparam is not None else abi.NumParam.default()
    k = complex(k)
    rc = _f(which, "pair_op")(op, cells.shape[1], n, abi.dptr(cells), abi.dptr(x), abi.dptr(j), k.real, k.imag,
                              C.byref(np_), abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"{which} pair_op failed: {rc}")
    return res


def integral_pnt(integrand, cells, x, kp, n_start, p_max, eps, which="port"):
    cells = _c(cells)
    x = _c(x)
    n = cells.shape[0]
    _, idim, cplx = abi.INTEGRANDS[integrand]
    res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
    rc = _f(which, "integral_pnt")(integrand, cells.shape[1], n, abi.dptr(cells), abi.dptr(x), kp, n_start, p_max,
                                   eps, abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"{which} integral_pnt failed: {rc}")
    return res


def integral_seg_pnt(integrand, a, b, x, kp, n_start, p_max, eps, which="port"):
    a, b, x = _c(a), _c(b), _c(x)
    n = a.shape[0]
    _, idim, cplx = abi.INTEGRANDS[integrand]
    res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
    rc = _f(which, "integral_seg_pnt")(integrand, n, abi.dptr(a), abi.dptr(b), abi.dptr(x), kp, n_start, p_max,
                                       eps, abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"{which} integral_seg_pnt failed: {rc}")
    return res


def integral(integrand, cells, kp, n_start, p_max, eps, which="port"):
    """IntegralUniversal, the F(x) form (integral_universal.h:252-431)."""
    cells = _c(cells)
    n = cells.shape[0]
    _, idim, cplx = abi.INTEGRANDS[integrand]
    res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
    rc = _f(which, "integral")(integrand, cells.shape[1], n, abi.dptr(cells), kp, n_start, p_max, eps, abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"{which} integral failed: {rc}")
    return res


def integral_seg(integrand, a, b, kp, n_start, p_max, eps, which="port"):
    """IntegralUniversalSegPnt, the F(x) overload (integral_universal_seg.h:120-179)."""
    a, b = _c(a), _c(b)
    n = a.shape[0]
    _, idim, cplx = abi.INTEGRANDS[integrand]
    res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
    rc = _f(which, "integral_seg")(integrand, n, abi.dptr(a), abi.dptr(b), kp, n_start, p_max, eps, abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"{which} integral_seg failed: {rc}")
    return res


def k0(integrand, common, cells, x, j, kp, n_seg, p_seg, eps, which="port"):
    cells, x = _c(cells), _c(x)
    j = _c(j, np.complex128)
    n = cells.shape[0]
    res = np.zeros((n, 3), np.complex128)
    rc = _f(which, "k0")(integrand, int(common), cells.shape[1], n, abi.dptr(cells), abi.dptr(x), abi.dptr(j), kp,
                         n_seg, p_seg, eps, abi.dptr(res))
    if rc != 0:
        raise RuntimeError(f"{which} k0 failed: {rc}")
    return res


def integral_1divr(cells, x, which="port"):
    cells, x = _c(cells), _c(x)
    res = np.zeros(cells.shape[0])
    _f(which, "integral_1divr")(cells.shape[1], cells.shape[0], abi.dptr(cells), abi.dptr(x), abi.dptr(res))
    return res


def integral_grad1divr_seg(a, b, x, which="port"):
    a, b, x = _c(a), _c(b), _c(x)
    res = np.zeros((a.shape[0], 3))
    _f(which, "integral_grad1divr_seg")(a.shape[0], abi.dptr(a), abi.dptr(b), abi.dptr(x), abi.dptr(res))
    return res


def integral_surf_simplepot_h_hs(cells, x, analytic_r, n_start, p_max, eps, k, which="port"):
    cells, x = _c(cells), _c(x)
    res = np.zeros(cells.shape[0], np.complex128)
    k = complex(k)
    _f(which, "integral_surf_simplepot_h_hs")(cells.shape[1], cells.shape[0], abi.dptr(cells), abi.dptr(x),
                                              analytic_r, n_start, p_max, eps, k.real, k.imag, abi.dptr(res))
    return res


def integral_seg_gradsimplepot_h_hs(a, b, x, analytic_r, n_start, p_max, eps, k, which="port"):
    a, b, x = _c(a), _c(b), _c(x)
    res = np.zeros((a.shape[0], 3), np.complex128)
    k = complex(k)
    _f(which, "integral_seg_gradsimplepot_h_hs")(a.shape[0], abi.dptr(a), abi.dptr(b), abi.dptr(x), analytic_r,
                                                 n_start, p_max, eps, k.real, k.imag, abi.dptr(res))
    return res


def area_by_quadrature(cell, n_start=8, p_max=1, eps=1e-6, which="port"):
    cell = _c(cell)
    res = np.zeros(1)
    _f(which, "area_by_quadrature")(cell.shape[0], abi.dptr(cell), n_start, p_max, eps, abi.dptr(res))
    return float(res[0])


def cell_geometry(cells, which="port"):
    """[N][14]: centre(3), diam, normal(3), tau1(3), tau2(3), area."""
    cells = _c(cells)
    out = np.zeros((cells.shape[0], 14))
    _f(which, "cell_geometry")(cells.shape[1], cells.shape[0], abi.dptr(cells), abi.dptr(out))
    return out


def assemble_K(cells, k, numparam=None, layout=abi.LAYOUT_TAU2, rows=None):
    """Rows [r0, r1) of the collocation matrix (complex128), port only."""
    cells = _c(cells)
    N = cells.shape[0]
    m = 2 if layout == abi.LAYOUT_TAU2 else 3
    r0, r1 = rows if rows is not None else (0, N)
    A = np.zeros(((r1 - r0) * m, N * m), np.complex128)
    np_ = numparam if numparam is not None else abi.NumParam.default()
    k = complex(k)
    rc = _f("port", "assemble_K")(cells.shape[1], N, abi.dptr(cells), k.real, k.imag, C.byref(np_), layout, r0, r1,
                                  abi.dptr(A))
    if rc != 0:
        raise RuntimeError(f"oracle assemble_K failed: {rc}")
    return A


def ref_material(freq, eps_r=1.0, mu_r=1.0, sigma=0.0, table=None):
    """The reference's MaterialParam::Calc and RadiationSource::CalcK at freq:
    dict of eps, mu (complex), skin_depth, k (CalcK) and calck_threw."""
    L, _ = lib("ref")
    out = np.zeros(7)
    t = None if table is None else _c(table).reshape(-1, 3)
    disp = abi.DISPERSION_NONE if t is None else abi.DISPERSION_REFRACT
    L.ref_material(disp, float(eps_r), float(mu_r), float(sigma), 0 if t is None else len(t),
                   None if t is None else abi.dptr(t), float(freq), abi.dptr(out))
    return {"eps": complex(out[0], out[1]), "mu": complex(out[2], out[3]), "skin_depth": out[4], "k": out[5],
            "calck_threw": bool(out[6])}


def ref_read_mesh(path, n_vert, fmt):
    """Cells [N][n_vert][3] as the reference's SurfMesh reader fills them
    (fmt "dat" or "vtk"); raises on a reader error."""
    L, _ = lib("ref")
    n = C.c_int(0)
    f = 0 if fmt == "dat" else 1
    rc = L.ref_read_mesh(f, n_vert, os.fsencode(path), C.byref(n), None)
    if rc != 0:
        raise RuntimeError(f"reference reader failed on {path}: {rc}")
    cells = np.zeros((n.value, n_vert, 3))
    rc = L.ref_read_mesh(f, n_vert, os.fsencode(path), C.byref(n), abi.dptr(cells))
    if rc != 0:
        raise RuntimeError(f"reference reader failed on {path}: {rc}")
    return cells


def ref_read_currents(path_re, path_im):
    """J [N][3] complex as SurfaceCurrentsC_fromFiles reads it."""
    L, _ = lib("ref")
    n = C.c_int(0)
    rc = L.ref_read_currents(os.fsencode(path_re), os.fsencode(path_im), C.byref(n), None)
    if rc != 0:
        raise RuntimeError(f"reference current reader failed: {rc}")
    J = np.zeros((n.value, 3), np.complex128)
    rc = L.ref_read_currents(os.fsencode(path_re), os.fsencode(path_im), C.byref(n), abi.dptr(J))
    if rc != 0:
        raise RuntimeError(f"reference current reader failed: {rc}")
    return J
