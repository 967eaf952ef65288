"""Python binding of libbielcc_gpu.so (include/bielcc_gpu.h) via ctypes.

There is no CPU fallback: if the library is missing or no CUDA device is
visible, constructing a Context raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbielcc_gpu.so")

_lib = None


class BielccError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"bielcc error {code}: {msg}")
        self.code = code


def load(path=LIB_PATH):
    """Loads the CUDA library (building it first when absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        from . import build as _b

        _b.build()
    L = C.CDLL(path)
    dp, vp, ip = C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int32)

    def d(name, args, res=C.c_int):
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res

    d("bielcc_abi_version", [])
    d("bielcc_last_error", [], C.c_char_p)
    d("bielcc_numparam_default", [C.POINTER(abi.NumParam)], None)
    d("bielcc_ctx_create", [C.c_int, C.POINTER(vp)])
    d("bielcc_ctx_destroy", [vp])
    d("bielcc_ctx_synchronize", [vp])
    d("bielcc_ctx_mem_used", [vp, C.POINTER(C.c_int64)])
    d("bielcc_mesh_create", [vp, C.c_int, C.c_int, dp, ip])
    d("bielcc_mesh_destroy", [vp, C.c_int32])
    d("bielcc_mesh_geometry", [vp, C.c_int32, dp])
    field_args = [vp, C.c_int32, C.c_int, dp, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.POINTER(abi.PlaneWave), C.POINTER(abi.NumParam), C.c_int, dp, dp, dp, C.c_int]
    d("bielcc_field_EH", field_args + [C.POINTER(abi.Report)])
    d("bielcc_field_EH_device", [vp, C.c_int32, C.c_int, vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(abi.PlaneWave), C.POINTER(abi.NumParam), C.c_int, vp, vp, vp, C.c_int, vp,
                                 C.POINTER(abi.Report)])
    d("bielcc_integrand_info", [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)])
    d("bielcc_solve_dense", [C.c_int, C.c_int, C.c_int, vp, vp, vp, C.POINTER(C.c_int)])
    d("bielcc_solve_pec", [vp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(abi.PlaneWave),
                           C.POINTER(abi.NumParam), C.c_int, dp, C.POINTER(abi.Report)])
    d("bielcc_read_mesh_dat", [C.c_char_p, C.c_int, C.POINTER(C.c_int), dp])
    d("bielcc_read_mesh_vtk", [C.c_char_p, C.c_int, C.POINTER(C.c_int), dp, C.POINTER(C.c_int)])
    d("bielcc_read_currents", [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), dp])
    full_args = [vp, C.c_int32, C.c_int, vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                 C.c_double, C.POINTER(abi.PlaneWave), C.POINTER(abi.NumParam), C.c_int, vp, vp, vp, C.c_int]
    d("bielcc_field_EH_full", full_args + [C.POINTER(abi.Report)])
    d("bielcc_field_EH_full_device", full_args + [vp, C.POINTER(abi.Report)])
    d("bielcc_assemble_K", [vp, C.c_int32, C.c_double, C.c_double, C.POINTER(abi.NumParam), C.c_int, C.c_int, C.c_int,
                            vp, C.POINTER(abi.Report)])
    d("bielcc_assemble_K_device", [vp, C.c_int32, C.c_double, C.c_double, C.POINTER(abi.NumParam), C.c_int, C.c_int,
                                   C.c_int, vp, vp, C.POINTER(abi.Report)])
    d("bielcc_field_EH_batch", [vp, C.c_int, C.POINTER(abi.FieldJob), C.POINTER(abi.NumParam), C.c_int, vp,
                                C.POINTER(abi.Report)])
    d("bielcc_batch_autotune", [vp, C.c_int, C.POINTER(abi.FieldJob), C.POINTER(abi.NumParam), C.c_int, vp,
                                C.POINTER(C.c_double)])
    d("bielcc_batch_plan_create", [vp, C.c_int, C.POINTER(abi.FieldJob), C.POINTER(abi.NumParam), C.c_int, vp,
                                   C.POINTER(vp), C.POINTER(abi.Report)])
    d("bielcc_batch_plan_launch", [vp, vp])
    d("bielcc_batch_plan_destroy", [vp])
    d("bielcc_ctx_set_timing", [vp, C.c_int])
    d("bielcc_ctx_set_batch_tensor_cores", [vp, C.c_int])
    d("bielcc_ctx_set_batch_split", [vp, C.c_int64, C.c_int])
    d("bielcc_medium_at", [C.POINTER(abi.Material), C.c_double, C.POINTER(abi.Medium)])
    d("bielcc_planewave_in_medium", [C.POINTER(abi.Medium), C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(abi.PlaneWave)])
    d("bielcc_measure_fma_peak", [C.c_int, C.POINTER(C.c_double)])
    d("bielcc_ctx_stats", [vp, C.POINTER(abi.Stats), C.c_int])
    d("bielcc_server_create", [vp, C.c_int64, C.c_int, C.POINTER(abi.NumParam), C.c_int, C.POINTER(vp)])
    d("bielcc_server_destroy", [vp])
    d("bielcc_server_set_item_cost", [vp, C.c_double])
    d("bielcc_server_set_max_batch", [vp, C.c_int])
    d("bielcc_server_set_preemptible", [vp, C.c_int])
    d("bielcc_server_reserve", [vp, C.c_int64, C.c_int64])
    d("bielcc_server_submit_field", [vp, C.POINTER(abi.FieldRequest), C.POINTER(C.c_int64)])
    d("bielcc_server_submit_assemble", [vp, C.POINTER(abi.AssembleRequest), C.POINTER(C.c_int64)])
    d("bielcc_server_poll", [vp, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)])
    d("bielcc_server_wait", [vp, C.c_int64, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)])
    d("bielcc_server_cancel", [vp, C.c_int64])
    d("bielcc_server_pause", [vp, C.c_int])
    d("bielcc_server_drain", [vp, C.c_double])
    d("bielcc_server_set_max_batch_pairs", [vp, C.c_int64])
    d("bielcc_server_trace", [vp, C.POINTER(abi.BatchTrace), C.c_int, C.POINTER(C.c_int)])
    d("bielcc_server_set_overtake", [vp, C.c_int])
    d("bielcc_server_set_priority_pairs", [vp, C.c_int64])
    d("bielcc_server_get_stats", [vp, C.POINTER(abi.ServerStats), C.c_int])
    abi.declare_common(L, "bielcc_")
    if L.bielcc_abi_version() != abi.ABI_VERSION:
        raise RuntimeError(f"{path}: ABI {L.bielcc_abi_version()} != {abi.ABI_VERSION}")
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise BielccError(rc, _lib.bielcc_last_error().decode(errors="replace"))
    return rc


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


PREC = {"fp64": abi.PREC_FP64, "mixed": abi.PREC_MIXED}

# cudaStreamLegacy: the legacy default stream as an explicit handle
_CUDA_STREAM_LEGACY = 0x1


def _stream_arg(stream):
    """cudaStream_t argument of the C ABI. None selects the context's own
    stream; a raw handle (e.g. torch.cuda.Stream.cuda_stream) is passed as is,
    except 0 — torch's handle of the legacy default stream — which is passed as
    cudaStreamLegacy, so the work is ordered with everything on that stream
    instead of going to the context's (non-blocking) stream."""
    if stream is None:
        return None
    return C.c_void_p(int(stream) if int(stream) != 0 else _CUDA_STREAM_LEGACY)


def read_mesh_dat(path, n_vert):
    """Cells [N][n_vert][3] of a geodat .dat mesh file (host reader, no GPU)."""
    load()
    n = C.c_int(0)
    _check(_lib.bielcc_read_mesh_dat(os.fsencode(path), n_vert, C.byref(n), None))
    cells = np.zeros((n.value, n_vert, 3))
    _check(_lib.bielcc_read_mesh_dat(os.fsencode(path), n_vert, C.byref(n), abi.dptr(cells)))
    return cells


def read_mesh_vtk(path, n_vert):
    """(cells [N][n_vert][3], polygons skipped) of a legacy ASCII VTK file."""
    load()
    n, sk = C.c_int(0), C.c_int(0)
    _check(_lib.bielcc_read_mesh_vtk(os.fsencode(path), n_vert, C.byref(n), None, C.byref(sk)))
    cells = np.zeros((n.value, n_vert, 3))
    _check(_lib.bielcc_read_mesh_vtk(os.fsencode(path), n_vert, C.byref(n), abi.dptr(cells), C.byref(sk)))
    return cells, sk.value


def read_currents(path_re, path_im):
    """J [N][3] complex128 from the real / imaginary current files."""
    load()
    n = C.c_int(0)
    _check(_lib.bielcc_read_currents(os.fsencode(path_re), os.fsencode(path_im), C.byref(n), None))
    J = np.zeros((n.value, 3), np.complex128)
    _check(_lib.bielcc_read_currents(os.fsencode(path_re), os.fsencode(path_im), C.byref(n), abi.dptr(J)))
    return J


def material(eps_r=1.0, mu_r=1.0, sigma=0.0, table=None):
    """bielcc_material: NonDispersive (eps_r, mu_r, sigma), or, with `table`
    rows (frequency, n, absorption index), DispersiveByRefractIndex. The
    returned record keeps its table alive."""
    m = abi.Material()
    m.eps_r, m.mu_r, m.sigma = float(eps_r), float(mu_r), float(sigma)
    if table is not None:
        t = _c(table).reshape(-1, 3)
        m.dispersion, m.n_table = abi.DISPERSION_REFRACT, len(t)
        m.table = abi.dptr(t)
        m._table = t
    else:
        m.dispersion, m.n_table = abi.DISPERSION_NONE, 0
    return m


def medium_at(mat, freq):
    """bielcc_medium of a material at a frequency (host only, no GPU)."""
    load()
    md = abi.Medium()
    _check(_lib.bielcc_medium_at(C.byref(mat), float(freq), C.byref(md)))
    return md


def planewave_in_medium(md, freq, direction=(0.0, 0.0, 1.0), e0=(1.0, 0.0, 0.0), add_E=True, add_H=True):
    """The incident plane wave of RadiationSource in that medium."""
    load()
    pw = abi.PlaneWave()
    d = (C.c_double * 3)(*direction)
    e = (C.c_double * 3)(*e0)
    _check(_lib.bielcc_planewave_in_medium(C.byref(md), float(freq), d, e, int(add_E), int(add_H), C.byref(pw)))
    return pw


class Mesh:
    def __init__(self, ctx, cells):
        self.ctx = ctx
        self.cells = _c(cells)
        if self.cells.ndim != 3 or self.cells.shape[1] not in (3, 4) or self.cells.shape[2] != 3:
            raise ValueError("cells must be [N][3|4][3]")
        h = C.c_int32(0)
        _check(_lib.bielcc_mesh_create(ctx.h, self.cells.shape[1], self.cells.shape[0], abi.dptr(self.cells),
                                       C.byref(h)))
        self.id = h.value
        self.n_cells = self.cells.shape[0]
        self.n_vert = self.cells.shape[1]

    def geometry(self):
        """[N][14]: centre(3), diam, normal(3), tau1(3), tau2(3), area computed on the device."""
        out = np.zeros((self.n_cells, 14))
        _check(_lib.bielcc_mesh_geometry(self.ctx.h, self.id, abi.dptr(out)))
        return out

    def close(self):
        if self.id:
            _check(_lib.bielcc_mesh_destroy(self.ctx.h, self.id))
            self.id = 0


class Context:
    """One CUDA device, its stream and the resident meshes (bielcc_ctx)."""

    def __init__(self, device=0):
        load()
        h = C.c_void_p()
        _check(_lib.bielcc_ctx_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            _lib.bielcc_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        _check(_lib.bielcc_ctx_synchronize(self.h))

    def mem_used(self):
        b = C.c_int64(0)
        _check(_lib.bielcc_ctx_mem_used(self.h, C.byref(b)))
        return b.value

    def set_timing(self, on=True):
        _check(_lib.bielcc_ctx_set_timing(self.h, int(bool(on))))

    def set_batch_tensor_cores(self, on=True):
        """Mixed batches contract moments and currents on the tensor cores or on the CUDA cores (default)."""
        _check(_lib.bielcc_ctx_set_batch_tensor_cores(self.h, int(bool(on))))

    def set_batch_split(self, moments_bytes, all_batches=False):
        """Moments-buffer cap (bytes) of the split batched pipeline: batch plans
        whose moments fit one wave keep them and replay only the contraction;
        all_batches splits every mixed batch; 0 always runs the fused kernel."""
        _check(_lib.bielcc_ctx_set_batch_split(self.h, int(moments_bytes), int(bool(all_batches))))

    def stats(self, reset=False):
        st = abi.Stats()
        _check(_lib.bielcc_ctx_stats(self.h, C.byref(st), int(bool(reset))))
        return {f: getattr(st, f) for f, _ in abi.Stats._fields_}

    def mesh(self, cells):
        return Mesh(self, cells)

    def measure_fma_peak(self, fp64=False, packed=False):
        """CUDA-core FMA peak of this device in TFLOP/s: FP32, FP64, or packed
        FP32 pairs (fma.rn.f32x2) with packed=True."""
        t = C.c_double(0)
        _check(_lib.bielcc_measure_fma_peak(2 if packed else int(bool(fp64)), C.byref(t)))
        return t.value

    # ------------------------------------------------------------------ field
    def field_EH(self, mesh, J, k, pts, numparam=None, mult=1.0, inc=None, with_H=True, precision="fp64",
                 check=True, out=None):
        """E, H [S][M][3] complex128 and the report; J [S][N][3] or [N][3].
        `out` = (E, H) preallocated C-contiguous complex128 arrays (e.g. pinned)."""
        J = _c(J, np.complex128)
        if J.ndim == 2:
            J = J[None]
        pts = _c(pts)
        S, M = J.shape[0], pts.shape[0]
        if J.shape[1] != mesh.n_cells:
            raise ValueError("J has %d cells, mesh %d" % (J.shape[1], mesh.n_cells))
        if out is not None:
            E, H = out
            assert E.shape == (S, M, 3) and E.dtype == np.complex128 and E.flags.c_contiguous
            assert H is None or (H.shape == (S, M, 3) and H.dtype == np.complex128 and H.flags.c_contiguous)
        else:
            E = np.zeros((S, M, 3), np.complex128)
            H = np.zeros((S, M, 3), np.complex128) if with_H else None
        rep = abi.Report()
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k = complex(k)
        mult = complex(mult)
        rc = _lib.bielcc_field_EH(self.h, mesh.id, S, abi.dptr(J), k.real, k.imag, mult.real, mult.imag,
                                  C.byref(inc) if inc is not None else None, C.byref(np_), M, abi.dptr(pts),
                                  abi.dptr(E), abi.dptr(H), PREC[precision], C.byref(rep))
        if rc != 0 and (check or rc != abi.ERR_NAN):
            _check(rc)
        return E, H, rep

    def field_EH_device(self, mesh, J_dev, k, pts_dev, E_dev, H_dev, n_rhs, n_pts, numparam=None, mult=1.0,
                        inc=None, precision="fp64", stream=None, report=True):
        """Device-buffer form: pointers are ints (e.g. torch tensor data_ptr()).
        report=False passes no report: no error sample, and the call returns
        once enqueued (None is returned)."""
        rep = abi.Report() if report else None
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k = complex(k)
        mult = complex(mult)
        _check(_lib.bielcc_field_EH_device(self.h, mesh.id, n_rhs, C.c_void_p(J_dev), k.real, k.imag, mult.real,
                                           mult.imag, C.byref(inc) if inc is not None else None, C.byref(np_),
                                           n_pts, C.c_void_p(pts_dev), C.c_void_p(E_dev),
                                           C.c_void_p(H_dev) if H_dev else None, PREC[precision],
                                           _stream_arg(stream), C.byref(rep) if rep is not None else None))
        return rep

    def field_EH_full(self, mesh, J_E, J_M, k, pts, multE=1.0, multH=1.0, inc=None, numparam=None,
                      precision="fp64"):
        """Full Stratton-Chu E, H [S][M][3] of electric and magnetic currents
        (bielcc_field_EH_full) and the report."""
        JE = _c(J_E, np.complex128)
        JM = _c(J_M, np.complex128)
        if JE.ndim == 2:
            JE, JM = JE[None], JM[None]
        if JE.shape != JM.shape or JE.shape[1] != mesh.n_cells:
            raise ValueError("J_E and J_M must both be [S][n_cells][3]")
        pts = _c(pts)
        S, P = JE.shape[0], pts.shape[0]
        E = np.zeros((S, P, 3), np.complex128)
        H = np.zeros_like(E)
        rep = abi.Report()
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k, multE, multH = complex(k), complex(multE), complex(multH)
        _check(_lib.bielcc_field_EH_full(self.h, mesh.id, S, JE.ctypes.data, JM.ctypes.data, k.real, k.imag,
                                         multE.real, multE.imag, multH.real, multH.imag,
                                         C.byref(inc) if inc is not None else None, C.byref(np_), P,
                                         pts.ctypes.data, E.ctypes.data, H.ctypes.data, PREC[precision],
                                         C.byref(rep)))
        return E, H, rep

    def field_EH_full_device(self, mesh, JE_dev, JM_dev, k, pts_dev, E_dev, H_dev, n_rhs, n_pts, multE=1.0,
                             multH=1.0, inc=None, numparam=None, precision="mixed", stream=None):
        rep = abi.Report()
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k, multE, multH = complex(k), complex(multE), complex(multH)
        _check(_lib.bielcc_field_EH_full_device(self.h, mesh.id, n_rhs, C.c_void_p(JE_dev), C.c_void_p(JM_dev),
                                                k.real, k.imag, multE.real, multE.imag, multH.real, multH.imag,
                                                C.byref(inc) if inc is not None else None, C.byref(np_), n_pts,
                                                C.c_void_p(pts_dev), C.c_void_p(E_dev), C.c_void_p(H_dev),
                                                PREC[precision], _stream_arg(stream), C.byref(rep)))
        return rep

    # ------------------------------------------------------------------ solving the collocation system
    def solve_pec(self, mesh, k, inc, multE, numparam=None, precision="fp64"):
        """Currents J [N][3] of a perfect conductor under the plane wave `inc`
        (bielcc_solve_pec): TAU2 assembly, LU solve, basis -> currents."""
        J = np.zeros((mesh.n_cells, 3), np.complex128)
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k, multE = complex(k), complex(multE)
        rep = abi.Report()
        _check(_lib.bielcc_solve_pec(self.h, mesh.id, k.real, k.imag, multE.real, multE.imag, C.byref(inc),
                                     C.byref(np_), PREC[precision], abi.dptr(J), C.byref(rep)))
        return J

    @staticmethod
    def solve_dense(n, nrhs, c64, A_dev, B_dev, stream=None):
        """A X = B on device buffers (row-major A, B = [nrhs][n]); returns cuSOLVER's info."""
        info = C.c_int(0)
        _check(_lib.bielcc_solve_dense(n, nrhs, int(bool(c64)), C.c_void_p(A_dev), C.c_void_p(B_dev),
                                       _stream_arg(stream), C.byref(info)))
        return info.value

    # ------------------------------------------------------------------ batched field
    @staticmethod
    def make_jobs(specs):
        """specs: dicts with mesh, n_rhs, n_pts, J, pts, E, H (device pointers as ints),
        k, mult (optional), inc (optional PlaneWave), est (optional device address of
        one double that receives the job's estimated mixed-precision error)."""
        arr = (abi.FieldJob * len(specs))()
        for i, sp in enumerate(specs):
            k = complex(sp["k"])
            mult = complex(sp.get("mult", 1.0))
            j = arr[i]
            j.mesh = sp["mesh"].id
            j.n_rhs = sp["n_rhs"]
            j.n_pts = sp["n_pts"]
            j.J_dev = sp["J"]
            j.pts_dev = sp["pts"]
            j.E_dev = sp["E"]
            j.H_dev = sp.get("H") or None
            j.k_re, j.k_im = k.real, k.imag
            j.mult_re, j.mult_im = mult.real, mult.imag
            if sp.get("inc") is not None:
                j.inc = sp["inc"]
            j.est_dev = sp.get("est") or None
        return arr

    def field_EH_batch(self, jobs, numparam=None, precision="mixed", stream=None, report=True):
        """Runs a batch built by make_jobs on device buffers; returns the report
        (report=False passes none: no error sample, the call returns once enqueued)."""
        rep = abi.Report()
        np_ = numparam if numparam is not None else abi.NumParam.default()
        _check(_lib.bielcc_field_EH_batch(self.h, len(jobs), jobs, C.byref(np_), PREC[precision],
                                          _stream_arg(stream), C.byref(rep) if report else None))
        return rep

    def batch_autotune(self, jobs, numparam=None, precision="mixed", stream=None):
        c = C.c_double(0)
        np_ = numparam if numparam is not None else abi.NumParam.default()
        _check(_lib.bielcc_batch_autotune(self.h, len(jobs), jobs, C.byref(np_), PREC[precision],
                                          _stream_arg(stream), C.byref(c)))
        return c.value

    def batch_plan(self, jobs, numparam=None, precision="mixed", stream=None):
        """Plans a batch for repeated evaluation (fixed geometry, new currents in
        place) and runs it once; returns a BatchPlan whose launch() replays the
        captured CUDA graph."""
        return BatchPlan(self, jobs, numparam, precision, stream)

    # ------------------------------------------------------------------ per-pair operators
    def pair_op(self, op, cells, x, j, k, numparam=None):
        cells, x = _c(cells), _c(x)
        j = _c(j, np.complex128)
        n = cells.shape[0]
        res = np.zeros((n, 3), np.complex128)
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k = complex(k)
        _check(_lib.bielcc_pair_op(self.h, op, cells.shape[1], n, abi.dptr(cells), abi.dptr(x), abi.dptr(j), k.real,
                                   k.imag, C.byref(np_), abi.dptr(res)))
        return res

    def integral_pnt(self, integrand, cells, x, kp, n_start, p_max, eps):
        cells, x = _c(cells), _c(x)
        n = cells.shape[0]
        _, idim, cplx = abi.INTEGRANDS[integrand]
        res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
        _check(_lib.bielcc_integral_pnt(self.h, integrand, cells.shape[1], n, abi.dptr(cells), abi.dptr(x), kp,
                                        n_start, p_max, eps, abi.dptr(res)))
        return res

    def integral_seg_pnt(self, integrand, a, b, x, kp, n_start, p_max, eps):
        a, b, x = _c(a), _c(b), _c(x)
        n = a.shape[0]
        _, idim, cplx = abi.INTEGRANDS[integrand]
        res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
        _check(_lib.bielcc_integral_seg_pnt(self.h, integrand, n, abi.dptr(a), abi.dptr(b), abi.dptr(x), kp, n_start,
                                            p_max, eps, abi.dptr(res)))
        return res

    def integral(self, integrand, cells, kp, n_start, p_max, eps):
        """IntegralUniversal, the F(x) form (F_ONE or F_PLANEWAVE_E), per cell."""
        cells = _c(cells)
        n = cells.shape[0]
        _, idim, cplx = abi.INTEGRANDS[integrand]
        res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
        _check(_lib.bielcc_integral(self.h, integrand, cells.shape[1], n, abi.dptr(cells), kp, n_start, p_max, eps,
                                    abi.dptr(res)))
        return res

    def integral_seg(self, integrand, a, b, kp, n_start, p_max, eps):
        """IntegralUniversalSegPnt, the F(x) overload, per segment [a, b]."""
        a, b = _c(a), _c(b)
        n = a.shape[0]
        _, idim, cplx = abi.INTEGRANDS[integrand]
        res = np.zeros((n, idim), np.complex128 if cplx else np.float64)
        _check(_lib.bielcc_integral_seg(self.h, integrand, n, abi.dptr(a), abi.dptr(b), kp, n_start, p_max, eps,
                                        abi.dptr(res)))
        return res

    def k0(self, integrand, common, cells, x, j, kp, n_seg, p_seg, eps):
        cells, x = _c(cells), _c(x)
        j = _c(j, np.complex128)
        n = cells.shape[0]
        res = np.zeros((n, 3), np.complex128)
        _check(_lib.bielcc_k0(self.h, integrand, int(common), cells.shape[1], n, abi.dptr(cells), abi.dptr(x),
                              abi.dptr(j), kp, n_seg, p_seg, eps, abi.dptr(res)))
        return res

    def integral_1divr(self, cells, x):
        cells, x = _c(cells), _c(x)
        res = np.zeros(cells.shape[0])
        _check(_lib.bielcc_integral_1divr(self.h, cells.shape[1], cells.shape[0], abi.dptr(cells), abi.dptr(x),
                                          abi.dptr(res)))
        return res

    def integral_grad1divr_seg(self, a, b, x):
        a, b, x = _c(a), _c(b), _c(x)
        res = np.zeros((a.shape[0], 3))
        _check(_lib.bielcc_integral_grad1divr_seg(self.h, a.shape[0], abi.dptr(a), abi.dptr(b), abi.dptr(x),
                                                  abi.dptr(res)))
        return res

    def integral_surf_simplepot_h_hs(self, cells, x, analytic_r, n_start, p_max, eps, k):
        cells, x = _c(cells), _c(x)
        res = np.zeros(cells.shape[0], np.complex128)
        k = complex(k)
        _check(_lib.bielcc_integral_surf_simplepot_h_hs(self.h, cells.shape[1], cells.shape[0], abi.dptr(cells),
                                                        abi.dptr(x), analytic_r, n_start, p_max, eps, k.real, k.imag,
                                                        abi.dptr(res)))
        return res

    def integral_seg_gradsimplepot_h_hs(self, a, b, x, analytic_r, n_start, p_max, eps, k):
        a, b, x = _c(a), _c(b), _c(x)
        res = np.zeros((a.shape[0], 3), np.complex128)
        k = complex(k)
        _check(_lib.bielcc_integral_seg_gradsimplepot_h_hs(self.h, a.shape[0], abi.dptr(a), abi.dptr(b), abi.dptr(x),
                                                           analytic_r, n_start, p_max, eps, k.real, k.imag,
                                                           abi.dptr(res)))
        return res

    # ------------------------------------------------------------------ assembly
    def assemble_K(self, mesh, k, numparam=None, layout=abi.LAYOUT_TAU2, c64=False, precision="fp64"):
        m = 2 if layout == abi.LAYOUT_TAU2 else 3
        dim = m * mesh.n_cells
        A = np.zeros((dim, dim), np.complex64 if c64 else np.complex128)
        rep = abi.Report()
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k = complex(k)
        _check(_lib.bielcc_assemble_K(self.h, mesh.id, k.real, k.imag, C.byref(np_), layout, int(c64),
                                      PREC[precision], A.ctypes.data_as(C.c_void_p), C.byref(rep)))
        return A, rep

    def assemble_K_device(self, mesh, k, A_dev, numparam=None, layout=abi.LAYOUT_TAU2, c64=True, precision="mixed",
                          stream=None):
        rep = abi.Report()
        np_ = numparam if numparam is not None else abi.NumParam.default()
        k = complex(k)
        _check(_lib.bielcc_assemble_K_device(self.h, mesh.id, k.real, k.imag, C.byref(np_), layout, int(c64),
                                             PREC[precision], C.c_void_p(A_dev), _stream_arg(stream),
                                             C.byref(rep)))
        return rep


class BatchPlan:
    """bielcc_batch_plan: a batch captured once in a CUDA graph."""

    def __init__(self, ctx, jobs, numparam=None, precision="mixed", stream=None):
        self.ctx, self.jobs = ctx, jobs
        np_ = numparam if numparam is not None else abi.NumParam.default()
        h = C.c_void_p()
        self.report = abi.Report()
        _check(_lib.bielcc_batch_plan_create(ctx.h, len(jobs), jobs, C.byref(np_), PREC[precision],
                                             _stream_arg(stream), C.byref(h),
                                             C.byref(self.report)))
        self.h = h

    def launch(self, stream=None):
        _check(_lib.bielcc_batch_plan_launch(self.h, _stream_arg(stream)))

    def close(self):
        if self.h:
            _check(_lib.bielcc_batch_plan_destroy(self.h))
            self.h = None


class Server:
    """Continuous-batching request loop over a Context's resident meshes
    (bielcc_server_*). Requests return a ticket at once; wait / poll hand back
    (status, latency_ms, outputs) once the request finished."""

    def __init__(self, ctx, hbm_budget=0, n_slots=2, numparam=None, precision="mixed", max_batch=None,
                 item_cost=None, preemptible=True, reserve=None, max_batch_pairs=None, overtake=True,
                 priority_pairs=None):
        self.ctx = ctx
        np_ = numparam if numparam is not None else abi.NumParam.default()
        h = C.c_void_p()
        _check(_lib.bielcc_server_create(ctx.h, int(hbm_budget), int(n_slots), C.byref(np_), PREC[precision],
                                         C.byref(h)))
        self.h = h
        self._live = {}
        if max_batch is not None:
            _check(_lib.bielcc_server_set_max_batch(self.h, int(max_batch)))
        if max_batch_pairs is not None:
            _check(_lib.bielcc_server_set_max_batch_pairs(self.h, int(max_batch_pairs)))
        if item_cost is not None:
            _check(_lib.bielcc_server_set_item_cost(self.h, float(item_cost)))
        _check(_lib.bielcc_server_set_preemptible(self.h, int(bool(preemptible))))
        _check(_lib.bielcc_server_set_overtake(self.h, int(bool(overtake))))
        if priority_pairs is not None:
            _check(_lib.bielcc_server_set_priority_pairs(self.h, int(priority_pairs)))
        if reserve is not None:
            _check(_lib.bielcc_server_reserve(self.h, int(reserve[0]), int(reserve[1])))

    def submit_field(self, mesh, J, pts, k, mult=1.0, inc=None, with_H=True, out_c64=True, J_dev=None, n_rhs=None,
                     out=None):
        """J: complex [S][N][3] host array, or J=None with J_dev (device pointer) and n_rhs.
        out: optional caller-owned (E, H) arrays ([S][P][3], complex64 or complex128 per out_c64)."""
        pts = _c(pts)
        if J is not None:
            J = _c(J, np.complex128).reshape(-1, mesh.n_cells, 3)
            n_rhs = J.shape[0]
        elif not J_dev or not n_rhs:
            raise ValueError("J or (J_dev, n_rhs) required")
        P = pts.shape[0]
        dt = np.complex64 if out_c64 else np.complex128
        if out is not None:
            E, H = out
            for a in (E, H):
                if a is not None and (a.dtype != dt or a.shape != (n_rhs, P, 3) or not a.flags.c_contiguous):
                    raise ValueError("out arrays must be C-contiguous [S][P][3] of the output dtype")
        else:
            E = np.zeros((n_rhs, P, 3), dt)
            H = np.zeros((n_rhs, P, 3), dt) if with_H else None
        r = abi.FieldRequest()
        r.mesh, r.n_rhs, r.n_pts, r.out_c64 = mesh.id, n_rhs, P, int(bool(out_c64))
        r.J = J.ctypes.data if J is not None else None
        r.J_dev = int(J_dev) if J is None else None
        r.pts = pts.ctypes.data
        r.E = E.ctypes.data
        r.H = H.ctypes.data if H is not None else None
        k, mult = complex(k), complex(mult)
        r.k_re, r.k_im, r.mult_re, r.mult_im = k.real, k.imag, mult.real, mult.imag
        if inc is not None:
            r.inc = inc
        est = C.c_double(0.0)  # the mixed form's estimated error, written on completion
        r.est = C.addressof(est)
        t = C.c_int64(0)
        _check(_lib.bielcc_server_submit_field(self.h, C.byref(r), C.byref(t)))
        self._live[t.value] = (r, J, pts, {"E": E, "H": H}, est)
        return t.value

    def submit_assemble(self, mesh, k, layout="tau2", out_c64=True, out=None, A_dev=None):
        """out: optional caller-owned host matrix; A_dev: a caller-owned device
        matrix (device pointer) written instead of a host one."""
        m = 2 if layout == "tau2" else 3
        dt = np.complex64 if out_c64 else np.complex128
        shape = (m * mesh.n_cells, m * mesh.n_cells)
        A = None
        if A_dev is None:
            if out is not None:
                if out.dtype != dt or out.shape != shape or not out.flags.c_contiguous:
                    raise ValueError("out must be a C-contiguous matrix of the output dtype")
                A = out
            else:
                A = np.zeros(shape, dt)
        r = abi.AssembleRequest()
        r.mesh = mesh.id
        r.layout = abi.LAYOUT_TAU2 if layout == "tau2" else abi.LAYOUT_FULL3
        r.out_c64 = int(bool(out_c64))
        r.A = A.ctypes.data if A is not None else None
        r.A_dev = int(A_dev) if A_dev is not None else None
        k = complex(k)
        r.k_re, r.k_im = k.real, k.imag
        t = C.c_int64(0)
        _check(_lib.bielcc_server_submit_assemble(self.h, C.byref(r), C.byref(t)))
        self._live[t.value] = (r, None, None, {"A": A})
        return t.value

    def poll(self, ticket):
        done, st, lat = C.c_int(0), C.c_int(0), C.c_double(0)
        _check(_lib.bielcc_server_poll(self.h, ticket, C.byref(done), C.byref(st), C.byref(lat)))
        if not done.value:
            return None
        return st.value, lat.value, self._live.pop(ticket)[3]

    def wait(self, ticket, timeout=120.0):
        st, lat = C.c_int(0), C.c_double(0)
        _check(_lib.bielcc_server_wait(self.h, ticket, float(timeout), C.byref(st), C.byref(lat)))
        live = self._live.pop(ticket)
        out = live[3]
        if len(live) > 4:
            out["est"] = live[4].value
        return st.value, lat.value, out

    def pause(self, paused=True):
        _check(_lib.bielcc_server_pause(self.h, int(bool(paused))))

    def cancel(self, ticket):
        _check(_lib.bielcc_server_cancel(self.h, ticket))

    def drain(self, timeout=600.0):
        _check(_lib.bielcc_server_drain(self.h, float(timeout)))

    def trace(self, capacity=4096):
        """The last batches served (bielcc_server_trace), oldest first, as dicts."""
        buf = (abi.BatchTrace * capacity)()
        n = C.c_int(0)
        _check(_lib.bielcc_server_trace(self.h, buf, capacity, C.byref(n)))
        return [buf[i].as_dict() for i in range(n.value)]

    def stats(self, reset=False):
        st = abi.ServerStats()
        _check(_lib.bielcc_server_get_stats(self.h, C.byref(st), int(bool(reset))))
        return st.as_dict()

    def close(self):
        if self.h:
            _check(_lib.bielcc_server_destroy(self.h))
            self.h = None
            self._live.clear()
