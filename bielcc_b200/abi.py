"""ctypes mirror of include/bielcc_gpu.h (structs, constants, prototypes).

The same definitions serve the GPU library (libbielcc_gpu.so) and any other
shared object exporting functions with these argument layouts.
"""
import ctypes as C

ABI_VERSION = 4

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_NAN = -4
ERR_TIMEOUT = -5
ERR_UNSUPPORTED = -6
ERR_NOT_FOUND = -7
ERR_BUSY = -8
ERR_CANCELLED = -9
ERR_IO = -10

PREC_FP64 = 0
PREC_MIXED = 1

LAYOUT_TAU2 = 0
LAYOUT_FULL3 = 1

# per-pair operators (electrodynamics/K.h, R.h)
OP_K_NEAR_SMOOTH = 0
OP_K_HS = 1
OP_K_HS_COLLOC = 2
OP_K_HS2_COLLOC = 3
OP_K_FAR = 4
OP_R_SMOOTH = 5
OP_R_COLLOC = 6
OP_R_NEAR = 7
OP_NAMES = {
    OP_K_NEAR_SMOOTH: "K_RotRot_Near_Smooth",
    OP_K_HS: "K_RotRot_HS",
    OP_K_HS_COLLOC: "K_RotRot_HS_Colloc",
    OP_K_HS2_COLLOC: "K_RotRot_HS2_Colloc",
    OP_K_FAR: "K_RotRot_Far",
    OP_R_SMOOTH: "R_Rot_Smooth",
    OP_R_COLLOC: "R_Rot_Colloc",
    OP_R_NEAR: "R_Rot_Near",
}

# kernel_lib integrands (electrodynamics/kernel_lib.h): id -> (name, idim, complex)
F_SIMPLEPOT_L = 0
F_GRADSIMPLEPOT_L = 1
F_DOUBLEPOT_L = 2
F_VECTORPOT_L = 3
F_SIMPLEPOT_H = 4
F_NU_SIMPLEPOT_H = 5
F_SIMPLEPOT_HM1 = 6
F_GRADSIMPLEPOT_H = 7
F_GRADSIMPLEPOT_HM1 = 8
F_DOUBLEPOT_H = 9
F_N_DOUBLEPOT_H = 10
F_ROTROTSIMPLEPOT_H = 11
F_ONE = 12
F_PLANEWAVE_E = 13
INTEGRANDS = {
    F_SIMPLEPOT_L: ("F_SimplePot_L", 1, False),
    F_GRADSIMPLEPOT_L: ("F_GradSimplePot_L", 3, False),
    F_DOUBLEPOT_L: ("F_DoublePot_L", 1, False),
    F_VECTORPOT_L: ("F_VectorPot_L", 3, False),
    F_SIMPLEPOT_H: ("F_SimplePot_H", 1, True),
    F_NU_SIMPLEPOT_H: ("nuF_SimplePot_H", 3, True),
    F_SIMPLEPOT_HM1: ("F_SimplePot_Hm1", 1, True),
    F_GRADSIMPLEPOT_H: ("F_GradSimplePot_H", 3, True),
    F_GRADSIMPLEPOT_HM1: ("F_GradSimplePot_Hm1", 3, True),
    F_DOUBLEPOT_H: ("F_DoublePot_H", 1, True),
    F_N_DOUBLEPOT_H: ("nF_DoublePot_H", 3, True),
    F_ROTROTSIMPLEPOT_H: ("F_RotRotSimplePot_H", 3, True),
    F_ONE: ("F_One", 1, False),
    F_PLANEWAVE_E: ("PlaneWaveFieldE", 3, True),
}
# integrands of one point, F(x): the form IntegralUniversal and the segment
# F(x) overload take (the rest are pair integrands F(x, y))
FX_INTEGRANDS = (F_ONE, F_PLANEWAVE_E)
# integrands the *_pnt and K0 forms take: the pair integrands and F = 1
PAIR_INTEGRANDS = tuple(i for i in INTEGRANDS if i != F_PLANEWAVE_E)


class NumParam(C.Structure):
    """bielcc_numparam; defaults = Calculation_Constants (electrodynamics/constants.h:17-27)."""

    _fields_ = [
        ("eps", C.c_double),
        ("rs", C.c_double),
        ("rs_seg", C.c_double),
        ("analytic_calc", C.c_double),
        ("n_start", C.c_int32),
        ("n_start_seg", C.c_int32),
        ("p_max", C.c_int32),
        ("p_max_seg", C.c_int32),
    ]

    @classmethod
    def default(cls, **kw):
        p = cls(1e-6, 2.0, 2.0, 3.0, 8, 10, 1, 1)
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class PlaneWave(C.Structure):
    _fields_ = [
        ("k_vec", C.c_double * 3),
        ("e0", C.c_double * 3),
        ("h_scale", C.c_double),
        ("add_E", C.c_int32),
        ("add_H", C.c_int32),
    ]

    @classmethod
    def make(cls, k_vec, e0, h_scale=0.0, add_E=True, add_H=False):
        return cls((C.c_double * 3)(*k_vec), (C.c_double * 3)(*e0), float(h_scale), int(add_E), int(add_H))


class KernelParam(C.Structure):
    _fields_ = [
        ("smoothR", C.c_double),
        ("smoothRMin", C.c_double),
        ("k_re", C.c_double),
        ("k_im", C.c_double),
        ("current", (C.c_double * 2) * 3),
        ("vec_dbl", C.c_double * 3),
        ("n", C.c_double * 3),
        ("e0", C.c_double * 3),
    ]


DISPERSION_NONE = 0
DISPERSION_REFRACT = 1


class Material(C.Structure):
    """bielcc_material: MaterialParam's description (electrodynamics/material.h)."""

    _fields_ = [
        ("dispersion", C.c_int32),
        ("n_table", C.c_int32),
        ("eps_r", C.c_double),
        ("mu_r", C.c_double),
        ("sigma", C.c_double),
        ("table", C.POINTER(C.c_double)),
    ]


class Medium(C.Structure):
    """bielcc_medium: eps, mu, k, multE, multH of a material at one frequency."""

    _fields_ = [
        ("eps", C.c_double * 2),
        ("mu", C.c_double * 2),
        ("k", C.c_double * 2),
        ("k_source", C.c_double),
        ("multE", C.c_double * 2),
        ("multH", C.c_double * 2),
        ("tand", C.c_double),
        ("skin_depth", C.c_double),
    ]

    def cplx(self, name):
        v = getattr(self, name)
        return complex(v[0], v[1])


class Report(C.Structure):
    _fields_ = [
        ("n_pairs", C.c_int64),
        ("n_near_pairs", C.c_int64),
        ("n_nonfinite", C.c_int64),
        ("est_rel_l2", C.c_double),
        ("est_sample", C.c_int32),
        ("status", C.c_int32),
    ]


class FieldJob(C.Structure):
    """bielcc_field_job: one field evaluation of a batch (device pointers)."""

    _fields_ = [
        ("mesh", C.c_int32),
        ("n_rhs", C.c_int32),
        ("n_pts", C.c_int32),
        ("J_dev", C.c_void_p),
        ("pts_dev", C.c_void_p),
        ("E_dev", C.c_void_p),
        ("H_dev", C.c_void_p),
        ("k_re", C.c_double),
        ("k_im", C.c_double),
        ("mult_re", C.c_double),
        ("mult_im", C.c_double),
        ("inc", PlaneWave),
        ("est_dev", C.c_void_p),
    ]


class FieldRequest(C.Structure):
    """bielcc_field_request: a serving request (host buffers, or resident J_dev)."""

    _fields_ = [
        ("mesh", C.c_int32),
        ("n_rhs", C.c_int32),
        ("n_pts", C.c_int32),
        ("out_c64", C.c_int32),
        ("J", C.c_void_p),
        ("J_dev", C.c_void_p),
        ("pts", C.c_void_p),
        ("E", C.c_void_p),
        ("H", C.c_void_p),
        ("k_re", C.c_double),
        ("k_im", C.c_double),
        ("mult_re", C.c_double),
        ("mult_im", C.c_double),
        ("inc", PlaneWave),
        ("est", C.c_void_p),
    ]


class AssembleRequest(C.Structure):
    _fields_ = [
        ("mesh", C.c_int32),
        ("layout", C.c_int32),
        ("out_c64", C.c_int32),
        ("A", C.c_void_p),
        ("A_dev", C.c_void_p),
        ("k_re", C.c_double),
        ("k_im", C.c_double),
    ]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "submitted", "completed", "failed", "cancelled", "rejected", "queued", "running", "batches", "priority_batches",
        "max_batch",
        "bytes_reserved", "peak_bytes_reserved", "bytes_allocated", "budget", "pairs_done", "pool_mapped_bytes",
        "pinned_bytes")] + \
        [(n, C.c_double) for n in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "wall_s", "pairs_per_s", "stage_in_s",
                                   "copy_out_s", "gpu_busy_s", "stage_alloc_s", "stage_copy_s", "stage_plan_s",
                                   "stage_launch_s")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchTrace(C.Structure):
    """bielcc_batch_trace: one served batch (times in ms from the first submission)."""
    _fields_ = [
        ("slot", C.c_int32),
        ("n_requests", C.c_int32),
        ("assembly", C.c_int32),
        ("high_priority", C.c_int32),
        ("pairs", C.c_int64),
        ("first_ticket", C.c_int64),
        ("admit_ms", C.c_double),
        ("stage1_ms", C.c_double),
        ("done_ms", C.c_double),
        ("complete_ms", C.c_double),
        ("oldest_wait_ms", C.c_double),
    ]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [
        ("kernel_launches", C.c_int64),
        ("far_launches", C.c_int64),
        ("far_pairs", C.c_int64),
        ("far_ms", C.c_double),
        ("far_ctas", C.c_int64),
    ]


def kernelparam_array(n, smoothR=0.0, smoothRMin=0.0, k=0.0, current=None, vec_dbl=None, normal=None, e0=None):
    """Array of n KernelParam records; array-valued arguments are per pair."""
    import numpy as np

    arr = (KernelParam * n)()
    kk = np.broadcast_to(np.asarray(k, dtype=np.complex128), (n,))
    sR = np.broadcast_to(np.asarray(smoothR, dtype=np.float64), (n,))
    sRm = np.broadcast_to(np.asarray(smoothRMin, dtype=np.float64), (n,))
    cur = None if current is None else np.broadcast_to(np.asarray(current, dtype=np.complex128), (n, 3))
    vd = None if vec_dbl is None else np.broadcast_to(np.asarray(vec_dbl, dtype=np.float64), (n, 3))
    nn = None if normal is None else np.broadcast_to(np.asarray(normal, dtype=np.float64), (n, 3))
    ee = None if e0 is None else np.broadcast_to(np.asarray(e0, dtype=np.float64), (n, 3))
    for i in range(n):
        a = arr[i]
        a.smoothR = float(sR[i])
        a.smoothRMin = float(sRm[i])
        a.k_re = float(kk[i].real)
        a.k_im = float(kk[i].imag)
        for g in range(3):
            if cur is not None:
                a.current[g][0] = float(cur[i, g].real)
                a.current[g][1] = float(cur[i, g].imag)
            if vd is not None:
                a.vec_dbl[g] = float(vd[i, g])
            if nn is not None:
                a.n[g] = float(nn[i, g])
            if ee is not None:
                a.e0[g] = float(ee[i, g])
    return arr


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p


def declare_common(lib, prefix):
    """Prototypes shared by the GPU library (prefix 'bielcc_', ctx-taking) and
    the CPU checkers (prefix 'oracle_' / 'ref_', no ctx)."""
    gpu = prefix == "bielcc_"
    ctx = [_vp] if gpu else []

    def d(name, args, res=C.c_int):
        f = getattr(lib, prefix + name)
        f.argtypes = args
        f.restype = res
        return f

    d("pair_op", ctx + [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, C.POINTER(NumParam), _dp])
    d("integral_pnt", ctx + [C.c_int, C.c_int, C.c_int, _dp, _dp, C.POINTER(KernelParam), C.c_int, C.c_int, C.c_double, _dp])
    d("integral_seg_pnt", ctx + [C.c_int, C.c_int, _dp, _dp, _dp, C.POINTER(KernelParam), C.c_int, C.c_int, C.c_double, _dp])
    d("integral", ctx + [C.c_int, C.c_int, C.c_int, _dp, C.POINTER(KernelParam), C.c_int, C.c_int, C.c_double, _dp])
    d("integral_seg", ctx + [C.c_int, C.c_int, _dp, _dp, C.POINTER(KernelParam), C.c_int, C.c_int, C.c_double, _dp])
    d("k0", ctx + [C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.POINTER(KernelParam), C.c_int, C.c_int, C.c_double, _dp])
    d("integral_1divr", ctx + [C.c_int, C.c_int, _dp, _dp, _dp])
    d("integral_grad1divr_seg", ctx + [C.c_int, _dp, _dp, _dp, _dp])
    d("integral_surf_simplepot_h_hs", ctx + [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp])
    d("integral_seg_gradsimplepot_h_hs", ctx + [C.c_int, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp])
    return lib


def dptr(a):
    """double* of a C-contiguous float64 / complex128 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)
