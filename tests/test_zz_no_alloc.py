"""bielcc_field_EH_noalloc: the field evaluation for callers that cannot
allocate device memory while they run (they reserved the GPU's memory in their
own pool, or cannot afford cudaMalloc's device-wide synchronisation). All of
its scratch lives in a static 64 MiB device array; the caller passes device
buffers only.

Checked through the C ABI against the allocating entry point
(bielcc_field_EH_device) on two calls in a row — the second with other points
and precision, so leftovers of the first call in the shared array would show —
plus the size limit and the free device memory around a call (unchanged). This
file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from bielcc_b200 import abi, gpu
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, TOL_MIXED, golden, rel_l2

pytestmark = pytest.mark.gpu


def _bind():
    L = gpu.load()
    f = L.bielcc_field_EH_noalloc
    vp = C.c_void_p
    f.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.POINTER(abi.PlaneWave), C.POINTER(abi.NumParam), C.c_int, vp, vp, vp, C.c_int, vp,
                  C.POINTER(abi.Report)]
    f.restype = C.c_int
    return L, f


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    L, noalloc = _bind()
    g = golden("field_quad512.npz")
    inc = abi.PlaneWave.make(g["kvec"], g["e0"], float(g["h_scale"]), True, True)
    cells, J, k = g["cells"], g["J"], float(g["k"])
    dev = torch.device("cuda:0")
    ctx = gpu.Context(0)
    mesh = ctx.mesh(cells)
    stream = torch.cuda.current_stream(dev)
    Cd = torch.from_numpy(np.ascontiguousarray(cells)).to(dev)
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    np_ = abi.NumParam.default()

    def run_both(pts, precision, numparam=None):
        nparam = np_ if numparam is None else numparam
        Pd = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
        shape = (1, len(pts), 3)
        Ea = torch.zeros(shape, dtype=torch.complex128, device=dev)
        Ha = torch.zeros_like(Ea)
        Eb = torch.full(shape, complex(7.0, 7.0), dtype=torch.complex128, device=dev)
        Hb = torch.full(shape, complex(7.0, 7.0), dtype=torch.complex128, device=dev)
        ctx.field_EH_device(mesh, Jd.data_ptr(), k, Pd.data_ptr(), Ea.data_ptr(), Ha.data_ptr(), 1, len(pts),
                            inc=inc, numparam=nparam, precision=precision, stream=stream.cuda_stream)
        rep = abi.Report()
        rc = noalloc(4, len(cells), Cd.data_ptr(), 1, Jd.data_ptr(), k, 0.0, 1.0, 0.0, C.byref(inc), C.byref(nparam),
                     len(pts), Pd.data_ptr(), Eb.data_ptr(), Hb.data_ptr(), gpu.PREC[precision], stream.cuda_stream,
                     C.byref(rep))
        assert rc == 0, L.bielcc_last_error().decode()
        torch.cuda.synchronize()
        assert rep.n_pairs == len(pts) * len(cells)
        return (Ea.cpu().numpy(), Ha.cpu().numpy()), (Eb.cpu().numpy(), Hb.cpu().numpy()), rep

    # call 1: the golden far + near points, FP64
    (Ea, Ha), (Eb, Hb), rep = run_both(g["pts"], "fp64")
    assert rep.n_near_pairs > 0
    assert rel_l2(Eb, Ea) < TOL_FP64 and rel_l2(Hb, Ha) < TOL_FP64
    assert rel_l2(Eb, g["E"]) < TOL_FP64 and rel_l2(Hb, g["H"]) < TOL_FP64

    # call 2: another point set and the mixed form, on the array call 1 left behind
    rng = np.random.default_rng(42)
    pts2 = np.concatenate([W.sphere_points(150, 2.2, 5), W.near_points(cells, 30, 0.03, 0.2, rng)])
    (Ea, Ha), (Eb, Hb), rep = run_both(pts2, "mixed")
    assert rep.n_near_pairs > 0
    assert rel_l2(Eb, Ea) < TOL_MIXED and rel_l2(Hb, Ha) < TOL_MIXED

    # call 3: adaptive quadrature with p_max = 2, whose far pass runs at 2 n_start
    # (node tables four times larger in the static array)
    np2 = abi.NumParam.default(p_max=2, p_max_seg=2)
    (Ea, Ha), (Eb, Hb), rep = run_both(pts2, "fp64", np2)
    assert rel_l2(Eb, Ea) < TOL_FP64 and rel_l2(Hb, Ha) < TOL_FP64

    # call 4: p_max = 3 (the n_start table of the convergence test joins the array)
    np3 = abi.NumParam.default(p_max=3, p_max_seg=2)
    (Ea, Ha), (Eb, Hb), rep = run_both(pts2, "fp64", np3)
    assert rel_l2(Eb, Ea) < TOL_FP64 and rel_l2(Hb, Ha) < TOL_FP64

    mesh.close()
    ctx.close()


def test_noalloc_large_far_point_set_fits():
    """8192 cells x 18,000 far points (no near pairs): the far partial sums are
    sized to the room the static array has left, so the call fits and matches
    the allocating entry point."""
    torch = pytest.importorskip("torch")
    L, noalloc = _bind()
    c = W.config2()
    cells, J, k = c["cells"], c["J"], c["k"]
    pts = c["pts"][:18000]
    dev = torch.device("cuda:0")
    ctx = gpu.Context(0)
    mesh = ctx.mesh(cells)
    stream = torch.cuda.current_stream(dev)
    Cd = torch.from_numpy(np.ascontiguousarray(cells)).to(dev)
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    shape = (1, len(pts), 3)
    Ea = torch.zeros(shape, dtype=torch.complex128, device=dev)
    Ha = torch.zeros_like(Ea)
    Eb = torch.zeros_like(Ea)
    Hb = torch.zeros_like(Ea)
    ctx.field_EH_device(mesh, Jd.data_ptr(), k, Pd.data_ptr(), Ea.data_ptr(), Ha.data_ptr(), 1, len(pts),
                        precision="mixed", stream=stream.cuda_stream)
    rep = abi.Report()
    rc = noalloc(4, len(cells), Cd.data_ptr(), 1, Jd.data_ptr(), k, 0.0, 1.0, 0.0, None, None, len(pts),
                 Pd.data_ptr(), Eb.data_ptr(), Hb.data_ptr(), gpu.PREC["mixed"], stream.cuda_stream, C.byref(rep))
    assert rc == 0, L.bielcc_last_error().decode()
    torch.cuda.synchronize()
    assert rep.n_near_pairs == 0
    assert rel_l2(Eb.cpu().numpy(), Ea.cpu().numpy()) < TOL_MIXED
    assert rel_l2(Hb.cpu().numpy(), Ha.cpu().numpy()) < TOL_MIXED
    mesh.close()
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    L, noalloc = _bind()
    dev = torch.device("cuda:0")
    cells = W.uv_sphere(128, 256)  # 32768 cells: node tables alone exceed 64 MiB
    Cd = torch.from_numpy(np.ascontiguousarray(cells)).to(dev)
    Jd = torch.zeros((1, len(cells), 3), dtype=torch.complex128, device=dev)
    Pd = torch.zeros((4, 3), dtype=torch.float64, device=dev)
    Ed = torch.zeros((1, 4, 3), dtype=torch.complex128, device=dev)
    rc = noalloc(4, len(cells), Cd.data_ptr(), 1, Jd.data_ptr(), 1.0, 0.0, 1.0, 0.0, None, None, 4, Pd.data_ptr(),
                 Ed.data_ptr(), None, 0, None, None)
    assert rc == abi.ERR_ARG
    assert "scratch" in L.bielcc_last_error().decode()


def test_noalloc_allocates_no_device_memory():
    """The point of the entry point: after a warm-up call (which may load the
    library's kernels into the context), a call on a fresh stream leaves the
    device's free memory unchanged, and so does a call rejected as too large."""
    torch = pytest.importorskip("torch")
    L, noalloc = _bind()
    g = golden("field_quad512.npz")
    cells, J, k = g["cells"], g["J"], float(g["k"])
    dev = torch.device("cuda:0")
    Cd = torch.from_numpy(np.ascontiguousarray(cells)).to(dev)
    Jd = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
    Pd = torch.from_numpy(np.ascontiguousarray(g["pts"])).to(dev)
    shape = (1, len(g["pts"]), 3)
    Ed = torch.zeros(shape, dtype=torch.complex128, device=dev)
    Hd = torch.zeros_like(Ed)
    big = W.uv_sphere(128, 256)
    Bd = torch.from_numpy(np.ascontiguousarray(big)).to(dev)
    Jb = torch.zeros((1, len(big), 3), dtype=torch.complex128, device=dev)
    stream = torch.cuda.Stream(dev)
    np_ = abi.NumParam.default()

    def call(precision):
        rep = abi.Report()
        rc = noalloc(4, len(cells), Cd.data_ptr(), 1, Jd.data_ptr(), k, 0.0, 1.0, 0.0, None, C.byref(np_),
                     len(g["pts"]), Pd.data_ptr(), Ed.data_ptr(), Hd.data_ptr(), gpu.PREC[precision],
                     stream.cuda_stream, C.byref(rep))
        assert rc == 0, L.bielcc_last_error().decode()
        stream.synchronize()
        return rep

    for prec in ("fp64", "mixed"):
        call(prec)  # warm-up: kernels of this precision are loaded
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(dev)
        rep = call(prec)
        free1, _ = torch.cuda.mem_get_info(dev)
        assert rep.n_near_pairs > 0
        assert free1 == free0, (prec, free0 - free1)

    free0, _ = torch.cuda.mem_get_info(dev)
    rc = noalloc(4, len(big), Bd.data_ptr(), 1, Jb.data_ptr(), 1.0, 0.0, 1.0, 0.0, None, None, 4, Pd.data_ptr(),
                 Ed.data_ptr(), None, 0, stream.cuda_stream, None)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert rc == abi.ERR_ARG
    assert free1 == free0, free0 - free1
