"""Full Stratton-Chu field of electric and magnetic currents
(bielcc_field_EH_full) against the combination that
examples/field/main0_field_test.cpp:313-319 forms from its four sums:
E = multE K[j_E] - R[j_M] + E_inc, H = multH K[j_M] + R[j_E] + H_inc. The sums
come from the reference compiled from its sources (or the C++ port when it is
absent), each a GetFieldE_Ideal-style evaluation of one current."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, TOL_MIXED, rel_l2

pytestmark = pytest.mark.gpu

MULT_E, MULT_H = complex(0.3, 1.2), complex(-0.7, 0.4)


def _case():
    cells = W.uv_sphere(16, 32)
    k = 2 * np.pi
    rng = np.random.default_rng(11)
    pts = np.concatenate([W.sphere_points(150, 3.0, 5), W.near_points(cells, 30, 0.02, 0.1, rng)])
    JE = W.po_currents(cells, k, directions=2, seed=1)
    JM = 0.5 * W.po_currents(cells, k, directions=2, seed=2)[:, ::-1].copy()  # a second, unrelated current
    return cells, k, pts, JE, JM


def _reference(cells, k, pts, JE, JM, inc, mult_e=MULT_E, mult_h=MULT_H):
    which = "ref" if oracle.available("ref") else "port"
    KE, RE = oracle.field_EH(cells, JE, k, pts, which=which)
    KM, RM = oracle.field_EH(cells, JM, k, pts, which=which)
    E = mult_e * KE - RM
    H = mult_h * KM + RE
    if inc is not None:
        kvec = np.array(inc.k_vec[:])
        e0 = np.array(inc.e0[:])
        ph = np.exp(1j * (pts @ kvec))[None, :, None]
        E = E + e0[None, None, :] * ph
        H = H + inc.h_scale * np.cross(kvec, e0)[None, None, :] * ph
    return E, H


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_full_field_matches_reference_sums(gctx, precision, tol):
    cells, k, pts, JE, JM = _case()
    kv, e0, hs = W.planewave(k)
    inc = abi.PlaneWave.make(kv, e0, hs, True, True)
    m = gctx.mesh(cells)
    E, H, rep = gctx.field_EH_full(m, JE, JM, k, pts, multE=MULT_E, multH=MULT_H, inc=inc, precision=precision)
    Er, Hr = _reference(cells, k, pts, JE, JM, inc)
    assert rep.n_near_pairs > 0 and rep.n_nonfinite == 0
    assert rel_l2(E, Er) < tol and rel_l2(H, Hr) < tol


def test_full_field_reduces_to_field_EH_and_device_form(gctx):
    torch = pytest.importorskip("torch")
    cells, k, pts, JE, JM = _case()
    m = gctx.mesh(cells)
    # no magnetic current: E = multE K[j_E], H = R[j_E], as bielcc_field_EH with mult = multE
    E0, H0, _ = gctx.field_EH_full(m, JE, np.zeros_like(JE), k, pts, multE=MULT_E, multH=MULT_H)
    E1, H1, _ = gctx.field_EH(m, JE, k, pts, mult=MULT_E)
    assert rel_l2(E0, E1) < 1e-13 and rel_l2(H0, H1) < 1e-13
    # device form = host form, bit for bit
    Eh, Hh, _ = gctx.field_EH_full(m, JE, JM, k, pts, multE=MULT_E, multH=MULT_H, precision="mixed")
    dev = torch.device("cuda:0")
    tJE = torch.from_numpy(np.ascontiguousarray(JE)).to(dev)
    tJM = torch.from_numpy(np.ascontiguousarray(JM)).to(dev)
    tP = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    tE = torch.zeros((JE.shape[0], len(pts), 3), dtype=torch.complex128, device=dev)
    tH = torch.zeros_like(tE)
    gctx.field_EH_full_device(m, tJE.data_ptr(), tJM.data_ptr(), k, tP.data_ptr(), tE.data_ptr(), tH.data_ptr(),
                              JE.shape[0], len(pts), multE=MULT_E, multH=MULT_H, precision="mixed",
                              stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(tE.cpu().numpy(), Eh) and np.array_equal(tH.cpu().numpy(), Hh)


def test_extinction_theorem_sphere(gctx):
    """The known answer of examples/field/main0_field_test.cpp (its header,
    steps 1-4): with j_E = -n x H_inc and j_M = n x E_inc on a closed surface,
    the Stratton-Chu field is E_inc inside the body and zero outside. Units
    with eps = mu = 1, omega = k (H_inc = k_hat x E_inc), so multE = multH =
    i / k. Piecewise-constant currents on 8192 quads: a few per cent of
    discretisation error."""
    cells = W.uv_sphere(64, 128)
    k = 2 * np.pi
    kv, e0, hs = W.planewave(k)
    c, n = W.centres(cells), W.normals(cells)
    ph = np.exp(1j * (c @ kv))[:, None]
    Einc = e0[None, :] * ph
    Hinc = hs * np.cross(kv, e0)[None, :] * ph
    JE = -np.cross(n, Hinc)[None]
    JM = np.cross(n, Einc)[None]
    rng = np.random.default_rng(3)
    inside = W.shell_points(200, 0.0, 0.5, rng)
    outside = W.shell_points(200, 2.0, 3.0, rng)
    m = gctx.mesh(cells)
    mult = 1j / k
    Ei, Hi, _ = gctx.field_EH_full(m, JE, JM, k, inside, multE=mult, multH=mult, precision="mixed")
    Eo, Ho, _ = gctx.field_EH_full(m, JE, JM, k, outside, multE=mult, multH=mult, precision="mixed")
    pin = np.exp(1j * (inside @ kv))[:, None]
    Ein = e0[None, :] * pin
    Hin = hs * np.cross(kv, e0)[None, :] * pin
    assert rel_l2(Ei[0], Ein) < 0.05 and rel_l2(Hi[0], Hin) < 0.05
    assert np.sqrt(np.mean(np.abs(Eo[0]) ** 2)) < 0.05 and np.sqrt(np.mean(np.abs(Ho[0]) ** 2)) < 0.05


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_full_field_in_lossy_medium(gctx, precision, tol):
    """A body in a lossy dielectric (eps_r = 2, sigma = 2 mS/m at the frequency
    where Re k = 2 pi): the medium's complex wave number (Im k > 0), multE =
    i / (omega eps), multH = i / (omega mu) and incident plane wave from
    bielcc_medium_at / bielcc_planewave_in_medium (MaterialParam::Calc,
    RadiationSource::CalcK, main0_field_test.cpp:185-199), through
    bielcc_field_EH_full, against the reference's own field sums with that
    complex k (KType = std::complex<double>) combined as the example does."""
    from bielcc_b200 import gpu

    c0 = 299792458.0
    freq = c0 / np.sqrt(2.0)  # Re k ~ 2 pi in eps_r = 2
    md = gpu.medium_at(gpu.material(eps_r=2.0, sigma=2e-3), freq)
    k = md.cplx("k")
    assert k.imag > 0.05 and abs(k.real - 2 * np.pi) < 0.2
    inc = gpu.planewave_in_medium(md, freq, direction=(0, 0, 1), e0=(1, 0, 0))
    cells, _, pts, JE, JM = _case()
    multE, multH = md.cplx("multE"), md.cplx("multH")
    m = gctx.mesh(cells)
    E, H, rep = gctx.field_EH_full(m, JE, JM, k, pts, multE=multE, multH=multH, inc=inc, precision=precision)
    Er, Hr = _reference(cells, k, pts, JE, JM, inc, multE, multH)
    assert rep.n_near_pairs > 0 and rep.n_nonfinite == 0
    assert rel_l2(E, Er) < tol and rel_l2(H, Hr) < tol
