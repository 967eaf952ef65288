"""Material constants at a frequency (bielcc_medium_at, host only) against the
reference's MaterialParam::Calc (electrodynamics/material.cpp:60-128) and
RadiationSource::CalcK (radiation_source.cpp:159-180): permittivity,
permeability, skin depth and wave number, for a lossless dielectric, a
conductor-loaded dielectric and refractive-index tables with and without
absorption; the multipliers of examples/field/main0_field_test.cpp:185-199.
Where the reference's CalcK throws (complex eps with its real mu), the wave
number is checked against omega sqrt(eps mu) instead."""
import cmath
import math

import numpy as np
import pytest

import oracle
from bielcc_b200 import abi, gpu

EPS0, MU0 = 8.8541878128e-12, 4 * math.pi * 1e-7

CASES = [
    dict(freq=3.0e8, eps_r=4.0, mu_r=1.0),                       # lossless dielectric
    dict(freq=1.5e8, eps_r=4.0, mu_r=1.5, sigma=0.05),           # lossy: complex eps
    dict(freq=2.0e8, table=[[1.0e8, 1.4, 0.0], [2.0e8, 1.5, 0.0]], mu_r=1.0),      # CalcEpsN
    dict(freq=2.0e8, table=[[1.0e8, 1.4, 0.1], [2.0e8, 1.6, 0.02]], mu_r=1.0),     # CalcEpsNK
]


def _mat(c):
    return gpu.material(eps_r=c.get("eps_r", 1.0), mu_r=c.get("mu_r", 1.0), sigma=c.get("sigma", 0.0),
                        table=c.get("table"))


@pytest.mark.parametrize("case", CASES)
def test_medium_against_reference(case):
    if not oracle.available("ref"):
        pytest.skip("reference build absent")
    md = gpu.medium_at(_mat(case), case["freq"])
    ref = oracle.ref_material(case["freq"], case.get("eps_r", 1.0), case.get("mu_r", 1.0), case.get("sigma", 0.0),
                              case.get("table"))
    assert abs(md.cplx("eps") - ref["eps"]) <= 1e-15 * abs(ref["eps"])
    assert abs(md.cplx("mu") - ref["mu"]) <= 1e-15 * abs(ref["mu"])
    if "table" not in case:  # the reference's refractive-index constructors leave _sigma uninitialised
        assert abs(md.skin_depth - ref["skin_depth"]) <= 1e-14 * max(ref["skin_depth"], 1e-300)
    else:
        assert md.skin_depth == 0.0
    omega = 2 * math.pi * case["freq"]
    k = omega * cmath.sqrt(ref["eps"] * ref["mu"])
    assert abs(md.cplx("k") - k) <= 1e-14 * abs(k)
    if ref["eps"].imag == 0.0:
        assert not ref["calck_threw"]
        assert abs(md.k_source - ref["k"]) <= 1e-14 * ref["k"] and md.k[1] == 0.0
    else:  # the reference's CalcK throws: it reads its real mu as complex
        assert ref["calck_threw"]
        assert md.k[1] > 0.0
    assert abs(md.cplx("multE") - 1j / (omega * ref["eps"])) <= 1e-14 * abs(1 / (omega * ref["eps"]))
    assert abs(md.cplx("multH") - 1j / (omega * ref["mu"])) <= 1e-14 * abs(1 / (omega * ref["mu"]))


def test_medium_host_rules():
    md = gpu.medium_at(gpu.material(eps_r=2.25), 1.0e9)
    assert md.k[1] == 0.0 and abs(md.k[0] - 2 * math.pi * 1e9 * math.sqrt(2.25 * EPS0 * MU0)) < 1e-9
    pw = gpu.planewave_in_medium(md, 1.0e9, direction=(0, 0, 2.0), e0=(1, 0, 0))
    assert np.allclose(pw.k_vec[:], [0, 0, md.k_source]) and pw.add_E == 1 and pw.add_H == 1
    assert abs(pw.h_scale - 1 / (2 * math.pi * 1e9 * MU0)) < 1e-12 / MU0
    with pytest.raises(gpu.BielccError) as e:  # the reference silently takes n = 0 here
        gpu.medium_at(gpu.material(table=[[1.0e8, 1.4, 0.0]]), 2.0e8)
    assert e.value.code == abi.ERR_ARG
    with pytest.raises(gpu.BielccError):
        gpu.medium_at(gpu.material(), 0.0)
