"""The C++ drop-in layer (include/bielcc_gpu.hpp) executed on the GPU next to
the reference's own templates: oracle/_ref/dropin_check (built from
oracle/dropin_check.cpp with the reference's sources, where they exist) calls
GetFieldE_Ideal with the reference's SurfMesh and PlaneWaveFieldE, the K / R
operators, the universal quadratures with kernel_lib pointers (incl. the
smoothR they leave behind), K0, the F(x) forms and the analytic integrals
through both namespaces and prints each relative error; every one must be
within 1e-12 and too few currents must throw."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "oracle", "_ref", "dropin_check")


@pytest.mark.skipif(not os.path.exists(EXE), reason="drop-in checker not built (reference sources were absent)")
def test_dropin_templates_match_the_reference():
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert lines[-1].startswith("ALL OK"), lines[-5:]
    checked = [l for l in lines if l.endswith(" ok")]
    assert len(checked) >= 60, len(checked)
