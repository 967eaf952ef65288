"""The C++ drop-in layer (include/bielcc_gpu.hpp) compiles against the
reference's own headers and types: the reference's NumParam, KernelParam,
IntegralParam, SurfMesh and kernel_lib function pointers are accepted by the
bielcc_gpu:: templates with the reference's call shapes. Compile and link
only (no GPU); skipped where the reference sources are absent."""
import os
import subprocess
import tempfile

import pytest

from conftest import ROOT

REF = os.environ.get("BIELCC_REF_SRC", "/root/reference")

SRC = r'''
#include "surf_mesh.h"
#include "kernel_lib.h"
#include "K.h"
#include "R.h"
#include "get_field.h"
#include "incident_field.h"
#include "integral_param.h"
#include "bielcc_gpu.hpp"

using namespace bielcc;

int main() {
    const double cell[4][3] = {{0, 0, 0}, {2, 0, 0}, {3, 2, 0}, {0, 2, 0}};
    const double tri[3][3] = {{0, 2, 0}, {0, 0, 0}, {2, 0, 0}};
    const double x[3] = {10, 10, 10};
    NumParam np(1e-6, 2, 2, 3, 8, 10, 1, 1);
    std::complex<double> j[3] = {1., 0., 0.}, res[3];
    bielcc_gpu::K_RotRot_Far(j, x, cell, np, 1.0, res);
    bielcc_gpu::K_RotRot_Near_Smooth(j, x, tri, np, std::complex<double>(1., 0.), res);
    bielcc_gpu::R_Rot_Colloc(j, x, cell, np, 1.0, res);
    KernelParam<double> kp;
    kp.smoothR = 0.1; kp.smoothRMin = 1e-6; kp.k = 1.0;
    IntegralParam ip(3, 8, 1, 1e-6);
    bielcc_gpu::IntegralUniversalPnt(x, cell, F_GradSimplePot_H<double>, kp, ip, res);
    bielcc_gpu::K0(j, x, cell, F_GradSimplePot_H<double>, kp, ip, res);
    double r = bielcc_gpu::integral1Divr(cell, x);
    (void)r;
    SurfMesh<CellQuad>* mesh = nullptr;
    std::vector<std::array<std::complex<double>, 3>> jE, fE;
    std::vector<std::array<double, 3>> pts;
    KernelParam<double> einc;
    if (mesh) bielcc_gpu::GetFieldE_Ideal(*mesh, jE, std::complex<double>(1., 0.), einc, PlaneWaveFieldE<double>, np,
                                          pts, fE);
    return 0;
}
'''


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference sources absent")
def test_dropin_header_compiles_against_reference_types():
    inc = []
    for d in ("electrodynamics", "geometry", "integrators", "io", "mesh"):
        inc += ["-I", os.path.join(REF, d)]
    objs = os.path.join(ROOT, "oracle", "_ref", "obj")
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "t.cpp")
        open(c, "w").write(SRC)
        cmd = ["/usr/bin/g++", "-std=c++17", "-fopenmp", "-I", os.path.join(ROOT, "include")] + inc + \
            ["-c", c, "-o", os.path.join(td, "t.o")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        if os.path.isdir(objs):
            lib = os.path.join(ROOT, "bielcc_b200")
            link = ["/usr/bin/g++", "-fopenmp", os.path.join(td, "t.o")] + \
                [os.path.join(objs, f) for f in sorted(os.listdir(objs))] + \
                ["-L", lib, "-lbielcc_gpu", "-o", os.path.join(td, "t")]
            r = subprocess.run(link, capture_output=True, text=True)
            assert r.returncode == 0, r.stderr[-3000:]
