// dropin_check.cpp — test infrastructure: runs the C++ drop-in templates of
// include/bielcc_gpu.hpp (namespace bielcc_gpu, GPU through the C ABI) and the
// reference's own templates (namespace bielcc, AlenaSetukha/BIELcc compiled
// from its sources) on the same inputs, with the reference's own types
// (SurfMesh<CellQuad>, NumParam, KernelParam<KType>, IntegralParam) and its
// kernel_lib / incident-field function pointers, and prints the relative
// error of every call. Exit status 0 when every FP64 result is within 1e-12
// (relative L2) of the reference and every mutated smoothR is equal.
//
// Built by oracle/Makefile (target dropin) into oracle/_ref/dropin_check,
// next to the reference objects; run by tests/test_gpu_dropin.py on a GPU.
// Calls covered: GetFieldE_Ideal (get_field.h:35-78) with PlaneWaveFieldE as
// EInc_Func; K_RotRot_Near_Smooth / _HS / _HS_Colloc / _HS2_Colloc / _Far
// (K.h); R_Rot_Smooth / _Colloc / _Near (R.h); IntegralUniversalPnt,
// IntegralUniversal (integral_universal.h); IntegralUniversalSegPnt, both
// overloads (integral_universal_seg.h); K0 / K0_Common (K0.h);
// integral1Divr, integralGrad1DivrSeg, IntegralSurf_SimplePot_H_HS,
// IntegralSeg_GradSimplePot_H_HS (integrals_analytic.h).
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "surf_mesh.h"  // get_field.h uses SurfMesh without including it
#include "K.h"
#include "K0.h"
#include "R.h"
#include "get_field.h"
#include "incident_field.h"
#include "integral_param.h"
#include "integral_universal.h"
#include "integral_universal_seg.h"
#include "integrals_analytic.h"
#include "kernel_lib.h"
#include "num_param.h"

#include "../include/bielcc_gpu.hpp"

using cd = std::complex<double>;

namespace {

// SurfMesh whose cells come from flat arrays (FillMeshFromVTK is protected,
// mesh/surf_mesh.h:65-66).
template <typename CellType>
struct ArrayMesh : public bielcc::SurfMesh<CellType> {
    ArrayMesh(int nv, const std::vector<double>& cells) {
        const int n = (int)(cells.size() / (3 * nv));
        std::vector<std::vector<int>> polys((size_t)n);
        std::vector<std::array<double, 3>> pts((size_t)n * nv);
        for (int c = 0; c < n; c++) {
            polys[c].resize(nv);
            for (int v = 0; v < nv; v++) {
                polys[c][v] = c * nv + v;
                for (int g = 0; g < 3; g++) pts[(size_t)c * nv + v][g] = cells[((size_t)c * nv + v) * 3 + g];
            }
        }
        this->_cell_list.clear();
        this->FillMeshFromVTK(polys, pts);
        this->_num_frm = (int)this->_cell_list.size();
        this->_num_obj = 1;
        this->_num_mod = 1;
    }
};

// UV sphere of radius r: nlat x nlon quads, the pole rows degenerate.
std::vector<double> uv_sphere(int nlat, int nlon, double r) {
    std::vector<double> out;
    auto pt = [&](int i, int j) {
        double th = M_PI * i / nlat, ph = 2 * M_PI * j / nlon;
        return std::array<double, 3>{r * std::sin(th) * std::cos(ph), r * std::sin(th) * std::sin(ph),
                                     r * std::cos(th)};
    };
    for (int i = 0; i < nlat; i++)
        for (int j = 0; j < nlon; j++) {
            const std::array<double, 3> q[4] = {pt(i, j), pt(i + 1, j), pt(i + 1, j + 1), pt(i, j + 1)};
            for (auto& v : q) out.insert(out.end(), v.begin(), v.end());
        }
    return out;
}

double rel(const cd* a, const cd* b, size_t n) {
    double num = 0, den = 0;
    for (size_t i = 0; i < n; i++) {
        num += std::norm(a[i] - b[i]);
        den += std::norm(b[i]);
    }
    return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}
double rel(const double* a, const double* b, size_t n) {
    double num = 0, den = 0;
    for (size_t i = 0; i < n; i++) {
        num += (a[i] - b[i]) * (a[i] - b[i]);
        den += b[i] * b[i];
    }
    return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}

int g_fail = 0;
void report(const std::string& name, double err, bool ok_extra = true) {
    const bool ok = err <= 1e-12 && ok_extra;
    if (!ok) g_fail++;
    std::printf("%-40s %.3e %s\n", name.c_str(), err, ok ? "ok" : "FAIL");
}

}  // namespace

int run() {
    const double k = 2 * M_PI;
    const cd kc(2 * M_PI, 0.3);
    bielcc::NumParam np(1e-6, 2, 2, 3, 8, 10, 1, 1);
    bielcc::NumParam np3(1e-6, 2, 2, 3, 8, 10, 3, 3);

    // ---- GetFieldE_Ideal on a 128-quad sphere, far and near points, host incident field
    std::vector<double> flat = uv_sphere(8, 16, 1.0);
    ArrayMesh<bielcc::CellQuad> mesh(4, flat);
    const int N = mesh.GetNFrm();
    std::vector<std::array<cd, 3>> jE((size_t)N);
    for (int c = 0; c < N; c++) {
        double y[3];
        bielcc::get_center_mass(mesh.GetCell(c).GetCellCoords(), y);
        jE[c] = {cd(std::cos(3 * y[2]), 0.2 * y[0]), cd(0.5 * y[1], std::sin(2 * y[0])), cd(0.1, -0.3 * y[2])};
    }
    std::vector<std::array<double, 3>> pts;
    for (int i = 0; i < 40; i++) {
        double th = std::acos(1 - 2 * (i + 0.5) / 40), ph = 2.399963 * i;
        pts.push_back({2.5 * std::sin(th) * std::cos(ph), 2.5 * std::sin(th) * std::sin(ph), 2.5 * std::cos(th)});
    }
    for (int c = 3; c < N; c += 13) {  // near points just above cell centres
        double y[3];
        bielcc::get_center_mass(mesh.GetCell(c).GetCellCoords(), y);
        const double s = 1.0 + 0.03 + 0.01 * (c % 5);
        pts.push_back({y[0] * s, y[1] * s, y[2] * s});
    }
    bielcc::KernelParam<double> einc;
    einc.k = k;
    einc.smoothR = 0;
    einc.smoothRMin = 0;
    einc.vec_dbl[0] = 0, einc.vec_dbl[1] = 0, einc.vec_dbl[2] = k;
    einc.e0[0] = 1, einc.e0[1] = 0, einc.e0[2] = 0;
    const cd mult(0.0, -1.7);
    std::vector<std::array<cd, 3>> Er(pts.size()), Eg(pts.size());
    bielcc::GetFieldE_Ideal(mesh, jE, mult, einc, bielcc::PlaneWaveFieldE<double>, np, pts, Er);
    bielcc_gpu::GetFieldE_Ideal(mesh, jE, mult, einc, bielcc::PlaneWaveFieldE<double>, np, pts, Eg);
    report("GetFieldE_Ideal (128 quads, " + std::to_string(pts.size()) + " pts)",
           rel(&Eg[0][0], &Er[0][0], 3 * pts.size()));
    // adaptive refinement: p_max = 2 (the far pass at 2 n_start) and 3 (the
    // per-integral convergence test and the third pass)
    {
        bielcc::NumParam np2(1e-6, 2, 2, 3, 8, 10, 2, 2);
        for (const bielcc::NumParam* npa : {&np2, &np3}) {
            std::vector<std::array<cd, 3>> Ra(pts.size()), Ga(pts.size());
            bielcc::GetFieldE_Ideal(mesh, jE, mult, einc, bielcc::PlaneWaveFieldE<double>, *npa, pts, Ra);
            bielcc_gpu::GetFieldE_Ideal(mesh, jE, mult, einc, bielcc::PlaneWaveFieldE<double>, *npa, pts, Ga);
            report("GetFieldE_Ideal, p_max " + std::to_string(npa->p_max), rel(&Ga[0][0], &Ra[0][0], 3 * pts.size()));
        }
    }
    // more currents than cells: the extra ones are ignored, as in the reference loop
    std::vector<std::array<cd, 3>> jLong = jE;
    jLong.push_back({cd(1e3, 0), cd(1e3, 0), cd(1e3, 0)});
    std::vector<std::array<cd, 3>> Eg2(pts.size());
    bielcc_gpu::GetFieldE_Ideal(mesh, jLong, mult, einc, bielcc::PlaneWaveFieldE<double>, np, pts, Eg2);
    report("GetFieldE_Ideal, one extra current", rel(&Eg2[0][0], &Er[0][0], 3 * pts.size()));
    // fewer currents than cells: an error, not a read past the end
    bool threw = false;
    try {
        std::vector<std::array<cd, 3>> jShort(jE.begin(), jE.end() - 1);
        bielcc_gpu::GetFieldE_Ideal(mesh, jShort, mult, einc, bielcc::PlaneWaveFieldE<double>, np, pts, Eg2);
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    report("GetFieldE_Ideal, one current short: throws", threw ? 0.0 : 1.0, threw);

    // ---- per-pair operators, quads and triangles, real and complex k
    const double quad[4][3] = {{0, 0, 0}, {2, 0, 0}, {3, 2, 0.2}, {0, 2, 0}};
    const double tri[3][3] = {{0, 2, 0}, {0, 0, 0}, {2, 0, 0.1}};
    const double xs[3][3] = {{1.2, 0.9, 0.05}, {1.0, 1.1, 0.6}, {9.0, 8.0, 7.0}};
    const cd jj[3] = {cd(1, 0.5), cd(-0.3, 0.2), cd(0.7, -1)};
    auto ops = [&](auto kk, const char* kt) {
        for (int xi = 0; xi < 3; xi++) {
            const double* x = xs[xi];
            cd r[3], g[3];
            const std::string sfx = std::string(" ") + kt + " x" + std::to_string(xi);
#define BIELCC_CMP(NAME, CELL, NP)                                  \
    bielcc::NAME(jj, x, CELL, NP, kk, r);                           \
    bielcc_gpu::NAME(jj, x, CELL, NP, kk, g);                       \
    report(std::string(#NAME " ") + (sizeof(CELL) == 96 ? "quad" : "tri") + sfx, rel(g, r, 3));
            BIELCC_CMP(K_RotRot_Near_Smooth, quad, np)
            BIELCC_CMP(K_RotRot_Near_Smooth, tri, np3)
            BIELCC_CMP(K_RotRot_HS, quad, np)
            BIELCC_CMP(K_RotRot_HS_Colloc, tri, np)
            BIELCC_CMP(K_RotRot_HS2_Colloc, quad, np)
            BIELCC_CMP(K_RotRot_Far, quad, np)
            BIELCC_CMP(R_Rot_Smooth, tri, np)
            BIELCC_CMP(R_Rot_Colloc, quad, np)
            BIELCC_CMP(R_Rot_Near, quad, np3)
#undef BIELCC_CMP
        }
    };
    ops(k, "k");
    ops(kc, "kc");

    // ---- integrators with kernel_lib pointers: result and the smoothR left behind
    const double x0[3] = {1.2, 0.9, 0.05};
    bielcc::IntegralParam ip3(3, 8, 3, 1e-6), ip1(1, 8, 3, 1e-6), ips(3, 10, 3, 1e-6);
    auto kp_make = [&]() {
        bielcc::KernelParam<double> p;
        p.k = k;
        p.smoothR = 0.4;
        p.smoothRMin = 0.001;
        p.vec_dbl[0] = 0.3, p.vec_dbl[1] = -0.2, p.vec_dbl[2] = 1.9;
        p.n[0] = 0, p.n[1] = 0, p.n[2] = 1;
        p.e0[0] = 0.2, p.e0[1] = 1, p.e0[2] = -0.4;
        for (int i = 0; i < 3; i++) p.current[i] = jj[i];
        return p;
    };
    {
        auto a = kp_make(), b = kp_make();
        cd r[3], g[3];
        bielcc::IntegralUniversalPnt(x0, quad, bielcc::F_GradSimplePot_H<double>, a, ip3, r);
        bielcc_gpu::IntegralUniversalPnt(x0, quad, bielcc::F_GradSimplePot_H<double>, b, ip3, g);
        report("IntegralUniversalPnt F_GradSimplePot_H quad", rel(g, r, 3), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        bielcc::IntegralUniversalPnt(x0, tri, bielcc::F_SimplePot_H<double>, a, ip1, r);
        bielcc_gpu::IntegralUniversalPnt(x0, tri, bielcc::F_SimplePot_H<double>, b, ip1, g);
        report("IntegralUniversalPnt F_SimplePot_H tri", rel(g, r, 1), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        double rl[3], gl[3];
        bielcc::IntegralUniversalPnt(x0, quad, bielcc::F_GradSimplePot_L<double>, a, ip3, rl);
        bielcc_gpu::IntegralUniversalPnt(x0, quad, bielcc::F_GradSimplePot_L<double>, b, ip3, gl);
        report("IntegralUniversalPnt F_GradSimplePot_L quad", rel(gl, rl, 3), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        bielcc::IntegralUniversalSegPnt(quad[0], quad[2], x0, bielcc::F_GradSimplePot_H<double>, a, ips, r);
        bielcc_gpu::IntegralUniversalSegPnt(quad[0], quad[2], x0, bielcc::F_GradSimplePot_H<double>, b, ips, g);
        report("IntegralUniversalSegPnt F_GradSimplePot_H", rel(g, r, 3), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        bielcc::K0(jj, x0, quad, bielcc::F_GradSimplePot_H<double>, a, ips, r);
        bielcc_gpu::K0(jj, x0, quad, bielcc::F_GradSimplePot_H<double>, b, ips, g);
        report("K0 F_GradSimplePot_H quad", rel(g, r, 3), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        bielcc::K0_Common(x0, tri, bielcc::nuF_SimplePot_H<double>, a, ips, r);
        bielcc_gpu::K0_Common(x0, tri, bielcc::nuF_SimplePot_H<double>, b, ips, g);
        report("K0_Common nuF_SimplePot_H tri", rel(g, r, 3), a.smoothR == b.smoothR);
        // the F(x) forms with the incident field as integrand
        a = kp_make(), b = kp_make();
        bielcc::IntegralUniversal(quad, bielcc::PlaneWaveFieldE<double>, a, ip3, r);
        bielcc_gpu::IntegralUniversal(quad, bielcc::PlaneWaveFieldE<double>, b, ip3, g);
        report("IntegralUniversal PlaneWaveFieldE quad", rel(g, r, 3), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        bielcc::IntegralUniversal(tri, bielcc::PlaneWaveFieldE<double>, a, ip3, r);
        bielcc_gpu::IntegralUniversal(tri, bielcc::PlaneWaveFieldE<double>, b, ip3, g);
        report("IntegralUniversal PlaneWaveFieldE tri", rel(g, r, 3), a.smoothR == b.smoothR);
        a = kp_make(), b = kp_make();
        bielcc::IntegralUniversalSegPnt(quad[1], quad[3], bielcc::PlaneWaveFieldE<double>, a, ips, r);
        bielcc_gpu::IntegralUniversalSegPnt(quad[1], quad[3], bielcc::PlaneWaveFieldE<double>, b, ips, g);
        report("IntegralUniversalSegPnt F(x) PlaneWaveFieldE", rel(g, r, 3), a.smoothR == b.smoothR);
    }

    // ---- analytic singular parts
    {
        double r = bielcc::integral1Divr(quad, x0), g = bielcc_gpu::integral1Divr(quad, x0);
        report("integral1Divr quad", rel(&g, &r, 1));
        r = bielcc::integral1Divr(tri, x0), g = bielcc_gpu::integral1Divr(tri, x0);
        report("integral1Divr tri", rel(&g, &r, 1));
        double rv[3], gv[3];
        bielcc::integralGrad1DivrSeg(quad[0], quad[1], x0, rv);
        bielcc_gpu::integralGrad1DivrSeg(quad[0], quad[1], x0, gv);
        report("integralGrad1DivrSeg", rel(gv, rv, 3));
        bielcc::IntegralParam ipa(1, 8, 1, 1e-6), ipb(3, 10, 1, 1e-6);
        cd rc = bielcc::IntegralSurf_SimplePot_H_HS(quad, x0, 3.0, ipa, k);
        cd gc = bielcc_gpu::IntegralSurf_SimplePot_H_HS(quad, x0, 3.0, ipa, k);
        report("IntegralSurf_SimplePot_H_HS quad", rel(&gc, &rc, 1));
        cd r3[3], g3[3];
        bielcc::IntegralSeg_GradSimplePot_H_HS(quad[0], quad[1], x0, 3.0, ipb, k, r3);
        bielcc_gpu::IntegralSeg_GradSimplePot_H_HS(quad[0], quad[1], x0, 3.0, ipb, k, g3);
        report("IntegralSeg_GradSimplePot_H_HS", rel(g3, r3, 3));
    }

    std::printf("%s: %d failed\n", g_fail ? "FAILED" : "ALL OK", g_fail);
    return g_fail ? 1 : 0;
}

int main() {
    try {
        return run();
    } catch (const std::exception& e) {
        std::printf("ERROR: %s\n", e.what());
        return 2;
    }
}
