// ref_glue.cpp — exposes the REFERENCE implementation (AlenaSetukha/BIELcc,
// compiled from its own sources by oracle/Makefile) through the same C
// signatures as the oracle (oracle/bielcc_oracle.cpp), prefixed ref_.
//
// Test infrastructure only: used by tests/ to pin the oracle, by
// tests/golden/make_golden.py to produce golden vectors, and by bench.py's
// reference arm (timed CPU baseline). The product never loads it.
//
// Everything computed here goes through the reference's public templates:
// GetFieldE_Ideal (electrodynamics/get_field.h:35-78), K_RotRot_* (K.h),
// R_Rot_* (R.h), K0 / K0_Common (K0.h), IntegralUniversalPnt /
// IntegralUniversal (integral_universal.h), IntegralUniversalSegPnt
// (integral_universal_seg.h) and integrals_analytic.{h,cpp}.

#include <array>
#include <complex>
#include <cstdint>
#include <vector>
#include <omp.h>

#include "surf_mesh.h"  // get_field.h uses SurfMesh without including it
#include "K.h"
#include "K0.h"
#include "R.h"
#include "get_field.h"
#include "integral_universal.h"
#include "integral_universal_seg.h"
#include "integrals_analytic.h"
#include "kernel_lib.h"
#include "num_param.h"
#include "incident_field.h"
#include "material.h"
#include "radiation_source.h"
#include "currents.h"
#include <fstream>
#include <stdexcept>

#include "../include/bielcc_gpu.h"

using namespace bielcc;
using cd = std::complex<double>;

namespace {

// SurfMesh whose cells come from flat arrays (FillMeshFromVTK is protected,
// mesh/surf_mesh.h:65-66, so a derived class feeds it polygons + points).
template <typename CellType>
struct ArrayMesh : public SurfMesh<CellType> {
    ArrayMesh(int nv, int n_cells, const double* cells) {
        std::vector<std::vector<int>> polys((size_t)n_cells);
        std::vector<std::array<double, 3>> pts((size_t)n_cells * nv);
        for (int c = 0; c < n_cells; c++) {
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

NumParam make_np(const bielcc_numparam* p) {
    if (!p)
        return NumParam(Calculation_Constants::INTEGRAL_ACCURACY, Calculation_Constants::SMOOTHING_DIST_SURF_INT,
                        Calculation_Constants::SMOOTHING_DIST_SEG_INT, Calculation_Constants::ANALYTIC_CALC_DIST,
                        Calculation_Constants::START_CELL_SPLIT, Calculation_Constants::START_SEG_SPLIT,
                        Calculation_Constants::PMAX_CELL_SPLIT, Calculation_Constants::PMAX_SEG_SPLIT);
    return NumParam(p->eps, p->rs, p->rs_seg, p->analytic_calc, p->n_start, p->n_start_seg, p->p_max,
                    p->p_max_seg);
}

template <typename KType>
void zero_inc(const double*, const KernelParam<KType>&, cd* e) { e[0] = e[1] = e[2] = 0.; }

template <typename KType> KType make_k(double re, double im);
template <> double make_k<double>(double re, double) { return re; }
template <> cd make_k<cd>(double re, double im) { return cd(re, im); }

template <typename KType, typename CellType, size_t NV>
int field_impl(int n_cells, const double* cells, int n_rhs, const double* J, double k_re, double k_im,
               double mult_re, double mult_im, const bielcc_planewave* inc, const bielcc_numparam* npp,
               int n_pts, const double* pts, double* E, double* H, int n_threads) {
    if (n_threads > 0) omp_set_num_threads(n_threads);
    ArrayMesh<CellType> mesh(NV, n_cells, cells);
    NumParam np = make_np(npp);
    KType k = make_k<KType>(k_re, k_im);
    std::vector<std::array<double, 3>> points((size_t)n_pts);
    for (int i = 0; i < n_pts; i++)
        for (int g = 0; g < 3; g++) points[i][g] = pts[3 * (size_t)i + g];
    KernelParam<KType> einc;
    einc.k = k;
    if (inc)
        for (int g = 0; g < 3; g++) { einc.vec_dbl[g] = inc->k_vec[g]; einc.e0[g] = inc->e0[g]; }
    void (*f_inc)(const double*, const KernelParam<KType>&, cd*) =
        (inc && inc->add_E) ? PlaneWaveFieldE<KType> : zero_inc<KType>;
    for (int s = 0; s < n_rhs; s++) {
        std::vector<std::array<cd, 3>> jE((size_t)n_cells), fE((size_t)n_pts);
        for (int c = 0; c < n_cells; c++)
            for (int g = 0; g < 3; g++) {
                size_t o = (((size_t)s * n_cells + c) * 3 + g) * 2;
                jE[c][g] = cd(J[o], J[o + 1]);
            }
        GetFieldE_Ideal(mesh, jE, cd(mult_re, mult_im), einc, f_inc, np, points, fE);
        for (int i = 0; i < n_pts; i++)
            for (int g = 0; g < 3; g++) {
                size_t o = (((size_t)s * n_pts + i) * 3 + g) * 2;
                E[o] = fE[i][g].real();
                E[o + 1] = fE[i][g].imag();
            }
        if (!H) continue;
        // H counterpart: the R-operator loop of examples/field/main0_field_test.cpp
        // (far R_Rot_Colloc :255/:271, near R_Rot_Smooth :291/:306) with the
        // per-cell near criterion of get_field.h:58.
#pragma omp parallel for
        for (int i = 0; i < n_pts; i++) {
            cd h[3] = {0., 0., 0.}, tmp[3];
            double y[3];
            for (int c = 0; c < n_cells; c++) {
                const auto& cell = mesh.GetCell(c);
                get_center_mass(cell.GetCellCoords(), y);
                if (dist(points[i].data(), y) < np.analytic_calc * get_diam(cell.GetCellCoords()))
                    R_Rot_Smooth(jE[c].data(), points[i].data(), cell.GetCellCoords(), np, k, tmp);
                else
                    R_Rot_Colloc(jE[c].data(), points[i].data(), cell.GetCellCoords(), np, k, tmp);
                for (int g = 0; g < 3; g++) h[g] += tmp[g];
            }
            if (inc && inc->add_H) {
                double kx0[3];
                vec_prod(inc->k_vec, inc->e0, kx0);
                cd ph = std::exp(cd(0., 1.) * scal_prod(inc->k_vec, points[i].data())) * inc->h_scale;
                for (int g = 0; g < 3; g++) h[g] += kx0[g] * ph;
            }
            for (int g = 0; g < 3; g++) {
                size_t o = (((size_t)s * n_pts + i) * 3 + g) * 2;
                H[o] = h[g].real();
                H[o + 1] = h[g].imag();
            }
        }
    }
    return BIELCC_OK;
}

template <typename KType, size_t NV>
void run_op(int op, const cd* j, const double* x, const double (&cell)[NV][3], const NumParam& np, KType k,
            cd* res) {
    switch (op) {
        case BIELCC_OP_K_NEAR_SMOOTH: K_RotRot_Near_Smooth(j, x, cell, np, k, res); break;
        case BIELCC_OP_K_HS: K_RotRot_HS(j, x, cell, np, k, res); break;
        case BIELCC_OP_K_HS_COLLOC: K_RotRot_HS_Colloc(j, x, cell, np, k, res); break;
        case BIELCC_OP_K_HS2_COLLOC: K_RotRot_HS2_Colloc(j, x, cell, np, k, res); break;
        case BIELCC_OP_K_FAR: K_RotRot_Far(j, x, cell, np, k, res); break;
        case BIELCC_OP_R_SMOOTH: R_Rot_Smooth(j, x, cell, np, k, res); break;
        case BIELCC_OP_R_COLLOC: R_Rot_Colloc(j, x, cell, np, k, res); break;
        case BIELCC_OP_R_NEAR: R_Rot_Near(j, x, cell, np, k, res); break;
    }
}

template <typename KType>
KernelParam<KType> make_kp(const bielcc_kernelparam& s) {
    KernelParam<KType> p;
    p.smoothR = s.smoothR;
    p.smoothRMin = s.smoothRMin;
    p.k = make_k<KType>(s.k_re, s.k_im);
    for (int i = 0; i < 3; i++) {
        p.current[i] = cd(s.current[i][0], s.current[i][1]);
        p.vec_dbl[i] = s.vec_dbl[i];
        p.n[i] = s.n[i];
        p.e0[i] = s.e0[i];
    }
    return p;
}

template <typename KType>
void f_one(const double*, const double*, const KernelParam<KType>&, double* ff) { ff[0] = 1.; }
template <typename KType>
void f_one_x(const double*, const KernelParam<KType>&, double* ff) { ff[0] = 1.; }

// Runs `fn(f_real, f_cplx, idim)` with the reference integrand for `id`.
template <typename KType, typename Fn>
int with_integrand(int id, Fn fn) {
    using FR = void (*)(const double*, const double*, const KernelParam<KType>&, double*);
    using FC = void (*)(const double*, const double*, const KernelParam<KType>&, cd*);
    FR fr = nullptr;
    FC fc = nullptr;
    int idim = 1;
    switch (id) {
        case BIELCC_F_SIMPLEPOT_L: fr = F_SimplePot_L<KType>; idim = 1; break;
        case BIELCC_F_GRADSIMPLEPOT_L: fr = F_GradSimplePot_L<KType>; idim = 3; break;
        case BIELCC_F_DOUBLEPOT_L: fr = F_DoublePot_L<KType>; idim = 1; break;
        case BIELCC_F_VECTORPOT_L: fr = F_VectorPot_L<KType>; idim = 3; break;
        case BIELCC_F_SIMPLEPOT_H: fc = F_SimplePot_H<KType>; idim = 1; break;
        case BIELCC_F_NU_SIMPLEPOT_H: fc = nuF_SimplePot_H<KType>; idim = 3; break;
        case BIELCC_F_SIMPLEPOT_HM1: fc = F_SimplePot_Hm1<KType>; idim = 1; break;
        case BIELCC_F_GRADSIMPLEPOT_H: fc = F_GradSimplePot_H<KType>; idim = 3; break;
        case BIELCC_F_GRADSIMPLEPOT_HM1: fc = F_GradSimplePot_Hm1<KType>; idim = 3; break;
        case BIELCC_F_DOUBLEPOT_H: fc = F_DoublePot_H<KType>; idim = 1; break;
        case BIELCC_F_N_DOUBLEPOT_H: fc = nF_DoublePot_H<KType>; idim = 3; break;
        case BIELCC_F_ROTROTSIMPLEPOT_H: fc = F_RotRotSimplePot_H<KType>; idim = 3; break;
        case BIELCC_F_ONE: fr = f_one<KType>; idim = 1; break;
        default: return BIELCC_ERR_ARG;
    }
    fn(fr, fc, idim);
    return BIELCC_OK;
}

template <typename KType>
int integral_pnt_impl(int integrand, int n_vert, int n_pairs, const double* cells, const double* x,
                      bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    return with_integrand<KType>(integrand, [&](auto fr, auto fc, int idim) {
        for (int p = 0; p < n_pairs; p++) {
            KernelParam<KType> k = make_kp<KType>(kp[p]);
            IntegralParam ip(idim, n_start, p_max, eps);
            const double* xp = x + 3 * (size_t)p;
            if (n_vert == 4) {
                const auto& c = *reinterpret_cast<const double(*)[4][3]>(cells + (size_t)p * 12);
                if (fc) IntegralUniversalPnt(xp, c, fc, k, ip, reinterpret_cast<cd*>(res) + (size_t)idim * p);
                else IntegralUniversalPnt(xp, c, fr, k, ip, res + (size_t)idim * p);
            } else {
                const auto& c = *reinterpret_cast<const double(*)[3][3]>(cells + (size_t)p * 9);
                if (fc) IntegralUniversalPnt(xp, c, fc, k, ip, reinterpret_cast<cd*>(res) + (size_t)idim * p);
                else IntegralUniversalPnt(xp, c, fr, k, ip, res + (size_t)idim * p);
            }
            kp[p].smoothR = k.smoothR;
        }
    });
}

template <typename KType>
int integral_seg_impl(int integrand, int n_pairs, const double* a, const double* b, const double* x,
                      bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    return with_integrand<KType>(integrand, [&](auto fr, auto fc, int idim) {
        for (int p = 0; p < n_pairs; p++) {
            KernelParam<KType> k = make_kp<KType>(kp[p]);
            IntegralParam ip(idim, n_start, p_max, eps);
            size_t o = 3 * (size_t)p;
            if (fc) IntegralUniversalSegPnt(a + o, b + o, x + o, fc, k, ip, reinterpret_cast<cd*>(res) + (size_t)idim * p);
            else IntegralUniversalSegPnt(a + o, b + o, x + o, fr, k, ip, res + (size_t)idim * p);
            kp[p].smoothR = k.smoothR;
        }
    });
}

template <typename KType>
int k0_impl(int integrand, int common, int n_vert, int n_pairs, const double* cells, const double* x,
            const double* j, bielcc_kernelparam* kp, int n_seg, int p_seg, double eps, double* res) {
    return with_integrand<KType>(integrand, [&](auto, auto fc, int idim) {
        if (!fc || idim != 3) return;
        for (int p = 0; p < n_pairs; p++) {
            KernelParam<KType> k = make_kp<KType>(kp[p]);
            IntegralParam ip(3, n_seg, p_seg, eps);
            const double* xp = x + 3 * (size_t)p;
            cd* r = reinterpret_cast<cd*>(res) + 3 * (size_t)p;
            const cd* jp = reinterpret_cast<const cd*>(j) + 3 * (size_t)p;
            if (n_vert == 4) {
                const auto& c = *reinterpret_cast<const double(*)[4][3]>(cells + (size_t)p * 12);
                if (common) K0_Common(xp, c, fc, k, ip, r);
                else K0(jp, xp, c, fc, k, ip, r);
            } else {
                const auto& c = *reinterpret_cast<const double(*)[3][3]>(cells + (size_t)p * 9);
                if (common) K0_Common(xp, c, fc, k, ip, r);
                else K0(jp, xp, c, fc, k, ip, r);
            }
            kp[p].smoothR = k.smoothR;
        }
    });
}

}  // namespace

namespace {
// IntegralUniversal (integral_universal.h:252-431) and the segment F(x)
// overload (integral_universal_seg.h:120-179) with F = 1 or PlaneWaveFieldE
// (incident_field.h:20-29), the reference's own templates.
template <typename KType>
int integral_fx_impl(int integrand, int n_vert, int n_items, const double* cells, const double* a, const double* b,
                     bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    const int idim = integrand == BIELCC_F_ONE ? 1 : 3;
    if (integrand != BIELCC_F_ONE && integrand != BIELCC_F_PLANEWAVE_E) return BIELCC_ERR_ARG;
    for (int p = 0; p < n_items; p++) {
        KernelParam<KType> k = make_kp<KType>(kp[p]);
        IntegralParam ip(idim, n_start, p_max, eps);
        double* rr = res + (size_t)idim * p;
        cd* rc = reinterpret_cast<cd*>(res) + (size_t)idim * p;
        if (cells && n_vert == 4) {
            const auto& c = *reinterpret_cast<const double(*)[4][3]>(cells + (size_t)p * 12);
            if (integrand == BIELCC_F_ONE) IntegralUniversal(c, f_one_x<KType>, k, ip, rr);
            else IntegralUniversal(c, PlaneWaveFieldE<KType>, k, ip, rc);
        } else if (cells) {
            const auto& c = *reinterpret_cast<const double(*)[3][3]>(cells + (size_t)p * 9);
            if (integrand == BIELCC_F_ONE) IntegralUniversal(c, f_one_x<KType>, k, ip, rr);
            else IntegralUniversal(c, PlaneWaveFieldE<KType>, k, ip, rc);
        } else {
            size_t o = 3 * (size_t)p;
            if (integrand == BIELCC_F_ONE) IntegralUniversalSegPnt(a + o, b + o, f_one_x<KType>, k, ip, rr);
            else IntegralUniversalSegPnt(a + o, b + o, PlaneWaveFieldE<KType>, k, ip, rc);
        }
        kp[p].smoothR = k.smoothR;
    }
    return BIELCC_OK;
}

}  // namespace

extern "C" {

int ref_field_EH(int n_vert, int n_cells, const double* cells, int n_rhs, const double* J, double k_re,
                 double k_im, double mult_re, double mult_im, const bielcc_planewave* inc,
                 const bielcc_numparam* np, int n_pts, const double* pts, double* E, double* H, int n_threads) {
    if (n_vert == 4) {
        if (k_im == 0.)
            return field_impl<double, CellQuad, 4>(n_cells, cells, n_rhs, J, k_re, k_im, mult_re, mult_im, inc,
                                                   np, n_pts, pts, E, H, n_threads);
        return field_impl<cd, CellQuad, 4>(n_cells, cells, n_rhs, J, k_re, k_im, mult_re, mult_im, inc, np,
                                           n_pts, pts, E, H, n_threads);
    }
    if (n_vert == 3) {
        if (k_im == 0.)
            return field_impl<double, CellTriangle, 3>(n_cells, cells, n_rhs, J, k_re, k_im, mult_re, mult_im,
                                                       inc, np, n_pts, pts, E, H, n_threads);
        return field_impl<cd, CellTriangle, 3>(n_cells, cells, n_rhs, J, k_re, k_im, mult_re, mult_im, inc, np,
                                               n_pts, pts, E, H, n_threads);
    }
    return BIELCC_ERR_ARG;
}

int ref_pair_op(int op, int n_vert, int n_pairs, const double* cells, const double* x, const double* j,
                double k_re, double k_im, const bielcc_numparam* npp, double* res) {
    if (op < 0 || op >= BIELCC_OP_COUNT || (n_vert != 3 && n_vert != 4)) return BIELCC_ERR_ARG;
    NumParam np = make_np(npp);
#pragma omp parallel for
    for (int p = 0; p < n_pairs; p++) {
        const cd* jp = reinterpret_cast<const cd*>(j) + 3 * (size_t)p;
        const double* xp = x + 3 * (size_t)p;
        cd* r = reinterpret_cast<cd*>(res) + 3 * (size_t)p;
        if (n_vert == 4) {
            const auto& c = *reinterpret_cast<const double(*)[4][3]>(cells + (size_t)p * 12);
            if (k_im == 0.) run_op<double, 4>(op, jp, xp, c, np, k_re, r);
            else run_op<cd, 4>(op, jp, xp, c, np, cd(k_re, k_im), r);
        } else {
            const auto& c = *reinterpret_cast<const double(*)[3][3]>(cells + (size_t)p * 9);
            if (k_im == 0.) run_op<double, 3>(op, jp, xp, c, np, k_re, r);
            else run_op<cd, 3>(op, jp, xp, c, np, cd(k_re, k_im), r);
        }
    }
    return BIELCC_OK;
}

int ref_integral_pnt(int integrand, int n_vert, int n_pairs, const double* cells, const double* x,
                     bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    if (n_vert != 3 && n_vert != 4) return BIELCC_ERR_ARG;
    bool cplx = false;
    for (int p = 0; p < n_pairs; p++) cplx = cplx || kp[p].k_im != 0.;
    if (cplx) return integral_pnt_impl<cd>(integrand, n_vert, n_pairs, cells, x, kp, n_start, p_max, eps, res);
    return integral_pnt_impl<double>(integrand, n_vert, n_pairs, cells, x, kp, n_start, p_max, eps, res);
}

int ref_integral_seg_pnt(int integrand, int n_pairs, const double* a, const double* b, const double* x,
                         bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    bool cplx = false;
    for (int p = 0; p < n_pairs; p++) cplx = cplx || kp[p].k_im != 0.;
    if (cplx) return integral_seg_impl<cd>(integrand, n_pairs, a, b, x, kp, n_start, p_max, eps, res);
    return integral_seg_impl<double>(integrand, n_pairs, a, b, x, kp, n_start, p_max, eps, res);
}

int ref_integral(int integrand, int n_vert, int n_cells, const double* cells, bielcc_kernelparam* kp, int n_start,
                 int p_max, double eps, double* res) {
    if (n_vert != 3 && n_vert != 4) return BIELCC_ERR_ARG;
    return integral_fx_impl<double>(integrand, n_vert, n_cells, cells, nullptr, nullptr, kp, n_start, p_max, eps, res);
}

int ref_integral_seg(int integrand, int n_segs, const double* a, const double* b, bielcc_kernelparam* kp, int n_start,
                     int p_max, double eps, double* res) {
    return integral_fx_impl<double>(integrand, 0, n_segs, nullptr, a, b, kp, n_start, p_max, eps, res);
}

int ref_k0(int integrand, int common, int n_vert, int n_pairs, const double* cells, const double* x,
           const double* j, bielcc_kernelparam* kp, int n_seg, int p_seg, double eps, double* res) {
    bool cplx = false;
    for (int p = 0; p < n_pairs; p++) cplx = cplx || kp[p].k_im != 0.;
    if (cplx) return k0_impl<cd>(integrand, common, n_vert, n_pairs, cells, x, j, kp, n_seg, p_seg, eps, res);
    return k0_impl<double>(integrand, common, n_vert, n_pairs, cells, x, j, kp, n_seg, p_seg, eps, res);
}

int ref_integral_1divr(int n_vert, int n_pairs, const double* cells, const double* x, double* res) {
    for (int p = 0; p < n_pairs; p++) {
        if (n_vert == 4) res[p] = integral1Divr(*reinterpret_cast<const double(*)[4][3]>(cells + (size_t)p * 12), x + 3 * (size_t)p);
        else res[p] = integral1Divr(*reinterpret_cast<const double(*)[3][3]>(cells + (size_t)p * 9), x + 3 * (size_t)p);
    }
    return BIELCC_OK;
}

int ref_integral_grad1divr_seg(int n_pairs, const double* a, const double* b, const double* x, double* res) {
    for (int p = 0; p < n_pairs; p++)
        integralGrad1DivrSeg(a + 3 * (size_t)p, b + 3 * (size_t)p, x + 3 * (size_t)p, res + 3 * (size_t)p);
    return BIELCC_OK;
}

int ref_integral_surf_simplepot_h_hs(int n_vert, int n_pairs, const double* cells, const double* x,
                                     double analytic_r, int n_start, int p_max, double eps, double k_re,
                                     double k_im, double* res) {
    IntegralParam ip(1, n_start, p_max, eps);
    for (int p = 0; p < n_pairs; p++) {
        cd v;
        const double* xp = x + 3 * (size_t)p;
        if (n_vert == 4) {
            const auto& c = *reinterpret_cast<const double(*)[4][3]>(cells + (size_t)p * 12);
            v = (k_im == 0.) ? IntegralSurf_SimplePot_H_HS(c, xp, analytic_r, ip, k_re)
                             : IntegralSurf_SimplePot_H_HS(c, xp, analytic_r, ip, cd(k_re, k_im));
        } else {
            const auto& c = *reinterpret_cast<const double(*)[3][3]>(cells + (size_t)p * 9);
            v = (k_im == 0.) ? IntegralSurf_SimplePot_H_HS(c, xp, analytic_r, ip, k_re)
                             : IntegralSurf_SimplePot_H_HS(c, xp, analytic_r, ip, cd(k_re, k_im));
        }
        res[2 * p] = v.real();
        res[2 * p + 1] = v.imag();
    }
    return BIELCC_OK;
}

int ref_integral_seg_gradsimplepot_h_hs(int n_pairs, const double* a, const double* b, const double* x,
                                        double analytic_r, int n_start, int p_max, double eps, double k_re,
                                        double k_im, double* res) {
    IntegralParam ip(3, n_start, p_max, eps);
    for (int p = 0; p < n_pairs; p++) {
        size_t o = 3 * (size_t)p;
        cd* r = reinterpret_cast<cd*>(res) + o;
        if (k_im == 0.) IntegralSeg_GradSimplePot_H_HS(a + o, b + o, x + o, analytic_r, ip, k_re, r);
        else IntegralSeg_GradSimplePot_H_HS(a + o, b + o, x + o, analytic_r, ip, cd(k_re, k_im), r);
    }
    return BIELCC_OK;
}

int ref_area_by_quadrature(int n_vert, const double* cell, int n_start, int p_max, double eps, double* res) {
    KernelParam<double> kp;
    IntegralParam ip(1, n_start, p_max, eps);
    if (n_vert == 4)
        IntegralUniversal(*reinterpret_cast<const double(*)[4][3]>(cell), f_one_x<double>, kp, ip, res);
    else
        IntegralUniversal(*reinterpret_cast<const double(*)[3][3]>(cell), f_one_x<double>, kp, ip, res);
    return BIELCC_OK;
}

// Cell geometry as the reference's CellFill / element_geom compute it:
// centre(3), diam, norm_func normal(3), tau1(3), tau2(3), CellFill area (14).
int ref_cell_geometry(int n_vert, int n_cells, const double* cells, double* out) {
    for (int c = 0; c < n_cells; c++) {
        double* o = out + 14 * (size_t)c;
        if (n_vert == 4) {
            const auto& v = *reinterpret_cast<const double(*)[4][3]>(cells + (size_t)c * 12);
            CellQuad q;
            q.CellFill(v);
            get_center_mass(v, o);
            o[3] = get_diam(v);
            norm_func(v, o + 4);
            for (int g = 0; g < 3; g++) { o[7 + g] = q.GetTau1()[g]; o[10 + g] = q.GetTau2()[g]; }
            o[13] = q.GetArea();
        } else {
            const auto& v = *reinterpret_cast<const double(*)[3][3]>(cells + (size_t)c * 9);
            CellTriangle t;
            t.CellFill(v);
            get_center_mass(v, o);
            o[3] = get_diam(v);
            norm_func(v, o + 4);
            for (int g = 0; g < 3; g++) { o[7 + g] = t.GetTau1()[g]; o[10 + g] = t.GetTau2()[g]; }
            o[13] = t.GetArea();
        }
    }
    return BIELCC_OK;
}

// The reference's own readers, through their public entry
// SurfMesh<CellType>::ReadFromFile (mesh/surf_mesh.h:352-363), which picks
// ReadFromDatFile (mesh/surf_mesh.cpp:18-175) or ReadFromVtkFile
// (mesh/surf_mesh.h:388-555) by the file's extension; cells as
// GetCell(i).GetCellCoords(). Counts when cells is NULL; returns -10 when the
// reader throws. (fmt is the caller's expectation of the format.)
int ref_read_mesh(int fmt, int n_vert, const char* path, int* n_cells, double* cells) {
    (void)fmt;
    try {
        auto run = [&](auto& m) {
            m.ReadFromFile(path);
            const int n = m.GetNFrm();
            if (cells && *n_cells < n) return BIELCC_ERR_ARG;
            *n_cells = n;
            if (cells)
                for (int c = 0; c < n; c++) {
                    const auto& v = m.GetCell(c).GetCellCoords();
                    for (int a = 0; a < n_vert; a++)
                        for (int g = 0; g < 3; g++) cells[((size_t)c * n_vert + a) * 3 + g] = v[a][g];
                }
            return BIELCC_OK;
        };
        if (n_vert == 4) {
            SurfMesh<CellQuad> m;
            return run(m);
        }
        SurfMesh<CellTriangle> m;
        return run(m);
    } catch (const std::exception&) {
        return BIELCC_ERR_IO;
    }
}

// SurfaceCurrentsC_fromFiles (electrodynamics/currents.cpp:74-109): J as
// interleaved complex [n][3]; the vector is presized from the files' header
// (n1 x n2 values), since the reference writes into it by index.
int ref_read_currents(const char* path_re, const char* path_im, int* n, double* J) {
    std::ifstream f(path_re);
    int n1 = 0, n2 = 0;
    if (!(f >> n1 >> n2)) return BIELCC_ERR_IO;
    const int cnt = n1 * n2;
    if (!J) {
        *n = cnt;
        return BIELCC_OK;
    }
    if (*n < cnt) return BIELCC_ERR_ARG;
    std::vector<std::array<cd, 3>> j((size_t)cnt);
    try {
        SurfaceCurrentsC_fromFiles(path_re, path_im, j);
    } catch (const std::exception&) {
        return BIELCC_ERR_IO;
    }
    for (int i = 0; i < cnt; i++)
        for (int g = 0; g < 3; g++) {
            J[(6 * (size_t)i) + 2 * g] = j[i][g].real();
            J[(6 * (size_t)i) + 2 * g + 1] = j[i][g].imag();
        }
    *n = cnt;
    return BIELCC_OK;
}

// MaterialParam::Calc (electrodynamics/material.cpp:60-128) and
// RadiationSource::CalcK (radiation_source.cpp:159-180) of the reference.
// out: eps (re, im), mu (re, im), skin depth (0 if none), k of CalcK, and
// 1 if CalcK threw (it does for complex eps with its real mu), else 0.
int ref_material(int dispersion, double eps_r, double mu_r, double sigma, int n_table, const double* table,
                 double freq, double* out) {
    MaterialParam m;
    if (dispersion == BIELCC_DISPERSION_REFRACT) {
        std::map<double, double> n, ka;
        bool absorb = false;
        for (int i = 0; i < n_table; i++) {
            n[table[3 * i]] = table[3 * i + 1];
            ka[table[3 * i]] = table[3 * i + 2];
            absorb = absorb || table[3 * i + 2] != 0.;
        }
        if (absorb)
            m = MaterialParam("m", ChangeMaterialTypeDir::Isotropic, ChangeMaterialTypeFreq::DispersiveByRefractIndex,
                              n, ka, mu_r);
        else
            m = MaterialParam("m", ChangeMaterialTypeDir::Isotropic, ChangeMaterialTypeFreq::DispersiveByRefractIndex,
                              n, mu_r);
    } else {
        m = MaterialParam("m", ChangeMaterialTypeDir::Isotropic, ChangeMaterialTypeFreq::NonDispersive, eps_r, mu_r,
                          sigma, 0., 0.);
    }
    m.Calc(freq);
    const auto eps = m.GetEps(), mu = m.GetMu();
    const cd e = std::holds_alternative<double>(eps) ? cd(std::get<double>(eps), 0.) : std::get<cd>(eps);
    const cd u = std::holds_alternative<double>(mu) ? cd(std::get<double>(mu), 0.) : std::get<cd>(mu);
    out[0] = e.real();
    out[1] = e.imag();
    out[2] = u.real();
    out[3] = u.imag();
    out[4] = m.GetSkinDepth() ? *m.GetSkinDepth() : 0.;
    const double ort[3] = {0., 0., 1.}, e0[3] = {1., 0., 0.};
    RadiationSource src(RadiationSourceType::PlaneWave, ort, e0);
    out[5] = 0.;
    out[6] = 0.;
    try {
        src.CalcK(freq, m);
        out[5] = src.GetK();
    } catch (const std::bad_variant_access&) {
        out[6] = 1.;
    }
    return BIELCC_OK;
}

}  // extern "C"
