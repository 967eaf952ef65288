// bielcc_gpu.hpp — C++ drop-in layer over the C ABI (bielcc_gpu.h).
//
// Same names, template parameters and argument meaning as the reference's
// operator API (AlenaSetukha/BIELcc), in namespace bielcc_gpu so that both can
// be included side by side:
//   K_RotRot_Near_Smooth / _HS / _HS_Colloc / _HS2_Colloc / _Far   electrodynamics/K.h:47-301
//   R_Rot_Smooth / R_Rot_Colloc / R_Rot_Near                          electrodynamics/R.h:46-175
//   K0 / K0_Common                                                    electrodynamics/K0.h:36-166
//   IntegralUniversalPnt (quad, triangle)                             integrators/integral_universal.h:38-220
//   IntegralUniversal, the F(x) form (quad, triangle)                 integrators/integral_universal.h:252-431
//   IntegralUniversalSegPnt (F(x, y) and F(x) overloads)              integrators/integral_universal_seg.h:38-179
//   integral1Divr / integralGrad1DivrSeg                              integrators/integrals_analytic.h:31-50
//   IntegralSurf_SimplePot_H_HS / IntegralSeg_GradSimplePot_H_HS      integrators/integrals_analytic.h:136-221
//   GetFieldE_Ideal                                                   electrodynamics/get_field.h:35-78
// The parameter records are duck-typed: any NumParam with the fields eps, rs,
// rs_seg, analytic_calc, n_start, n_start_seg, p_max, p_max_seg; any
// KernelParam<KType> with smoothR, smoothRMin, k, current, vec_dbl, n, e0; any
// IntegralParam with GetIDim/GetNStart/GetPMax/GetEpsAccur; any SurfMesh with
// GetNFrm() and GetCell(i).GetCellCoords(). The reference's own types work.
//
// Integrands are the kernel_lib functions. When the reference's kernel_lib.h
// is included before this header, its function pointers (bielcc::F_*<KType>)
// are recognised, and so is bielcc::PlaneWaveFieldE<KType> (incident_field.h)
// as the F(x) integrand of IntegralUniversal; otherwise pass the BIELCC_F_* id.
// A user-written integrand cannot run on the device: such a call throws
// std::invalid_argument.
//
// Every call below is one batched GPU launch (the per-pair forms with a batch
// of one); for throughput use the *_batch forms or bielcc_field_EH directly.
// Errors from the C ABI are thrown as bielcc_gpu::Error (the reference has no
// error reporting; NaN results still propagate as NaN values).
#pragma once

#include <array>
#include <complex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "bielcc_gpu.h"

namespace bielcc_gpu {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != BIELCC_OK) throw Error(rc, std::string("bielcc: ") + bielcc_last_error());
}

// Process-wide context on device 0 unless set_context() installs another.
inline bielcc_ctx& context_slot() {
    static bielcc_ctx c = nullptr;
    return c;
}
inline bielcc_ctx context() {
    bielcc_ctx& c = context_slot();
    if (!c) check(bielcc_ctx_create(0, &c));
    return c;
}
inline void set_context(bielcc_ctx c) { context_slot() = c; }

template <typename NP>
inline bielcc_numparam to_numparam(const NP& n) {
    bielcc_numparam p;
    p.eps = n.eps;
    p.rs = n.rs;
    p.rs_seg = n.rs_seg;
    p.analytic_calc = n.analytic_calc;
    p.n_start = n.n_start;
    p.n_start_seg = n.n_start_seg;
    p.p_max = n.p_max;
    p.p_max_seg = n.p_max_seg;
    return p;
}

inline void split_k(double k, double* re, double* im) { *re = k; *im = 0.; }
inline void split_k(std::complex<double> k, double* re, double* im) { *re = k.real(); *im = k.imag(); }

template <typename JType>
inline std::complex<double> as_c(const JType& v) { return std::complex<double>(v); }

template <typename KP>
inline bielcc_kernelparam to_kernelparam(const KP& k) {
    bielcc_kernelparam p{};
    p.smoothR = k.smoothR;
    p.smoothRMin = k.smoothRMin;
    split_k(k.k, &p.k_re, &p.k_im);
    for (int i = 0; i < 3; i++) {
        std::complex<double> c(k.current[i]);
        p.current[i][0] = c.real();
        p.current[i][1] = c.imag();
        p.vec_dbl[i] = k.vec_dbl[i];
        p.n[i] = k.n[i];
        p.e0[i] = k.e0[i];
    }
    return p;
}

// ---------------------------------------------------------------- per-pair operators
template <int OP, typename JType, typename KType, size_t CellPoints, typename NP>
inline void pair_op(const JType* j, const double* x, const double (&cell)[CellPoints][3], const NP& num_param,
                    const KType k, std::complex<double>* res) {
    static_assert(CellPoints == 3 || CellPoints == 4, "cells have 3 or 4 vertices");
    double kr, ki;
    split_k(k, &kr, &ki);
    double jj[6];
    for (int i = 0; i < 3; i++) {
        std::complex<double> c = as_c(j[i]);
        jj[2 * i] = c.real();
        jj[2 * i + 1] = c.imag();
    }
    bielcc_numparam np = to_numparam(num_param);
    check(bielcc_pair_op(context(), OP, (int)CellPoints, 1, &cell[0][0], x, jj, kr, ki, &np,
                         reinterpret_cast<double*>(res)));
}

#define BIELCC_GPU_OPERATOR(NAME, OP)                                                                         \
    template <typename JType, typename KType, size_t CellPoints, typename NP>                                \
    inline void NAME(const JType* j, const double* x, const double (&cell)[CellPoints][3], const NP& num_param, \
                     const KType k, std::complex<double>* res) {                                               \
        pair_op<OP>(j, x, cell, num_param, k, res);                                                          \
    }
BIELCC_GPU_OPERATOR(K_RotRot_Near_Smooth, BIELCC_OP_K_NEAR_SMOOTH)
BIELCC_GPU_OPERATOR(K_RotRot_HS, BIELCC_OP_K_HS)
BIELCC_GPU_OPERATOR(K_RotRot_HS_Colloc, BIELCC_OP_K_HS_COLLOC)
BIELCC_GPU_OPERATOR(K_RotRot_HS2_Colloc, BIELCC_OP_K_HS2_COLLOC)
BIELCC_GPU_OPERATOR(K_RotRot_Far, BIELCC_OP_K_FAR)
BIELCC_GPU_OPERATOR(R_Rot_Smooth, BIELCC_OP_R_SMOOTH)
BIELCC_GPU_OPERATOR(R_Rot_Colloc, BIELCC_OP_R_COLLOC)
BIELCC_GPU_OPERATOR(R_Rot_Near, BIELCC_OP_R_NEAR)
#undef BIELCC_GPU_OPERATOR

// Batched form: one launch for many (cell, x, j) triples of one operator.
template <size_t CellPoints, typename NP, typename KType>
inline void pair_op_batch(int op, const std::vector<std::array<std::array<double, 3>, CellPoints>>& cells,
                          const std::vector<std::array<double, 3>>& x,
                          const std::vector<std::array<std::complex<double>, 3>>& j, const NP& num_param, KType k,
                          std::vector<std::array<std::complex<double>, 3>>& res) {
    if (cells.size() != x.size() || cells.size() != j.size()) throw std::invalid_argument("batch sizes differ");
    res.resize(cells.size());
    double kr, ki;
    split_k(k, &kr, &ki);
    bielcc_numparam np = to_numparam(num_param);
    check(bielcc_pair_op(context(), op, (int)CellPoints, (int)cells.size(), cells.empty() ? nullptr : &cells[0][0][0],
                         x.empty() ? nullptr : &x[0][0], j.empty() ? nullptr : reinterpret_cast<const double*>(&j[0][0]),
                         kr, ki, &np, res.empty() ? nullptr : reinterpret_cast<double*>(&res[0][0])));
}

// ---------------------------------------------------------------- integrands
// Maps a kernel_lib function pointer to its BIELCC_F_* id (needs the
// reference's kernel_lib.h included first), or passes an id through.
inline int integrand_id(int id) { return id; }
#ifdef _KERNEL_LIB_H_
template <typename KType, typename P>
inline int integrand_id(void (*f)(const double*, const double*, const bielcc::KernelParam<KType>&, P*)) {
    using F = void (*)(const double*, const double*, const bielcc::KernelParam<KType>&, P*);
    if constexpr (std::is_same<P, double>::value) {
        if (f == (F)bielcc::F_SimplePot_L<KType>) return BIELCC_F_SIMPLEPOT_L;
        if (f == (F)bielcc::F_GradSimplePot_L<KType>) return BIELCC_F_GRADSIMPLEPOT_L;
        if (f == (F)bielcc::F_DoublePot_L<KType>) return BIELCC_F_DOUBLEPOT_L;
        if (f == (F)bielcc::F_VectorPot_L<KType>) return BIELCC_F_VECTORPOT_L;
    } else {
        if (f == (F)bielcc::F_SimplePot_H<KType>) return BIELCC_F_SIMPLEPOT_H;
        if (f == (F)bielcc::nuF_SimplePot_H<KType>) return BIELCC_F_NU_SIMPLEPOT_H;
        if (f == (F)bielcc::F_SimplePot_Hm1<KType>) return BIELCC_F_SIMPLEPOT_HM1;
        if (f == (F)bielcc::F_GradSimplePot_H<KType>) return BIELCC_F_GRADSIMPLEPOT_H;
        if (f == (F)bielcc::F_GradSimplePot_Hm1<KType>) return BIELCC_F_GRADSIMPLEPOT_HM1;
        if (f == (F)bielcc::F_DoublePot_H<KType>) return BIELCC_F_DOUBLEPOT_H;
        if (f == (F)bielcc::nF_DoublePot_H<KType>) return BIELCC_F_N_DOUBLEPOT_H;
        if (f == (F)bielcc::F_RotRotSimplePot_H<KType>) return BIELCC_F_ROTROTSIMPLEPOT_H;
    }
    throw std::invalid_argument("integrand is not a kernel_lib function: it cannot run on the GPU");
}
#endif
#ifdef _INCIDENT_FIELD_H_
// F(x) integrands of IntegralUniversal: PlaneWaveFieldE (incident_field.h:20-29).
template <typename KType, typename P>
inline int integrand_id(void (*f)(const double*, const bielcc::KernelParam<KType>&, P*)) {
    using F = void (*)(const double*, const bielcc::KernelParam<KType>&, P*);
    if constexpr (std::is_same<P, std::complex<double>>::value) {
        if (f == (F)bielcc::PlaneWaveFieldE<KType>) return BIELCC_F_PLANEWAVE_E;
    }
    throw std::invalid_argument("F(x) integrand is not PlaneWaveFieldE: it cannot run on the GPU "
                                "(pass BIELCC_F_ONE for F = 1)");
}
#endif

// IntegralUniversalPnt: res receives idim values (double or complex); the
// kernel parameter's smoothR is left as the reference leaves it.
template <typename F, typename KP, typename IP, size_t CellPoints, typename P>
inline void IntegralUniversalPnt(const double* x, const double (&cell)[CellPoints][3], F f_0, KP& ker_param,
                                 const IP& int_param, P* res) {
    int id = integrand_id(f_0);
    bielcc_kernelparam kp = to_kernelparam(ker_param);
    check(bielcc_integral_pnt(context(), id, (int)CellPoints, 1, &cell[0][0], x, &kp, int_param.GetNStart(),
                              int_param.GetPMax(), int_param.GetEpsAccur(), reinterpret_cast<double*>(res)));
    ker_param.smoothR = kp.smoothR;
}

template <typename F, typename KP, typename IP, typename P>
inline void IntegralUniversalSegPnt(const double* a, const double* b, const double* x, F f_0, KP& ker_param,
                                    const IP& int_param, P* res) {
    int id = integrand_id(f_0);
    bielcc_kernelparam kp = to_kernelparam(ker_param);
    check(bielcc_integral_seg_pnt(context(), id, 1, a, b, x, &kp, int_param.GetNStart(), int_param.GetPMax(),
                                  int_param.GetEpsAccur(), reinterpret_cast<double*>(res)));
    ker_param.smoothR = kp.smoothR;
}

// IntegralUniversal, the F(x) form: f_0 is PlaneWaveFieldE or BIELCC_F_ONE.
template <typename F, typename KP, typename IP, size_t CellPoints, typename P>
inline void IntegralUniversal(const double (&cell)[CellPoints][3], F f_0, KP& ker_param, const IP& int_param,
                              P* res) {
    int id = integrand_id(f_0);
    bielcc_kernelparam kp = to_kernelparam(ker_param);
    check(bielcc_integral(context(), id, (int)CellPoints, 1, &cell[0][0], &kp, int_param.GetNStart(),
                          int_param.GetPMax(), int_param.GetEpsAccur(), reinterpret_cast<double*>(res)));
    ker_param.smoothR = kp.smoothR;
}

// IntegralUniversalSegPnt, the F(x) overload (integral_universal_seg.h:120-179).
template <typename F, typename KP, typename IP, typename P>
inline void IntegralUniversalSegPnt(const double* a, const double* b, F f_0, KP& ker_param, const IP& int_param,
                                    P* res) {
    int id = integrand_id(f_0);
    bielcc_kernelparam kp = to_kernelparam(ker_param);
    check(bielcc_integral_seg(context(), id, 1, a, b, &kp, int_param.GetNStart(), int_param.GetPMax(),
                              int_param.GetEpsAccur(), reinterpret_cast<double*>(res)));
    ker_param.smoothR = kp.smoothR;
}

template <typename P, typename F, typename KP, typename IP, size_t CellPoints>
inline void K0(const P* j, const double* x, const double (&cell)[CellPoints][3], F f_0, KP& ker_param,
               const IP& int_param, P* res) {
    int id = integrand_id(f_0);
    bielcc_kernelparam kp = to_kernelparam(ker_param);
    double jj[6];
    for (int i = 0; i < 3; i++) {
        std::complex<double> c = as_c(j[i]);
        jj[2 * i] = c.real();
        jj[2 * i + 1] = c.imag();
    }
    check(bielcc_k0(context(), id, 0, (int)CellPoints, 1, &cell[0][0], x, jj, &kp, int_param.GetNStart(),
                    int_param.GetPMax(), int_param.GetEpsAccur(), reinterpret_cast<double*>(res)));
    ker_param.smoothR = kp.smoothR;
}

template <typename P, typename F, typename KP, typename IP, size_t CellPoints>
inline void K0_Common(const double* x, const double (&cell)[CellPoints][3], F f_0, KP& ker_param, const IP& int_param,
                      P* res) {
    int id = integrand_id(f_0);
    bielcc_kernelparam kp = to_kernelparam(ker_param);
    check(bielcc_k0(context(), id, 1, (int)CellPoints, 1, &cell[0][0], x, nullptr, &kp, int_param.GetNStart(),
                    int_param.GetPMax(), int_param.GetEpsAccur(), reinterpret_cast<double*>(res)));
    ker_param.smoothR = kp.smoothR;
}

// ---------------------------------------------------------------- analytic integrals
template <size_t CellPoints>
inline double integral1Divr(const double (&cell)[CellPoints][3], const double* x) {
    double r = 0.;
    check(bielcc_integral_1divr(context(), (int)CellPoints, 1, &cell[0][0], x, &r));
    return r;
}
inline void integralGrad1DivrSeg(const double* A, const double* B, const double* x, double* res) {
    check(bielcc_integral_grad1divr_seg(context(), 1, A, B, x, res));
}
template <size_t CellPoints, typename IP, typename KType>
inline std::complex<double> IntegralSurf_SimplePot_H_HS(const double (&cell)[CellPoints][3], const double* x,
                                                        double analyticR_r, const IP& int_param, KType k_wave) {
    double kr, ki, r[2];
    split_k(k_wave, &kr, &ki);
    check(bielcc_integral_surf_simplepot_h_hs(context(), (int)CellPoints, 1, &cell[0][0], x, analyticR_r,
                                              int_param.GetNStart(), int_param.GetPMax(), int_param.GetEpsAccur(),
                                              kr, ki, r));
    return {r[0], r[1]};
}
template <typename IP, typename KType>
inline void IntegralSeg_GradSimplePot_H_HS(const double* A, const double* B, const double* x, double analyticR_r,
                                           const IP& int_param, KType k_wave, std::complex<double>* res) {
    double kr, ki;
    split_k(k_wave, &kr, &ki);
    check(bielcc_integral_seg_gradsimplepot_h_hs(context(), 1, A, B, x, analyticR_r, int_param.GetNStart(),
                                                 int_param.GetPMax(), int_param.GetEpsAccur(), kr, ki,
                                                 reinterpret_cast<double*>(res)));
}

// ---------------------------------------------------------------- field driver
// Flattens a SurfMesh-like container into [N][nv][3].
template <typename Mesh>
inline std::vector<double> mesh_cells(const Mesh& surf_mesh, int* nv_out) {
    int n = surf_mesh.GetNFrm();
    std::vector<double> out;
    int nv = 0;
    for (int c = 0; c < n; c++) {
        const auto& v = surf_mesh.GetCell(c).GetCellCoords();
        nv = (int)(sizeof(v) / sizeof(v[0]));
        for (int a = 0; a < nv; a++)
            for (int g = 0; g < 3; g++) out.push_back(v[a][g]);
    }
    *nv_out = nv;
    return out;
}

// GetFieldE_Ideal (electrodynamics/get_field.h:35-78): field_E[i] =
// mult * sum_j K[cell_j, j_E[j]](points[i]) + EInc_Func(points[i]). The
// incident term is evaluated by EInc_Func on the host (O(points), not the
// O(points x cells) hot path); the reference's PlaneWaveFieldE can be passed
// as is. field_E must be presized to points.size() (written by index).
template <typename Mesh, typename KP, typename P, typename NP>
inline void GetFieldE_Ideal(const Mesh& surf_mesh, const std::vector<std::array<std::complex<double>, 3>>& j_E,
                            std::complex<double> mult, const KP& EInc_param,
                            void (*EInc_Func)(const double*, const KP&, P*), const NP& num_param,
                            const std::vector<std::array<double, 3>>& points,
                            std::vector<std::array<std::complex<double>, 3>>& field_E) {
    // the reference sums over the mesh's GetNFrm() cells, reading j_E[j] for each
    // (get_field.h:47-55): extra currents are ignored, missing ones are an error
    const int n_frm = surf_mesh.GetNFrm();
    if (j_E.size() < (size_t)n_frm) throw std::invalid_argument("j_E holds fewer currents than the mesh has cells");
    if (field_E.size() < points.size()) throw std::invalid_argument("field_E must be presized to points.size()");
    int nv = 0;
    std::vector<double> cells = mesh_cells(surf_mesh, &nv);
    if (n_frm == 0) {  // no cells: the incident field alone
        for (size_t i = 0; i < points.size(); i++) {
            P e_inc[3] = {};
            EInc_Func(points[i].data(), EInc_param, e_inc);
            for (int g = 0; g < 3; g++) field_E[i][g] = e_inc[g];
        }
        return;
    }
    bielcc_ctx ctx = context();
    bielcc_mesh m = 0;
    check(bielcc_mesh_create(ctx, nv, n_frm, cells.data(), &m));
    double kr, ki;
    split_k(EInc_param.k, &kr, &ki);
    bielcc_numparam np = to_numparam(num_param);
    int rc = bielcc_field_EH(ctx, m, 1, reinterpret_cast<const double*>(j_E.data()), kr, ki, mult.real(), mult.imag(),
                             nullptr, &np, (int)points.size(), points.empty() ? nullptr : &points[0][0],
                             field_E.empty() ? nullptr : reinterpret_cast<double*>(&field_E[0][0]), nullptr,
                             BIELCC_PREC_FP64, nullptr);
    bielcc_mesh_destroy(ctx, m);
    if (rc != BIELCC_ERR_NAN) check(rc);
    for (size_t i = 0; i < points.size(); i++) {
        P e_inc[3] = {};
        EInc_Func(points[i].data(), EInc_param, e_inc);
        for (int g = 0; g < 3; g++) field_E[i][g] += e_inc[g];
    }
}

}  // namespace bielcc_gpu
