// ops.cuh — generic FP64 per-pair device operators: the kernel_lib integrands,
// the adaptive universal quadratures (cell and segment), the contour
// operators, the analytic singular integrals and the K / R operators.
//
// One (point, cell) pair is evaluated by one thread, with the adaptive
// n -> 2n refinement and smoothing-radius schedule of the reference, nodes
// generated on the fly. These serve the per-pair C-ABI calls, the FP64 near
// pairs of the field driver and the near / singular entries of the
// collocation assembly. The far bulk uses the precomputed-node kernels in
// field.cu / assemble.cu instead.
#pragma once
#include "common.cuh"

namespace bielcc_gpu {

// Cell held in registers / local memory: nv = 4 (CellQuad) or 3 (CellTriangle).
struct DCell {
    int nv;
    double v[4][3];
};

// KernelParam<KType> (integrators/kernel_param.h:25-57), the fields read here.
struct DKP {
    double smoothR, smoothRMin;
    cplx k;
    cplx current[3];
    double vec_dbl[3];
    double n[3];
    double e0[3];
};

BIELCC_D void dkp_zero(DKP& p) {
    p.smoothR = p.smoothRMin = 0.;
    p.k = mk(0, 0);
    for (int i = 0; i < 3; i++) {
        p.current[i] = mk(0, 0);
        p.vec_dbl[i] = p.n[i] = p.e0[i] = 0.;
    }
}

// ------------------------------------------------------------------ cell geometry
// get_center_mass (geometry/element_geom.cpp:320-342)
BIELCC_D void cell_centre(const DCell& c, double* y) {
    for (int i = 0; i < 3; i++) {
        if (c.nv == 4) y[i] = (c.v[0][i] + c.v[1][i] + c.v[2][i] + c.v[3][i]) * 0.25;
        else y[i] = (c.v[0][i] + c.v[1][i] + c.v[2][i]) / 3.;
    }
}
// get_diam (element_geom.cpp:275-317)
BIELCC_D double cell_diam(const DCell& c) {
    if (c.nv == 4) {
        double d1[3], d2[3];
        for (int g = 0; g < 3; g++) { d1[g] = c.v[2][g] - c.v[0][g]; d2[g] = c.v[3][g] - c.v[1][g]; }
        double l1 = len3(d1), l2 = len3(d2);
        double best = l1 > l2 ? l1 : l2;
        for (int s = 0; s < 4; s++) {
            double e[3];
            for (int g = 0; g < 3; g++) e[g] = c.v[(s + 1) & 3][g] - c.v[s][g];
            double l = len3(e);
            if (l > best) best = l;
        }
        return best;
    }
    double l1 = dist3(c.v[0], c.v[1]), l2 = dist3(c.v[1], c.v[2]), l3 = dist3(c.v[2], c.v[0]);
    return fmax(fmax(l1, l2), l3);
}
// norm_func (element_geom.cpp:130-156)
BIELCC_D void cell_normal(const DCell& c, double* nrm) {
    double a[3], b[3], v[3];
    if (c.nv == 4) {
        for (int i = 0; i < 3; i++) { a[i] = c.v[2][i] - c.v[0][i]; b[i] = c.v[3][i] - c.v[1][i]; }
    } else {
        for (int i = 0; i < 3; i++) { a[i] = c.v[1][i] - c.v[0][i]; b[i] = c.v[2][i] - c.v[0][i]; }
    }
    cross3(a, b, v);
    double l = len3(v);
    for (int i = 0; i < 3; i++) nrm[i] = v[i] / l;
}
// tr_square (element_geom.cpp:54-66)
BIELCC_D double tri_area(const double* p1, const double* p2, const double* p3) {
    double ab[3], ac[3], n[3];
    for (int i = 0; i < 3; i++) { ab[i] = p2[i] - p1[i]; ac[i] = p3[i] - p1[i]; }
    cross3(ab, ac, n);
    return sqrt(dot3(n, n)) / 2.;
}
// Edge nu of K0 (electrodynamics/K0.h:72-80): (B - A) x n, normalised unless
// its length is <= MACHINE_ZERO.
BIELCC_D void edge_nu(const double* A, const double* B, const double* nrm, double* nu) {
    double d[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    cross3(d, nrm, nu);
    double l = len3(nu);
    if (l > kMachineZero)
        for (int g = 0; g < 3; g++) nu[g] /= l;
}

// ------------------------------------------------------------------ integrands
// kernel_lib.h, "all functions without 1/4pi" (kernel_lib.h:38). The smoothed
// weights keep the reference's 0/1 arithmetic so NaN/Inf behave the same.
enum Integrand {
    F_SIMPLEPOT_L = 0, F_GRADSIMPLEPOT_L, F_DOUBLEPOT_L, F_VECTORPOT_L, F_SIMPLEPOT_H, F_NU_SIMPLEPOT_H,
    F_SIMPLEPOT_HM1, F_GRADSIMPLEPOT_H, F_GRADSIMPLEPOT_HM1, F_DOUBLEPOT_H, F_N_DOUBLEPOT_H,
    F_ROTROTSIMPLEPOT_H, F_ONE, F_PLANEWAVE_E, F_COUNT
};
// Integrands of one point, F(x) (IntegralUniversal, integral_universal.h:252-431):
// evaluated at the node y, the pair point x unused.
BIELCC_HD bool integrand_one_point(int id) { return id == F_ONE || id == F_PLANEWAVE_E; }
BIELCC_HD int integrand_dim(int id) {
    return (id == F_SIMPLEPOT_L || id == F_DOUBLEPOT_L || id == F_SIMPLEPOT_H || id == F_SIMPLEPOT_HM1 ||
            id == F_DOUBLEPOT_H || id == F_ONE) ? 1 : 3;
}
BIELCC_HD bool integrand_complex(int id) {
    return !(id == F_SIMPLEPOT_L || id == F_GRADSIMPLEPOT_L || id == F_DOUBLEPOT_L || id == F_VECTORPOT_L ||
             id == F_ONE);
}

BIELCC_D double w_pot(double t, double r, double R) {  // F_SimplePot_* bracket
    return (double)(t < 1) * (t * (3. - 2. * t) / R) + (double)(t >= 1) / r;
}
BIELCC_D double w_grad(double t, double r, double R) {  // gradient / double-layer bracket
    return (double)(t < 1) * (3. - 2. * t) / (r * (R * R)) + (double)(t >= 1) / ((r * r) * r);
}

// Real-valued integrands (kernel_lib.h:62-177, + F = 1).
BIELCC_D void eval_real(int id, const double* x, const double* y, const DKP& p, double* out) {
    switch (id) {
        case F_SIMPLEPOT_L: {  // kernel_lib.h:62-69
            double r = dist3(x, y), t = r / p.smoothR;
            out[0] = w_pot(t, r, p.smoothR);
        } break;
        case F_GRADSIMPLEPOT_L: {  // kernel_lib.h:87-98
            double r = dist3(x, y), t = r / p.smoothR, w = w_grad(t, r, p.smoothR);
            for (int i = 0; i < 3; i++) out[i] = (y[i] - x[i]) * w;
        } break;
        case F_DOUBLEPOT_L: {  // kernel_lib.h:117-129
            double r = dist3(x, y), t = r / p.smoothR;
            double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
            out[0] = dot3(p.n, d) * w_grad(t, r, p.smoothR);
        } break;
        case F_VECTORPOT_L: {  // kernel_lib.h:149-177
            double r = dist3(x, y);
            if (r < kMachineZero) { out[0] = out[1] = out[2] = 0.; break; }
            double f = 1. / r / r / r;
            double d[3] = {(y[0] - x[0]) * f, (y[1] - x[1]) * f, (y[2] - x[2]) * f};
            cross3(d, p.vec_dbl, out);
            if (r < p.smoothR) {
                double t = r / p.smoothR;
                for (int i = 0; i < 3; i++) out[i] = out[i] * (3 * t * t - 2 * t * t * t);
            }
        } break;
        default: out[0] = 1.; break;  // F = 1
    }
}

// Complex-valued integrands (kernel_lib.h:209-492).
BIELCC_D void eval_cplx(int id, const double* x, const double* y, const DKP& p, cplx* out) {
    double r = dist3(x, y);
    switch (id) {
        case F_SIMPLEPOT_H: {  // kernel_lib.h:209-217
            double t = r / p.smoothR;
            out[0] = eikr(r, p.k) * w_pot(t, r, p.smoothR);
        } break;
        case F_NU_SIMPLEPOT_H: {  // kernel_lib.h:235-245
            double t = r / p.smoothR;
            cplx f = eikr(r, p.k) * w_pot(t, r, p.smoothR);
            for (int i = 0; i < 3; i++) out[i] = p.vec_dbl[i] * f;
        } break;
        case F_SIMPLEPOT_HM1: {  // kernel_lib.h:262-278
            cplx ikr = mk(-r * p.k.im, r * p.k.re);
            if (cabs(ikr) < 1e-7) {
                out[0] = mk(-p.k.im, p.k.re) - (p.k * p.k) * r / 2.;
            } else {
                double t = r / p.smoothR;
                cplx e = eikr(r, p.k);
                out[0] = mk(e.re - 1., e.im) * w_pot(t, r, p.smoothR);
            }
        } break;
        case F_GRADSIMPLEPOT_H: {  // kernel_lib.h:295-313
            double t = r / p.smoothR, w = w_grad(t, r, p.smoothR);
            cplx e = eikr(r, p.k);
            cplx ikr_m1 = mk(-r * p.k.im - 1., r * p.k.re);
            for (int i = 0; i < 3; i++) out[i] = ((x[i] - y[i]) * e) * ikr_m1 * w;
        } break;
        case F_GRADSIMPLEPOT_HM1: {  // kernel_lib.h:332-356
            cplx ikr = mk(-r * p.k.im, r * p.k.re);
            double a = cabs(ikr);
            if (a < 1e-6) {
                out[0] = out[1] = out[2] = mk(0, 0);
            } else if (a < 1e-4) {
                for (int i = 0; i < 3; i++) out[i] = ((y[i] - x[i]) * p.k) * p.k / (2. * r);
            } else {
                cplx e = eikr(r, p.k);
                cplx num = mk(1., 0.) + mk(ikr.re - 1., ikr.im) * e;
                for (int i = 0; i < 3; i++) out[i] = (x[i] - y[i]) * num / (r * r * r);
            }
        } break;
        case F_DOUBLEPOT_H:      // kernel_lib.h:375-390
        case F_N_DOUBLEPOT_H: {  // kernel_lib.h:409-419
            double t = r / p.smoothR;
            double d[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
            cplx ikr_m1 = mk(-r * p.k.im - 1., r * p.k.re);
            cplx v = dot3(p.n, d) * eikr(r, p.k) * ikr_m1 * w_grad(t, r, p.smoothR);
            if (id == F_DOUBLEPOT_H) out[0] = v;
            else for (int i = 0; i < 3; i++) out[i] = p.n[i] * v;
        } break;
        case F_PLANEWAVE_E: {  // PlaneWaveFieldE (electrodynamics/incident_field.h:20-29), at the node y
            double sn, cs;
            sincos(dot3(p.vec_dbl, y), &sn, &cs);
            for (int i = 0; i < 3; i++) out[i] = mk(p.e0[i] * cs, p.e0[i] * sn);
        } break;
        case F_ROTROTSIMPLEPOT_H: {  // kernel_lib.h:453-492
            if (r < kMachineZero) { out[0] = out[1] = out[2] = mk(0, 0); break; }
            cplx ik = mk(-p.k.im, p.k.re);
            cplx k2 = p.k * p.k;
            double dh[3];
            for (int i = 0; i < 3; i++) dh[i] = (x[i] - y[i]) / r;
            double ir3 = 1.0 / (r * r) / r, r2 = r * r;
            cplx f1 = mk(-ir3, 0.) + ik / r2 + k2 / r;
            cplx f2 = mk(3.0 * ir3, 0.) - (3.0 * ik) / r2 - k2 / r;
            cplx e = eikr(r, p.k);
            f2 *= cdot_cr(p.current, dh);
            for (int i = 0; i < 3; i++) out[i] = (dh[i] * f2 + p.current[i] * f1) * e;
            if (r < p.smoothR) {
                double t = r / p.smoothR;
                for (int i = 0; i < 3; i++) out[i] *= (t * t * (3 - 2 * t));
            }
        } break;
        default: out[0] = out[1] = out[2] = mk(0, 0); break;
    }
}

// F_SimplePot_H and F_GradSimplePot_H at one node together: the same r, t and
// e^{ikr}, each output by the expression eval_cplx uses for it alone.
BIELCC_D void eval_pot_and_grad(const double* x, const double* y, const DKP& p, cplx* f, cplx* g) {
    double r = dist3(x, y);
    double t = r / p.smoothR;
    cplx e = eikr(r, p.k);
    f[0] = e * w_pot(t, r, p.smoothR);
    double w = w_grad(t, r, p.smoothR);
    cplx ikr_m1 = mk(-r * p.k.im - 1., r * p.k.re);
    for (int i = 0; i < 3; i++) g[i] = ((x[i] - y[i]) * e) * ikr_m1 * w;
}

template <typename T> struct Eval;
template <> struct Eval<double> {
    BIELCC_D static void run(int id, const double* x, const double* y, const DKP& p, double* o) { eval_real(id, x, y, p, o); }
    BIELCC_D static double zero() { return 0.; }
    BIELCC_D static double absdiff2(double a, double b) { return (a - b) * (a - b); }
};
template <> struct Eval<cplx> {
    BIELCC_D static void run(int id, const double* x, const double* y, const DKP& p, cplx* o) { eval_cplx(id, x, y, p, o); }
    BIELCC_D static cplx zero() { return mk(0, 0); }
    BIELCC_D static double absdiff2(cplx a, cplx b) { return cabs2(a - b); }
};
BIELCC_D double madd(double acc, double f, double s) { return acc + f * s; }
BIELCC_D cplx madd(cplx acc, cplx f, double s) { return acc + f * s; }

// ------------------------------------------------------------------ universal quadrature
// Shared adaptive driver (integral_universal.h:58-119, :160-219;
// integral_universal_seg.h:57-97): pass at n; stop when the L2 change is
// below eps (never after the first pass); else n -> 2n and the smoothing
// radius is halved once per component while above smoothRMin and p < 8; an
// exhausted budget returns the previous pass.
template <typename T, typename Pass>
BIELCC_D void adaptive(int n_start, int p_max, double eps, int idim, DKP& kp, T* res, Pass pass) {
    T prev[3] = {Eval<T>::zero(), Eval<T>::zero(), Eval<T>::zero()};
    for (int g = 0; g < idim; g++) res[g] = Eval<T>::zero();
    int n = n_start, p;
    for (p = 0; p < p_max; p++) {
        pass(n, res);
        double delta = 0.;
        for (int g = 0; g < idim; g++) {
            double a = sqrt(Eval<T>::absdiff2(res[g], prev[g]));
            delta += a * a;
        }
        if (delta < eps * eps && p != 0) break;
        n *= 2;
        for (int g = 0; g < idim; g++) {
            prev[g] = res[g];
            res[g] = Eval<T>::zero();
            if (p < 8 && kp.smoothR > kp.smoothRMin) kp.smoothR /= 2.;
        }
    }
    if (p == p_max)
        for (int g = 0; g < idim; g++) res[g] = prev[g];
}

// Bilinear sub-cell (i, j) of an n x n split of a quad: centre y and area s
// (integral_universal.h:59-87).
BIELCC_D void quad_node(const double (*c)[3], int i, int j, int n, double* y, double* s) {
    double p0 = (double)i / (double)n, q0 = (double)j / (double)n;
    double p1 = ((double)i + 1.) / (double)n, q1 = ((double)j + 1.) / (double)n;
    double c1[3], c2[3], c3[3], c4[3], m1[3], m2[3], nr[3];
    for (int k = 0; k < 3; k++) {
        double lo = q0 * c[1][k] + (1 - q0) * c[0][k];
        double hi = q0 * c[2][k] + (1 - q0) * c[3][k];
        c1[k] = p0 * hi + (1 - p0) * lo;
        c4[k] = p1 * hi + (1 - p1) * lo;
        lo = q1 * c[1][k] + (1 - q1) * c[0][k];
        hi = q1 * c[2][k] + (1 - q1) * c[3][k];
        c2[k] = p0 * hi + (1 - p0) * lo;
        c3[k] = p1 * hi + (1 - p1) * lo;
    }
    for (int k = 0; k < 3; k++) {
        y[k] = (c1[k] + c2[k] + c3[k] + c4[k]) / 4.0;
        m1[k] = ((c2[k] + c3[k]) - (c1[k] + c4[k])) / 2.0;
        m2[k] = ((c3[k] + c4[k]) - (c1[k] + c2[k])) / 2.0;
    }
    cross3(m1, m2, nr);
    *s = len3(nr);
}

// IntegralUniversalPnt over a quad (integral_universal.h:38-120).
template <typename T>
BIELCC_D void integral_quad(int id, const double* x, const double (*c)[3], DKP& kp, int idim, int n_start, int p_max,
                            double eps, T* res) {
    adaptive<T>(n_start, p_max, eps, idim, kp, res, [&](int n, T* acc) {
        T ff[3];
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double y[3], s;
                quad_node(c, i, j, n, y, &s);
                Eval<T>::run(id, x, y, kp, ff);
                for (int g = 0; g < idim; g++) acc[g] = madd(acc[g], ff[g], s);
            }
    });
}

// IntegralUniversalPnt over a triangle (integral_universal.h:136-220): n^2
// sub-triangle centroids summed, then scaled by area / n / n.
template <typename T>
BIELCC_D void integral_tri(int id, const double* x, const double (*c)[3], DKP& kp, int idim, int n_start, int p_max,
                           double eps, T* res) {
    double area = tri_area(c[0], c[1], c[2]);
    adaptive<T>(n_start, p_max, eps, idim, kp, res, [&](int n, T* acc) {
        double pv[3], qv[3], rv[3];
        for (int k = 0; k < 3; k++) {
            pv[k] = (c[1][k] - c[0][k]) / n;
            qv[k] = (c[2][k] - c[0][k]) / n;
            rv[k] = (c[2][k] - c[1][k]) / n;
        }
        T ff[3];
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n - i; j++) {
                double B[3], y[3];
                for (int k = 0; k < 3; k++) {
                    B[k] = c[0][k] + (i + 1) * pv[k] + j * qv[k];
                    double A = B[k] - pv[k];
                    y[k] = (B[k] + A + (A + qv[k])) / 3.0;
                }
                Eval<T>::run(id, x, y, kp, ff);
                for (int g = 0; g < idim; g++) acc[g] = madd(acc[g], ff[g], 1.0);
                if (j < n - 1 - i) {
                    for (int k = 0; k < 3; k++) y[k] = (B[k] + (B[k] + rv[k]) + (B[k] + qv[k])) / 3.0;
                    Eval<T>::run(id, x, y, kp, ff);
                    for (int g = 0; g < idim; g++) acc[g] = madd(acc[g], ff[g], 1.0);
                }
            }
        for (int g = 0; g < idim; g++) acc[g] = acc[g] * area / (double)n / (double)n;
    });
}

template <typename T>
BIELCC_D void integral_cell(int id, const double* x, const DCell& c, DKP& kp, int idim, int n_start, int p_max,
                            double eps, T* res) {
    if (c.nv == 4) integral_quad<T>(id, x, c.v, kp, idim, n_start, p_max, eps, res);
    else integral_tri<T>(id, x, c.v, kp, idim, n_start, p_max, eps, res);
}

// One pass (p_max = 1) of IntegralUniversalPnt for F_SimplePot_H (F) and
// F_GradSimplePot_H (G) over one cell with the same smoothing radius: the
// nodes, weights and accumulation order of integral_quad / integral_tri, with
// each node evaluated once for both integrands.
BIELCC_D void integral_cell_pot_and_grad(const double* x, const DCell& c, const DKP& kp, int n, cplx* F, cplx* G) {
    F[0] = mk(0, 0);
    for (int g = 0; g < 3; g++) G[g] = mk(0, 0);
    cplx f[1], gg[3];
    if (c.nv == 4) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double y[3], s;
                quad_node(c.v, i, j, n, y, &s);
                eval_pot_and_grad(x, y, kp, f, gg);
                F[0] = madd(F[0], f[0], s);
                for (int g = 0; g < 3; g++) G[g] = madd(G[g], gg[g], s);
            }
        return;
    }
    const double(*cv)[3] = c.v;
    double area = tri_area(cv[0], cv[1], cv[2]);
    double pv[3], qv[3], rv[3];
    for (int k = 0; k < 3; k++) {
        pv[k] = (cv[1][k] - cv[0][k]) / n;
        qv[k] = (cv[2][k] - cv[0][k]) / n;
        rv[k] = (cv[2][k] - cv[1][k]) / n;
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n - i; j++) {
            double B[3], y[3];
            for (int k = 0; k < 3; k++) {
                B[k] = cv[0][k] + (i + 1) * pv[k] + j * qv[k];
                double A = B[k] - pv[k];
                y[k] = (B[k] + A + (A + qv[k])) / 3.0;
            }
            eval_pot_and_grad(x, y, kp, f, gg);
            F[0] = madd(F[0], f[0], 1.0);
            for (int g = 0; g < 3; g++) G[g] = madd(G[g], gg[g], 1.0);
            if (j < n - 1 - i) {
                for (int k = 0; k < 3; k++) y[k] = (B[k] + (B[k] + rv[k]) + (B[k] + qv[k])) / 3.0;
                eval_pot_and_grad(x, y, kp, f, gg);
                F[0] = madd(F[0], f[0], 1.0);
                for (int g = 0; g < 3; g++) G[g] = madd(G[g], gg[g], 1.0);
            }
        }
    F[0] = F[0] * area / (double)n / (double)n;
    for (int g = 0; g < 3; g++) G[g] = G[g] * area / (double)n / (double)n;
}

// IntegralUniversalSegPnt (integral_universal_seg.h:38-98).
template <typename T>
BIELCC_D void integral_seg(int id, const double* a, const double* b, const double* x, DKP& kp, int idim, int n_start,
                           int p_max, double eps, T* res) {
    adaptive<T>(n_start, p_max, eps, idim, kp, res, [&](int n, T* acc) {
        double d[3], y[3];
        for (int k = 0; k < 3; k++) d[k] = (b[k] - a[k]) / n;
        double dl = len3(d);
        T ff[3];
        for (int i = 0; i < n; i++) {
            for (int k = 0; k < 3; k++) y[k] = a[k] + (i + 0.5) * d[k];
            Eval<T>::run(id, x, y, kp, ff);
            for (int g = 0; g < idim; g++) acc[g] = madd(acc[g], ff[g], dl);
        }
    });
}

// ------------------------------------------------------------------ contour operators
// K0 (electrodynamics/K0.h:36-86): -sum_e (j . nu_e) int_e F; kp shared across
// edges (its smoothR keeps shrinking from edge to edge, as in the reference).
// When `mat` is given, the j-independent 3x3 matrix M = -sum_e ks_e nu_e^T is
// accumulated instead (K0 = M j).
BIELCC_D void K0_dev(int id, const cplx* j, const double* x, const DCell& c, DKP& kp, int n_seg, int p_seg, double eps,
                     cplx* res, cplx (*mat)[3] = nullptr) {
    double nrm[3];
    cell_normal(c, nrm);
    for (int g = 0; g < 3; g++) {
        res[g] = mk(0, 0);
        if (mat) mat[g][0] = mat[g][1] = mat[g][2] = mk(0, 0);
    }
    for (int s = 0; s < c.nv; s++) {
        const double* A = c.v[s];
        const double* B = c.v[(s + 1) % c.nv];
        cplx ks[3];
        integral_seg<cplx>(id, A, B, x, kp, 3, n_seg, p_seg, eps, ks);
        double nu[3];
        edge_nu(A, B, nrm, nu);
        if (mat) {
            for (int g = 0; g < 3; g++)
                for (int h = 0; h < 3; h++) mat[g][h] += ks[g] * (-nu[h]);
        } else {
            cplx jn = cdot_cr(j, nu);
            cplx m = -jn;
            for (int g = 0; g < 3; g++) res[g] += ks[g] * m;
        }
    }
}

// K0_Common (K0.h:112-166): sum_e int_e F(x, y) with vec_dbl = nu_e.
BIELCC_D void K0_common_dev(int id, const double* x, const DCell& c, DKP& kp, int n_seg, int p_seg, double eps,
                            cplx* res) {
    double nrm[3];
    cell_normal(c, nrm);
    for (int g = 0; g < 3; g++) res[g] = mk(0, 0);
    for (int s = 0; s < c.nv; s++) {
        const double* A = c.v[s];
        const double* B = c.v[(s + 1) % c.nv];
        double nu[3];
        edge_nu(A, B, nrm, nu);
        for (int g = 0; g < 3; g++) kp.vec_dbl[g] = nu[g];
        cplx ks[3];
        integral_seg<cplx>(id, A, B, x, kp, 3, n_seg, p_seg, eps, ks);
        for (int g = 0; g < 3; g++) res[g] += ks[g];
    }
}

// ------------------------------------------------------------------ analytic integrals
// Exact integral of 1/|x - y| over a triangle from the classical closed form
// (D. R. Wilton et al., IEEE Trans. AP-32(3), 1984):
//   sum_e P0 ln((R+ + l+)/(R- + l-)) - |h| sum_e [atan(P0 l+ / (R0^2 + |h| R+))
//                                             - atan(P0 l- / (R0^2 + |h| R-))]
// Same value as integral1Divr (integrators/integrals_analytic.cpp:37-235).
BIELCC_D double int_1divr_tri(const double* P1, const double* P2, const double* P3, const double* x) {
    const double* P[3] = {P1, P2, P3};
    double e1[3], e2[3], nrm[3];
    for (int i = 0; i < 3; i++) { e1[i] = P2[i] - P1[i]; e2[i] = P3[i] - P1[i]; }
    cross3(e1, e2, nrm);
    double nl = len3(nrm);
    // zero-area triangle (collapsed half of a pole quad): the integral vanishes;
    // relative test because e1 x e1 is rounding noise under FMA contraction
    if (!(nl > 1e-13 * len3(e1) * len3(e2))) return 0.;
    for (int i = 0; i < 3; i++) nrm[i] /= nl;
    double w[3] = {x[0] - P1[0], x[1] - P1[1], x[2] - P1[2]};
    double h = dot3(w, nrm), ah = fabs(h);
    double rho[3] = {x[0] - h * nrm[0], x[1] - h * nrm[1], x[2] - h * nrm[2]};
    double sum = 0.;
    for (int e = 0; e < 3; e++) {
        const double* A = P[e];
        const double* B = P[(e + 1) % 3];
        double lv[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
        double L = len3(lv);
        if (!(L > 0)) continue;
        for (int i = 0; i < 3; i++) lv[i] /= L;
        double u[3];
        cross3(lv, nrm, u);
        double am[3] = {A[0] - rho[0], A[1] - rho[1], A[2] - rho[2]};
        double bm[3] = {B[0] - rho[0], B[1] - rho[1], B[2] - rho[2]};
        double P0 = dot3(am, u), lm = dot3(am, lv), lp = dot3(bm, lv);
        double Rm = dist3(x, A), Rp = dist3(x, B);
        double R02 = P0 * P0 + h * h;
        if (fabs(P0) > 1e-14 * (L + Rm + Rp)) {
            double num = Rp + lp, den = Rm + lm;
            if (num > 0 && den > 0) sum += P0 * log(num / den);
            sum -= ah * (atan2(P0 * lp, R02 + ah * Rp) - atan2(P0 * lm, R02 + ah * Rm));
        }
    }
    return sum;
}
// integral1Divr (integrals_analytic.cpp:218-235): quad = triangles 012 + 230
BIELCC_D double integral_1divr_dev(const DCell& c, const double* x) {
    if (c.nv == 3) return int_1divr_tri(c.v[0], c.v[1], c.v[2], x);
    return int_1divr_tri(c.v[0], c.v[1], c.v[2], x) + int_1divr_tri(c.v[2], c.v[3], c.v[0], x);
}
// integralGrad1DivrSeg (integrals_analytic.cpp:240-257), closed form
BIELCC_D void grad_1divr_seg_dev(const double* A, const double* B, const double* x, double* res) {
    double xa[3] = {x[0] - A[0], x[1] - A[1], x[2] - A[2]};
    double xb[3] = {x[0] - B[0], x[1] - B[1], x[2] - B[2]};
    double ra = dist3(x, A), rb = dist3(x, B), ab = dist3(A, B);
    double den = dot3(xa, xb) + ra * rb;
    for (int i = 0; i < 3; i++) res[i] = -ab * (xa[i] / ra + xb[i] / rb) / den;
}
// IntegralSurf_SimplePot_H_HS (integrals_analytic.h:136-164)
BIELCC_D cplx surf_simplepot_h_hs_dev(const DCell& c, const double* x, double analytic_r, int n_start, int p_max,
                                      double eps, cplx k) {
    double y[3];
    cell_centre(c, y);
    DKP kp;
    dkp_zero(kp);
    kp.k = k;
    kp.smoothR = kMachineZero;
    kp.smoothRMin = kMachineZero;
    cplx tmp[1];
    if (dist3(x, y) < analytic_r * cell_diam(c)) {
        double a = integral_1divr_dev(c, x);
        integral_cell<cplx>(F_SIMPLEPOT_HM1, x, c, kp, 1, n_start, p_max, eps, tmp);
        return mk(a, 0.) + tmp[0];
    }
    integral_cell<cplx>(F_SIMPLEPOT_H, x, c, kp, 1, n_start, p_max, eps, tmp);
    return tmp[0];
}
// IntegralSeg_GradSimplePot_H_HS (integrals_analytic.h:193-221); the
// reference leaves smoothRMin unset (never read at p_max_seg = 1); 0 here.
BIELCC_D void seg_gradsimplepot_h_hs_dev(const double* A, const double* B, const double* x, double analytic_r,
                                         int n_seg, int p_seg, double eps, cplx k, cplx* res) {
    DKP kp;
    dkp_zero(kp);
    kp.k = k;
    kp.smoothR = kMachineZero;
    double y[3] = {(B[0] + A[0]) / 2., (B[1] + A[1]) / 2., (B[2] + A[2]) / 2.};
    if (dist3(x, y) < analytic_r * dist3(A, B)) {
        double t[3];
        grad_1divr_seg_dev(A, B, x, t);
        integral_seg<cplx>(F_GRADSIMPLEPOT_HM1, A, B, x, kp, 3, n_seg, p_seg, eps, res);
        for (int i = 0; i < 3; i++) res[i] += mk(t[i], 0.);
    } else {
        integral_seg<cplx>(F_GRADSIMPLEPOT_H, A, B, x, kp, 3, n_seg, p_seg, eps, res);
    }
}
// K0_GradSimplePot_H_HS (K0.h:197-249); `mat` as in K0_dev.
BIELCC_D void K0_grad_hs_dev(const cplx* j, const double* x, const DCell& c, int n_seg, int p_seg, double eps,
                             double analytic_r, cplx k, cplx* res, cplx (*mat)[3] = nullptr) {
    double nrm[3];
    cell_normal(c, nrm);
    for (int g = 0; g < 3; g++) {
        res[g] = mk(0, 0);
        if (mat) mat[g][0] = mat[g][1] = mat[g][2] = mk(0, 0);
    }
    for (int s = 0; s < c.nv; s++) {
        const double* A = c.v[s];
        const double* B = c.v[(s + 1) % c.nv];
        cplx ks[3];
        seg_gradsimplepot_h_hs_dev(A, B, x, analytic_r, n_seg, p_seg, eps, k, ks);
        double nu[3];
        edge_nu(A, B, nrm, nu);
        if (mat) {
            for (int g = 0; g < 3; g++)
                for (int h = 0; h < 3; h++) mat[g][h] += ks[g] * (-nu[h]);
        } else {
            cplx m = -cdot_cr(j, nu);
            for (int g = 0; g < 3; g++) res[g] += ks[g] * m;
        }
    }
}

// ------------------------------------------------------------------ K and R operators
struct DNP {
    double eps, rs, rs_seg, analytic_calc;
    int n_start, n_start_seg, p_max, p_max_seg;
};

// K_RotRot_Near_Smooth (electrodynamics/K.h:47-79)
BIELCC_D void K_near_smooth_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    double dm = cell_diam(c);
    DKP pF, pG;
    dkp_zero(pF);
    dkp_zero(pG);
    pF.smoothR = np.rs * dm / np.n_start;
    pF.smoothRMin = np.eps;
    pF.k = k;
    pG.smoothR = np.rs_seg * dm / np.n_start_seg;
    pG.smoothRMin = np.eps;
    pG.k = k;
    cplx s[1];
    integral_cell<cplx>(F_SIMPLEPOT_H, x, c, pF, 1, np.n_start, np.p_max, np.eps, s);
    cplx surf = s[0] * k * k / kFourPi;
    cplx c3[3];
    K0_dev(F_GRADSIMPLEPOT_H, j, x, c, pG, np.n_start_seg, np.p_max_seg, np.eps, c3);
    for (int i = 0; i < 3; i++) res[i] = surf * j[i] + c3[i] / kFourPi;
}
// K_RotRot_HS (K.h:119-145)
BIELCC_D void K_hs_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    cplx I = surf_simplepot_h_hs_dev(c, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    for (int i = 0; i < 3; i++) res[i] = I * k * k * j[i] / kFourPi;
    DKP ps;
    dkp_zero(ps);
    ps.smoothR = np.rs_seg * cell_diam(c) / np.n_start_seg;
    ps.smoothRMin = np.eps;
    ps.k = k;
    cplx c3[3];
    K0_dev(F_GRADSIMPLEPOT_H, j, x, c, ps, np.n_start_seg, np.p_max_seg, np.eps, c3);
    for (int i = 0; i < 3; i++) res[i] += c3[i] / kFourPi;
}
// K_RotRot_HS_Colloc (K.h:179-204)
BIELCC_D void K_hs_colloc_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    cplx I = surf_simplepot_h_hs_dev(c, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    for (int i = 0; i < 3; i++) res[i] = I * k * k * j[i] / kFourPi;
    DKP ps;
    dkp_zero(ps);
    ps.smoothR = kMachineZero;
    ps.smoothRMin = kMachineZero;
    ps.k = k;
    cplx c3[3];
    K0_dev(F_GRADSIMPLEPOT_H, j, x, c, ps, np.n_start_seg, np.p_max_seg, np.eps, c3);
    for (int i = 0; i < 3; i++) res[i] += c3[i] / kFourPi;
}
// K_RotRot_HS2_Colloc (K.h:230-252)
BIELCC_D void K_hs2_colloc_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    cplx I = surf_simplepot_h_hs_dev(c, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    for (int i = 0; i < 3; i++) res[i] = I * k * k * j[i] / kFourPi;
    cplx c3[3];
    K0_grad_hs_dev(j, x, c, np.n_start_seg, np.p_max_seg, np.eps, np.analytic_calc, k, c3);
    for (int i = 0; i < 3; i++) res[i] += c3[i] / kFourPi;
}
// K_RotRot_Far (K.h:288-301)
BIELCC_D void K_far_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    DKP p;
    dkp_zero(p);
    p.smoothR = kMachineZero;
    p.smoothRMin = kMachineZero;
    p.k = k;
    for (int i = 0; i < 3; i++) p.current[i] = j[i];
    integral_cell<cplx>(F_ROTROTSIMPLEPOT_H, x, c, p, 3, np.n_start, np.p_max, np.eps, res);
    for (int i = 0; i < 3; i++) res[i] = res[i] / kFourPi;
}
// R_Rot_Smooth (electrodynamics/R.h:46-61)
BIELCC_D void R_smooth_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    double dm = cell_diam(c);
    DKP p;
    dkp_zero(p);
    p.smoothR = np.rs * dm / np.n_start;
    p.smoothRMin = dm / 100.;
    p.k = k;
    cplx g[3];
    integral_cell<cplx>(F_GRADSIMPLEPOT_H, x, c, p, 3, np.n_start, np.p_max, np.eps, g);
    ccross_cc(g, j, res);
    for (int i = 0; i < 3; i++) res[i] = res[i] / kFourPi;
}
// R_Rot_Colloc (R.h:89-111)
BIELCC_D void R_colloc_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    double y[3];
    cell_centre(c, y);
    if (dist3(x, y) < kMachineZero) {
        res[0] = res[1] = res[2] = mk(0, 0);
        return;
    }
    DKP p;
    dkp_zero(p);
    p.smoothR = kMachineZero;
    p.smoothRMin = kMachineZero;
    p.k = k;
    cplx g[3];
    integral_cell<cplx>(F_GRADSIMPLEPOT_H, x, c, p, 3, np.n_start, np.p_max, np.eps, g);
    ccross_cc(g, j, res);
    for (int i = 0; i < 3; i++) res[i] = res[i] / kFourPi;
}
// R_Rot_Near (R.h:140-175)
BIELCC_D void R_near_dev(const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    double nrm[3];
    cell_normal(c, nrm);
    double dm = cell_diam(c);
    DKP p;
    dkp_zero(p);
    p.smoothR = np.rs * dm / np.n_start;
    p.smoothRMin = dm / 100.;
    p.k = k;
    for (int i = 0; i < 3; i++) p.n[i] = nrm[i];
    cplx surf[3];
    integral_cell<cplx>(F_N_DOUBLEPOT_H, x, c, p, 3, np.n_start, np.p_max, np.eps, surf);
    DKP ps;
    dkp_zero(ps);
    ps.smoothR = kMachineZero;
    ps.smoothRMin = kMachineZero;
    ps.k = k;
    cplx curl[3];
    K0_common_dev(F_NU_SIMPLEPOT_H, x, c, ps, np.n_start_seg, np.p_max_seg, np.eps, curl);
    cplx t[3];
    for (int i = 0; i < 3; i++) t[i] = (surf[i] + curl[i]) / kFourPi;
    ccross_cc(j, t, res);
}

// J-independent parts of the near-field pair (x, cell) of the field driver,
// scaled by 1/4pi: out[13] = { surf * k^2 / 4pi, M (3x3) / 4pi, g (3) / 4pi }
// so that K_RotRot_Near_Smooth (K.h:47-79) = out0 * J + M J and
// R_Rot_Smooth (R.h:46-61) = g x J.
BIELCC_D void near_pair_moments(const double* x, const DCell& cl, cplx k, const DNP& np, cplx* o) {
    double dm = cell_diam(cl);
    if (np.p_max == 1) {
        // one quadrature pass for both surface integrals: K_RotRot_Near_Smooth's
        // int F (K.h:51-67) and R_Rot_Smooth's int grad F (R.h:46-61) start from
        // the same smoothing radius rs diam / n_start, and without refinement
        // their different smoothRMin never applies
        DKP pS;
        dkp_zero(pS);
        pS.smoothR = np.rs * dm / np.n_start;
        pS.k = k;
        cplx sF[1], g[3];
        integral_cell_pot_and_grad(x, cl, pS, np.n_start, sF, g);
        o[0] = sF[0] * k * k / kFourPi;
        DKP pG;
        dkp_zero(pG);
        pG.smoothR = np.rs_seg * dm / np.n_start_seg;
        pG.smoothRMin = np.eps;
        pG.k = k;
        cplx M[3][3], dummy[3];
        K0_dev(F_GRADSIMPLEPOT_H, nullptr, x, cl, pG, np.n_start_seg, np.p_max_seg, np.eps, dummy, M);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) o[1 + 3 * a + b] = M[a][b] / kFourPi;
        for (int a = 0; a < 3; a++) o[10 + a] = g[a] / kFourPi;
        return;
    }
    // surface part of K_RotRot_Near_Smooth (K.h:51-67)
    DKP pF;
    dkp_zero(pF);
    pF.smoothR = np.rs * dm / np.n_start;
    pF.smoothRMin = np.eps;
    pF.k = k;
    cplx s[1];
    integral_cell<cplx>(F_SIMPLEPOT_H, x, cl, pF, 1, np.n_start, np.p_max, np.eps, s);
    o[0] = s[0] * k * k / kFourPi;
    // contour part (K.h:56-72): K0 with the shared, shrinking segment radius
    DKP pG;
    dkp_zero(pG);
    pG.smoothR = np.rs_seg * dm / np.n_start_seg;
    pG.smoothRMin = np.eps;
    pG.k = k;
    cplx M[3][3], dummy[3];
    K0_dev(F_GRADSIMPLEPOT_H, nullptr, x, cl, pG, np.n_start_seg, np.p_max_seg, np.eps, dummy, M);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) o[1 + 3 * a + b] = M[a][b] / kFourPi;
    // R_Rot_Smooth (R.h:46-61)
    DKP pR;
    dkp_zero(pR);
    pR.smoothR = np.rs * dm / np.n_start;
    pR.smoothRMin = dm / 100.;
    pR.k = k;
    cplx g[3];
    integral_cell<cplx>(F_GRADSIMPLEPOT_H, x, cl, pR, 3, np.n_start, np.p_max, np.eps, g);
    for (int a = 0; a < 3; a++) o[10 + a] = g[a] / kFourPi;
}

BIELCC_D void run_pair_op(int op, const cplx* j, const double* x, const DCell& c, const DNP& np, cplx k, cplx* res) {
    switch (op) {
        case 0: K_near_smooth_dev(j, x, c, np, k, res); break;
        case 1: K_hs_dev(j, x, c, np, k, res); break;
        case 2: K_hs_colloc_dev(j, x, c, np, k, res); break;
        case 3: K_hs2_colloc_dev(j, x, c, np, k, res); break;
        case 4: K_far_dev(j, x, c, np, k, res); break;
        case 5: R_smooth_dev(j, x, c, np, k, res); break;
        case 6: R_colloc_dev(j, x, c, np, k, res); break;
        default: R_near_dev(j, x, c, np, k, res); break;
    }
}

}  // namespace bielcc_gpu
