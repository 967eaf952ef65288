// bielcc_oracle.cpp — CPU ORACLE (test infrastructure only).
//
// A plain C++17 restatement of AlenaSetukha/BIELcc's Stratton-Chu hot path,
// used ONLY by tests/, by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg as the checker. The product (bielcc_b200/, libbielcc_gpu.so)
// never links, loads or calls this file.
//
// Parity is pinned two ways: (1) tests/test_oracle_reference.py compares every
// exported function against the reference compiled from its own sources
// (oracle/_ref/libbielcc_ref.so, built by oracle/Makefile), and (2) against the
// golden vectors in tests/golden/ that tests/golden/make_golden.py generated by
// running that compiled reference.
//
// Every function cites the reference file:line whose behaviour it restates.
// Complex numbers cross the C boundary as interleaved (re, im) doubles.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/bielcc_gpu.h"

namespace orc {

using cd = std::complex<double>;
static const double kEps = std::numeric_limits<double>::epsilon();  // Tolerance_Constants::MACHINE_ZERO
static const double kFourPi = 4.0 * M_PI;

// ---------------------------------------------------------------- geometry
// geometry/element_geom.h:91-108 (dist, vec_length), element_geom.cpp:9-56
static inline double dist3(const double* a, const double* b) {
    double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}
static inline double len3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const double* a, const double* b, double* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline cd cdot_cr(const cd* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void ccross_cr(const cd* a, const double* b, cd* r) {  // complex x real
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline void ccross_cc(const cd* a, const cd* b, cd* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

// Cell view: nv = 4 (CellQuad) or 3 (CellTriangle).
struct Cell {
    int nv;
    const double (*v)[3];
};

// get_center_mass, element_geom.cpp:320-342
static void centre(const Cell& c, double* y) {
    for (int i = 0; i < 3; i++) {
        if (c.nv == 4) y[i] = (c.v[0][i] + c.v[1][i] + c.v[2][i] + c.v[3][i]) * 0.25;
        else y[i] = (c.v[0][i] + c.v[1][i] + c.v[2][i]) / 3.;
    }
}

// get_diam, element_geom.cpp:275-317 (quad: diagonals then sides; tri: sides)
static double diam(const Cell& c) {
    if (c.nv == 4) {
        double d1[3], d2[3];
        for (int g = 0; g < 3; g++) { d1[g] = c.v[2][g] - c.v[0][g]; d2[g] = c.v[3][g] - c.v[1][g]; }
        double best = len3(d1) > len3(d2) ? len3(d1) : len3(d2);
        for (int s = 0; s < 4; s++) {
            double e[3];
            int a = s, b = (s + 1) % 4;
            for (int g = 0; g < 3; g++) e[g] = c.v[b][g] - c.v[a][g];
            if (len3(e) > best) best = len3(e);
        }
        return best;
    }
    double l1 = dist3(c.v[0], c.v[1]), l2 = dist3(c.v[1], c.v[2]), l3 = dist3(c.v[2], c.v[0]);
    return std::max(std::max(l1, l2), l3);
}

// norm_func, element_geom.cpp:130-156 (quad: diagonal cross product, tri: ab x ac)
static void normal(const Cell& c, double* nrm) {
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

// tangent basis of CellQuad::CellFill (mesh/cell.cpp:8-51) / CellTriangle::CellFill
// (mesh/cell.cpp:60-99)
static void tangents(const Cell& c, double* t1, double* t2) {
    double nrm[3], base[3], len;
    if (c.nv == 4) {
        double ma[3], mb[3], mc[3], md[3], ac[3], bd[3];
        for (int i = 0; i < 3; i++) {
            ma[i] = (c.v[0][i] + c.v[1][i]) / 2.0;
            mb[i] = (c.v[1][i] + c.v[2][i]) / 2.0;
            mc[i] = (c.v[2][i] + c.v[3][i]) / 2.0;
            md[i] = (c.v[3][i] + c.v[0][i]) / 2.0;
            ac[i] = mc[i] - ma[i];
            bd[i] = md[i] - mb[i];
        }
        cross3(ac, bd, nrm);
        len = len3(nrm);
        for (int i = 0; i < 3; i++) nrm[i] /= len;
        for (int i = 0; i < 3; i++) base[i] = ac[i];
    } else {
        double ab[3], ac[3];
        for (int i = 0; i < 3; i++) { ab[i] = c.v[1][i] - c.v[0][i]; ac[i] = c.v[2][i] - c.v[0][i]; }
        cross3(ab, ac, nrm);
        len = len3(nrm);
        for (int i = 0; i < 3; i++) nrm[i] /= len;
        for (int i = 0; i < 3; i++) base[i] = ab[i];
    }
    len = len3(base);
    for (int i = 0; i < 3; i++) t1[i] = base[i] / len;
    cross3(nrm, t1, t2);
    len = len3(t2);
    for (int i = 0; i < 3; i++) t2[i] /= len;
}

// tr_square, element_geom.cpp:54-66
static double tri_area(const double* p1, const double* p2, const double* p3) {
    double ab[3], ac[3], n[3];
    for (int i = 0; i < 3; i++) { ab[i] = p2[i] - p1[i]; ac[i] = p3[i] - p1[i]; }
    cross3(ab, ac, n);
    return std::sqrt(dot3(n, n)) / 2.;
}

// ---------------------------------------------------------------- integrand parameters
// KernelParam<KType>, integrators/kernel_param.h:25-57 (fields the integrands read)
struct KP {
    double smoothR = 0, smoothRMin = 0;
    cd k = 0;
    cd current[3] = {0., 0., 0.};
    double vec_dbl[3] = {0, 0, 0};
    double n[3] = {0, 0, 0};
    double e0[3] = {0, 0, 0};
};

// ---------------------------------------------------------------- integrands
// All "without 1/4pi" (electrodynamics/kernel_lib.h:38). `out` holds idim values.
// Bracket weight shared by the smoothed kernels:
//   (t < 1) * A + (t >= 1) * B, kept as arithmetic on 0/1 so NaN/Inf behave as in
//   the reference (e.g. 0/0 at r = 0).
static inline double pick(double t, double a, double b) {
    return (double)(t < 1) * a + (double)(t >= 1) * b;
}

// F_SimplePot_L, kernel_lib.h:62-69
static void F_SimplePot_L(const double* x, const double* y, const KP& p, double* out) {
    double r = dist3(x, y), R = p.smoothR, t = r / R;
    out[0] = (double)(t < 1) * (t * (3. - 2. * t) / R) + (double)(t >= 1) / r;
}
// F_GradSimplePot_L, kernel_lib.h:87-98
static void F_GradSimplePot_L(const double* x, const double* y, const KP& p, double* out) {
    double r = dist3(x, y), R = p.smoothR, t = r / R;
    double w = (double)(t < 1) * (3. - 2. * t) / (r * (R * R)) + (double)(t >= 1) / ((r * r) * r);
    for (int i = 0; i < 3; i++) out[i] = (y[i] - x[i]) * w;
}
// F_DoublePot_L, kernel_lib.h:117-129
static void F_DoublePot_L(const double* x, const double* y, const KP& p, double* out) {
    double r = dist3(x, y), R = p.smoothR, t = r / R;
    double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
    double w = (double)(t < 1) * (3. - 2. * t) / (r * (R * R)) + (double)(t >= 1) / ((r * r) * r);
    out[0] = dot3(p.n, d) * w;
}
// F_VectorPot_L, kernel_lib.h:149-177
static void F_VectorPot_L(const double* x, const double* y, const KP& p, double* out) {
    double r = dist3(x, y);
    if (r < kEps) { out[0] = out[1] = out[2] = 0.; return; }
    double f = 1. / r / r / r;
    double d[3] = {(y[0] - x[0]) * f, (y[1] - x[1]) * f, (y[2] - x[2]) * f};
    cross3(d, p.vec_dbl, out);
    if (r < p.smoothR) {
        double t = r / p.smoothR;
        for (int i = 0; i < 3; i++) out[i] = out[i] * (3 * t * t - 2 * t * t * t);
    }
}
// exp(i r k) as the reference writes it: std::exp(complex(0, r) * k)
static inline cd eikr(double r, cd k) { return std::exp(cd(0., r) * k); }

// F_SimplePot_H, kernel_lib.h:209-217
static void F_SimplePot_H(const double* x, const double* y, const KP& p, cd* out) {
    double r = dist3(x, y), R = p.smoothR, t = r / R;
    out[0] = eikr(r, p.k) * pick(t, t * (3. - 2. * t) / R, 1. / r);
}
// nuF_SimplePot_H, kernel_lib.h:235-245
static void nuF_SimplePot_H(const double* x, const double* y, const KP& p, cd* out) {
    cd f[1];
    F_SimplePot_H(x, y, p, f);
    for (int i = 0; i < 3; i++) out[i] = p.vec_dbl[i] * f[0];
}
// F_SimplePot_Hm1, kernel_lib.h:262-278
static void F_SimplePot_Hm1(const double* x, const double* y, const KP& p, cd* out) {
    double r = dist3(x, y);
    if (std::abs(cd(0., r) * p.k) < 1e-7) {
        out[0] = cd(0., 1.) * p.k - p.k * p.k * r / 2.;
    } else {
        double R = p.smoothR, t = r / R;
        out[0] = (eikr(r, p.k) - 1.) * pick(t, t * (3. - 2. * t) / R, 1. / r);
    }
}
// F_GradSimplePot_H, kernel_lib.h:295-313
static void F_GradSimplePot_H(const double* x, const double* y, const KP& p, cd* out) {
    double r = dist3(x, y), R = p.smoothR, t = r / R;
    cd ikr = cd(0., r) * p.k;
    cd e = std::exp(ikr);
    double w = (double)(t < 1) * (3. - 2. * t) / (r * (R * R)) + (double)(t >= 1) / ((r * r) * r);
    for (int i = 0; i < 3; i++) out[i] = ((x[i] - y[i]) * e) * (ikr - 1.) * w;
}
// F_GradSimplePot_Hm1, kernel_lib.h:332-356
static void F_GradSimplePot_Hm1(const double* x, const double* y, const KP& p, cd* out) {
    double r = dist3(x, y);
    double a = std::abs(cd(0., r) * p.k);
    if (a < 1e-6) {
        out[0] = out[1] = out[2] = 0.;
    } else if (a < 1e-4) {
        for (int i = 0; i < 3; i++) out[i] = (y[i] - x[i]) * p.k * p.k / (2. * r);
    } else {
        cd ikr = cd(0., r) * p.k;
        cd num = 1. + (ikr - 1.) * std::exp(ikr);
        for (int i = 0; i < 3; i++) out[i] = (x[i] - y[i]) * num / (r * r * r);
    }
}
// F_DoublePot_H, kernel_lib.h:375-390
static void F_DoublePot_H(const double* x, const double* y, const KP& p, cd* out) {
    double r = dist3(x, y), R = p.smoothR, t = r / R;
    double d[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
    cd ikr = cd(0., r) * p.k;
    double w = (double)(t < 1) * (3 - 2 * t) / (r * (R * R)) + (double)(t >= 1) / ((r * r) * r);
    out[0] = dot3(p.n, d) * std::exp(ikr) * (ikr - 1.) * w;
}
// nF_DoublePot_H, kernel_lib.h:409-419
static void nF_DoublePot_H(const double* x, const double* y, const KP& p, cd* out) {
    cd f[1];
    F_DoublePot_H(x, y, p, f);
    for (int i = 0; i < 3; i++) out[i] = p.n[i] * f[0];
}
// F_RotRotSimplePot_H, kernel_lib.h:453-492
static void F_RotRotSimplePot_H(const double* x, const double* y, const KP& p, cd* out) {
    double r = dist3(x, y);
    if (r < kEps) { out[0] = out[1] = out[2] = 0.; return; }
    cd ik = cd(0., 1.) * p.k;
    cd k2 = p.k * p.k;
    double dh[3];
    for (int i = 0; i < 3; i++) dh[i] = (x[i] - y[i]) / r;
    cd f1 = (-1.0 / (r * r) / r) + (ik / (r * r)) + (k2 / r);
    cd f2 = (3.0 / (r * r) / r) - (3.0 * ik / (r * r)) - (k2 / r);
    cd e = std::exp(ik * r);
    f2 *= cdot_cr(p.current, dh);
    for (int i = 0; i < 3; i++) out[i] = (dh[i] * f2 + p.current[i] * f1) * e;
    if (r < p.smoothR) {
        double t = r / p.smoothR;
        for (int i = 0; i < 3; i++) out[i] *= (t * t * (3 - 2 * t));
    }
}
// F = 1 (the f1 integrand of examples/integrators/main0_integrals.cpp:77-81)
static void F_One(const double*, const double*, const KP&, double* out) { out[0] = 1.; }
// PlaneWaveFieldE (electrodynamics/incident_field.h:20-29) as a one-point
// integrand F(y) = e0 exp(i vec_dbl . y); the pair point is unused.
static void PlaneWave_E(const double*, const double* y, const KP& p, cd* out) {
    cd deg = std::exp(cd(0., 1.) * dot3(p.vec_dbl, y));
    for (int i = 0; i < 3; i++) out[i] = p.e0[i] * deg;
}

// ---------------------------------------------------------------- universal quadrature
// The adaptive driver shared by the three rules (integral_universal.h:58-119,
// :160-219; integral_universal_seg.h:57-97): run a pass at n, stop once two
// successive passes differ by less than eps (L2 over idim, not at the first
// pass), else n -> 2n and the smoothing radius is halved once PER COMPONENT
// (idim times) while above smoothRMin and p < 8; when the pass budget runs
// out the previous pass is returned.
template <typename T, typename Pass>
static void adaptive(int n_start, int p_max, double eps, int idim, KP& kp, T* res, Pass pass) {
    T prev[3] = {T(0), T(0), T(0)};
    for (int g = 0; g < idim; g++) res[g] = T(0);
    int n = n_start, p;
    for (p = 0; p < p_max; p++) {
        pass(n, res);
        double delta = 0.;
        for (int g = 0; g < idim; g++) delta += std::abs(res[g] - prev[g]) * std::abs(res[g] - prev[g]);
        if (delta < eps * eps && p != 0) break;
        n *= 2;
        for (int g = 0; g < idim; g++) {
            prev[g] = res[g];
            res[g] = T(0);
            if (p < 8 && kp.smoothR > kp.smoothRMin) kp.smoothR /= 2.;
        }
    }
    if (p == p_max)
        for (int g = 0; g < idim; g++) res[g] = prev[g];
}

template <typename T>
using Integrand = void (*)(const double*, const double*, const KP&, T*);

// IntegralUniversalPnt over a quad: midpoint rule on the n x n bilinear
// sub-cells, integral_universal.h:38-120
template <typename T>
static void integral_quad(const double* x, const double (*c)[3], Integrand<T> f, KP& kp, int idim,
                          int n_start, int p_max, double eps, T* res) {
    adaptive<T>(n_start, p_max, eps, idim, kp, res, [&](int n, T* acc) {
        T ff[3];
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < n; j++) {
                double p0 = (double)i / (double)n, q0 = (double)j / (double)n;
                double p1 = ((double)i + 1.) / (double)n, q1 = ((double)j + 1.) / (double)n;
                double c1[3], c2[3], c3[3], c4[3], m1[3], m2[3], y[3], nr[3];
                for (int k = 0; k < 3; k++) {
                    double lo = q0 * c[1][k] + (1 - q0) * c[0][k];
                    double hi = q0 * c[2][k] + (1 - q0) * c[3][k];
                    c1[k] = p0 * hi + (1 - p0) * lo;
                    c4[k] = p1 * hi + (1 - p1) * lo;
                }
                for (int k = 0; k < 3; k++) {
                    double lo = q1 * c[1][k] + (1 - q1) * c[0][k];
                    double hi = q1 * c[2][k] + (1 - q1) * c[3][k];
                    c2[k] = p0 * hi + (1 - p0) * lo;
                    c3[k] = p1 * hi + (1 - p1) * lo;
                }
                for (int k = 0; k < 3; k++) {
                    y[k] = (c1[k] + c2[k] + c3[k] + c4[k]) / 4.0;
                    m1[k] = ((c2[k] + c3[k]) - (c1[k] + c4[k])) / 2.0;
                    m2[k] = ((c3[k] + c4[k]) - (c1[k] + c2[k])) / 2.0;
                }
                cross3(m1, m2, nr);
                double s = len3(nr);
                f(x, y, kp, ff);
                for (int g = 0; g < idim; g++) acc[g] += ff[g] * s;
            }
        }
    });
}

// IntegralUniversalPnt over a triangle: n^2 congruent sub-triangle centroids,
// weight area/n^2 applied after the sum, integral_universal.h:136-220
template <typename T>
static void integral_tri(const double* x, const double (*c)[3], Integrand<T> f, KP& kp, int idim,
                         int n_start, int p_max, double eps, T* res) {
    double area = tri_area(c[0], c[1], c[2]);
    adaptive<T>(n_start, p_max, eps, idim, kp, res, [&](int n, T* acc) {
        double pv[3], qv[3], rv[3];
        for (int k = 0; k < 3; k++) {
            pv[k] = (c[1][k] - c[0][k]) / n;
            qv[k] = (c[2][k] - c[0][k]) / n;
            rv[k] = (c[2][k] - c[1][k]) / n;
        }
        T ff[3];
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < n - i; j++) {
                double B[3], y[3];
                for (int k = 0; k < 3; k++) {
                    B[k] = c[0][k] + (i + 1) * pv[k] + j * qv[k];
                    double A = B[k] - pv[k];
                    double C = A + qv[k];
                    y[k] = (B[k] + A + C) / 3.0;
                }
                f(x, y, kp, ff);
                for (int g = 0; g < idim; g++) acc[g] += ff[g];
                if (j < n - 1 - i) {
                    for (int k = 0; k < 3; k++) {
                        double A = B[k] + rv[k];
                        double C = B[k] + qv[k];
                        y[k] = (B[k] + A + C) / 3.0;
                    }
                    f(x, y, kp, ff);
                    for (int g = 0; g < idim; g++) acc[g] += ff[g];
                }
            }
        }
        for (int g = 0; g < idim; g++) acc[g] = acc[g] * area / (double)n / (double)n;
    });
}

template <typename T>
static void integral_cell(const double* x, const Cell& c, Integrand<T> f, KP& kp, int idim,
                          int n_start, int p_max, double eps, T* res) {
    if (c.nv == 4) integral_quad<T>(x, c.v, f, kp, idim, n_start, p_max, eps, res);
    else integral_tri<T>(x, c.v, f, kp, idim, n_start, p_max, eps, res);
}

// IntegralUniversalSegPnt: midpoint rule on n sub-segments,
// integral_universal_seg.h:38-98
template <typename T>
static void integral_seg(const double* a, const double* b, const double* x, Integrand<T> f, KP& kp,
                         int idim, int n_start, int p_max, double eps, T* res) {
    adaptive<T>(n_start, p_max, eps, idim, kp, res, [&](int n, T* acc) {
        double d[3], y[3];
        for (int k = 0; k < 3; k++) d[k] = (b[k] - a[k]) / n;
        double dl = len3(d);
        T ff[3];
        for (int i = 0; i < n; i++) {
            for (int k = 0; k < 3; k++) y[k] = a[k] + (i + 0.5) * d[k];
            f(x, y, kp, ff);
            for (int g = 0; g < idim; g++) acc[g] += ff[g] * dl;
        }
    });
}

// IntegralUniversal with F(x) = 1 (integral_universal.h:252-334 quad,
// :347-431 triangle): the same node sets without an observation point.
static double area_by_quadrature(const Cell& c, int n_start, int p_max, double eps) {
    KP kp;
    double r[1];
    double dummy[3] = {0, 0, 0};
    integral_cell<double>(dummy, c, F_One, kp, 1, n_start, p_max, eps, r);
    return r[0];
}

// ---------------------------------------------------------------- contour operators
// Edge s of a cell runs from vertex s to vertex s+1 (last -> 0), K0.h:64-71.
static inline void edge_ends(const Cell& c, int s, const double*& A, const double*& B) {
    A = c.v[s];
    B = c.v[(s + 1) % c.nv];
}
// nu = (B - A) x n, normalised unless its length is <= MACHINE_ZERO (K0.h:72-80)
static inline void edge_nu(const double* A, const double* B, const double* nrm, double* nu) {
    double d[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    cross3(d, nrm, nu);
    double l = len3(nu);
    if (l > kEps)
        for (int g = 0; g < 3; g++) nu[g] /= l;
}

// K0, K0.h:36-86: -sum_e (j . nu_e) int_e F; kp shared (and mutated) across edges.
static void K0(const cd* j, const double* x, const Cell& c, Integrand<cd> f, KP& kp, int n_seg,
               int p_seg, double eps, cd* res) {
    double nrm[3];
    normal(c, nrm);
    for (int g = 0; g < 3; g++) res[g] = 0.;
    for (int s = 0; s < c.nv; s++) {
        const double *A, *B;
        edge_ends(c, s, A, B);
        cd ks[3];
        integral_seg<cd>(A, B, x, f, kp, 3, n_seg, p_seg, eps, ks);
        double nu[3];
        edge_nu(A, B, nrm, nu);
        cd jn = cdot_cr(j, nu);
        for (int g = 0; g < 3; g++) {
            ks[g] *= -jn;
            res[g] += ks[g];
        }
    }
}

// K0_Common, K0.h:112-166: sum_e int_e F(x, y) with vec_dbl = nu_e.
static void K0_Common(const double* x, const Cell& c, Integrand<cd> f, KP& kp, int n_seg, int p_seg,
                      double eps, cd* res) {
    double nrm[3];
    normal(c, nrm);
    for (int g = 0; g < 3; g++) res[g] = 0.;
    for (int s = 0; s < c.nv; s++) {
        const double *A, *B;
        edge_ends(c, s, A, B);
        double nu[3];
        edge_nu(A, B, nrm, nu);
        for (int g = 0; g < 3; g++) kp.vec_dbl[g] = nu[g];
        cd ks[3];
        integral_seg<cd>(A, B, x, f, kp, 3, n_seg, p_seg, eps, ks);
        for (int g = 0; g < 3; g++) res[g] += ks[g];
    }
}

// ---------------------------------------------------------------- analytic integrals
// Exact integral of 1/|x - y| over the triangle (P1, P2, P3), written from the
// classical closed form (D. R. Wilton et al., IEEE Trans. AP-32, 1984):
//   sum_e P0_e ln((R+ + l+)/(R- + l-)) - |h| sum_e [atan(P0 l+/(R0^2 + |h|R+))
//                                                - atan(P0 l-/(R0^2 + |h|R-))]
// Same value as _Integral1Divr_inv (integrators/integrals_analytic.cpp:37-200),
// which reaches it through Givens rotations.
static double int_1divr_tri(const double* P1, const double* P2, const double* P3, const double* x) {
    const double* P[3] = {P1, P2, P3};
    double e1[3], e2[3], nrm[3];
    for (int i = 0; i < 3; i++) { e1[i] = P2[i] - P1[i]; e2[i] = P3[i] - P1[i]; }
    cross3(e1, e2, nrm);
    double nl = len3(nrm);
    // zero-area triangle (a pole quad's collapsed half): the integral vanishes.
    // Relative test: with FMA contraction e x e is rounding noise, not 0.
    if (!(nl > 1e-13 * len3(e1) * len3(e2))) return 0.;
    for (int i = 0; i < 3; i++) nrm[i] /= nl;
    double w[3] = {x[0] - P1[0], x[1] - P1[1], x[2] - P1[2]};
    double h = dot3(w, nrm);
    double ah = std::fabs(h);
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
        cross3(lv, nrm, u);  // in-plane outward normal of the edge
        double am[3] = {A[0] - rho[0], A[1] - rho[1], A[2] - rho[2]};
        double bm[3] = {B[0] - rho[0], B[1] - rho[1], B[2] - rho[2]};
        double P0 = dot3(am, u);
        double lm = dot3(am, lv), lp = dot3(bm, lv);
        double Rm = dist3(x, A), Rp = dist3(x, B);
        double R02 = P0 * P0 + h * h;
        double scale = L + Rm + Rp;
        if (std::fabs(P0) > 1e-14 * scale) {
            double num = Rp + lp, den = Rm + lm;
            if (num > 0 && den > 0) sum += P0 * std::log(num / den);
            double tp = std::atan2(P0 * lp, R02 + ah * Rp);
            double tm = std::atan2(P0 * lm, R02 + ah * Rm);
            sum -= ah * (tp - tm);
        }
    }
    return sum;
}

// integral1Divr, integrals_analytic.cpp:218-235 (quad = triangles 012 + 230)
static double integral_1divr(const Cell& c, const double* x) {
    if (c.nv == 3) return int_1divr_tri(c.v[0], c.v[1], c.v[2], x);
    return int_1divr_tri(c.v[0], c.v[1], c.v[2], x) + int_1divr_tri(c.v[2], c.v[3], c.v[0], x);
}

// integralGrad1DivrSeg, integrals_analytic.cpp:240-257: closed form of
// int_AB grad_x 1/|x - y| dl.
static void grad_1divr_seg(const double* A, const double* B, const double* x, double* res) {
    double xa[3] = {x[0] - A[0], x[1] - A[1], x[2] - A[2]};
    double xb[3] = {x[0] - B[0], x[1] - B[1], x[2] - B[2]};
    double ra = dist3(x, A), rb = dist3(x, B), ab = dist3(A, B);
    double den = dot3(xa, xb) + ra * rb;
    for (int i = 0; i < 3; i++) res[i] = -ab * (xa[i] / ra + xb[i] / rb) / den;
}

// IntegralSurf_SimplePot_H_HS, integrals_analytic.h:136-164
static cd surf_simplepot_h_hs(const Cell& c, const double* x, double analytic_r, int n_start, int p_max,
                              double eps, cd k) {
    double y[3];
    centre(c, y);
    KP kp;
    kp.k = k;
    kp.smoothR = kEps;
    kp.smoothRMin = kEps;
    cd tmp[1];
    if (dist3(x, y) < analytic_r * diam(c)) {
        cd ff = cd(integral_1divr(c, x));
        integral_cell<cd>(x, c, F_SimplePot_Hm1, kp, 1, n_start, p_max, eps, tmp);
        return ff + tmp[0];
    }
    integral_cell<cd>(x, c, F_SimplePot_H, kp, 1, n_start, p_max, eps, tmp);
    return tmp[0];
}

// IntegralSeg_GradSimplePot_H_HS, integrals_analytic.h:193-221. The reference
// leaves smoothRMin of its local KernelParam unset; with p_max_seg = 1 (the
// default) it is never read. Here it is 0.
static void seg_gradsimplepot_h_hs(const double* A, const double* B, const double* x, double analytic_r,
                                   int n_seg, int p_seg, double eps, cd k, cd* res) {
    KP kp;
    kp.k = k;
    kp.smoothR = kEps;
    kp.smoothRMin = 0.;
    double y[3] = {(B[0] + A[0]) / 2., (B[1] + A[1]) / 2., (B[2] + A[2]) / 2.};
    if (dist3(x, y) < analytic_r * dist3(A, B)) {
        double t[3];
        grad_1divr_seg(A, B, x, t);
        integral_seg<cd>(A, B, x, F_GradSimplePot_Hm1, kp, 3, n_seg, p_seg, eps, res);
        for (int i = 0; i < 3; i++) res[i] += cd(t[i]);
    } else {
        integral_seg<cd>(A, B, x, F_GradSimplePot_H, kp, 3, n_seg, p_seg, eps, res);
    }
}

// K0_GradSimplePot_H_HS, K0.h:197-249
static void K0_grad_hs(const cd* j, const double* x, const Cell& c, int n_seg, int p_seg, double eps,
                       double analytic_r, cd k, cd* res) {
    double nrm[3];
    normal(c, nrm);
    for (int g = 0; g < 3; g++) res[g] = 0.;
    for (int s = 0; s < c.nv; s++) {
        const double *A, *B;
        edge_ends(c, s, A, B);
        cd ks[3];
        seg_gradsimplepot_h_hs(A, B, x, analytic_r, n_seg, p_seg, eps, k, ks);
        double nu[3];
        edge_nu(A, B, nrm, nu);
        cd jn = cdot_cr(j, nu);
        for (int g = 0; g < 3; g++) {
            ks[g] *= -jn;
            res[g] += ks[g];
        }
    }
}

// ---------------------------------------------------------------- K and R operators
struct NP {
    double eps, rs, rs_seg, analytic_calc;
    int n_start, n_start_seg, p_max, p_max_seg;
};
static NP np_from(const bielcc_numparam* p) {
    NP n;
    if (!p) {
        n.eps = 1e-6; n.rs = 2.; n.rs_seg = 2.; n.analytic_calc = 3.;
        n.n_start = 8; n.n_start_seg = 10; n.p_max = 1; n.p_max_seg = 1;
        return n;
    }
    n.eps = p->eps; n.rs = p->rs; n.rs_seg = p->rs_seg; n.analytic_calc = p->analytic_calc;
    n.n_start = p->n_start; n.n_start_seg = p->n_start_seg; n.p_max = p->p_max; n.p_max_seg = p->p_max_seg;
    return n;
}

// K_RotRot_Near_Smooth, K.h:47-79
static void K_near_smooth(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    double dm = diam(c);
    KP pF;
    pF.smoothR = np.rs * dm / np.n_start;
    pF.smoothRMin = np.eps;
    pF.k = k;
    KP pG;
    pG.smoothR = np.rs_seg * dm / np.n_start_seg;
    pG.smoothRMin = np.eps;
    pG.k = k;
    cd s[1];
    integral_cell<cd>(x, c, F_SimplePot_H, pF, 1, np.n_start, np.p_max, np.eps, s);
    cd surf = s[0] * k * k / kFourPi;
    cd c3[3];
    K0(j, x, c, F_GradSimplePot_H, pG, np.n_start_seg, np.p_max_seg, np.eps, c3);
    for (int i = 0; i < 3; i++) res[i] = surf * j[i] + c3[i] / kFourPi;
}

// K_RotRot_HS, K.h:119-145
static void K_hs(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    cd I = surf_simplepot_h_hs(c, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    for (int i = 0; i < 3; i++) res[i] = I * k * k * j[i] / kFourPi;
    KP ps;
    ps.smoothR = np.rs_seg * diam(c) / np.n_start_seg;
    ps.smoothRMin = np.eps;
    ps.k = k;
    cd c3[3];
    K0(j, x, c, F_GradSimplePot_H, ps, np.n_start_seg, np.p_max_seg, np.eps, c3);
    for (int i = 0; i < 3; i++) res[i] += c3[i] / kFourPi;
}

// K_RotRot_HS_Colloc, K.h:179-204
static void K_hs_colloc(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    cd I = surf_simplepot_h_hs(c, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    for (int i = 0; i < 3; i++) res[i] = I * k * k * j[i] / kFourPi;
    KP ps;
    ps.smoothR = kEps;
    ps.smoothRMin = kEps;
    ps.k = k;
    cd c3[3];
    K0(j, x, c, F_GradSimplePot_H, ps, np.n_start_seg, np.p_max_seg, np.eps, c3);
    for (int i = 0; i < 3; i++) res[i] += c3[i] / kFourPi;
}

// K_RotRot_HS2_Colloc, K.h:230-252
static void K_hs2_colloc(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    cd I = surf_simplepot_h_hs(c, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    for (int i = 0; i < 3; i++) res[i] = I * k * k * j[i] / kFourPi;
    cd c3[3];
    K0_grad_hs(j, x, c, np.n_start_seg, np.p_max_seg, np.eps, np.analytic_calc, k, c3);
    for (int i = 0; i < 3; i++) res[i] += c3[i] / kFourPi;
}

// K_RotRot_Far, K.h:288-301
static void K_far(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    KP p;
    p.smoothR = kEps;
    p.smoothRMin = kEps;
    p.k = k;
    for (int i = 0; i < 3; i++) p.current[i] = j[i];
    integral_cell<cd>(x, c, F_RotRotSimplePot_H, p, 3, np.n_start, np.p_max, np.eps, res);
    for (int i = 0; i < 3; i++) res[i] /= kFourPi;
}

// R_Rot_Smooth, R.h:46-61
static void R_smooth(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    double dm = diam(c);
    KP p;
    p.smoothR = np.rs * dm / np.n_start;
    p.smoothRMin = dm / 100.;
    p.k = k;
    cd g[3];
    integral_cell<cd>(x, c, F_GradSimplePot_H, p, 3, np.n_start, np.p_max, np.eps, g);
    ccross_cc(g, j, res);
    for (int i = 0; i < 3; i++) res[i] /= kFourPi;
}

// R_Rot_Colloc, R.h:89-111
static void R_colloc(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    double y[3];
    centre(c, y);
    if (dist3(x, y) < kEps) { res[0] = res[1] = res[2] = 0.; return; }
    KP p;
    p.smoothR = kEps;
    p.smoothRMin = kEps;
    p.k = k;
    cd g[3];
    integral_cell<cd>(x, c, F_GradSimplePot_H, p, 3, np.n_start, np.p_max, np.eps, g);
    ccross_cc(g, j, res);
    for (int i = 0; i < 3; i++) res[i] /= kFourPi;
}

// R_Rot_Near, R.h:140-175
static void R_near(const cd* j, const double* x, const Cell& c, const NP& np, cd k, cd* res) {
    double nrm[3];
    normal(c, nrm);
    double dm = diam(c);
    KP p;
    p.smoothR = np.rs * dm / np.n_start;
    p.smoothRMin = dm / 100.;
    p.k = k;
    for (int i = 0; i < 3; i++) p.n[i] = nrm[i];
    cd surf[3];
    integral_cell<cd>(x, c, nF_DoublePot_H, p, 3, np.n_start, np.p_max, np.eps, surf);
    KP ps;
    ps.smoothR = kEps;
    ps.smoothRMin = kEps;
    ps.k = k;
    cd curl[3];
    K0_Common(x, c, nuF_SimplePot_H, ps, np.n_start_seg, np.p_max_seg, np.eps, curl);
    cd t[3];
    for (int i = 0; i < 3; i++) t[i] = (surf[i] + curl[i]) / kFourPi;
    ccross_cc(j, t, res);
}

typedef void (*PairOp)(const cd*, const double*, const Cell&, const NP&, cd, cd*);
static PairOp op_table(int op) {
    switch (op) {
        case BIELCC_OP_K_NEAR_SMOOTH: return K_near_smooth;
        case BIELCC_OP_K_HS: return K_hs;
        case BIELCC_OP_K_HS_COLLOC: return K_hs_colloc;
        case BIELCC_OP_K_HS2_COLLOC: return K_hs2_colloc;
        case BIELCC_OP_K_FAR: return K_far;
        case BIELCC_OP_R_SMOOTH: return R_smooth;
        case BIELCC_OP_R_COLLOC: return R_colloc;
        case BIELCC_OP_R_NEAR: return R_near;
        default: return nullptr;
    }
}

static void kp_from(const bielcc_kernelparam* s, KP& d) {
    d.smoothR = s->smoothR;
    d.smoothRMin = s->smoothRMin;
    d.k = cd(s->k_re, s->k_im);
    for (int i = 0; i < 3; i++) {
        d.current[i] = cd(s->current[i][0], s->current[i][1]);
        d.vec_dbl[i] = s->vec_dbl[i];
        d.n[i] = s->n[i];
        d.e0[i] = s->e0[i];
    }
}

static Integrand<cd> cplx_integrand(int id) {
    switch (id) {
        case BIELCC_F_SIMPLEPOT_H: return F_SimplePot_H;
        case BIELCC_F_NU_SIMPLEPOT_H: return nuF_SimplePot_H;
        case BIELCC_F_SIMPLEPOT_HM1: return F_SimplePot_Hm1;
        case BIELCC_F_GRADSIMPLEPOT_H: return F_GradSimplePot_H;
        case BIELCC_F_GRADSIMPLEPOT_HM1: return F_GradSimplePot_Hm1;
        case BIELCC_F_DOUBLEPOT_H: return F_DoublePot_H;
        case BIELCC_F_N_DOUBLEPOT_H: return nF_DoublePot_H;
        case BIELCC_F_ROTROTSIMPLEPOT_H: return F_RotRotSimplePot_H;
        case BIELCC_F_PLANEWAVE_E: return PlaneWave_E;
        default: return nullptr;
    }
}
static Integrand<double> real_integrand(int id) {
    switch (id) {
        case BIELCC_F_SIMPLEPOT_L: return F_SimplePot_L;
        case BIELCC_F_GRADSIMPLEPOT_L: return F_GradSimplePot_L;
        case BIELCC_F_DOUBLEPOT_L: return F_DoublePot_L;
        case BIELCC_F_VECTORPOT_L: return F_VectorPot_L;
        case BIELCC_F_ONE: return F_One;
        default: return nullptr;
    }
}
static int integrand_dim(int id) {
    switch (id) {
        case BIELCC_F_SIMPLEPOT_L: case BIELCC_F_DOUBLEPOT_L: case BIELCC_F_SIMPLEPOT_H:
        case BIELCC_F_SIMPLEPOT_HM1: case BIELCC_F_DOUBLEPOT_H: case BIELCC_F_ONE: return 1;
        default: return 3;
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

// Field driver: GetFieldE_Ideal (electrodynamics/get_field.h:35-78) for E plus
// the H loop of examples/field/main0_field_test.cpp:237-311 (far R_Rot_Colloc,
// near R_Rot_Smooth) with get_field's per-cell near criterion. Points are
// split over `n_threads` OpenMP threads (0 = runtime default), as get_field.h:49.
int oracle_field_EH(int n_vert, int n_cells, const double* cells, int n_rhs, const double* J,
                    double k_re, double k_im, double mult_re, double mult_im,
                    const bielcc_planewave* inc, const bielcc_numparam* npp, int n_pts,
                    const double* pts, double* E, double* H, int n_threads) {
    if ((n_vert != 3 && n_vert != 4) || n_cells < 0 || n_pts < 0 || n_rhs < 1) return BIELCC_ERR_ARG;
    NP np = np_from(npp);
    cd k(k_re, k_im), mult(mult_re, mult_im);
    const cd* Jc = reinterpret_cast<const cd*>(J);
    cd* Ec = reinterpret_cast<cd*>(E);
    cd* Hc = reinterpret_cast<cd*>(H);
    // per-cell geometry the reference recomputes per pair (identical values)
    std::vector<double> ctr(3 * (size_t)n_cells), thr((size_t)n_cells);
    for (int c = 0; c < n_cells; c++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)c * n_vert * 3)};
        centre(cl, &ctr[3 * (size_t)c]);
        thr[c] = np.analytic_calc * diam(cl);
    }
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int i = 0; i < n_pts; i++) {
        const double* x = pts + 3 * (size_t)i;
        for (int s = 0; s < n_rhs; s++) {
            cd e[3] = {0., 0., 0.}, h[3] = {0., 0., 0.};
            for (int c = 0; c < n_cells; c++) {
                Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)c * n_vert * 3)};
                const cd* j = Jc + ((size_t)s * n_cells + c) * 3;
                cd tk[3], tr[3];
                if (dist3(x, &ctr[3 * (size_t)c]) < thr[c]) {
                    K_near_smooth(j, x, cl, np, k, tk);
                    R_smooth(j, x, cl, np, k, tr);
                } else {
                    K_far(j, x, cl, np, k, tk);
                    R_colloc(j, x, cl, np, k, tr);
                }
                for (int g = 0; g < 3; g++) { e[g] += tk[g]; h[g] += tr[g]; }
            }
            for (int g = 0; g < 3; g++) e[g] *= mult;
            if (inc) {
                cd ph = std::exp(cd(0., 1.) * dot3(inc->k_vec, x));
                double kx0[3];
                cross3(inc->k_vec, inc->e0, kx0);
                if (inc->add_E)
                    for (int g = 0; g < 3; g++) e[g] += inc->e0[g] * ph;
                if (inc->add_H)
                    for (int g = 0; g < 3; g++) h[g] += kx0[g] * (ph * inc->h_scale);
            }
            cd* eo = Ec + ((size_t)s * n_pts + i) * 3;
            for (int g = 0; g < 3; g++) eo[g] = e[g];
            if (Hc) {
                cd* ho = Hc + ((size_t)s * n_pts + i) * 3;
                for (int g = 0; g < 3; g++) ho[g] = h[g];
            }
        }
    }
    return BIELCC_OK;
}

int oracle_pair_op(int op, int n_vert, int n_pairs, const double* cells, const double* x, const double* j,
                   double k_re, double k_im, const bielcc_numparam* npp, double* res) {
    PairOp f = op_table(op);
    if (!f || (n_vert != 3 && n_vert != 4) || n_pairs < 0) return BIELCC_ERR_ARG;
    NP np = np_from(npp);
    cd k(k_re, k_im);
#ifdef _OPENMP
#pragma omp parallel for
#endif
    for (int p = 0; p < n_pairs; p++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)p * n_vert * 3)};
        f(reinterpret_cast<const cd*>(j) + 3 * (size_t)p, x + 3 * (size_t)p, cl, np, k,
          reinterpret_cast<cd*>(res) + 3 * (size_t)p);
    }
    return BIELCC_OK;
}

int oracle_integral_pnt(int integrand, int n_vert, int n_pairs, const double* cells, const double* x,
                        bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    if ((n_vert != 3 && n_vert != 4) || integrand < 0 || integrand >= BIELCC_F_COUNT) return BIELCC_ERR_ARG;
    int idim = integrand_dim(integrand);
    for (int p = 0; p < n_pairs; p++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)p * n_vert * 3)};
        KP k;
        kp_from(kp + p, k);
        if (auto fc = cplx_integrand(integrand))
            integral_cell<cd>(x + 3 * (size_t)p, cl, fc, k, idim, n_start, p_max, eps,
                              reinterpret_cast<cd*>(res) + (size_t)idim * p);
        else
            integral_cell<double>(x + 3 * (size_t)p, cl, real_integrand(integrand), k, idim, n_start, p_max,
                                  eps, res + (size_t)idim * p);
        kp[p].smoothR = k.smoothR;  // the reference leaves its KernelParam mutated
    }
    return BIELCC_OK;
}

int oracle_integral_seg_pnt(int integrand, int n_pairs, const double* a, const double* b, const double* x,
                            bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    if (integrand < 0 || integrand >= BIELCC_F_COUNT) return BIELCC_ERR_ARG;
    int idim = integrand_dim(integrand);
    for (int p = 0; p < n_pairs; p++) {
        KP k;
        kp_from(kp + p, k);
        if (auto fc = cplx_integrand(integrand))
            integral_seg<cd>(a + 3 * (size_t)p, b + 3 * (size_t)p, x + 3 * (size_t)p, fc, k, idim, n_start,
                             p_max, eps, reinterpret_cast<cd*>(res) + (size_t)idim * p);
        else
            integral_seg<double>(a + 3 * (size_t)p, b + 3 * (size_t)p, x + 3 * (size_t)p,
                                 real_integrand(integrand), k, idim, n_start, p_max, eps,
                                 res + (size_t)idim * p);
        kp[p].smoothR = k.smoothR;
    }
    return BIELCC_OK;
}

// IntegralUniversal, the F(x) form (integrators/integral_universal.h:252-334
// quad, :347-431 triangle): the nodes and weights of IntegralUniversalPnt with
// a one-point integrand (F = 1 or PlaneWaveFieldE).
static bool one_point(int id) { return id == BIELCC_F_ONE || id == BIELCC_F_PLANEWAVE_E; }

int oracle_integral(int integrand, int n_vert, int n_cells, const double* cells, bielcc_kernelparam* kp,
                    int n_start, int p_max, double eps, double* res) {
    if ((n_vert != 3 && n_vert != 4) || !one_point(integrand)) return BIELCC_ERR_ARG;
    int idim = integrand_dim(integrand);
    const double none[3] = {0, 0, 0};
    for (int p = 0; p < n_cells; p++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)p * n_vert * 3)};
        KP k;
        kp_from(kp + p, k);
        if (auto fc = cplx_integrand(integrand))
            integral_cell<cd>(none, cl, fc, k, idim, n_start, p_max, eps, reinterpret_cast<cd*>(res) + (size_t)idim * p);
        else
            integral_cell<double>(none, cl, real_integrand(integrand), k, idim, n_start, p_max, eps,
                                  res + (size_t)idim * p);
        kp[p].smoothR = k.smoothR;
    }
    return BIELCC_OK;
}

// IntegralUniversalSegPnt, the F(x) overload (integral_universal_seg.h:120-179).
int oracle_integral_seg(int integrand, int n_segs, const double* a, const double* b, bielcc_kernelparam* kp,
                        int n_start, int p_max, double eps, double* res) {
    if (!one_point(integrand)) return BIELCC_ERR_ARG;
    int idim = integrand_dim(integrand);
    const double none[3] = {0, 0, 0};
    for (int p = 0; p < n_segs; p++) {
        KP k;
        kp_from(kp + p, k);
        if (auto fc = cplx_integrand(integrand))
            integral_seg<cd>(a + 3 * (size_t)p, b + 3 * (size_t)p, none, fc, k, idim, n_start, p_max, eps,
                             reinterpret_cast<cd*>(res) + (size_t)idim * p);
        else
            integral_seg<double>(a + 3 * (size_t)p, b + 3 * (size_t)p, none, real_integrand(integrand), k, idim,
                                 n_start, p_max, eps, res + (size_t)idim * p);
        kp[p].smoothR = k.smoothR;
    }
    return BIELCC_OK;
}

int oracle_k0(int integrand, int common, int n_vert, int n_pairs, const double* cells, const double* x,
              const double* j, bielcc_kernelparam* kp, int n_seg, int p_seg, double eps, double* res) {
    auto f = cplx_integrand(integrand);
    if (!f || integrand_dim(integrand) != 3) return BIELCC_ERR_ARG;
    for (int p = 0; p < n_pairs; p++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)p * n_vert * 3)};
        KP k;
        kp_from(kp + p, k);
        cd* r = reinterpret_cast<cd*>(res) + 3 * (size_t)p;
        if (common) K0_Common(x + 3 * (size_t)p, cl, f, k, n_seg, p_seg, eps, r);
        else K0(reinterpret_cast<const cd*>(j) + 3 * (size_t)p, x + 3 * (size_t)p, cl, f, k, n_seg, p_seg, eps, r);
        kp[p].smoothR = k.smoothR;
    }
    return BIELCC_OK;
}

int oracle_integral_1divr(int n_vert, int n_pairs, const double* cells, const double* x, double* res) {
    for (int p = 0; p < n_pairs; p++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)p * n_vert * 3)};
        res[p] = integral_1divr(cl, x + 3 * (size_t)p);
    }
    return BIELCC_OK;
}

int oracle_integral_grad1divr_seg(int n_pairs, const double* a, const double* b, const double* x, double* res) {
    for (int p = 0; p < n_pairs; p++)
        grad_1divr_seg(a + 3 * (size_t)p, b + 3 * (size_t)p, x + 3 * (size_t)p, res + 3 * (size_t)p);
    return BIELCC_OK;
}

int oracle_integral_surf_simplepot_h_hs(int n_vert, int n_pairs, const double* cells, const double* x,
                                        double analytic_r, int n_start, int p_max, double eps, double k_re,
                                        double k_im, double* res) {
    for (int p = 0; p < n_pairs; p++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)p * n_vert * 3)};
        reinterpret_cast<cd*>(res)[p] =
            surf_simplepot_h_hs(cl, x + 3 * (size_t)p, analytic_r, n_start, p_max, eps, cd(k_re, k_im));
    }
    return BIELCC_OK;
}

int oracle_integral_seg_gradsimplepot_h_hs(int n_pairs, const double* a, const double* b, const double* x,
                                           double analytic_r, int n_start, int p_max, double eps, double k_re,
                                           double k_im, double* res) {
    for (int p = 0; p < n_pairs; p++)
        seg_gradsimplepot_h_hs(a + 3 * (size_t)p, b + 3 * (size_t)p, x + 3 * (size_t)p, analytic_r, n_start,
                               p_max, eps, cd(k_re, k_im), reinterpret_cast<cd*>(res) + 3 * (size_t)p);
    return BIELCC_OK;
}

int oracle_area_by_quadrature(int n_vert, const double* cell, int n_start, int p_max, double eps, double* res) {
    Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cell)};
    res[0] = area_by_quadrature(cl, n_start, p_max, eps);
    return BIELCC_OK;
}

// Per-cell geometry rows as SurfMesh / CellFill expose them:
// out[c] = centre(3), diam, normal(3), tau1(3), tau2(3), area = 14 doubles.
int oracle_cell_geometry(int n_vert, int n_cells, const double* cells, double* out) {
    for (int c = 0; c < n_cells; c++) {
        Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)c * n_vert * 3)};
        double* o = out + 14 * (size_t)c;
        centre(cl, o);
        o[3] = diam(cl);
        normal(cl, o + 4);
        tangents(cl, o + 7, o + 10);
        // cell area as CellFill stores it (_s): quad = |mid-edge cross|, tri = |ab x ac|/2
        if (n_vert == 4) {
            double ma[3], mb[3], mc[3], md[3], ac[3], bd[3], v[3];
            for (int i = 0; i < 3; i++) {
                ma[i] = (cl.v[0][i] + cl.v[1][i]) / 2.0; mb[i] = (cl.v[1][i] + cl.v[2][i]) / 2.0;
                mc[i] = (cl.v[2][i] + cl.v[3][i]) / 2.0; md[i] = (cl.v[3][i] + cl.v[0][i]) / 2.0;
                ac[i] = mc[i] - ma[i]; bd[i] = md[i] - mb[i];
            }
            cross3(ac, bd, v);
            o[13] = len3(v);
        } else {
            o[13] = tri_area(cl.v[0], cl.v[1], cl.v[2]);
        }
    }
    return BIELCC_OK;
}

// Collocation assembly rows [row_begin, row_end) of
//   A[(i,a),(j,b)] = tau_a(i) . K[cell_j, tau_b(j)](c_i)       (layout TAU2)
//   A[(i,p),(j,q)] = e_p . K[cell_j, e_q](c_i)                  (layout FULL3)
// near (|c_i - c_j| < analytic_calc*diam_j): K_RotRot_HS_Colloc (K.h:179-204),
// far: K_RotRot_Far (K.h:288-301). A is complex128, row-major over ALL columns,
// holding only the requested rows.
int oracle_assemble_K(int n_vert, int n_cells, const double* cells, double k_re, double k_im,
                      const bielcc_numparam* npp, int layout, int row_begin, int row_end, double* A) {
    if (layout != BIELCC_LAYOUT_TAU2 && layout != BIELCC_LAYOUT_FULL3) return BIELCC_ERR_ARG;
    NP np = np_from(npp);
    cd k(k_re, k_im);
    int m = layout == BIELCC_LAYOUT_TAU2 ? 2 : 3;
    size_t ncols = (size_t)m * n_cells;
    std::vector<double> geo(14 * (size_t)n_cells);
    oracle_cell_geometry(n_vert, n_cells, cells, geo.data());
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int i = row_begin; i < row_end; i++) {
        const double* ci = &geo[14 * (size_t)i];
        for (int j = 0; j < n_cells; j++) {
            Cell cl{n_vert, reinterpret_cast<const double(*)[3]>(cells + (size_t)j * n_vert * 3)};
            const double* gj = &geo[14 * (size_t)j];
            bool near = dist3(ci, gj) < np.analytic_calc * gj[3];
            for (int b = 0; b < m; b++) {
                cd jv[3];
                for (int g = 0; g < 3; g++) {
                    double comp = (layout == BIELCC_LAYOUT_TAU2) ? gj[7 + 3 * b + g] : (g == b ? 1. : 0.);
                    jv[g] = comp;
                }
                cd kv[3];
                if (near) K_hs_colloc(jv, ci, cl, np, k, kv);
                else K_far(jv, ci, cl, np, k, kv);
                for (int a = 0; a < m; a++) {
                    cd v;
                    if (layout == BIELCC_LAYOUT_TAU2) v = kv[0] * ci[7 + 3 * a] + kv[1] * ci[8 + 3 * a] + kv[2] * ci[9 + 3 * a];
                    else v = kv[a];
                    size_t row = (size_t)(i - row_begin) * m + a;
                    size_t col = (size_t)j * m + b;
                    A[2 * (row * ncols + col)] = v.real();
                    A[2 * (row * ncols + col) + 1] = v.imag();
                }
            }
        }
    }
    return BIELCC_OK;
}

}  // extern "C"
