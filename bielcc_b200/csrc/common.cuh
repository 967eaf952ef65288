// common.cuh — device complex types, constants and small helpers shared by
// every kernel of libbielcc_gpu.so (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define BIELCC_HD __host__ __device__ __forceinline__
#define BIELCC_D __device__ __forceinline__

namespace bielcc_gpu {

constexpr double kMachineZero = 2.220446049250313080847e-16;  // DBL_EPSILON (Tolerance_Constants::MACHINE_ZERO)
constexpr double kFourPi = 12.566370614359172953850;          // 4 * M_PI
constexpr double kInvFourPi = 0.079577471545947667884;        // 1 / (4 pi)

// ------------------------------------------------------------------ complex FP64
struct cplx {
    double re, im;
};
BIELCC_HD cplx mk(double r, double i) { return cplx{r, i}; }
BIELCC_HD cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
BIELCC_HD cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
BIELCC_HD cplx operator-(cplx a) { return {-a.re, -a.im}; }
BIELCC_HD cplx operator*(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
BIELCC_HD cplx operator*(cplx a, double s) { return {a.re * s, a.im * s}; }
BIELCC_HD cplx operator*(double s, cplx a) { return {a.re * s, a.im * s}; }
BIELCC_HD cplx operator/(cplx a, double s) { return {a.re / s, a.im / s}; }
BIELCC_HD cplx& operator+=(cplx& a, cplx b) { a.re += b.re; a.im += b.im; return a; }
BIELCC_HD cplx& operator*=(cplx& a, cplx b) { a = a * b; return a; }
BIELCC_HD cplx& operator*=(cplx& a, double s) { a.re *= s; a.im *= s; return a; }
BIELCC_HD double cabs2(cplx a) { return a.re * a.re + a.im * a.im; }
BIELCC_D double cabs(cplx a) { return hypot(a.re, a.im); }
// exp(z) for complex z
BIELCC_D cplx cexp(cplx z) {
    double s, c;
    sincos(z.im, &s, &c);
    double m = exp(z.re);
    return {m * c, m * s};
}
// exp(i r k): the reference's std::exp(complex(0, r) * k); (0 + i r)(kr + i ki)
BIELCC_D cplx eikr(double r, cplx k) {
    double s, c;
    sincos(r * k.re, &s, &c);
    if (k.im == 0.0) return {c, s};
    double m = exp(-r * k.im);
    return {m * c, m * s};
}

// ------------------------------------------------------------------ complex FP32
struct cplxf {
    float re, im;
};
BIELCC_D cplxf operator*(cplxf a, cplxf b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
BIELCC_D cplxf operator+(cplxf a, cplxf b) { return {a.re + b.re, a.im + b.im}; }

// ------------------------------------------------------------------ vectors
BIELCC_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
BIELCC_HD void cross3(const double* a, const double* b, double* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
BIELCC_D double len3(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
BIELCC_D double dist3(const double* a, const double* b) {
    double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}
// |a - b| rounded exactly as the reference's dist() on a CPU without FMA
// contraction (geometry/element_geom.h:91-98). Used wherever a near/far
// decision is taken, so every kernel takes the same decision for a pair.
BIELCC_D double dist3_rn(const double* a, const double* b) {
    double d0 = __dsub_rn(a[0], b[0]), d1 = __dsub_rn(a[1], b[1]), d2 = __dsub_rn(a[2], b[2]);
    double s = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
    return __dsqrt_rn(s);
}
BIELCC_D cplx cdot_cr(const cplx* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
BIELCC_D void ccross_cc(const cplx* a, const cplx* b, cplx* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

// Per-cell geometry row written by the mesh preparation kernel (16 doubles,
// 128 B): centre(3), diam, normal(3), tau1(3), tau2(3), area, rho, pad.
// rho = largest distance of a vertex from the centre.
struct CellGeo {
    double c[3];
    double diam;
    double n[3];
    double t1[3];
    double t2[3];
    double area;
    double rho;
    double pad;
};
static_assert(sizeof(CellGeo) == 128, "CellGeo must stay 128 B");

}  // namespace bielcc_gpu
