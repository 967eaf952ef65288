// farnode.cuh — the per-node far-field integrand shared by the far kernels
// (field.cu, batch.cu): F_RotRotSimplePot_H (kernel_lib.h:453-492) and
// F_GradSimplePot_H (kernel_lib.h:295-313) evaluated together at one
// quadrature node and accumulated as J-independent moments of one cell:
//   A1 = sum w e f1,  T = sum w e f2 d^ d^T (6),  G = sum w e (ikr - 1)/r^3 d (3)
// so that K_RotRot_Far = (A1 J + T J)/4pi and R_Rot_Colloc = (G x J)/4pi.
// FP64 and FP32 (phase split relative to the cell centre) forms.
//
// Real k: with alpha = 1/r^3 - i k/r^2 and u = k^2/r,
//   f1 = u - alpha, f2 = 3 alpha - u, (ikr - 1)/r^3 = -alpha.
// The node loop accumulates S = sum w e alpha in place of A1 and T/3 in place
// of T; since |d|^2 = r^2, tr T = 3 S - sum w e u, so A1 = 2 S - tr T, which
// finish_real_k recovers once per cell (two accumulators and the k^2/r
// product leave the per-node work).
#pragma once
#include "common.cuh"

namespace bielcc_gpu {

// Near decision of get_field.h:58 with the reference's rounding.
BIELCC_D bool is_near(const double* x, const double* c, double diam, double analytic_calc, double* d_out) {
    double d = dist3_rn(x, c);
    *d_out = d;
    return d < __dmul_rn(analytic_calc, diam);
}

// Per-thread moment accumulators of one cell.
template <typename F>
struct Moments {
    F a1r, a1i;
    F t[6][2];  // xx, xy, xz, yy, yz, zz
    F g[3][2];
    BIELCC_D void zero() {
        a1r = a1i = 0;
        for (int i = 0; i < 6; i++) t[i][0] = t[i][1] = 0;
        for (int i = 0; i < 3; i++) g[i][0] = g[i][1] = 0;
    }
    BIELCC_D void finish_real_k();
};

// Real-k node loops leave (S, T/3) in (a1, t): turn them into (A1, T).
template <typename F>
BIELCC_D void finish_real_k(F& a1r, F& a1i, F (&t)[6][2]) {
    const F trr = t[0][0] + t[3][0] + t[5][0], tri = t[0][1] + t[3][1] + t[5][1];
    a1r = F(2) * a1r - F(3) * trr;
    a1i = F(2) * a1i - F(3) * tri;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        t[q][0] *= F(3);
        t[q][1] *= F(3);
    }
}

template <typename F>
BIELCC_D void Moments<F>::finish_real_k() {
    bielcc_gpu::finish_real_k<F>(a1r, a1i, t);
}

// FP32 wavenumber constants of one launch (or one job).
struct KF32 {
    float kr, ki;    // k
    float k2r, k2i;  // k^2
    float ikr;       // 1 / Re k, 1e30 for Re k = 0 (phase k (r - r0) = q / ((r + r0) ikr) then rounds to 0)
    float k2r3;      // Re k^2 / 3
    static BIELCC_D KF32 make(double kre, double kim) {
        KF32 f;
        const double k2r = kre * kre - kim * kim;
        f.kr = (float)kre;
        f.ki = (float)kim;
        f.k2r = (float)k2r;
        f.k2i = (float)(2.0 * kre * kim);
        f.ikr = kre != 0.0 ? (float)(1.0 / kre) : 1e30f;
        f.k2r3 = (float)(k2r / 3.0);
        return f;
    }
};

// e^{i t} in FP64 from its Taylor series; the length follows a bound on |t|
// (a template level, uniform over a cell): TD 0 |t| <= 0.5 (sin to t^13, cos
// to t^14), TD 1 |t| <= 0.25 (t^11, t^12), TD 2 |t| <= 0.125 (t^9, t^10);
// truncation below 3e-17 in each case. Coefficients are +-1/n!.
template <int TD = 0>
BIELCC_D void sincos_taylor64(double t, double* s, double* c) {
    double t2 = t * t;
    double ps;
    if (TD == 0) ps = fma(fma(t2, -1.6059043836821613e-10, 2.5052108385441720e-08), t2, -2.7557319223985893e-06);
    else if (TD == 1) ps = fma(t2, 2.5052108385441720e-08, -2.7557319223985893e-06);
    else ps = -2.7557319223985893e-06;
    ps = fma(t2, ps, 1.9841269841269841e-04);
    ps = fma(t2, ps, -8.3333333333333333e-03);
    ps = fma(t2, ps, 1.6666666666666667e-01);
    *s = t - t * t2 * ps;
    double pc;
    if (TD == 0) pc = fma(fma(t2, 1.1470745597729725e-11, -2.0876756987868099e-09), t2, 2.7557319223985891e-07);
    else if (TD == 1) pc = fma(t2, -2.0876756987868099e-09, 2.7557319223985891e-07);
    else pc = 2.7557319223985891e-07;
    pc = fma(t2, pc, -2.4801587301587302e-05);
    pc = fma(t2, pc, 1.3888888888888889e-03);
    pc = fma(t2, pc, -4.1666666666666667e-02);
    pc = fma(t2, pc, 0.5);
    *c = 1.0 - t2 * pc;
}

// One far node, FP64. dx = x - y; w = node weight. Real k (CK = false) or
// complex k. F_RotRotSimplePot_H (kernel_lib.h:453-492) and
// F_GradSimplePot_H (kernel_lib.h:295-313) share r, 1/r and e^{ikr}.
// SPLIT: the phase is taken relative to r0 = |x - centre| (the moments are
// multiplied by e^{ik r0} once per cell) and e^{ik (r - r0)} comes from the
// Taylor series; otherwise e^{ikr} from sincos per node.
template <bool CK, bool SPLIT, int TD = 0>
BIELCC_D void far_node_f64(Moments<double>& m, double dx, double dy, double dz, double w, cplx k, double k2r,
                           double k2i, double r0) {
    double r2 = dx * dx + dy * dy + dz * dz;
    double ir = rsqrt(r2);
    double r = r2 * ir;
    double s, c;
    if (SPLIT) {
        sincos_taylor64<TD>(k.re * (r - r0), &s, &c);
    } else {
        sincos(k.re * r, &s, &c);
        if (CK) {
            double a = exp(-k.im * r);
            s *= a;
            c *= a;
        }
    }
    double ir2 = ir * ir, ir3 = ir2 * ir;
    double er = w * c, ei = w * s;
    if (!CK) {
        // real k: S += e alpha, T/3 += e (alpha - u/3)/r^2 d d^T, G -= e alpha d
        const double beta = k.re * ir2;
        const double ear = fma(ei, beta, er * ir3), eai = fma(-er, beta, ei * ir3);
        if (r >= kMachineZero) {  // F_RotRotSimplePot_H is 0 below MACHINE_ZERO
            m.a1r += ear;
            m.a1i += eai;
            const double u3 = k2r * (1.0 / 3.0) * ir3;
            const double a2r = fma(ear, ir2, -er * u3), a2i = fma(eai, ir2, -ei * u3);
            const double dd[6] = {dx * dx, dx * dy, dx * dz, dy * dy, dy * dz, dz * dz};
#pragma unroll
            for (int q = 0; q < 6; q++) {
                m.t[q][0] += a2r * dd[q];
                m.t[q][1] += a2i * dd[q];
            }
        }
        m.g[0][0] -= ear * dx;
        m.g[0][1] -= eai * dx;
        m.g[1][0] -= ear * dy;
        m.g[1][1] -= eai * dy;
        m.g[2][0] -= ear * dz;
        m.g[2][1] -= eai * dz;
        return;
    }
    if (r >= kMachineZero) {  // F_RotRotSimplePot_H is 0 below MACHINE_ZERO
        double f1r, f1i, f2r, f2i;
        if (CK) {
            f1r = k2r * ir - ir3 - k.im * ir2;
            f1i = k.re * ir2 + k2i * ir;
            f2r = 3.0 * ir3 + 3.0 * k.im * ir2 - k2r * ir;
            f2i = -3.0 * k.re * ir2 - k2i * ir;
        } else {
            f1r = k2r * ir - ir3;
            f1i = k.re * ir2;
            f2r = 3.0 * ir3 - k2r * ir;
            f2i = -3.0 * k.re * ir2;
        }
        m.a1r += er * f1r - ei * f1i;
        m.a1i += er * f1i + ei * f1r;
        double a2r = (er * f2r - ei * f2i) * ir2, a2i = (er * f2i + ei * f2r) * ir2;
        double dd[6] = {dx * dx, dx * dy, dx * dz, dy * dy, dy * dz, dz * dz};
#pragma unroll
        for (int q = 0; q < 6; q++) {
            m.t[q][0] += a2r * dd[q];
            m.t[q][1] += a2i * dd[q];
        }
    }
    // (ikr - 1) with ikr = (-k.im r, k.re r)
    double ur = CK ? (-k.im * r - 1.0) : -1.0, ui = k.re * r;
    double gr = (er * ur - ei * ui) * ir3, gi = (er * ui + ei * ur) * ir3;
    m.g[0][0] += gr * dx;
    m.g[0][1] += gi * dx;
    m.g[1][0] += gr * dy;
    m.g[1][1] += gi * dy;
    m.g[2][0] += gr * dz;
    m.g[2][1] += gi * dz;
}

// Taylor sine / cosine on |t| <= 1 (truncation below 2.6e-8), FP32.
BIELCC_D void sincos_poly(float t, float* s, float* c) {
    float t2 = t * t;
    float ps = fmaf(t2, 2.7557319e-6f, -1.9841270e-4f);
    ps = fmaf(t2, ps, 8.3333333e-3f);
    ps = fmaf(t2, ps, -1.6666667e-1f);
    ps = fmaf(t2, ps, 1.0f);
    *s = t * ps;
    float pc = fmaf(t2, -2.7557319e-7f, 2.4801587e-5f);
    pc = fmaf(t2, pc, -1.3888889e-3f);
    pc = fmaf(t2, pc, 4.1666667e-2f);
    pc = fmaf(t2, pc, -0.5f);
    *c = fmaf(t2, pc, 1.0f);
}

// Short Taylor sine / cosine for |t| <= 0.25 (truncation below 1.3e-8).
BIELCC_D void sincos_short(float t, float* s, float* c) {
    float t2 = t * t;
    float ps = fmaf(t2, 8.3333333e-3f, -1.6666667e-1f);
    *s = t * fmaf(t2, ps, 1.0f);
    float pc = fmaf(t2, -1.3888889e-3f, 4.1666667e-2f);
    pc = fmaf(t2, pc, -0.5f);
    *c = fmaf(t2, pc, 1.0f);
}

// e^{i theta} for a per-cell bound on |theta| (uniform over the CTA, so the
// mode is a template argument of the node loop): 0 -> |theta| <= 0.25 short
// polynomial; 1 -> <= 1; 2 -> <= 2 (half angle, one doubling); 3 -> <= 4 (two
// doublings); 4 -> accurate sincosf.
template <int MODE>
BIELCC_D void phase_f32(float th, float* s, float* c) {
    if constexpr (MODE == 0) {
        sincos_short(th, s, c);
    } else if constexpr (MODE == 4) {
        sincosf(th, s, c);
    } else {
        constexpr int H = MODE - 1;
        float ss, cc;
        sincos_poly(th * (H == 0 ? 1.f : (H == 1 ? 0.5f : 0.25f)), &ss, &cc);
#pragma unroll
        for (int h = 0; h < H; h++) {
            float ns = 2.f * ss * cc;
            cc = fmaf(cc, cc, -ss * ss);
            ss = ns;
        }
        *s = ss;
        *c = cc;
    }
}

BIELCC_HD int phase_mode(float th) {
    return th <= 0.25f ? 0 : (th <= 1.f ? 1 : (th <= 2.f ? 2 : (th <= 4.f ? 3 : 4)));
}

// Per-pair FP32 state of the mixed far node, relative to the cell centre:
// X = x - centre, X2 = -2 X, r0 = |X| (FP64 rounded), r0sq = r0^2, r0k = r0 / Re k.
struct PairF32 {
    float X[3], X2[3], r0, r0sq, r0k;
    BIELCC_D void set(const double* x, const double* centre, double d, const KF32& kf) {
        for (int g = 0; g < 3; g++) {
            X[g] = (float)(x[g] - centre[g]);
            X2[g] = -2.f * X[g];
        }
        r0 = (float)d;
        r0sq = (float)(d * d);
        r0k = r0 * kf.ikr;
    }
};

// |y - centre|^2 of a staged node (computed once per node and CTA).
BIELCC_D float node_yy(float4 nd) { return fmaf(nd.x, nd.x, fmaf(nd.y, nd.y, nd.z * nd.z)); }

// Shared head of the FP32 far node: nd = (y - centre, w), yy = |y - centre|^2.
// q = |x - y|^2 - r0^2 = yy - 2 (y - centre).X carries no cancellation.
// Returns 1/r and sets r, the weighted phase factor e = w e^{ik(r - r0)} and d = x - y.
template <bool CK, int MODE>
BIELCC_D float far_head_f32(const PairF32& p, float4 nd, float yy, const KF32& kf, float& r_out, float& er, float& ei,
                            float& dx, float& dy, float& dz) {
    const float q = fmaf(nd.x, p.X2[0], fmaf(nd.y, p.X2[1], fmaf(nd.z, p.X2[2], yy)));
    const float r2 = p.r0sq + q;
    const float ir = rsqrtf(r2);
    const float r = r2 * ir;
    float s, c, w = nd.w;
    if (CK) {
        const float dr = __fdividef(q, r + p.r0);  // r - r0 without cancellation
        phase_f32<MODE>(kf.kr * dr, &s, &c);
        w *= __expf(-kf.ki * dr);
    } else {
        phase_f32<MODE>(__fdividef(q, fmaf(r, kf.ikr, p.r0k)), &s, &c);  // k (r - r0)
    }
    dx = p.X[0] - nd.x;
    dy = p.X[1] - nd.y;
    dz = p.X[2] - nd.z;
    er = w * c;
    ei = w * s;
    r_out = r;
    return ir;
}

// T += b d^T over the 6 symmetric entries, b = a2 d (complex a2).
BIELCC_D void acc_sym6(float (&t)[6][2], float a2r, float a2i, float dx, float dy, float dz) {
    const float bx_r = a2r * dx, bx_i = a2i * dx, by_r = a2r * dy, by_i = a2i * dy, bz_r = a2r * dz, bz_i = a2i * dz;
    t[0][0] = fmaf(bx_r, dx, t[0][0]);
    t[0][1] = fmaf(bx_i, dx, t[0][1]);
    t[1][0] = fmaf(bx_r, dy, t[1][0]);
    t[1][1] = fmaf(bx_i, dy, t[1][1]);
    t[2][0] = fmaf(bx_r, dz, t[2][0]);
    t[2][1] = fmaf(bx_i, dz, t[2][1]);
    t[3][0] = fmaf(by_r, dy, t[3][0]);
    t[3][1] = fmaf(by_i, dy, t[3][1]);
    t[4][0] = fmaf(by_r, dz, t[4][0]);
    t[4][1] = fmaf(by_i, dz, t[4][1]);
    t[5][0] = fmaf(bz_r, dz, t[5][0]);
    t[5][1] = fmaf(bz_i, dz, t[5][1]);
}

// One far node, FP32 (E and H moments). Real k leaves (S, T/3) in (a1, t):
// the caller runs finish_real_k once the cell's nodes are summed.
template <bool CK, int MODE>
BIELCC_D void far_node_f32(Moments<float>& m, const PairF32& p, float4 nd, float yy, const KF32& kf) {
    float r, er, ei, dx, dy, dz;
    const float ir = far_head_f32<CK, MODE>(p, nd, yy, kf, r, er, ei, dx, dy, dz);
    const float ir2 = ir * ir, ir3 = ir2 * ir;
    if (!CK) {
        const float beta = kf.kr * ir2;
        const float ear = fmaf(ei, beta, er * ir3), eai = fmaf(-er, beta, ei * ir3);  // e alpha
        m.a1r += ear;  // S
        m.a1i += eai;
        const float u3 = kf.k2r3 * ir3;                                               // k^2 / (3 r^3)
        const float a2r = fmaf(ear, ir2, -er * u3), a2i = fmaf(eai, ir2, -ei * u3);  // e (alpha - u/3) / r^2
        acc_sym6(m.t, a2r, a2i, dx, dy, dz);
        m.g[0][0] = fmaf(-ear, dx, m.g[0][0]);
        m.g[0][1] = fmaf(-eai, dx, m.g[0][1]);
        m.g[1][0] = fmaf(-ear, dy, m.g[1][0]);
        m.g[1][1] = fmaf(-eai, dy, m.g[1][1]);
        m.g[2][0] = fmaf(-ear, dz, m.g[2][0]);
        m.g[2][1] = fmaf(-eai, dz, m.g[2][1]);
        return;
    }
    const float f1r = kf.k2r * ir - ir3 - kf.ki * ir2;
    const float f1i = kf.kr * ir2 + kf.k2i * ir;
    const float f2r = 3.f * ir3 + 3.f * kf.ki * ir2 - kf.k2r * ir;
    const float f2i = -3.f * kf.kr * ir2 - kf.k2i * ir;
    m.a1r = fmaf(er, f1r, fmaf(-ei, f1i, m.a1r));
    m.a1i = fmaf(er, f1i, fmaf(ei, f1r, m.a1i));
    const float a2r = (er * f2r - ei * f2i) * ir2, a2i = (er * f2i + ei * f2r) * ir2;
    acc_sym6(m.t, a2r, a2i, dx, dy, dz);
    const float ur = -kf.ki * r - 1.f, ui = kf.kr * r;
    const float gr = (er * ur - ei * ui) * ir3, gi = (er * ui + ei * ur) * ir3;
    m.g[0][0] = fmaf(gr, dx, m.g[0][0]);
    m.g[0][1] = fmaf(gi, dx, m.g[0][1]);
    m.g[1][0] = fmaf(gr, dy, m.g[1][0]);
    m.g[1][1] = fmaf(gi, dy, m.g[1][1]);
    m.g[2][0] = fmaf(gr, dz, m.g[2][0]);
    m.g[2][1] = fmaf(gi, dz, m.g[2][1]);
}

// The K moments only (A1, T; no grad F) of one far node, FP32: the node
// arithmetic of far_node_f32 for the collocation matrix, whose entries need
// K_RotRot_Far alone. Real k leaves (S, T/3) as far_node_f32 does.
template <bool CK, int MODE>
BIELCC_D void far_node_f32_K(float& a1r, float& a1i, float (&t)[6][2], const PairF32& p, float4 nd, float yy,
                             const KF32& kf) {
    float r, er, ei, dx, dy, dz;
    const float ir = far_head_f32<CK, MODE>(p, nd, yy, kf, r, er, ei, dx, dy, dz);
    const float ir2 = ir * ir, ir3 = ir2 * ir;
    if (!CK) {
        const float beta = kf.kr * ir2;
        const float ear = fmaf(ei, beta, er * ir3), eai = fmaf(-er, beta, ei * ir3);
        a1r += ear;
        a1i += eai;
        const float u3 = kf.k2r3 * ir3;
        acc_sym6(t, fmaf(ear, ir2, -er * u3), fmaf(eai, ir2, -ei * u3), dx, dy, dz);
        return;
    }
    const float f1r = kf.k2r * ir - ir3 - kf.ki * ir2;
    const float f1i = kf.kr * ir2 + kf.k2i * ir;
    const float f2r = 3.f * ir3 + 3.f * kf.ki * ir2 - kf.k2r * ir;
    const float f2i = -3.f * kf.kr * ir2 - kf.k2i * ir;
    a1r = fmaf(er, f1r, fmaf(-ei, f1i, a1r));
    a1i = fmaf(er, f1i, fmaf(ei, f1r, a1i));
    acc_sym6(t, (er * f2r - ei * f2i) * ir2, (er * f2i + ei * f2r) * ir2, dx, dy, dz);
}

}  // namespace bielcc_gpu
