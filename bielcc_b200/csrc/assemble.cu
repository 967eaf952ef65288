// assemble.cu — collocation-matrix assembly of the K operator:
//   A[(i,a),(j,b)] = tau_a(i) . K[cell_j, tau_b(j)](c_i),  c_i = centre of cell i
// (layout TAU2, 2N x 2N) or the full 3x3 blocks (layout FULL3, 3N x 3N).
// K is linear in the cell current, so each (i, j) block is the 3x3 operator
// matrix projected on the tangent bases (CellFill, mesh/cell.cpp).
//   far  (|c_i - c_j| >= analytic_calc * diam_j): K_RotRot_Far (K.h:288-301)
//        = (A1 I + T) / 4pi from the precomputed node tables; FP64 or FP32
//        (phase split as in field.cu);
//   near: K_RotRot_HS_Colloc (K.h:179-204) in FP64 = I_hs k^2/4pi I + M / 4pi,
//        I_hs = IntegralSurf_SimplePot_H_HS (integrals_analytic.h:136-164),
//        M = -sum_e ks_e nu_e^T from the unsmoothed K0 (K0.h:36-86).
// Every entry is written exactly once (far kernel skips near pairs).
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "farnode.cuh"
#include "grid.h"
#include "internal.h"
#include "ops.cuh"
#include "scan.cuh"

namespace bielcc_gpu {

constexpr int kAsmThreads = 128;
constexpr int kAsmStageNodes = 256;
constexpr int kAsmMaxCells = 32;

struct AsmArgs {
    const CellGeo* geo;
    int n_cells;
    const double4* nodes64;
    const float4* nodes32;
    const float* rho32;
    int nn;
    cplx k;
    double analytic_calc;
    int cols_per_split;
    int m;  // 2 (tau) or 3 (full)
    int c64;
    void* A;
    unsigned* mask;  // [ceil(N/32)][N] near bits of (row i, column word) written by the far kernel, or null
};

// p_max >= 3, the far kernel's marks-reading variant: mark[b] [ceil(N/32)][N]
// is set for the (row, column) blocks whose column-b integral failed the
// convergence test at the second pass; take_marked 0 writes the columns that
// passed, 1 the ones that failed. (A separate type, so that the plain
// variants keep AsmArgs' parameter block.)
struct AsmArgsMarks : AsmArgs {
    const unsigned* mark;
    int take_marked;
};
template <bool MARKS>
using AsmArgsOf = typename std::conditional<MARKS, AsmArgsMarks, AsmArgs>::type;

BIELCC_D bool asm_is_near(const double* x, const CellGeo& g, double analytic_calc, double* d) {
    *d = dist3_rn(x, g.c);
    return *d < __dmul_rn(analytic_calc, g.diam);
}

// Writes the M x M block of (row cell i, column cell j) from the 3x3 complex
// operator matrix K (already / 4pi): M = 2 projects on tau1, tau2 of both
// cells, M = 3 keeps the Cartesian block. M is a template argument so that the
// block stays in registers.
template <int M>
BIELCC_D void write_block_m(const AsmArgs& a, int i, int j, const double (&Kr)[3][3], const double (&Ki)[3][3],
                            const double* ti1, const double* ti2, const double* tj1, const double* tj2,
                            unsigned cols = ~0u) {
    const size_t dim = (size_t)M * a.n_cells;
#pragma unroll
    for (int aa = 0; aa < M; aa++) {
        double rv[M][2];
#pragma unroll
        for (int b = 0; b < M; b++) {
            double vr = 0., vi = 0.;
            if constexpr (M == 3) {
                vr = Kr[aa][b];
                vi = Ki[aa][b];
            } else {
                const double* ta = aa == 0 ? ti1 : ti2;
                const double* tb = b == 0 ? tj1 : tj2;
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    double kr = Kr[p][0] * tb[0] + Kr[p][1] * tb[1] + Kr[p][2] * tb[2];
                    double ki = Ki[p][0] * tb[0] + Ki[p][1] * tb[1] + Ki[p][2] * tb[2];
                    vr += ta[p] * kr;
                    vi += ta[p] * ki;
                }
            }
            rv[b][0] = vr;
            rv[b][1] = vi;
        }
        const size_t off = ((size_t)i * M + aa) * dim + (size_t)j * M;
        if (a.c64) {
            float2* dst = reinterpret_cast<float2*>(a.A) + off;
#pragma unroll
            for (int b = 0; b < M; b++)
                if ((cols >> b) & 1u) dst[b] = make_float2((float)rv[b][0], (float)rv[b][1]);
        } else {
            double2* dst = reinterpret_cast<double2*>(a.A) + off;
#pragma unroll
            for (int b = 0; b < M; b++)
                if ((cols >> b) & 1u) dst[b] = make_double2(rv[b][0], rv[b][1]);
        }
    }
}

// The mixed form's far block, in FP32 (the moments are FP32 sums already):
// K = A1 I + T with T symmetric (xx, xy, xz, yy, yz, zz), projected on the two
// cells' tangents (M = 2: u_b = K t_b, A_ab = t_a . u_b) or kept Cartesian
// (M = 3), times ph = e^{ik r0} / 4pi.
// cols: bit b writes column b of the block (the convergence-test passes of
// p_max >= 3; all otherwise).
template <int M>
BIELCC_D void write_block_f32(const AsmArgs& a, int i, int j, float a1r, float a1i, const float (&t)[6][2], float phr,
                              float phi, const float (&ti)[2][3], const double* tj1, const double* tj2,
                              unsigned cols = ~0u) {
    const size_t dim = (size_t)M * a.n_cells;
    const int sym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    float kr[6], ki[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const bool diag = q == 0 || q == 3 || q == 5;
        kr[q] = diag ? t[q][0] + a1r : t[q][0];
        ki[q] = diag ? t[q][1] + a1i : t[q][1];
    }
    float out[M][M][2];
    if constexpr (M == 3) {
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < 3; q++) {
                out[p][q][0] = kr[sym[p][q]] * phr - ki[sym[p][q]] * phi;
                out[p][q][1] = kr[sym[p][q]] * phi + ki[sym[p][q]] * phr;
            }
    } else {
        const float tb[2][3] = {{(float)tj1[0], (float)tj1[1], (float)tj1[2]},
                                {(float)tj2[0], (float)tj2[1], (float)tj2[2]}};
#pragma unroll
        for (int b = 0; b < 2; b++) {
            float ur[3], ui[3];
#pragma unroll
            for (int p = 0; p < 3; p++) {
                ur[p] = kr[sym[p][0]] * tb[b][0] + kr[sym[p][1]] * tb[b][1] + kr[sym[p][2]] * tb[b][2];
                ui[p] = ki[sym[p][0]] * tb[b][0] + ki[sym[p][1]] * tb[b][1] + ki[sym[p][2]] * tb[b][2];
            }
#pragma unroll
            for (int aa = 0; aa < 2; aa++) {
                const float vr = ti[aa][0] * ur[0] + ti[aa][1] * ur[1] + ti[aa][2] * ur[2];
                const float vi = ti[aa][0] * ui[0] + ti[aa][1] * ui[1] + ti[aa][2] * ui[2];
                out[aa][b][0] = vr * phr - vi * phi;
                out[aa][b][1] = vr * phi + vi * phr;
            }
        }
    }
#pragma unroll
    for (int aa = 0; aa < M; aa++) {
        const size_t off = ((size_t)i * M + aa) * dim + (size_t)j * M;
        if (a.c64) {
            float2* dst = reinterpret_cast<float2*>(a.A) + off;
#pragma unroll
            for (int b = 0; b < M; b++)
                if ((cols >> b) & 1u) dst[b] = make_float2(out[aa][b][0], out[aa][b][1]);
        } else {
            double2* dst = reinterpret_cast<double2*>(a.A) + off;
#pragma unroll
            for (int b = 0; b < M; b++)
                if ((cols >> b) & 1u) dst[b] = make_double2(out[aa][b][0], out[aa][b][1]);
        }
    }
}

BIELCC_D void write_block(const AsmArgs& a, int i, int j, const double (&Kr)[3][3], const double (&Ki)[3][3],
                          const double* ti1, const double* ti2, const double* tj1, const double* tj2,
                          unsigned cols = ~0u) {
    if (a.m == 2) write_block_m<2>(a, i, j, Kr, Ki, ti1, ti2, tj1, tj2, cols);
    else write_block_m<3>(a, i, j, Kr, Ki, ti1, ti2, tj1, tj2, cols);
}

// Minimum resident CTAs per SM asked of the real-k mixed far kernel (0: the
// compiler's own register choice, which the other variants keep). 5 gives 96
// registers without spills (20,480 triangles: 65.0 -> 62.4 ms).
#ifndef BIELCC_ASM_MINB
#define BIELCC_ASM_MINB 5
#endif
template <bool CK, bool MIXED, bool MARKS = false>
__global__ void __launch_bounds__(kAsmThreads, (!CK && MIXED) ? BIELCC_ASM_MINB : 0)
    assemble_far_kernel(AsmArgsOf<MARKS> a) {
    using NodeT = typename std::conditional<MIXED, float4, double4>::type;
    __shared__ __align__(16) NodeT s_nodes[kAsmStageNodes];
    __shared__ float s_yy[MIXED ? kAsmStageNodes : 1];  // |y - centre|^2 of the staged nodes (mixed form)
    __shared__ CellGeo s_geo[kAsmMaxCells];
    __shared__ float s_rho[kAsmMaxCells];

    const int i = blockIdx.x * kAsmThreads + threadIdx.x;
    const bool live = i < a.n_cells;
    CellGeo gi;
    if (live) gi = a.geo[i];
    else gi = a.geo[0];
    const double* x = gi.c;
    const int cb = blockIdx.y * a.cols_per_split;
    const int ce = min(a.n_cells, cb + a.cols_per_split);
    const int nn = a.nn;
    const int cps = nn <= kAsmStageNodes ? max(1, min(kAsmMaxCells, kAsmStageNodes / nn)) : 1;
    const int kchunk = nn <= kAsmStageNodes ? nn : kAsmStageNodes;
    const double k2r = a.k.re * a.k.re - a.k.im * a.k.im, k2i = 2.0 * a.k.re * a.k.im;

    using F = typename std::conditional<MIXED, float, double>::type;
    F a1r = 0, a1i = 0, t[6][2];
    bool far = false;
    unsigned cols = ~0u;  // MARKS: the block columns this pass writes
    PairF32 pf{};
    const KF32 kf = KF32::make(a.k.re, a.k.im);
    // the row cell's tangents in FP32 (mixed-form block projection)
    const float tif[2][3] = {{(float)gi.t1[0], (float)gi.t1[1], (float)gi.t1[2]},
                             {(float)gi.t2[0], (float)gi.t2[1], (float)gi.t2[2]}};
    double P0r = 1., P0i = 0.;
    int mode = 0;  // phase polynomial of the current cell (farnode.cuh phase_mode)
    bool split64 = false;
    double r0d = 0.;
    unsigned nbits = 0;  // near bits of the current 32-column word

    for (int c0 = cb; c0 < ce; c0 += cps) {
        const int nc = min(cps, ce - c0);
        for (int k0 = 0; k0 < nn; k0 += kchunk) {
            const int kc = min(kchunk, nn - k0);
            __syncthreads();
            const int tot = nc * kc;
            if constexpr (MIXED) {
                const float4* src = a.nodes32 + (size_t)c0 * nn + k0;
                for (int q = threadIdx.x; q < tot; q += kAsmThreads) {
                    int cc = q / kc, kk = q - cc * kc;
                    const float4 v = __ldg(src + (size_t)cc * nn + kk);
                    s_nodes[q] = v;
                    s_yy[q] = node_yy(v);
                }
            } else {
                const double2* src = reinterpret_cast<const double2*>(a.nodes64 + (size_t)c0 * nn + k0);
                double2* dst = reinterpret_cast<double2*>(s_nodes);
                for (int q = threadIdx.x; q < 2 * tot; q += kAsmThreads) {
                    int node = q >> 1, cc = node / kc, kk = node - cc * kc;
                    dst[q] = __ldg(src + 2 * ((size_t)cc * nn + kk) + (q & 1));
                }
            }
            if (k0 == 0)
                for (int q = threadIdx.x; q < nc; q += kAsmThreads) {
                    s_geo[q] = a.geo[c0 + q];
                    s_rho[q] = a.rho32[c0 + q];
                }
            __syncthreads();
            for (int cc = 0; cc < nc; cc++) {
                const CellGeo& gj = s_geo[cc];
                if (k0 == 0) {
                    double d;
                    const bool nr = asm_is_near(x, gj, a.analytic_calc, &d);
                    far = live && !nr;
                    if constexpr (MARKS) {
                        if (far) {
                            const int c = c0 + cc;
                            const size_t wi = (size_t)(c >> 5) * a.n_cells + i;
                            const size_t plane = (size_t)((a.n_cells + 31) >> 5) * a.n_cells;
                            cols = 0u;
                            for (int b = 0; b < a.m; b++)
                                if ((((a.mark[b * plane + wi] >> (c & 31)) & 1u) != 0) == (a.take_marked != 0))
                                    cols |= 1u << b;
                            far = cols != 0u;
                        }
                    }
                    if (a.mask) {
                        const int c = c0 + cc;
                        nbits |= (nr ? 1u : 0u) << (c & 31);
                        if ((c & 31) == 31 || c == ce - 1) {
                            if (live) a.mask[(size_t)(c >> 5) * a.n_cells + i] = nbits;
                            nbits = 0;
                        }
                    }
                    a1r = a1i = 0;
                    for (int q = 0; q < 6; q++) t[q][0] = t[q][1] = 0;
                    if (!MIXED && far) {  // FP64 phase split when the cell's phase range is small
                        split64 = !CK && fabs(a.k.re) * (double)s_rho[cc] * (1.0 + 1e-6) <= 0.5;
                        r0d = d;
                        if (split64) {
                            double sn, cs;
                            sincos(a.k.re * d, &sn, &cs);
                            P0r = cs;
                            P0i = sn;
                        } else {
                            P0r = 1.0;
                            P0i = 0.0;
                        }
                    }
                    if (MIXED && far) {
                        pf.set(x, gj.c, d, kf);
                        double sn, cs;
                        sincos(a.k.re * d, &sn, &cs);
                        if (CK) {
                            double am = exp(-a.k.im * d);
                            sn *= am;
                            cs *= am;
                        }
                        P0r = cs;
                        P0i = sn;
                        mode = phase_mode((float)fabs(a.k.re) * s_rho[cc]);
                    }
                }
                if (far) {
                    const NodeT* nd = s_nodes + cc * kc;
                    if constexpr (MIXED) {
                        const float* yy = s_yy + cc * kc;
#define BIELCC_ASM_LOOP(MODE_)         \
    _Pragma("unroll 4") for (int q = 0; q < kc; q++) \
        far_node_f32_K<CK, MODE_>(a1r, a1i, t, pf, nd[q], yy[q], kf);
                        switch (mode) {
                            case 0: BIELCC_ASM_LOOP(0) break;
                            case 1: BIELCC_ASM_LOOP(1) break;
                            case 2: BIELCC_ASM_LOOP(2) break;
                            case 3: BIELCC_ASM_LOOP(3) break;
                            default: BIELCC_ASM_LOOP(4) break;
                        }
#undef BIELCC_ASM_LOOP
                    } else {
                        // FP64: the field kernel's node (phase relative to r0 with the Taylor
                        // series when |k| rho <= 0.5); its grad-F moments are unused here
                        Moments<double> mm;
                        mm.zero();
                        if (split64) {
#pragma unroll 2
                            for (int q = 0; q < kc; q++) {
                                const double4 v = nd[q];
                                far_node_f64<CK, true>(mm, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, a.k, k2r, k2i,
                                                       r0d);
                            }
                        } else {
#pragma unroll 2
                            for (int q = 0; q < kc; q++) {
                                const double4 v = nd[q];
                                far_node_f64<CK, false>(mm, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, a.k, k2r, k2i,
                                                        r0d);
                            }
                        }
                        if (!CK) mm.finish_real_k();
                        a1r += mm.a1r;
                        a1i += mm.a1i;
#pragma unroll
                        for (int p = 0; p < 6; p++) {
                            t[p][0] += mm.t[p][0];
                            t[p][1] += mm.t[p][1];
                        }
                    }
                }
                if (k0 + kc == nn && far) {
                    if constexpr (MIXED) {
                        if constexpr (!CK) finish_real_k<F>(a1r, a1i, t);
                        const float phr = (float)(P0r * kInvFourPi), phi = (float)(P0i * kInvFourPi);
                        if constexpr (MARKS) {
                            if (a.m == 2) write_block_f32<2>(a, i, c0 + cc, a1r, a1i, t, phr, phi, tif, gj.t1, gj.t2, cols);
                            else write_block_f32<3>(a, i, c0 + cc, a1r, a1i, t, phr, phi, tif, gj.t1, gj.t2, cols);
                        } else {
                            if (a.m == 2) write_block_f32<2>(a, i, c0 + cc, a1r, a1i, t, phr, phi, tif, gj.t1, gj.t2);
                            else write_block_f32<3>(a, i, c0 + cc, a1r, a1i, t, phr, phi, tif, gj.t1, gj.t2);
                        }
                    } else {
                        // K = (A1 I + T) * P0 / 4pi
                        const int ti[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
                        double Kr[3][3], Ki[3][3];
                        for (int p = 0; p < 3; p++)
                            for (int q = 0; q < 3; q++) {
                                double vr = (double)t[ti[p][q]][0] + (p == q ? (double)a1r : 0.);
                                double vi = (double)t[ti[p][q]][1] + (p == q ? (double)a1i : 0.);
                                Kr[p][q] = (vr * P0r - vi * P0i) * kInvFourPi;
                                Ki[p][q] = (vr * P0i + vi * P0r) * kInvFourPi;
                            }
                        if constexpr (MARKS) write_block(a, i, c0 + cc, Kr, Ki, gi.t1, gi.t2, gj.t1, gj.t2, cols);
                        else write_block(a, i, c0 + cc, Kr, Ki, gi.t1, gi.t2, gj.t1, gj.t2);
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------- adaptive far blocks (p_max >= 3)
// The reference runs one refinement loop per matrix column: K_RotRot_Far
// (K.h:288-301) of the column's basis current J_b (tau_b of the column cell, or
// e_b) at the row cell's centre, which stops at the first pass after the first
// whose squared change is below eps^2 (integral_universal.h:58-119), else
// returns its last pass. asm_refine_decide_kernel runs the test at the second
// pass for every far block and column from the FP64 node tables at n_start and
// 2 n_start, writes the near mask, and marks the failing columns in
// mark[b]. The marks-reading far kernel then writes the columns that passed
// from the 2 n_start tables and, with p_max = 3, the failing ones from the
// 4 n_start tables; with p_max > 3 the failing ones run the whole loop in
// assemble_far_refine_kernel.

// One FP64 pass over a cell's node table row (the field kernels' FP64 node,
// K moments only), finished and ready for K = (A1 I + T) J.
template <bool CK>
BIELCC_D void asm_pass_f64(Moments<double>& m, const double4* __restrict__ nd, int nn, const double* x, cplx k,
                           double k2r, double k2i, double r0, bool split) {
    m.zero();
    if (split) {
#pragma unroll 8
        for (int q = 0; q < nn; q++) {
            const double4 v = nd[q];
            far_node_f64<CK, true>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, k, k2r, k2i, r0);
        }
    } else {
#pragma unroll 8
        for (int q = 0; q < nn; q++) {
            const double4 v = nd[q];
            far_node_f64<CK, false>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, k, k2r, k2i, r0);
        }
    }
    if (!CK) m.finish_real_k();
}

// The squared change of column b's raw integral (A1 J + T J) P0 between two
// passes, |.| taken first as in integral_universal.h:96-99.
BIELCC_D double asm_delta2(const Moments<double>& m0, const Moments<double>& m1, const double* J, double pr,
                           double pi) {
    const int ti[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    double d = 0.;
    for (int p = 0; p < 3; p++) {
        double e0r = m0.a1r * J[p], e0i = m0.a1i * J[p], e1r = m1.a1r * J[p], e1i = m1.a1i * J[p];
        for (int q = 0; q < 3; q++) {
            e0r += m0.t[ti[p][q]][0] * J[q];
            e0i += m0.t[ti[p][q]][1] * J[q];
            e1r += m1.t[ti[p][q]][0] * J[q];
            e1i += m1.t[ti[p][q]][1] * J[q];
        }
        const cplx k0 = mk(e0r, e0i) * mk(pr, pi), k1 = mk(e1r, e1i) * mk(pr, pi);
        const double t = sqrt(cabs2(k1 - k0));
        d += t * t;
    }
    return d;
}

// STAGED: the CTA stages each column cell's two node rows in shared memory
// ((nn_lo + nn) double4, dynamic); otherwise every thread reads them from
// global memory (rows too long to stage).
template <bool STAGED>
__global__ void asm_refine_decide_kernel(AsmArgs a, const double4* __restrict__ lo, int nn_lo, double eps2,
                                         unsigned* __restrict__ mark) {
    extern __shared__ double4 s_rows[];
    const int i = blockIdx.x * kAsmThreads + threadIdx.x;
    const bool live = i < a.n_cells;
    if (!STAGED && !live) return;
    const CellGeo gi = a.geo[live ? i : 0];
    const double* x = gi.c;
    const int cb = blockIdx.y * a.cols_per_split;
    const int ce = min(a.n_cells, cb + a.cols_per_split);
    const bool ck = a.k.im != 0.0;
    const double k2r = a.k.re * a.k.re - a.k.im * a.k.im, k2i = 2.0 * a.k.re * a.k.im;
    const size_t plane = (size_t)((a.n_cells + 31) >> 5) * a.n_cells;
    unsigned nbits = 0, mb[3] = {0u, 0u, 0u};
    for (int j = cb; j < ce; j++) {
        const double4* row_lo = lo + (size_t)j * nn_lo;
        const double4* row_hi = a.nodes64 + (size_t)j * a.nn;
        if constexpr (STAGED) {
            __syncthreads();  // the previous column's rows are no longer read
            for (int q = threadIdx.x; q < nn_lo; q += kAsmThreads) s_rows[q] = row_lo[q];
            for (int q = threadIdx.x; q < a.nn; q += kAsmThreads) s_rows[nn_lo + q] = row_hi[q];
            __syncthreads();
            row_lo = s_rows;
            row_hi = s_rows + nn_lo;
            if (!live) continue;  // after the barriers: every thread stages
        }
        const CellGeo& gj = a.geo[j];
        double d;
        const bool nr = asm_is_near(x, gj, a.analytic_calc, &d);
        if (!nr) {
            const bool split = !ck && fabs(a.k.re) * (double)a.rho32[j] * (1.0 + 1e-6) <= 0.5;
            double pr = 1.0, pi = 0.0;
            if (split) sincos(a.k.re * d, &pi, &pr);
            Moments<double> m0, m1;
            if (ck) {
                asm_pass_f64<true>(m0, row_lo, nn_lo, x, a.k, k2r, k2i, d, false);
                asm_pass_f64<true>(m1, row_hi, a.nn, x, a.k, k2r, k2i, d, false);
            } else {
                asm_pass_f64<false>(m0, row_lo, nn_lo, x, a.k, k2r, k2i, d, split);
                asm_pass_f64<false>(m1, row_hi, a.nn, x, a.k, k2r, k2i, d, split);
            }
            for (int b = 0; b < a.m; b++) {
                double J[3];
                for (int g = 0; g < 3; g++) J[g] = a.m == 3 ? (g == b ? 1. : 0.) : (b == 0 ? gj.t1[g] : gj.t2[g]);
                if (!(asm_delta2(m0, m1, J, pr, pi) < eps2)) mb[b] |= 1u << (j & 31);
            }
        }
        nbits |= (nr ? 1u : 0u) << (j & 31);
        if ((j & 31) == 31 || j == ce - 1) {
            const size_t wi = (size_t)(j >> 5) * a.n_cells + i;
            if (a.mask) a.mask[wi] = nbits;
            for (int b = 0; b < a.m; b++) mark[b * plane + wi] = mb[b];
            nbits = 0;
            mb[0] = mb[1] = mb[2] = 0u;
        }
    }
}

// p_max > 3: the marked (row, column, basis) far entries through the whole
// loop (integral_cell, ops.cuh: nodes on the fly).
__global__ void assemble_far_refine_kernel(AsmArgs a, const unsigned* __restrict__ mark, const double* __restrict__ verts,
                                           int nv, DNP np) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_cells) return;
    const CellGeo gi = a.geo[i];
    const int cb = blockIdx.y * a.cols_per_split;
    const int ce = min(a.n_cells, cb + a.cols_per_split);
    const int m = a.m;
    const size_t plane = (size_t)((a.n_cells + 31) >> 5) * a.n_cells;
    for (int j = cb; j < ce; j++) {
        const size_t wi = (size_t)(j >> 5) * a.n_cells + i;
        unsigned cols = 0u;
        for (int b = 0; b < m; b++) cols |= ((mark[b * plane + wi] >> (j & 31)) & 1u) << b;
        if (!cols) continue;
        const CellGeo& gj = a.geo[j];
        DCell cl;
        cl.nv = nv;
        for (int v = 0; v < nv; v++)
            for (int g = 0; g < 3; g++) cl.v[v][g] = verts[((size_t)j * nv + v) * 3 + g];
        cplx v[3][3];  // v[b] = K[J_b], J_b = tau_b(j) (TAU2) or e_b (FULL3)
        for (int b = 0; b < m; b++) {
            if (!((cols >> b) & 1u)) continue;
            DKP kp;
            dkp_zero(kp);
            kp.smoothR = kMachineZero;
            kp.smoothRMin = kMachineZero;
            kp.k = a.k;
            for (int g = 0; g < 3; g++)
                kp.current[g] = mk(m == 3 ? (g == b ? 1. : 0.) : (b == 0 ? gj.t1[g] : gj.t2[g]), 0.);
            integral_cell<cplx>(F_ROTROTSIMPLEPOT_H, gi.c, cl, kp, 3, np.n_start, np.p_max, np.eps, v[b]);
        }
        const size_t dim = (size_t)m * a.n_cells;
        for (int aa = 0; aa < m; aa++) {
            size_t off = ((size_t)i * m + aa) * dim + (size_t)j * m;
            for (int b = 0; b < m; b++) {
                if (!((cols >> b) & 1u)) continue;
                cplx e = m == 3 ? v[b][aa]
                                : (aa == 0 ? v[b][0] * gi.t1[0] + v[b][1] * gi.t1[1] + v[b][2] * gi.t1[2]
                                           : v[b][0] * gi.t2[0] + v[b][1] * gi.t2[1] + v[b][2] * gi.t2[2]);
                e = e * kInvFourPi;
                if (a.c64) reinterpret_cast<float2*>(a.A)[off + b] = make_float2((float)e.re, (float)e.im);
                else reinterpret_cast<double2*>(a.A)[off + b] = make_double2(e.re, e.im);
            }
        }
    }
}

__global__ void asm_near_count_kernel(const CellGeo* __restrict__ geo, int n_cells, double analytic_calc,
                                      long long* __restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cells) return;
    const double* x = geo[i].c;
    long long n = 0;
    for (int j = 0; j < n_cells; j++) {
        double d;
        n += asm_is_near(x, geo[j], analytic_calc, &d);
    }
    counts[i] = n;
}

__global__ void asm_near_fill_kernel(const CellGeo* __restrict__ geo, int n_cells, double analytic_calc,
                                     const long long* __restrict__ offs, int* __restrict__ pr, int* __restrict__ pc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cells) return;
    const double* x = geo[i].c;
    long long o = offs[i];
    for (int j = 0; j < n_cells; j++) {
        double d;
        if (asm_is_near(x, geo[j], analytic_calc, &d)) {
            pr[o] = i;
            pc[o] = j;
            o++;
        }
    }
}

// Near pairs from the far kernel's bit mask (row i, word w: the near test of
// get_field.h:58 for columns 32w..32w+31, evaluated there with the same
// non-contracted FP64 arithmetic): counts per row, then the (row, column)
// pairs in ascending column order.
__global__ void asm_mask_count_kernel(const unsigned* __restrict__ mask, int n_words, int n_cells,
                                      long long* __restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cells) return;
    long long n = 0;
    for (int w = 0; w < n_words; w++) n += __popc(mask[(size_t)w * n_cells + i]);
    counts[i] = n;
}

__global__ void asm_mask_fill_kernel(const unsigned* __restrict__ mask, int n_words, int n_cells,
                                     const long long* __restrict__ offs, int* __restrict__ pr, int* __restrict__ pc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cells) return;
    long long o = offs[i];
    for (int w = 0; w < n_words; w++) {
        unsigned b = mask[(size_t)w * n_cells + i];
        while (b) {
            const int bit = __ffs(b) - 1;
            b &= b - 1;
            pr[o] = i;
            pc[o] = w * 32 + bit;
            o++;
        }
    }
}

// K_RotRot_HS_Colloc (electrodynamics/K.h:179-204) at x as a 3x3 operator, FP64.
BIELCC_D void near_operator(const DCell& cl, const double* x, cplx k, const DNP& np, double (&Kr)[3][3],
                            double (&Ki)[3][3]) {
    cplx I = surf_simplepot_h_hs_dev(cl, x, np.analytic_calc, np.n_start, np.p_max, np.eps, k);
    cplx sI = I * k * k / kFourPi;
    DKP ps;
    dkp_zero(ps);
    ps.smoothR = kMachineZero;
    ps.smoothRMin = kMachineZero;
    ps.k = k;
    cplx M[3][3], dummy[3];
    K0_dev(F_GRADSIMPLEPOT_H, nullptr, x, cl, ps, np.n_start_seg, np.p_max_seg, np.eps, dummy, M);
    for (int p = 0; p < 3; p++)
        for (int r = 0; r < 3; r++) {
            cplx v = M[p][r] / kFourPi;
            if (p == r) v += sI;
            Kr[p][r] = v.re;
            Ki[p][r] = v.im;
        }
}

// Near entries: K_RotRot_HS_Colloc as a 3x3 operator, FP64.
__global__ void asm_near_kernel(AsmArgs a, const double* __restrict__ verts, int nv, const int* __restrict__ pr,
                                const int* __restrict__ pc, long long n_pairs, DNP np) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_pairs) return;
    int i = pr[q], j = pc[q];
    const CellGeo gi = a.geo[i], gj = a.geo[j];
    DCell cl;
    cl.nv = nv;
    for (int v = 0; v < nv; v++)
        for (int g = 0; g < 3; g++) cl.v[v][g] = verts[((size_t)j * nv + v) * 3 + g];
    const double* x = gi.c;
    double Kr[3][3], Ki[3][3];
    near_operator(cl, x, a.k, np, Kr, Ki);
    write_block(a, i, j, Kr, Ki, gi.t1, gi.t2, gj.t1, gj.t2);
}

// Error sample of a mixed assembly: rows of the cells i_r = r N / R
// (r < R), every column, recomputed in FP64 with the per-pair operators
// (K_RotRot_HS_Colloc near, K_RotRot_Far far, electrodynamics/K.h) and
// projected as the stored entries are; each block sums |stored - FP64|^2
// and |FP64|^2 of its (row, column) pairs into part[block] (fixed order).
__global__ void asm_error_sample_kernel(AsmArgs a, const double* __restrict__ verts, int nv, int R, DNP np,
                                        double2* __restrict__ part) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int N = a.n_cells, M = a.m;
    double num = 0., den = 0.;
    if (q < (long long)R * N) {
        const int r = (int)(q / N), j = (int)(q - (long long)r * N);
        const int i = (int)((long long)r * N / R);
        const CellGeo gi = a.geo[i], gj = a.geo[j];
        DCell cl;
        cl.nv = nv;
        for (int v = 0; v < nv; v++)
            for (int g = 0; g < 3; g++) cl.v[v][g] = verts[((size_t)j * nv + v) * 3 + g];
        const double* x = gi.c;
        double d;
        double Kr[3][3], Ki[3][3];
        if (asm_is_near(x, gj, a.analytic_calc, &d)) {
            near_operator(cl, x, a.k, np, Kr, Ki);
        } else {
            for (int b = 0; b < 3; b++) {  // K_RotRot_Far is linear in the current: one column per basis vector
                cplx e[3] = {mk(b == 0, 0.), mk(b == 1, 0.), mk(b == 2, 0.)}, col[3];
                K_far_dev(e, x, cl, np, a.k, col);
                for (int p = 0; p < 3; p++) {
                    Kr[p][b] = col[p].re;
                    Ki[p][b] = col[p].im;
                }
            }
        }
        const size_t dim = (size_t)M * N;
        for (int aa = 0; aa < M; aa++)
            for (int b = 0; b < M; b++) {
                double vr = 0., vi = 0.;
                if (M == 3) {
                    vr = Kr[aa][b];
                    vi = Ki[aa][b];
                } else {
                    const double* ta = aa == 0 ? gi.t1 : gi.t2;
                    const double* tb = b == 0 ? gj.t1 : gj.t2;
                    for (int p = 0; p < 3; p++) {
                        vr += ta[p] * (Kr[p][0] * tb[0] + Kr[p][1] * tb[1] + Kr[p][2] * tb[2]);
                        vi += ta[p] * (Ki[p][0] * tb[0] + Ki[p][1] * tb[1] + Ki[p][2] * tb[2]);
                    }
                }
                const size_t off = ((size_t)i * M + aa) * dim + (size_t)j * M + b;
                double sr, si;
                if (a.c64) {
                    const float2 v = reinterpret_cast<const float2*>(a.A)[off];
                    sr = v.x;
                    si = v.y;
                } else {
                    const double2 v = reinterpret_cast<const double2*>(a.A)[off];
                    sr = v.x;
                    si = v.y;
                }
                num += (sr - vr) * (sr - vr) + (si - vi) * (si - vi);
                den += vr * vr + vi * vi;
            }
    }
    __shared__ double sn[128], sd[128];
    sn[threadIdx.x] = num;
    sd[threadIdx.x] = den;
    __syncthreads();
    for (int w = 64; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sn[threadIdx.x] += sn[threadIdx.x + w];
            sd[threadIdx.x] += sd[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = make_double2(sn[0], sd[0]);
}

__global__ void asm_error_sum_kernel(const double2* __restrict__ part, int n, double* __restrict__ sums) {
    double a = 0., b = 0.;
    for (int i = 0; i < n; i++) {
        a += part[i].x;
        b += part[i].y;
    }
    sums[0] = a;
    sums[1] = b;
}

static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// Column blocks of the (row, column word) marks of p_max >= 3: one per basis vector.
static int asm_mark_planes(const AssembleLaunch& a) { return far_adaptive(a.np) ? (a.layout == 1 ? 3 : 2) : 0; }

size_t assemble_ws_base_bytes(const AssembleLaunch& a) {
    size_t N = a.mesh->n_cells;
    return 2 * al256((N + 1) * sizeof(long long)) + al256((N + 31) / 32 * N * sizeof(unsigned)) + 256 +
           al256((size_t)asm_mark_planes(a) * ((N + 31) / 32) * N * sizeof(unsigned));
}

// The near mask is written by the far kernel (p_max <= 2) or the decision
// kernel (p_max >= 3); count / fill read it.
static bool uses_mask(const AssembleLaunch&) { return true; }

static AsmArgs make_args(const AssembleLaunch& a) {
    const MeshDev& m = *a.mesh;
    AsmArgs g;
    g.geo = m.geo;
    g.n_cells = m.n_cells;
    g.nodes64 = m.nodes64;
    g.nodes32 = m.nodes32;
    g.rho32 = m.rho32;
    g.nn = far_split_n(a.np) * far_split_n(a.np);
    g.k = a.k;
    g.analytic_calc = a.np.analytic_calc;
    g.m = a.layout == 1 ? 3 : 2;
    g.c64 = a.out_c64;
    g.A = a.A;
    g.mask = nullptr;
    return g;
}

// Resident CTAs (whole GPU) of the far assembly kernel variant.
static int asm_slots(bool ck, bool mixed) {
    static std::atomic<int> cache[2][2];
    std::atomic<int>& c = cache[ck][mixed];
    int v = c.load(std::memory_order_relaxed);
    if (v) return v;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn = ck ? (mixed ? (const void*)assemble_far_kernel<true, true>
                                 : (const void*)assemble_far_kernel<true, false>)
                        : (mixed ? (const void*)assemble_far_kernel<false, true>
                                 : (const void*)assemble_far_kernel<false, false>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kAsmThreads, 0);
    v = std::max(1, sms * std::max(1, per));
    c.store(v, std::memory_order_relaxed);
    return v;
}

cudaError_t assemble_stage1(const AssembleLaunch& a, void* ws, long long* d_total, cudaStream_t s) {
    const MeshDev& m = *a.mesh;
    const int N = m.n_cells;
    long long* counts = (long long*)ws;
    long long* offs = (long long*)((char*)ws + al256((size_t)(N + 1) * sizeof(long long)));
    unsigned* mask = (unsigned*)((char*)offs + al256((size_t)(N + 1) * sizeof(long long)));
    const int n_words = (N + 31) / 32;
    AsmArgs g = make_args(a);
    g.mask = uses_mask(a) ? mask : nullptr;
    int tiles = (N + kAsmThreads - 1) / kAsmThreads;
    bool ck = a.k.im != 0.;
    // column splits in whole 32-column words, so every mask word has one writer
    if (m.table_n != far_split_n(a.np))
        return cudaErrorInvalidValue;  // node tables of another split: the caller builds far_split_n's
    if (far_adaptive(a.np) && (m.table_lo_n != a.np.n_start || !m.nodes64_lo))
        return cudaErrorInvalidValue;  // no n_start table for the convergence test
    if (far_third_pass(a.np) && (m.table_hi_n != 4 * a.np.n_start || !m.nodes64_hi))
        return cudaErrorInvalidValue;  // no 4 n_start tables for the third pass
    int splits = choose_cell_splits(tiles, N, asm_slots(ck, a.precision == 1), N);
    g.cols_per_split = round_cells_per_split(N, splits);
    dim3 grid(tiles, splits);
    if (far_adaptive(a.np)) {
        unsigned* mark = (unsigned*)((char*)mask + al256((size_t)n_words * N * sizeof(unsigned)) + 256);
        const int nn_lo = a.np.n_start * a.np.n_start;
        const size_t rows = (size_t)(nn_lo + g.nn) * sizeof(double4);
        if (rows <= 48 * 1024)
            asm_refine_decide_kernel<true><<<grid, kAsmThreads, rows, s>>>(g, m.nodes64_lo, nn_lo, a.np.eps * a.np.eps,
                                                                           mark);
        else
            asm_refine_decide_kernel<false><<<grid, kAsmThreads, 0, s>>>(g, m.nodes64_lo, nn_lo, a.np.eps * a.np.eps,
                                                                         mark);
        AsmArgsMarks gm;
        static_cast<AsmArgs&>(gm) = g;
        gm.mask = nullptr;  // written by the decision kernel
        gm.mark = mark;
        gm.take_marked = 0;  // the columns that passed: the pass at 2 n_start
        if (a.precision == 1) {
            if (ck) assemble_far_kernel<true, true, true><<<grid, kAsmThreads, 0, s>>>(gm);
            else assemble_far_kernel<false, true, true><<<grid, kAsmThreads, 0, s>>>(gm);
        } else {
            if (ck) assemble_far_kernel<true, false, true><<<grid, kAsmThreads, 0, s>>>(gm);
            else assemble_far_kernel<false, false, true><<<grid, kAsmThreads, 0, s>>>(gm);
        }
        if (far_third_pass(a.np)) {  // p_max = 3: the failing columns return the pass at 4 n_start
            gm.nodes64 = m.nodes64_hi;
            gm.nodes32 = m.nodes32_hi;
            gm.rho32 = m.rho32_hi;
            gm.nn = 16 * a.np.n_start * a.np.n_start;
            gm.take_marked = 1;
            if (a.precision == 1) {
                if (ck) assemble_far_kernel<true, true, true><<<grid, kAsmThreads, 0, s>>>(gm);
                else assemble_far_kernel<false, true, true><<<grid, kAsmThreads, 0, s>>>(gm);
            } else {
                if (ck) assemble_far_kernel<true, false, true><<<grid, kAsmThreads, 0, s>>>(gm);
                else assemble_far_kernel<false, false, true><<<grid, kAsmThreads, 0, s>>>(gm);
            }
        } else {
            DNP np{a.np.eps, a.np.rs, a.np.rs_seg, a.np.analytic_calc, a.np.n_start, a.np.n_start_seg, a.np.p_max,
                   a.np.p_max_seg};
            assemble_far_refine_kernel<<<grid, kAsmThreads, 0, s>>>(g, mark, m.verts, m.nv, np);
        }
    } else if (a.precision == 1) {
        if (ck) assemble_far_kernel<true, true><<<grid, kAsmThreads, 0, s>>>(g);
        else assemble_far_kernel<false, true><<<grid, kAsmThreads, 0, s>>>(g);
    } else {
        if (ck) assemble_far_kernel<true, false><<<grid, kAsmThreads, 0, s>>>(g);
        else assemble_far_kernel<false, false><<<grid, kAsmThreads, 0, s>>>(g);
    }
    if (g.mask) asm_mask_count_kernel<<<tiles, kAsmThreads, 0, s>>>(mask, n_words, N, counts);
    else asm_near_count_kernel<<<tiles, kAsmThreads, 0, s>>>(m.geo, N, a.np.analytic_calc, counts);
    scan_kernel<<<1, 1024, 0, s>>>(counts, N, offs, d_total);
    return cudaGetLastError();
}

cudaError_t assemble_stage2(const AssembleLaunch& a, void* ws, long long n_near, void* pair_ws, cudaStream_t s) {
    if (n_near <= 0) return cudaSuccess;
    const MeshDev& m = *a.mesh;
    const int N = m.n_cells;
    long long* offs = (long long*)((char*)ws + al256((size_t)(N + 1) * sizeof(long long)));
    const unsigned* mask = (const unsigned*)((char*)offs + al256((size_t)(N + 1) * sizeof(long long)));
    int* pr = (int*)pair_ws;
    int* pc = pr + n_near;
    int tiles = (N + kAsmThreads - 1) / kAsmThreads;
    if (uses_mask(a))
        asm_mask_fill_kernel<<<tiles, kAsmThreads, 0, s>>>(mask, (N + 31) / 32, N, offs, pr, pc);
    else
        asm_near_fill_kernel<<<tiles, kAsmThreads, 0, s>>>(m.geo, N, a.np.analytic_calc, offs, pr, pc);
    AsmArgs g = make_args(a);
    DNP np{a.np.eps, a.np.rs, a.np.rs_seg, a.np.analytic_calc, a.np.n_start, a.np.n_start_seg, a.np.p_max,
           a.np.p_max_seg};
    asm_near_kernel<<<(int)((n_near + 127) / 128), 128, 0, s>>>(g, m.verts, m.nv, pr, pc, n_near, np);
    return cudaGetLastError();
}

size_t assemble_error_ws_bytes(const AssembleLaunch& a, int R) {
    return al256((size_t)(((long long)R * a.mesh->n_cells + 127) / 128) * sizeof(double2)) + 256;
}

cudaError_t assemble_error_sample(const AssembleLaunch& a, int R, void* ws, double* sums, cudaStream_t s) {
    const MeshDev& m = *a.mesh;
    const long long tot = (long long)R * m.n_cells;
    const int blocks = (int)((tot + 127) / 128);
    AsmArgs g = make_args(a);
    DNP np{a.np.eps, a.np.rs, a.np.rs_seg, a.np.analytic_calc, a.np.n_start, a.np.n_start_seg, a.np.p_max,
           a.np.p_max_seg};
    double2* part = (double2*)ws;
    asm_error_sample_kernel<<<blocks, 128, 0, s>>>(g, m.verts, m.nv, R, np, part);
    asm_error_sum_kernel<<<1, 1, 0, s>>>(part, blocks, sums);
    return cudaGetLastError();
}

}  // namespace bielcc_gpu
