// field.cu — E/H field over every observation-point x cell pair: the
// GetFieldE_Ideal driver (electrodynamics/get_field.h:35-78) and its H
// counterpart (examples/field/main0_field_test.cpp:237-311) on sm_100a.
//
// Pipeline (one stream, deterministic summation order):
//   1. far kernel   — one observation point per thread, cell node tiles staged
//                     in shared memory with 128-bit loads, cells split across
//                     gridDim.y (the split count is chosen per launch so that
//                     the last wave of CTAs fills the GPU: grid.h);
//                     far cells only (near cells skipped). Per cell
//                     the J-independent moments A1 = sum w e f1,
//                     T = sum w e f2 d^d^T, G = sum w grad F are accumulated and
//                     contracted with each right-hand side once per cell:
//                       K_RotRot_Far  (K.h:288-301)  = (A1 J + T J) / 4pi
//                       R_Rot_Colloc  (R.h:89-111)   = (G x J) / 4pi
//                     FP64 form: FP64 everywhere. Mixed form: nodes relative to
//                     the cell centre in FP32, phase split e^{ikr} =
//                     e^{ik r0} e^{ik (r - r0)} with r0 = |x - centre| and
//                     e^{ik r0} in FP64, r - r0 = q / (r + r0) with
//                     q = |delta|^2 - 2 delta.X (no cancellation), FP32 cell sums,
//                     FP64 accumulation across cells.
//   2. near count + scan + fill — per point, the cells with
//                     |x - centre| < analytic_calc * diam (get_field.h:58), in
//                     cell order.
//   3. near pair kernel — FP64, one pair per thread: the J-independent parts of
//                     K_RotRot_Near_Smooth (K.h:47-79) and R_Rot_Smooth
//                     (R.h:46-61) with the reference's adaptive quadrature.
//   4. near sums    — one warp per (point, RHS): the point's near pairs
//                     contracted with J, lane-strided in cell order, fixed
//                     butterfly across the lanes.
//   5. finalize     — per (point, RHS): far partials over splits (in order;
//                     lane-strided with a fixed butterfly beyond 32 splits) +
//                     the near sum, x mult, + incident field.
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "farnode.cuh"
#include "grid.h"
#include "internal.h"
#include "ops.cuh"
#include "scan.cuh"

namespace bielcc_gpu {

#ifndef BIELCC_FAR_THREADS
#define BIELCC_FAR_THREADS 128
#endif
constexpr int kFarThreads = BIELCC_FAR_THREADS;
// Unrolling of the mixed node loop (far launch on 8192 cells x 20,000 points:
// x2 26.07 ms, x4 25.41 ms, x8 25.93 ms).
#ifndef BIELCC_FAR_UNROLL
#define BIELCC_FAR_UNROLL 4
#endif
#define BIELCC_FAR_STR(x) #x
#define BIELCC_FAR_PRAGMA(x) _Pragma(BIELCC_FAR_STR(unroll x))
#define BIELCC_FAR_UNROLL_PRAGMA BIELCC_FAR_PRAGMA(BIELCC_FAR_UNROLL)
// Unrolling of the FP64 split node loop (FP64 step on 8192 cells x 20,000
// points: x1 57.7, x2 56.4, x4 54.6, x8 53.3, x16 52.8 ms; registers 152-166).
#ifndef BIELCC_FAR64_UNROLL
#define BIELCC_FAR64_UNROLL 16
#endif
#define BIELCC_FAR64_UNROLL_PRAGMA BIELCC_FAR_PRAGMA(BIELCC_FAR64_UNROLL)
// Minimum resident CTAs per SM asked of the 1-RHS real-k mixed far kernel
// (0: none, the compiler's own register choice, which the other variants
// keep). 5 caps it at 96 registers without spills: 20 warps per SM instead of
// 16 (far launch on 8192 cells x 20,000 points 25.87 -> 25.42 ms).
#ifndef BIELCC_FAR_MINB
#define BIELCC_FAR_MINB 5
#endif
// The same for the 1-RHS real-k FP64 far kernel: 4 (127 registers) measured
// slower than the compiler's own 152 (FP64 step 63.1 against 58.7 ms).
#ifndef BIELCC_FAR64_MINB
#define BIELCC_FAR64_MINB 0
#endif
#define BIELCC_FAR_BOUNDS(NRHS_, CK_, MIXED_) \
    __launch_bounds__(kFarThreads, NRHS_ == 1 && !CK_ ? (MIXED_ ? BIELCC_FAR_MINB : BIELCC_FAR64_MINB) : 0)
constexpr int kStageNodes = 256;
constexpr int kMaxStageCells = 32;

struct FarArgs {
    const double* pts;
    int n_pts;
    const CellGeo* geo;
    int n_cells;
    const double4* nodes64;
    const float4* nodes32;
    const float* rho32;
    int nn;  // nodes per cell
    const cplx* J;  // [S][N][3]
    int n_rhs, rhs0;
    cplx k;
    double analytic_calc;
    int cells_per_split;  // a multiple of 32: near-mask words never straddle splits
    double* partial;      // [split][S][12][P]
    unsigned* nearmask;   // [ceil(N/32)][P]: bit c%32 of word c/32 set iff (p, c) is near
};
// p_max >= 3, the far kernel's marks-reading variant: the integrals that failed
// the convergence test at the second pass, grad F per pair [ceil(N/32)][P] and
// F . J per RHS [S][ceil(N/32)][P]; take_marked 1 adds the integrals that
// failed (the third pass, at 4 n_start), 0 the ones that passed (which the
// decision kernel adds itself on the field path). (A separate type: the plain variants keep
// FarArgs' parameter block, whose size the FP64 kernel's register allocation
// follows.)
struct FarArgsMarks : FarArgs {
    const unsigned* markG;
    const unsigned* markK;
    int take_marked;
};
template <bool MARKS>
using FarArgsOf = typename std::conditional<MARKS, FarArgsMarks, FarArgs>::type;

// Contract one cell's moments (times the phase P = pr + i pi) with the RHS
// currents and add into the FP64 accumulators acc[r][12] =
// (Ex, Ey, Ez, Hx, Hy, Hz) x (re, im).
// takeE: bit r adds RHS r's E; takeH: the H of every RHS (convergence-test
// marks, p_max >= 3; all set otherwise).
template <int NRHS, typename F>
BIELCC_D void contract(const Moments<F>& m, F pr, F pi, const cplx (*sj)[3], bool zeroR, double (*acc)[12],
                       unsigned takeE = ~0u, bool takeH = true) {
    // moments x phase
    F A1r = m.a1r * pr - m.a1i * pi, A1i = m.a1r * pi + m.a1i * pr;
    F T[6][2], G[3][2];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        T[q][0] = m.t[q][0] * pr - m.t[q][1] * pi;
        T[q][1] = m.t[q][0] * pi + m.t[q][1] * pr;
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
        G[q][0] = m.g[q][0] * pr - m.g[q][1] * pi;
        G[q][1] = m.g[q][0] * pi + m.g[q][1] * pr;
    }
    const int ti[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
    for (int rr = 0; rr < NRHS; rr++) {
        F jr[3], ji[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            jr[a] = (F)sj[rr][a].re;
            ji[a] = (F)sj[rr][a].im;
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            F er = A1r * jr[a] - A1i * ji[a], ei = A1r * ji[a] + A1i * jr[a];
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const F* t = T[ti[a][b]];
                er += t[0] * jr[b] - t[1] * ji[b];
                ei += t[0] * ji[b] + t[1] * jr[b];
            }
            if ((takeE >> rr) & 1u) {
                acc[rr][2 * a] += (double)er;
                acc[rr][2 * a + 1] += (double)ei;
            }
        }
        if (!zeroR && takeH) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                int b = (a + 1) % 3, c = (a + 2) % 3;  // (G x J)_a = G_b J_c - G_c J_b
                F hr = (G[b][0] * jr[c] - G[b][1] * ji[c]) - (G[c][0] * jr[b] - G[c][1] * ji[b]);
                F hi = (G[b][0] * ji[c] + G[b][1] * jr[c]) - (G[c][0] * ji[b] + G[c][1] * jr[b]);
                acc[rr][6 + 2 * a] += (double)hr;
                acc[rr][6 + 2 * a + 1] += (double)hi;
            }
        }
    }
}

// The far kernel. MIXED = false: FP64 nodes; true: FP32 nodes. MARKS: the
// convergence-test marks of p_max >= 3 select the integrals this pass adds
// (FarArgs::markG / markK); the other variants read no marks.
template <int NRHS, bool CK, bool MIXED, bool MARKS = false>
__global__ void BIELCC_FAR_BOUNDS(NRHS, CK, MIXED) far_kernel(FarArgsOf<MARKS> a) {
    using NodeT = typename std::conditional<MIXED, float4, double4>::type;
    __shared__ __align__(16) NodeT s_nodes[kStageNodes];
    __shared__ float s_yy[MIXED ? kStageNodes : 1];  // |y - centre|^2 of the staged nodes (mixed form)
    __shared__ double4 s_cell[kMaxStageCells];  // centre xyz, near threshold
    __shared__ cplx s_j[kMaxStageCells][NRHS][3];
    __shared__ float s_rho[kMaxStageCells];
    __shared__ double s_rho64[kMaxStageCells];

    const int p = blockIdx.x * kFarThreads + threadIdx.x;
    const bool live = p < a.n_pts;
    double x[3] = {0., 0., 0.};
    if (live)
        for (int g = 0; g < 3; g++) x[g] = a.pts[3 * (size_t)p + g];
    const int cb = blockIdx.y * a.cells_per_split;
    const int ce = min(a.n_cells, cb + a.cells_per_split);
    const int nn = a.nn;
    const int cps = nn <= kStageNodes ? max(1, min(kMaxStageCells, kStageNodes / nn)) : 1;
    const int kchunk = nn <= kStageNodes ? nn : kStageNodes;
    const double k2r = a.k.re * a.k.re - a.k.im * a.k.im, k2i = 2.0 * a.k.re * a.k.im;

    double acc[NRHS][12];
#pragma unroll
    for (int r = 0; r < NRHS; r++)
#pragma unroll
        for (int q = 0; q < 12; q++) acc[r][q] = 0.;

    using F = typename std::conditional<MIXED, float, double>::type;
    Moments<F> m;
    m.zero();
    bool far = false, zeroR = false;
    unsigned takeE = ~0u;  // convergence-test marks (p_max >= 3): the RHS whose E this pass adds
    bool takeH = true;     // and whether it adds H
    unsigned nbits = 0;  // near bits of the current 32-cell word
    // mixed-form per-pair state
    PairF32 pf{};
    const KF32 kf = KF32::make(a.k.re, a.k.im);
    double P0r = 1.0, P0i = 0.0, r0d = 0.0;
    int mode = 0;
    bool split64 = false;
    int td64 = 0;  // Taylor length of the FP64 phase split (farnode.cuh sincos_taylor64)

    for (int c0 = cb; c0 < ce; c0 += cps) {
        const int nc = min(cps, ce - c0);
        for (int k0 = 0; k0 < nn; k0 += kchunk) {
            const int kc = min(kchunk, nn - k0);
            __syncthreads();
            // stage nodes (contiguous when kc == nn) with 128-bit loads
            {
                const int tot = nc * kc;
                if constexpr (MIXED) {
                    const float4* src = a.nodes32 + (size_t)c0 * nn + k0;
                    for (int i = threadIdx.x; i < tot; i += kFarThreads) {
                        int cc = i / kc, kk = i - cc * kc;
                        const float4 v = __ldg(src + (size_t)cc * nn + kk);
                        s_nodes[i] = v;
                        s_yy[i] = node_yy(v);
                    }
                } else {
                    const double2* src = reinterpret_cast<const double2*>(a.nodes64 + (size_t)c0 * nn + k0);
                    double2* dst = reinterpret_cast<double2*>(s_nodes);
                    for (int i = threadIdx.x; i < 2 * tot; i += kFarThreads) {
                        int node = i >> 1, cc = node / kc, kk = node - cc * kc;
                        dst[i] = __ldg(src + 2 * ((size_t)cc * nn + kk) + (i & 1));
                    }
                }
            }
            if (k0 == 0) {
                for (int i = threadIdx.x; i < nc; i += kFarThreads) {
                    const CellGeo& gg = a.geo[c0 + i];
                    s_cell[i] = make_double4(gg.c[0], gg.c[1], gg.c[2], gg.diam);
                    if (MIXED) s_rho[i] = a.rho32[c0 + i];
                    else s_rho64[i] = (double)a.rho32[c0 + i] * (1.0 + 1e-6);
                }
                for (int i = threadIdx.x; i < nc * NRHS * 3; i += kFarThreads) {
                    int cc = i / (NRHS * 3), rem = i - cc * NRHS * 3, rr = rem / 3, g = rem - rr * 3;
                    int rhs = min(a.rhs0 + rr, a.n_rhs - 1);
                    s_j[cc][rr][g] = a.J[((size_t)rhs * a.n_cells + (c0 + cc)) * 3 + g];
                }
            }
            __syncthreads();
            for (int cc = 0; cc < nc; cc++) {
                if (k0 == 0) {
                    double4 ci = s_cell[cc];
                    double cen[3] = {ci.x, ci.y, ci.z}, d;
                    const bool nr = is_near(x, cen, ci.w, a.analytic_calc, &d);
                    far = !nr && live;
                    if constexpr (MARKS) {
                      if (far) {  // each integral's convergence test decides which pass adds it
                        const int c = c0 + cc, nw = (a.n_cells + 31) >> 5;
                        const size_t wi = (size_t)(c >> 5) * a.n_pts + p;
                        const bool want = a.take_marked != 0;
                        takeH = (((a.markG[wi] >> (c & 31)) & 1u) != 0) == want;
                        takeE = 0u;
                        for (int rr = 0; rr < NRHS && a.rhs0 + rr < a.n_rhs; rr++) {
                            const unsigned mk = a.markK[(size_t)(a.rhs0 + rr) * nw * a.n_pts + wi];
                            if ((((mk >> (c & 31)) & 1u) != 0) == want) takeE |= 1u << rr;
                        }
                        far = takeE != 0u || takeH;
                      }
                    }
                    zeroR = d < kMachineZero;  // R_Rot_Colloc: R = 0 at the cell centre
                    m.zero();
                    const int c = c0 + cc;
                    nbits |= (nr ? 1u : 0u) << (c & 31);
                    if ((c & 31) == 31 || c == ce - 1) {
                        if (live && a.nearmask) a.nearmask[(size_t)(c >> 5) * a.n_pts + p] = nbits;
                        nbits = 0;
                    }
                    if (!MIXED && far) {  // FP64 phase split when the cell's phase range is small
                        const double th64 = fabs(a.k.re) * s_rho64[cc];
                        split64 = !CK && th64 <= 0.5;
                        td64 = th64 <= 0.125 ? 2 : (th64 <= 0.25 ? 1 : 0);
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
                    if (MIXED && far) {  // per-pair FP64 set-up of the phase split
                        pf.set(x, cen, d, kf);
                        double s, c;
                        sincos(a.k.re * d, &s, &c);
                        if (CK) {
                            double am = exp(-a.k.im * d);
                            s *= am;
                            c *= am;
                        }
                        P0r = c;
                        P0i = s;
                        mode = phase_mode((float)fabs(a.k.re) * s_rho[cc]);
                    }
                }
                if (far) {
                    const NodeT* nd = s_nodes + cc * kc;
                    if constexpr (MIXED) {
                        const float* yy = s_yy + cc * kc;
#define BIELCC_NODE_LOOP(MODE_)                                                                        \
    BIELCC_FAR_UNROLL_PRAGMA for (int i = 0; i < kc; i++) far_node_f32<CK, MODE_>(m, pf, nd[i], yy[i], kf);
                        switch (mode) {
                            case 0: BIELCC_NODE_LOOP(0) break;
                            case 1: BIELCC_NODE_LOOP(1) break;
                            case 2: BIELCC_NODE_LOOP(2) break;
                            case 3: BIELCC_NODE_LOOP(3) break;
                            default: BIELCC_NODE_LOOP(4) break;
                        }
#undef BIELCC_NODE_LOOP
                    } else {
                        if (split64) {
#define BIELCC_NODE64_LOOP(TD_)                                                                       \
    BIELCC_FAR64_UNROLL_PRAGMA for (int i = 0; i < kc; i++) {                                          \
        const double4 v = nd[i];                                                                       \
        far_node_f64<CK, true, TD_>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, a.k, k2r, k2i, r0d); \
    }
                            switch (td64) {
                                case 2: BIELCC_NODE64_LOOP(2) break;
                                case 1: BIELCC_NODE64_LOOP(1) break;
                                default: BIELCC_NODE64_LOOP(0) break;
                            }
#undef BIELCC_NODE64_LOOP
                        } else {
#pragma unroll 2
                            for (int i = 0; i < kc; i++) {
                                double4 v = nd[i];
                                far_node_f64<CK, false>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, a.k, k2r, k2i,
                                                        r0d);
                            }
                        }
                    }
                }
                if (k0 + kc == nn && far) {
                    if (!CK) m.finish_real_k();
                    if constexpr (MARKS) {
                        if constexpr (MIXED)
                            contract<NRHS, float>(m, (float)P0r, (float)P0i, s_j[cc], zeroR, acc, takeE, takeH);
                        else contract<NRHS, double>(m, P0r, P0i, s_j[cc], zeroR, acc, takeE, takeH);
                    } else {
                        if constexpr (MIXED) contract<NRHS, float>(m, (float)P0r, (float)P0i, s_j[cc], zeroR, acc);
                        else contract<NRHS, double>(m, P0r, P0i, s_j[cc], zeroR, acc);
                    }
                }
            }
        }
    }
    if (!live) return;
    const size_t P = a.n_pts;
#pragma unroll
    for (int r = 0; r < NRHS; r++) {
        if (a.rhs0 + r >= a.n_rhs) break;
        double* dst = a.partial + (((size_t)blockIdx.y * a.n_rhs + (a.rhs0 + r)) * 12) * P + p;
#pragma unroll
        for (int q = 0; q < 12; q++) dst[(size_t)q * P] = acc[r][q];
    }
}

// ---------------------------------------------------------------- adaptive far pairs (p_max >= 3)
// The reference's loop (integral_universal.h:58-119) stops at the first pass
// after the first whose squared L2 change is below eps^2, else returns its last
// pass. far_refine_decide_kernel runs that test between the passes at n_start
// and 2 n_start for every far pair, from node tables: K_RotRot_Far's integral
// of F_RotRotSimplePot_H . J for every right-hand side (K.h:288-301) and
// R_Rot_Colloc's integral of grad F (R.h:89-111; none at the cell centre).
// Each integral is tested on its own, as the reference runs one loop per
// integral: an integral that passes returns the pass at 2 n_start, which the
// decision kernel has just run for the test and adds to the split sums itself
// (in FP64, in the mixed form too); one that fails is marked (markG per pair,
// markK per pair and RHS) and takes the pass at 4 n_start when p_max = 3
// (far_kernel with take_marked = 1 on those tables), else the whole loop in
// far_refine_sum_kernel.

// Unrolling of the decision kernel's node loops (the node rows come from
// global memory: unrolled, their loads issue ahead of the arithmetic).
// 2000 x 8192 at p_max = 3, mixed / FP64: x1 ~92 / 131 ms, x4 88.3 / 129.3 ms,
// x8 88.4 / 127.9 ms.
#ifndef BIELCC_DECIDE_UNROLL
#define BIELCC_DECIDE_UNROLL 8
#endif

// One pass of the FP64 far node loop over a cell's node table row (far_kernel's
// FP64 arithmetic: the phase split below |k| rho = 0.5, else sincos per node).
template <bool CK>
BIELCC_D void far_pass_f64(Moments<double>& m, const double4* __restrict__ nd, int nn, const double* x, cplx k,
                           double k2r, double k2i, double r0, bool split, int td) {
    m.zero();
    if (split) {
#define BIELCC_PASS64(TD_)                                                                              \
    BIELCC_FAR_PRAGMA(BIELCC_DECIDE_UNROLL) for (int i = 0; i < nn; i++) {                              \
        const double4 v = nd[i];                                                                \
        far_node_f64<CK, true, TD_>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, k, k2r, k2i, r0);       \
    }
        switch (td) {
            case 2: BIELCC_PASS64(2) break;
            case 1: BIELCC_PASS64(1) break;
            default: BIELCC_PASS64(0) break;
        }
#undef BIELCC_PASS64
    } else {
        BIELCC_FAR_PRAGMA(BIELCC_DECIDE_UNROLL) for (int i = 0; i < nn; i++) {
            const double4 v = nd[i];
            far_node_f64<CK, false>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, k, k2r, k2i, r0);
        }
    }
    if (!CK) m.finish_real_k();
}

// Raw integrals of one pass (before the 1/4pi of K_RotRot_Far / R_Rot_Colloc),
// times the phase P: K = A1 J + T J, G = grad F.
BIELCC_D void far_raw_K(const Moments<double>& m, double pr, double pi, const cplx* j, cplx* K) {
    const int ti[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int a = 0; a < 3; a++) {
        cplx e = mk(m.a1r, m.a1i) * j[a];
        for (int b = 0; b < 3; b++) e = e + mk(m.t[ti[a][b]][0], m.t[ti[a][b]][1]) * j[b];
        K[a] = e * mk(pr, pi);
    }
}

// The reference's squared change: sum of |res - prev|^2 with |.| taken first
// (integral_universal.h:96-99).
BIELCC_D double far_delta2(const cplx* a, const cplx* b) {
    double d = 0.;
    for (int g = 0; g < 3; g++) {
        const double t = sqrt(cabs2(a[g] - b[g]));
        d += t * t;
    }
    return d;
}

// markK and this split's slot of a.partial must be zero on entry (set bits
// only; the passing integrals are added); markG is written in full.
// STAGED: the CTA stages each cell's two node rows in shared memory
// ((nn_lo + nn) double4, dynamic) before its threads use them; otherwise every
// thread reads them from global memory (rows too long to stage).
template <bool STAGED>
__global__ void far_refine_decide_kernel(FarArgs a, const double4* __restrict__ lo, int nn_lo, double eps2,
                                         unsigned* __restrict__ markG, unsigned* __restrict__ markK) {
    extern __shared__ double4 s_rows[];  // STAGED: [nn_lo] then [nn] of the current cell
    const int p = blockIdx.x * kFarThreads + threadIdx.x;
    const bool live = p < a.n_pts;
    if (!STAGED && !live) return;
    double x[3] = {0., 0., 0.};
    if (live)
        for (int g = 0; g < 3; g++) x[g] = a.pts[3 * (size_t)p + g];
    const int cb = blockIdx.y * a.cells_per_split;
    const int ce = min(a.n_cells, cb + a.cells_per_split);
    const bool ck = a.k.im != 0.0;
    const double k2r = a.k.re * a.k.re - a.k.im * a.k.im, k2i = 2.0 * a.k.re * a.k.im;
    const int nw = (a.n_cells + 31) >> 5;
    const size_t P = a.n_pts;
    unsigned nbits = 0, gbits = 0;
    for (int c = cb; c < ce; c++) {
        const double4* row_lo = lo + (size_t)c * nn_lo;
        const double4* row_hi = a.nodes64 + (size_t)c * a.nn;
        if constexpr (STAGED) {
            __syncthreads();  // the previous cell's rows are no longer read
            for (int i = threadIdx.x; i < nn_lo; i += kFarThreads) s_rows[i] = row_lo[i];
            for (int i = threadIdx.x; i < a.nn; i += kFarThreads) s_rows[nn_lo + i] = row_hi[i];
            __syncthreads();
            row_lo = s_rows;
            row_hi = s_rows + nn_lo;
            if (!live) continue;  // after the barriers: every thread stages
        }
        const CellGeo& gg = a.geo[c];
        double d;
        const bool nr = is_near(x, gg.c, gg.diam, a.analytic_calc, &d);
        bool gfail = false;
        if (!nr) {
            const double th64 = fabs(a.k.re) * (double)a.rho32[c] * (1.0 + 1e-6);
            const bool split = !ck && th64 <= 0.5;
            const int td = th64 <= 0.125 ? 2 : (th64 <= 0.25 ? 1 : 0);
            double pr = 1.0, pi = 0.0;
            if (split) sincos(a.k.re * d, &pi, &pr);
            Moments<double> m0, m1;
            if (ck) {
                far_pass_f64<true>(m0, row_lo, nn_lo, x, a.k, k2r, k2i, d, false, 0);
                far_pass_f64<true>(m1, row_hi, a.nn, x, a.k, k2r, k2i, d, false, 0);
            } else {
                far_pass_f64<false>(m0, row_lo, nn_lo, x, a.k, k2r, k2i, d, split, td);
                far_pass_f64<false>(m1, row_hi, a.nn, x, a.k, k2r, k2i, d, split, td);
            }
            const bool zeroR = d < kMachineZero;  // R_Rot_Colloc integrates grad F away from the centre only
            cplx g1[3];
            if (!zeroR) {
                cplx g0[3];
                for (int q = 0; q < 3; q++) {
                    g0[q] = mk(m0.g[q][0], m0.g[q][1]) * mk(pr, pi);
                    g1[q] = mk(m1.g[q][0], m1.g[q][1]) * mk(pr, pi);
                }
                gfail = !(far_delta2(g1, g0) < eps2);
            }
            for (int s = 0; s < a.n_rhs; s++) {
                const cplx* j = a.J + ((size_t)s * a.n_cells + c) * 3;
                const cplx jj[3] = {j[0], j[1], j[2]};
                cplx k0[3], k1[3];
                far_raw_K(m0, pr, pi, jj, k0);
                far_raw_K(m1, pr, pi, jj, k1);
                const bool kfail = !(far_delta2(k1, k0) < eps2);
                if (kfail) atomicOr(markK + ((size_t)s * nw + (c >> 5)) * a.n_pts + p, 1u << (c & 31));
                // the integrals that passed return the pass at 2 n_start: added
                // here, in cell order, to this split's raw sums (the thread owns them)
                double* dst = a.partial + ((size_t)blockIdx.y * a.n_rhs + s) * 12 * P + p;
                if (!kfail)
                    for (int q = 0; q < 3; q++) {
                        dst[(size_t)(2 * q) * P] += k1[q].re;
                        dst[(size_t)(2 * q + 1) * P] += k1[q].im;
                    }
                if (!zeroR && !gfail)
                    for (int q = 0; q < 3; q++) {  // (G x J)_q = G_b J_c - G_c J_b
                        const int b = (q + 1) % 3, cc = (q + 2) % 3;
                        const cplx h = g1[b] * jj[cc] - g1[cc] * jj[b];
                        dst[(size_t)(6 + 2 * q) * P] += h.re;
                        dst[(size_t)(6 + 2 * q + 1) * P] += h.im;
                    }
            }
        }
        nbits |= (nr ? 1u : 0u) << (c & 31);
        gbits |= (gfail ? 1u : 0u) << (c & 31);
        if ((c & 31) == 31 || c == ce - 1) {
            if (a.nearmask) a.nearmask[(size_t)(c >> 5) * a.n_pts + p] = nbits;
            markG[(size_t)(c >> 5) * a.n_pts + p] = gbits;
            nbits = gbits = 0;
        }
    }
}

// p_max > 3: the integrals that failed the test, through the whole loop
// (integral_cell, ops.cuh: the reference's passes, test and budget), one warp
// per (point, RHS, range of mask words): F . J where markK is set, grad F where
// markG is set. In round r lane l takes the range's marked cell of rank
// 32 r + l (cell order; each lane walks the mask words with its own cursor), so
// the lanes run their loops side by side; lane sums are in cell order and
// combined by a fixed xor butterfly. The marked cells gather on the few
// near-field points, so gridDim.z ranges per point give the GPU that many more
// warps. Writes the raw E, H sums (before 1/4pi) of every point and range,
// zero without marked cells, into partial-sum slot blockIdx.z of `out`
// [gridDim.z][S][12][P].
__global__ void far_refine_sum_kernel(FarArgs a, const unsigned* __restrict__ markG, const unsigned* __restrict__ markK,
                                      const double* __restrict__ verts, int nv, DNP np, double* __restrict__ out) {
    const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    const int s = blockIdx.y;
    if (p >= a.n_pts) return;  // whole warps
    const size_t P = a.n_pts;
    const int n_words = (a.n_cells + 31) / 32;
    // this warp's range of mask words (blockIdx.z of gridDim.z parts) and output slot
    const int wpp = (n_words + gridDim.z - 1) / gridDim.z;
    const int w_end = min(n_words, (int)(blockIdx.z + 1) * wpp);
    out += (size_t)blockIdx.z * a.n_rhs * 12 * P;
    const unsigned* mK = markK + (size_t)s * n_words * P;
    const double x[3] = {a.pts[3 * (size_t)p], a.pts[3 * (size_t)p + 1], a.pts[3 * (size_t)p + 2]};
    double v[12];
#pragma unroll
    for (int q = 0; q < 12; q++) v[q] = 0.;
    int w = blockIdx.z * wpp;
    unsigned bits = w < w_end ? (markG[(size_t)w * P + p] | mK[(size_t)w * P + p]) : 0u;
    long long base = 0;  // rank (within the range) of the first flagged cell of word w
    for (long long t = lane;; t += 32) {
        while (w < w_end && base + __popc(bits) <= t) {
            base += __popc(bits);
            w++;
            bits = w < w_end ? (markG[(size_t)w * P + p] | mK[(size_t)w * P + p]) : 0u;
        }
        const bool have = w < w_end;
        if (!__any_sync(0xffffffffu, have)) break;
        if (!have) continue;
        unsigned b = bits;
        for (long long r = base; r < t; r++) b &= b - 1;  // drop the lower-ranked cells of the word
        const int c = w * 32 + __ffs(b) - 1;
        const bool doK = (mK[(size_t)w * P + p] >> (c & 31)) & 1u, doG = (markG[(size_t)w * P + p] >> (c & 31)) & 1u;
        DCell cl;
        cl.nv = nv;
        for (int vv = 0; vv < nv; vv++)
            for (int g = 0; g < 3; g++) cl.v[vv][g] = verts[((size_t)c * nv + vv) * 3 + g];
        const cplx* j = a.J + ((size_t)s * a.n_cells + c) * 3;
        DKP kp;
        dkp_zero(kp);
        kp.smoothR = kMachineZero;
        kp.smoothRMin = kMachineZero;
        kp.k = a.k;
        for (int g = 0; g < 3; g++) kp.current[g] = j[g];
        if (doK) {
            cplx K[3];
            integral_cell<cplx>(F_ROTROTSIMPLEPOT_H, x, cl, kp, 3, np.n_start, np.p_max, np.eps, K);
            for (int g = 0; g < 3; g++) {
                v[2 * g] += K[g].re;
                v[2 * g + 1] += K[g].im;
            }
        }
        double d;
        is_near(x, a.geo[c].c, a.geo[c].diam, a.analytic_calc, &d);
        if (doG && !(d < kMachineZero)) {  // R_Rot_Colloc: 0 at the cell centre
            DKP kr;
            dkp_zero(kr);
            kr.smoothR = kMachineZero;
            kr.smoothRMin = kMachineZero;
            kr.k = a.k;
            cplx G[3], h[3], jj[3] = {j[0], j[1], j[2]};
            integral_cell<cplx>(F_GRADSIMPLEPOT_H, x, cl, kr, 3, np.n_start, np.p_max, np.eps, G);
            ccross_cc(G, jj, h);
            for (int g = 0; g < 3; g++) {
                v[6 + 2 * g] += h[g].re;
                v[7 + 2 * g] += h[g].im;
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int q = 0; q < 12; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
    if (lane < 12) {
        double r = v[0];
#pragma unroll
        for (int q = 1; q < 12; q++)
            if (lane == q) r = v[q];
        out[((size_t)s * 12 + lane) * P + p] = r;
    }
}

// ---------------------------------------------------------------- near classification
// The far kernels record, per point, which cells failed the far test
// (get_field.h:58) in a bit mask; these two kernels turn it into per-point
// counts and the cell lists in ascending cell order.
__global__ void near_count_kernel(const unsigned* __restrict__ mask, int n_words, int n_pts,
                                  long long* __restrict__ counts) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_pts) return;
    long long n = 0;
    for (int w = 0; w < n_words; w++) n += __popc(mask[(size_t)w * n_pts + p]);
    counts[p] = n;
}

// Near list of a point in ascending cell order: one warp per point. Lane l
// takes a contiguous run of the point's mask words, counts its bits, and
// writes its cells after those of the lanes before it (warp prefix sum), so a
// point with hundreds of near cells does not run 256 words in one thread.
__global__ void near_fill_kernel(const unsigned* __restrict__ mask, int n_words, int n_pts,
                                 const long long* __restrict__ offs, int* __restrict__ pair_cell,
                                 int* __restrict__ pair_pt) {
    const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (p >= n_pts) return;  // whole warps
    const long long o0 = offs[p];
    if (offs[p + 1] == o0) return;
    const int run = (n_words + 31) / 32, w0 = min(n_words, lane * run), w1 = min(n_words, w0 + run);
    int cnt = 0;
    for (int w = w0; w < w1; w++) cnt += __popc(mask[(size_t)w * n_pts + p]);
    int incl = cnt;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
    }
    long long o = o0 + (incl - cnt);
    for (int w = w0; w < w1; w++) {
        unsigned b = mask[(size_t)w * n_pts + p];
        while (b) {
            const int bit = __ffs(b) - 1;
            b &= b - 1;
            pair_cell[o] = w * 32 + bit;
            pair_pt[o] = p;
            o++;
        }
    }
}

// Near pair: the J-independent parts of K_RotRot_Near_Smooth and R_Rot_Smooth
// (near_pair_moments, ops.cuh), one pair per thread.
__global__ void near_pair_kernel(const double* __restrict__ pts, const double* __restrict__ verts, int nv,
                                 const int* __restrict__ pair_cell, const int* __restrict__ pair_pt, long long n_pairs,
                                 cplx k, DNP np, cplx* __restrict__ out) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_pairs) return;
    int c = pair_cell[q], p = pair_pt[q];
    DCell cl;
    cl.nv = nv;
    for (int v = 0; v < nv; v++)
        for (int g = 0; g < 3; g++) cl.v[v][g] = verts[((size_t)c * nv + v) * 3 + g];
    double x[3] = {pts[3 * (size_t)p], pts[3 * (size_t)p + 1], pts[3 * (size_t)p + 2]};
    near_pair_moments(x, cl, k, np, out + q * 13);
}

// Near pairs of a point contracted with one RHS: one warp per (point, RHS).
// Lane l takes the point's pairs l, l + 32, ... (cell order) and sums them in
// order; the 32 lane sums are combined by a fixed xor butterfly. The result
// depends only on the point's own pair list, whatever else runs, and a point
// with hundreds of near cells (small cells near a pole) no longer holds up a
// whole point tile in one thread. near[s][12][p] = E, H (re, im), already / 4pi.
__global__ void near_sum_kernel(const long long* __restrict__ offs, const int* __restrict__ pair_cell,
                                const cplx* __restrict__ moments, const cplx* __restrict__ J, int n_pts, int n_cells,
                                double* __restrict__ near) {
    const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    const int s = blockIdx.y;
    if (p >= n_pts) return;  // whole warps
    const long long q0 = offs[p], q1 = offs[p + 1];
    if (q0 == q1) return;
    double v[12];
#pragma unroll
    for (int i = 0; i < 12; i++) v[i] = 0.;
    for (long long q = q0 + lane; q < q1; q += 32) {
        const int c = pair_cell[q];
        const cplx* o = moments + q * 13;
        const cplx* j = J + ((size_t)s * n_cells + c) * 3;
#pragma unroll
        for (int g = 0; g < 3; g++) {
            const cplx kv = o[0] * j[g] + o[1 + 3 * g] * j[0] + o[2 + 3 * g] * j[1] + o[3 + 3 * g] * j[2];
            v[2 * g] += kv.re;
            v[2 * g + 1] += kv.im;
        }
        cplx h[3];
        ccross_cc(o + 10, j, h);
#pragma unroll
        for (int g = 0; g < 3; g++) {
            v[6 + 2 * g] += h[g].re;
            v[7 + 2 * g] += h[g].im;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int i = 0; i < 12; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i], off);
    if (lane < 12) {
        double x = v[0];
#pragma unroll
        for (int i = 1; i < 12; i++)
            if (lane == i) x = v[i];
        near[((size_t)s * 12 + lane) * n_pts + p] = x;
    }
}

struct FinalArgs {
    const double* pts;
    int n_pts, n_rhs, n_cells, splits;
    const double* partial;
    const long long* offs;  // near-pair offsets per point, or null without near pairs
    const double* near;     // near_sum_kernel's sums
    cplx mult;
    double kvec[3], e0[3], h_scale;
    int add_E, add_H;
    double* E;
    double* H;
    unsigned long long* nonfinite;
};

// Per (point, RHS): far partials over the splits, near sum, mult, incident
// field. One thread per point sums the splits in order (coalesced over the
// points); with many splits (a small point set spread over the whole GPU) one
// warp per point takes splits lane-strided and combines the lanes with a fixed
// xor butterfly, so the serial chain is splits / 32 loads long instead of splits.
template <bool WARP>
__global__ void finalize_kernel(FinalArgs a) {
    const int s = blockIdx.y;
    const size_t P = a.n_pts;
    double v[12];
#pragma unroll
    for (int q = 0; q < 12; q++) v[q] = 0.;
    int p;
    if constexpr (WARP) {
        p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
        const int lane = threadIdx.x & 31;
        if (p >= a.n_pts) return;  // whole warps
        for (int sp = lane; sp < a.splits; sp += 32) {
            const double* src = a.partial + (((size_t)sp * a.n_rhs + s) * 12) * P + p;
#pragma unroll
            for (int q = 0; q < 12; q++) v[q] += src[(size_t)q * P];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
#pragma unroll
            for (int q = 0; q < 12; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
        if (lane != 0) return;
    } else {
        p = blockIdx.x * blockDim.x + threadIdx.x;
        if (p >= a.n_pts) return;
        for (int sp = 0; sp < a.splits; sp++) {
            const double* src = a.partial + (((size_t)sp * a.n_rhs + s) * 12) * P + p;
            for (int q = 0; q < 12; q++) v[q] += src[(size_t)q * P];
        }
    }
    cplx E[3], H[3];
    for (int g = 0; g < 3; g++) {
        E[g] = mk(v[2 * g], v[2 * g + 1]) * kInvFourPi;
        H[g] = mk(v[6 + 2 * g], v[6 + 2 * g + 1]) * kInvFourPi;
    }
    if (a.offs && a.offs[p + 1] > a.offs[p]) {
        const double* nv = a.near + (size_t)s * 12 * P + p;
        for (int g = 0; g < 3; g++) {
            E[g] += mk(nv[(size_t)(2 * g) * P], nv[(size_t)(2 * g + 1) * P]);
            H[g] += mk(nv[(size_t)(6 + 2 * g) * P], nv[(size_t)(7 + 2 * g) * P]);
        }
    }
    for (int g = 0; g < 3; g++) E[g] = E[g] * a.mult;
    const double* x = a.pts + 3 * (size_t)p;
    if (a.add_E || a.add_H) {
        double ph = a.kvec[0] * x[0] + a.kvec[1] * x[1] + a.kvec[2] * x[2];
        double sn, cs;
        sincos(ph, &sn, &cs);
        if (a.add_E)
            for (int g = 0; g < 3; g++) E[g] += mk(a.e0[g] * cs, a.e0[g] * sn);
        if (a.add_H) {
            double kx0[3];
            cross3(a.kvec, a.e0, kx0);
            for (int g = 0; g < 3; g++) H[g] += mk(kx0[g] * cs * a.h_scale, kx0[g] * sn * a.h_scale);
        }
    }
    bool bad = false;
    cplx* eo = reinterpret_cast<cplx*>(a.E) + ((size_t)s * P + p) * 3;
    for (int g = 0; g < 3; g++) {
        eo[g] = E[g];
        bad |= !isfinite(E[g].re) || !isfinite(E[g].im);
    }
    if (a.H) {
        cplx* ho = reinterpret_cast<cplx*>(a.H) + ((size_t)s * P + p) * 3;
        for (int g = 0; g < 3; g++) {
            ho[g] = H[g];
            bad |= !isfinite(H[g].re) || !isfinite(H[g].im);
        }
    }
    if (bad && a.nonfinite) atomicAdd(a.nonfinite, 1ull);
}

// ---------------------------------------------------------------- host launchers
static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
static size_t mask_words(int n_cells) { return (size_t)(n_cells + 31) / 32; }
// Mask-word ranges per point of far_refine_sum_kernel (p_max > 3).
static int refine_parts(const FieldLaunch& f) {
    return (int)std::min<size_t>(8, std::max<size_t>(1, mask_words(f.mesh->n_cells)));
}
// Partial-sum slots [slot][S][12][P]: one per cell split; with p_max = 3 as
// many again for the third pass of the pairs that fail the convergence test;
// with p_max > 3 one per mask-word range of the pairs that take the whole
// refinement loop.
static int partial_slots(const FieldLaunch& f, int splits) {
    return splits + (far_third_pass(f.np) ? splits : (far_adaptive(f.np) ? refine_parts(f) : 0));
}
// Resident CTAs (whole GPU) of the far-kernel variant a launch starts with:
// NRHS 4 / 2 / 1 (the first RHS chunk), real / complex k, FP64 / mixed.
static int far_slots(int n_rhs, bool ck, bool mixed) {
    static std::atomic<int> cache[2][3][2];
    const int ri = n_rhs >= 4 ? 0 : (n_rhs >= 2 ? 1 : 2);
    std::atomic<int>& c = cache[ck][ri][mixed];
    int v = c.load(std::memory_order_relaxed);
    if (v) return v;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn;
#define BIELCC_FK(R, C, M) (const void*)far_kernel<R, C, M>
    if (ri == 0) fn = ck ? (mixed ? BIELCC_FK(4, true, true) : BIELCC_FK(4, true, false))
                              : (mixed ? BIELCC_FK(4, false, true) : BIELCC_FK(4, false, false));
    else if (ri == 1) fn = ck ? (mixed ? BIELCC_FK(2, true, true) : BIELCC_FK(2, true, false))
                              : (mixed ? BIELCC_FK(2, false, true) : BIELCC_FK(2, false, false));
    else fn = ck ? (mixed ? BIELCC_FK(1, true, true) : BIELCC_FK(1, true, false))
                 : (mixed ? BIELCC_FK(1, false, true) : BIELCC_FK(1, false, false));
#undef BIELCC_FK
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kFarThreads, 0);
    v = std::max(1, sms * std::max(1, per));
    c.store(v, std::memory_order_relaxed);
    return v;
}

size_t field_ws_base_bytes(const FieldLaunch& f, int* splits_out, size_t partial_cap) {
    const int tiles = (f.n_pts + kFarThreads - 1) / kFarThreads;
    const int N = f.mesh->n_cells;
    const size_t P = f.n_pts;
    const size_t per_split = (size_t)f.n_rhs * 12 * P * sizeof(double);
    const int slots = far_slots(f.n_rhs, f.k.im != 0.0, f.precision == 1);
    const int max_splits = (int)std::max<size_t>(1, partial_cap / std::max<size_t>(1, per_split));
    int splits = choose_cell_splits(tiles, N, slots, max_splits);
    if (far_third_pass(f.np)) {
        // p_max = 3: the third pass's work sits on the points whose integrals
        // failed the test (near-field points, a few tiles), so a grid balanced
        // for the plain far kernel leaves most SMs idle. Cells split as finely
        // as the near mask allows (32 per split), within partial_cap for both
        // slot sets: 2000 x 8192 cells, FP64 94.6 -> 78.0 ms, mixed 61.8 -> 53.7 ms.
        const int want = (int)std::min<size_t>((N + 31) / 32, partial_cap / std::max<size_t>(1, 2 * per_split));
        if (want > splits) {
            const int cps = round_cells_per_split(N, want);
            splits = (N + cps - 1) / cps;
        }
    }
    *splits_out = splits;
    return align256((size_t)partial_slots(f, splits) * per_split) + 2 * align256((P + 1) * sizeof(long long)) +
           align256(sizeof(long long)) + align256(mask_words(N) * P * sizeof(unsigned)) +
           align256((size_t)f.n_rhs * 12 * P * sizeof(double)) +
           (far_adaptive(f.np) ? align256((size_t)(1 + f.n_rhs) * mask_words(N) * P * sizeof(unsigned)) : 0);
}

template <int NRHS, bool CK, bool MIXED>
static void launch_far_t(const FarArgs& a, int tiles, int splits, cudaStream_t s) {
    far_kernel<NRHS, CK, MIXED><<<dim3(tiles, splits), kFarThreads, 0, s>>>(a);
}

// p_max >= 3: one RHS per launch of the marks-reading variant.
template <bool CK, bool MIXED>
static int launch_far_marks(FarArgsMarks a, int tiles, int splits, cudaStream_t s) {
    for (int r = 0; r < a.n_rhs; r++) {
        a.rhs0 = r;
        far_kernel<1, CK, MIXED, true><<<dim3(tiles, splits), kFarThreads, 0, s>>>(a);
    }
    return a.n_rhs;
}

template <bool CK, bool MIXED>
static int launch_far_rhs(FarArgs a, int tiles, int splits, cudaStream_t s) {
    int n = 0;
    for (int r0 = 0; r0 < a.n_rhs; n++) {
        a.rhs0 = r0;
        int left = a.n_rhs - r0;
        if (left >= 4) { launch_far_t<4, CK, MIXED>(a, tiles, splits, s); r0 += 4; }
        else if (left >= 2) { launch_far_t<2, CK, MIXED>(a, tiles, splits, s); r0 += 2; }
        else { launch_far_t<1, CK, MIXED>(a, tiles, splits, s); r0 += 1; }
    }
    return n;
}

cudaError_t field_stage1(const FieldLaunch& f, void* ws, int splits, long long* d_total, cudaStream_t s,
                         int* launches, cudaEvent_t far_begin, cudaEvent_t far_end, int* far_launches) {
    const MeshDev& m = *f.mesh;
    const size_t P = f.n_pts;
    char* w = (char*)ws;
    double* partial = (double*)w;
    w += align256((size_t)partial_slots(f, splits) * f.n_rhs * 12 * P * sizeof(double));
    long long* counts = (long long*)w;
    w += align256((P + 1) * sizeof(long long));
    long long* offs = (long long*)w;
    w += align256((P + 1) * sizeof(long long)) + align256(sizeof(long long));
    unsigned* mask = (unsigned*)w;
    const int n_words = (int)mask_words(m.n_cells);
    w += align256(mask_words(m.n_cells) * P * sizeof(unsigned)) + align256((size_t)f.n_rhs * 12 * P * sizeof(double));
    // p_max >= 3, after the near sums: the marks of grad F, then of F . J per RHS
    unsigned* markG = far_adaptive(f.np) ? (unsigned*)w : nullptr;
    unsigned* markK = markG ? markG + mask_words(m.n_cells) * P : nullptr;

    FarArgs a;
    a.pts = f.pts;
    a.n_pts = f.n_pts;
    a.geo = m.geo;
    a.n_cells = m.n_cells;
    a.nodes64 = m.nodes64;
    a.nodes32 = m.nodes32;
    a.rho32 = m.rho32;
    a.nn = far_split_n(f.np) * far_split_n(f.np);
    a.J = reinterpret_cast<const cplx*>(f.J);
    a.n_rhs = f.n_rhs;
    a.rhs0 = 0;
    a.k = f.k;
    a.analytic_calc = f.np.analytic_calc;
    a.cells_per_split = round_cells_per_split(m.n_cells, splits);
    a.partial = partial;
    a.nearmask = mask;
    int tiles = (f.n_pts + kFarThreads - 1) / kFarThreads;
    bool ck = f.k.im != 0.0;
    bool mixed = f.precision == 1;
    int nl = 0;
    if (tiles > 0 && m.table_n != far_split_n(f.np))
        return cudaErrorInvalidValue;  // node tables of another split: the caller builds far_split_n's
    if (tiles > 0 && far_adaptive(f.np) && (m.table_lo_n != f.np.n_start || !m.nodes64_lo))
        return cudaErrorInvalidValue;  // no n_start table for the convergence test
    if (tiles > 0 && far_third_pass(f.np) && (m.table_hi_n != 4 * f.np.n_start || !m.nodes64_hi))
        return cudaErrorInvalidValue;  // no 4 n_start tables for the third pass
    if (far_begin) cudaEventRecord(far_begin, s);
    if (tiles > 0 && far_adaptive(f.np)) {
        // the convergence test of every far pair's integrals; the failing ones
        // are marked, the passing ones added to the split sums (slots [0, splits))
        cudaError_t e = cudaMemsetAsync(markK, 0, (size_t)f.n_rhs * n_words * P * sizeof(unsigned), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(partial, 0, (size_t)splits * f.n_rhs * 12 * P * sizeof(double), s);
        if (e != cudaSuccess) return e;
        const int nn_lo = f.np.n_start * f.np.n_start;
        const size_t rows = (size_t)(nn_lo + a.nn) * sizeof(double4);
        if (rows <= 48 * 1024)
            far_refine_decide_kernel<true><<<dim3(tiles, splits), kFarThreads, rows, s>>>(
                a, m.nodes64_lo, nn_lo, f.np.eps * f.np.eps, markG, markK);
        else
            far_refine_decide_kernel<false><<<dim3(tiles, splits), kFarThreads, 0, s>>>(
                a, m.nodes64_lo, nn_lo, f.np.eps * f.np.eps, markG, markK);
        nl++;
    }
    FarArgsMarks am;
    static_cast<FarArgs&>(am) = a;
    am.markG = markG;
    am.markK = markK;
    if (tiles > 0 && !markG) {
        if (mixed) nl += ck ? launch_far_rhs<true, true>(a, tiles, splits, s) : launch_far_rhs<false, true>(a, tiles, splits, s);
        else nl += ck ? launch_far_rhs<true, false>(a, tiles, splits, s) : launch_far_rhs<false, false>(a, tiles, splits, s);
    }
    if (tiles > 0 && far_third_pass(f.np)) {
        // p_max = 3: the marked pairs return the third pass, at 4 n_start, into
        // their own partial slots
        FarArgsMarks a3 = am;
        a3.nodes64 = m.nodes64_hi;
        a3.nodes32 = m.nodes32_hi;
        a3.rho32 = m.rho32_hi;
        a3.nn = 16 * f.np.n_start * f.np.n_start;
        a3.partial = partial + (size_t)splits * f.n_rhs * 12 * P;
        a3.take_marked = 1;
        if (mixed) nl += ck ? launch_far_marks<true, true>(a3, tiles, splits, s) : launch_far_marks<false, true>(a3, tiles, splits, s);
        else nl += ck ? launch_far_marks<true, false>(a3, tiles, splits, s) : launch_far_marks<false, false>(a3, tiles, splits, s);
    } else if (tiles > 0 && f.n_rhs > 0 && far_adaptive(f.np)) {
        DNP np{f.np.eps, f.np.rs, f.np.rs_seg, f.np.analytic_calc, f.np.n_start, f.np.n_start_seg, f.np.p_max,
               f.np.p_max_seg};
        far_refine_sum_kernel<<<dim3((f.n_pts + 7) / 8, f.n_rhs, refine_parts(f)), 256, 0, s>>>(
            a, markG, markK, m.verts, m.nv, np, partial + (size_t)splits * f.n_rhs * 12 * P);
        nl++;
    }
    if (far_end) cudaEventRecord(far_end, s);
    if (tiles > 0) near_count_kernel<<<tiles, kFarThreads, 0, s>>>(mask, n_words, f.n_pts, counts);
    *far_launches = nl;
    *launches = nl + (tiles > 0 ? 1 : 0) + 1;
    scan_kernel<<<1, 1024, 0, s>>>(counts, f.n_pts, offs, d_total);
    return cudaGetLastError();
}

cudaError_t field_stage2(const FieldLaunch& f, void* ws, int splits, long long n_near, void* pair_ws,
                         unsigned long long* d_nonfinite, cudaStream_t s, int* launches) {
    *launches = 0;
    const MeshDev& m = *f.mesh;
    const size_t P = f.n_pts;
    char* w = (char*)ws;
    double* partial = (double*)w;
    w += align256((size_t)partial_slots(f, splits) * f.n_rhs * 12 * P * sizeof(double));
    w += align256((P + 1) * sizeof(long long));
    long long* offs = (long long*)w;
    w += align256((P + 1) * sizeof(long long)) + align256(sizeof(long long));
    const unsigned* mask = (const unsigned*)w;
    const int n_words = (int)mask_words(m.n_cells);
    w += align256(mask_words(m.n_cells) * P * sizeof(unsigned));
    double* near = (double*)w;

    int* pair_cell = nullptr;
    int* pair_pt = nullptr;
    cplx* moments = nullptr;
    int tiles = (f.n_pts + kFarThreads - 1) / kFarThreads;
    if (n_near > 0) {
        char* pw = (char*)pair_ws;
        moments = (cplx*)pw;
        pw += align256((size_t)n_near * 13 * sizeof(cplx));
        pair_cell = (int*)pw;
        pw += align256((size_t)n_near * sizeof(int));
        pair_pt = (int*)pw;
        near_fill_kernel<<<(f.n_pts + 7) / 8, 256, 0, s>>>(mask, n_words, f.n_pts, offs, pair_cell, pair_pt);
        DNP np{f.np.eps, f.np.rs, f.np.rs_seg, f.np.analytic_calc, f.np.n_start, f.np.n_start_seg, f.np.p_max,
               f.np.p_max_seg};
        int blocks = (int)((n_near + 127) / 128);
        near_pair_kernel<<<blocks, 128, 0, s>>>(f.pts, m.verts, m.nv, pair_cell, pair_pt, n_near, f.k, np, moments);
        near_sum_kernel<<<dim3((f.n_pts + 7) / 8, f.n_rhs), 256, 0, s>>>(
            offs, pair_cell, moments, reinterpret_cast<const cplx*>(f.J), f.n_pts, m.n_cells, near);
        *launches += 3;
    }
    FinalArgs fa;
    fa.pts = f.pts;
    fa.n_pts = f.n_pts;
    fa.n_rhs = f.n_rhs;
    fa.n_cells = m.n_cells;
    fa.splits = partial_slots(f, splits);
    fa.partial = partial;
    fa.offs = n_near > 0 ? offs : nullptr;
    fa.near = near;
    fa.mult = f.mult;
    for (int g = 0; g < 3; g++) {
        fa.kvec[g] = f.kvec[g];
        fa.e0[g] = f.e0[g];
    }
    fa.h_scale = f.h_scale;
    fa.add_E = f.add_E;
    fa.add_H = f.add_H;
    fa.E = f.E;
    fa.H = f.H;
    fa.nonfinite = d_nonfinite;
    if (tiles > 0 && f.n_rhs > 0) {
        if (fa.splits > 32) finalize_kernel<true><<<dim3((f.n_pts + 7) / 8, f.n_rhs), 256, 0, s>>>(fa);
        else finalize_kernel<false><<<dim3(tiles, f.n_rhs), kFarThreads, 0, s>>>(fa);
        *launches += 1;
    }
    return cudaGetLastError();
}

// Bytes of the stage-2 pair workspace for n_near pairs (matches the carving).
size_t field_pair_ws_bytes(long long n_near) {
    return align256((size_t)n_near * 13 * sizeof(cplx)) + 2 * align256((size_t)n_near * sizeof(int));
}

}  // namespace bielcc_gpu
