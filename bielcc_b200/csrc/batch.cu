// batch.cu — many field evaluations (meshes of uneven sizes, each with its own
// points, wave number and 1..S right-hand sides) in ONE persistent launch.
//
// Work is cut into items (job, 32-point tile, cell range) and ordered by
// estimated cost (largest first); each CTA of the persistent grid pulls the
// next item from a device counter. An item walks its cell range in chunks:
//   phase A — warp w evaluates the far-field moments (A1, T, G: 20 values,
//             farnode.cuh) of cells w, w+4, ... of the chunk for its 32 points
//             and stores them in shared memory (node tiles staged with 128-bit
//             loads, one observation point per lane);
//   phase B — the same threads contract the chunk's moments with the
//             right-hand sides, staged in shared memory a pass of kSP at a time
//             (the moments stay), R RHS per thread held in registers, and add
//             the result into the job's partial sums.
// Extra right-hand sides therefore cost ~72 FP32 operations per pair instead
// of the 64-node integrand. Near cells (get_field.h:58) are flagged in the
// job's near mask and handled by the FP64 near-pair path afterwards, exactly
// as in the single-job pipeline. Summation order depends only on the job
// itself (its ranges and chunks), never on the other jobs of the batch.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../../include/bielcc_gpu.h"
#include "farnode.cuh"
#include "internal.h"
#include "ops.cuh"
#include "scan.cuh"
#include "umma.cuh"

namespace bielcc_gpu {

constexpr int kBT = 128;  // threads per CTA: 4 warps x 32 points
constexpr int kBP = 32;   // points per item tile
constexpr int kBW = 4;    // warps
// Mixed form: cells per chunk at n_start <= 8 (CH32), right-hand sides staged
// per pass (SP; a chunk's moments are computed once and contracted pass by
// pass), and resident CTAs per SM the kernel is compiled for (MINB).
// Measured on the 256-mesh batch (B200), cells / RHS per pass / CTAs per SM:
// 16 / 16 / 3 (168 registers, 73 KB smem) 680 ms; 12 / 16 / 3 709 ms;
// 16 / 64 / 2 (234 registers, 109 KB) 760 ms; 12 / 16 / 4 787 ms;
// 8 / 16 / 4 (128 registers) 888 ms.
#ifndef BIELCC_BATCH_CH32
#define BIELCC_BATCH_CH32 16
#endif
#ifndef BIELCC_BATCH_SP
#define BIELCC_BATCH_SP 16
#endif
#ifndef BIELCC_BATCH_MINB
#define BIELCC_BATCH_MINB 3
#endif
// Mixed form: phase A two cells per warp at a time (TWO = 1) or one; RHS per
// thread in phase B (R; SP a multiple of 4 R). Measured on the 256-mesh batch
// (cells / SP / CTAs per SM / TWO / R): 16 / 16 / 3 / 1 / 4 (164 registers)
// 659 ms; 16 / 16 / 3 / 0 / 4 707 ms; 12 / 8 / 4 / 0 / 2 (128 registers)
// 705 ms; 8 / 8 / 4 / 1 / 2 734 ms; 8 / 8 / 5 / 0 / 2 (96 registers, 20 warps
// per SM) 865 ms: the two-cell node loop's second dependency chain is worth
// more than extra warps.
#ifndef BIELCC_BATCH_TWO
#define BIELCC_BATCH_TWO 1
#endif
#ifndef BIELCC_BATCH_R
#define BIELCC_BATCH_R 4
#endif
constexpr int kSP = BIELCC_BATCH_SP;  // right-hand sides staged per pass (a multiple of kBW x R)
// Unrolling of the one-cell and two-cell phase-A node loops. Three CTAs of
// different jobs (different phase polynomials) share an SM's instruction
// cache: the two-cell loop, already two dependency chains wide, is not
// unrolled (256-mesh batch: 681 ms unrolled x2, 661 ms not unrolled).
#ifndef BIELCC_BATCH_U1
#define BIELCC_BATCH_U1 4
#endif
#ifndef BIELCC_BATCH_U2
#define BIELCC_BATCH_U2 1
#endif
// FP64 form: unrolling of the node loop and resident CTAs per SM asked of the
// kernel. Measured on 64 meshes of the batched workload (unroll / CTAs per SM):
// 1 / 3 (168 registers, no spills) 284 ms; 2 / 3 284 ms; 4 / 3 322-327 ms;
// 1 / 2 (206 registers) 338 ms; 8 / 2 388 ms; 8 / 3 436 ms; 16 / 3 491 ms.
// Unrolling costs instruction-cache misses (CTAs of different jobs share an
// SM); a third CTA hides the FP64 latency better.
#ifndef BIELCC_BATCH64_UNROLL
#define BIELCC_BATCH64_UNROLL 1
#endif
#ifndef BIELCC_BATCH64_MINB
#define BIELCC_BATCH64_MINB 3
#endif
#define BIELCC_PRAGMA_STR(x) #x
#define BIELCC_UNROLL(n) _Pragma(BIELCC_PRAGMA_STR(unroll n))

template <bool MIXED>
struct BatchCfg {
    using F = typename std::conditional<MIXED, float, double>::type;
    using NodeT = typename std::conditional<MIXED, float4, double4>::type;
    static constexpr int CH = MIXED ? BIELCC_BATCH_CH32 : 8;            // cells per chunk (n_start <= 8)
    static constexpr int NODES = MIXED ? 64 * BIELCC_BATCH_CH32 : 512;  // staged nodes
    static constexpr int R = MIXED ? BIELCC_BATCH_R : 2;  // RHS per thread in phase B
    // currents per (cell, RHS, component): FP32 (re, im, im, re) for the packed
    // contraction, FP64 (re, im)
    static constexpr int JW = MIXED ? 4 : 2;
    static constexpr size_t YY = MIXED ? NODES : 0;  // |y - centre|^2 of the staged nodes (mixed form)
    static constexpr size_t smem_bytes() {
        return sizeof(NodeT) * NODES + sizeof(float) * YY + sizeof(F) * CH * 20 * kBP + sizeof(F) * JW * CH * kSP * 3 +
               sizeof(double4) * CH + sizeof(double) * CH + CH * kBP + 64;
    }
};
static_assert(kSP % (kBW * BatchCfg<true>::R) == 0, "a phase-B pass covers whole groups of kBW x R RHS");


// acc[12] += contraction of one cell's moments m[20] (a1r, a1i, t[6][2], g[3][2])
// with the current J = (jr, ji): E = (A1 I + T) J, H = G x J. The caller has
// folded A1 into T's diagonal (m[2..3], m[8..9], m[12..13]) once per cell, so
// E is one complex 3x3 matrix-vector product per right-hand side.
template <typename F>
BIELCC_D void contract12(const F* m, const F* jr, const F* ji, F* acc) {
    const int ti[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        F er = 0, ei = 0;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const F tr = m[2 + 2 * ti[a][b]], tim = m[3 + 2 * ti[a][b]];
            er += tr * jr[b] - tim * ji[b];
            ei += tr * ji[b] + tim * jr[b];
        }
        acc[2 * a] += er;
        acc[2 * a + 1] += ei;
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        const F gbr = m[14 + 2 * b], gbi = m[15 + 2 * b], gcr = m[14 + 2 * c], gci = m[15 + 2 * c];
        acc[6 + 2 * a] += (gbr * jr[c] - gbi * ji[c]) - (gcr * jr[b] - gci * ji[b]);
        acc[6 + 2 * a + 1] += (gbr * ji[c] + gbi * jr[c]) - (gcr * ji[b] + gci * jr[b]);
    }
}

// The FP32 contraction of one cell's moments (A1 already on T's diagonal) with
// the RHS sl = sl0 + step * j (j < R, sl < sp), two lanes of a packed
// fma.rn.f32x2 per complex multiply-add: (mr + i mi)(jr + i ji) =
// (mr, mr) * (jr, ji) + (-mi, mi) * (ji, jr). The currents are staged as
// (re, im, im, re), so both operand pairs come from one 128-bit load. The
// accumulators are (re, im) pairs: E x, y, z then H x, y, z. ALL: every one of
// the R right-hand sides is staged (no per-RHS test, so the R RHS's
// multiply-add chains interleave freely).
BIELCC_D float2 f2(float v) { return make_float2(v, v); }

template <int R, bool ALL>
BIELCC_D void contract_packed_cell(const float* m, const float4* __restrict__ sj, int sl0, int step, int sp,
                                   float2 (&acc)[R][6]) {
    float2 P[9], Q[9];  // T (6 entries), G (3): (mr, mr), (-mi, mi)
#pragma unroll
    for (int q = 0; q < 6; q++) {
        P[q] = f2(m[2 + 2 * q]);
        Q[q] = make_float2(-m[3 + 2 * q], m[3 + 2 * q]);
    }
    float2 NP[3], NQ[3];  // -G as pairs, for the subtracted half of G x J
#pragma unroll
    for (int q = 0; q < 3; q++) {
        P[6 + q] = f2(m[14 + 2 * q]);
        Q[6 + q] = make_float2(-m[15 + 2 * q], m[15 + 2 * q]);
        NP[q] = f2(-m[14 + 2 * q]);
        NQ[q] = make_float2(m[15 + 2 * q], -m[15 + 2 * q]);
    }
    const int ti[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    // Component b of the currents of all R right-hand sides at a time: every
    // accumulator takes one multiply-add in turn, so consecutive multiply-adds
    // into one accumulator are 12 (E) or 8 (H) instructions apart.
#pragma unroll
    for (int b = 0; b < 3; b++) {
        float2 jp[R], js[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (!ALL && sl0 + step * j >= sp) continue;
            const float4 v = sj[(size_t)(sl0 + step * j) * 3 + b];
            jp[j] = make_float2(v.x, v.y);
            js[j] = make_float2(v.z, v.w);
        }
        // E_a += W_ab J_b: the (mr, mr) halves, then the (-mi, mi) halves
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (!ALL && sl0 + step * j >= sp) continue;
#pragma unroll
            for (int a = 0; a < 3; a++) acc[j][a] = __ffma2_rn(P[ti[a][b]], jp[j], acc[j][a]);
        }
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (!ALL && sl0 + step * j >= sp) continue;
#pragma unroll
            for (int a = 0; a < 3; a++) acc[j][a] = __ffma2_rn(Q[ti[a][b]], js[j], acc[j][a]);
        }
        // H_a = G_(a+1) J_(a+2) - G_(a+2) J_(a+1): J_b adds G_(b+2) J_b to
        // H_(b+1) and takes G_(b+1) J_b from H_(b+2)
        const int a1 = (b + 1) % 3, a2 = (b + 2) % 3;
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (!ALL && sl0 + step * j >= sp) continue;
            acc[j][3 + a1] = __ffma2_rn(P[6 + a2], jp[j], acc[j][3 + a1]);
            acc[j][3 + a2] = __ffma2_rn(NP[a1], jp[j], acc[j][3 + a2]);
        }
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (!ALL && sl0 + step * j >= sp) continue;
            acc[j][3 + a1] = __ffma2_rn(Q[6 + a2], js[j], acc[j][3 + a1]);
            acc[j][3 + a2] = __ffma2_rn(NQ[a1], js[j], acc[j][3 + a2]);
        }
    }
}

// One cell's 20 moments from the staged chunk (s_mom[cc][20][32]), A1 folded
// onto T's diagonal (t_xx, t_yy, t_zz): W = A1 I + T.
template <typename F>
BIELCC_D void load_cell_moments(const F* s_mom, int cc, int lane, F (&m)[20]) {
#pragma unroll
    for (int q = 0; q < 20; q++) m[q] = s_mom[(cc * 20 + q) * kBP + lane];
    m[2] += m[0];
    m[3] += m[1];
    m[8] += m[0];
    m[9] += m[1];
    m[12] += m[0];
    m[13] += m[1];
}

// Moments of one cell, real-k form finished, times e^{ik r0} into mom[20];
// R_Rot_Colloc is 0 at the cell centre.
template <bool CK, typename F>
BIELCC_D void store_moments(Moments<F>& m, double P0r, double P0i, double d, F* mom) {
    if (!CK) m.finish_real_k();
    const F pr = (F)P0r, pi = (F)P0i;
    mom[0] = m.a1r * pr - m.a1i * pi;
    mom[1] = m.a1r * pi + m.a1i * pr;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        mom[2 + 2 * q] = m.t[q][0] * pr - m.t[q][1] * pi;
        mom[3 + 2 * q] = m.t[q][0] * pi + m.t[q][1] * pr;
    }
    if (!(d < kMachineZero)) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            mom[14 + 2 * q] = m.g[q][0] * pr - m.g[q][1] * pi;
            mom[15 + 2 * q] = m.g[q][0] * pi + m.g[q][1] * pr;
        }
    }
}

// Mixed-form set-up of one (point, cell) pair: FP32 pair state, e^{ik r0} in
// FP64, and the phase polynomial for the cell's phase range |k| rho.
template <bool CK>
BIELCC_D int mixed_pair_setup(const double* x, const double4& ci, double d, double rho, cplx k, const KF32& kf,
                              PairF32& pf, double& P0r, double& P0i) {
    const double cen[3] = {ci.x, ci.y, ci.z};
    pf.set(x, cen, d, kf);
    double sn, cs;
    sincos(k.re * d, &sn, &cs);
    if (CK) {
        const double am = exp(-k.im * d);
        sn *= am;
        cs *= am;
    }
    P0r = cs;
    P0i = sn;
    return phase_mode((float)fabs(k.re) * (float)rho);
}

// Phase A of one (point, cell) pair: the 20 far moments times e^{ik r0}.
// CK (complex k) is a property of the job, so every item of a job takes the
// same code path whatever else is in the batch.
template <bool MIXED, bool CK>
BIELCC_D void batch_moments(const typename BatchCfg<MIXED>::NodeT* nd, const float* yy, int nn, const double* x,
                            const double4& ci, double d, double rho, cplx k, double k2r, double k2i,
                            typename BatchCfg<MIXED>::F* mom) {
    using F = typename BatchCfg<MIXED>::F;
    double P0r = 1.0, P0i = 0.0;
    Moments<F> m;
    m.zero();
    if constexpr (MIXED) {
        const KF32 kf = KF32::make(k.re, k.im);
        PairF32 pf;
        const int mode = mixed_pair_setup<CK>(x, ci, d, rho, k, kf, pf, P0r, P0i);
#define BIELCC_BNODE(MODE_) \
    BIELCC_UNROLL(BIELCC_BATCH_U1) for (int i = 0; i < nn; i++) far_node_f32<CK, MODE_>(m, pf, nd[i], yy[i], kf);
        switch (mode) {
            case 0: BIELCC_BNODE(0) break;
            case 1: BIELCC_BNODE(1) break;
            case 2: BIELCC_BNODE(2) break;
            case 3: BIELCC_BNODE(3) break;
            default: BIELCC_BNODE(4) break;
        }
#undef BIELCC_BNODE
    } else {
        const bool split = !CK && fabs(k.re) * rho * (1.0 + 1e-6) <= 0.5;
        if (split) {
            double sn, cs;
            sincos(k.re * d, &sn, &cs);
            P0r = cs;
            P0i = sn;
            BIELCC_UNROLL(BIELCC_BATCH64_UNROLL)
            for (int i = 0; i < nn; i++) {
                const double4 v = nd[i];
                far_node_f64<CK, true>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, k, k2r, k2i, d);
            }
        } else {
            BIELCC_UNROLL(BIELCC_BATCH64_UNROLL)
            for (int i = 0; i < nn; i++) {
                const double4 v = nd[i];
                far_node_f64<CK, false>(m, x[0] - v.x, x[1] - v.y, x[2] - v.z, v.w, k, k2r, k2i, d);
            }
        }
    }
    store_moments<CK, F>(m, P0r, P0i, d, mom);
}

// Phase A of two far pairs of the same point (cells A and B of one job, equal
// node counts), mixed form: the two node loops are interleaved, so each thread
// has two independent dependency chains per node. A cell's moments do not
// depend on the other cell; the phase polynomial is the one for the larger
// phase range of the two (exact over the smaller range too).
template <bool CK>
BIELCC_D void batch_moments2(const float4* ndA, const float* yyA, const float4* ndB, const float* yyB, int nn,
                             const double* x, const double4& ciA, double dA, double rhoA, const double4& ciB,
                             double dB, double rhoB, cplx k, float* momA, float* momB) {
    const KF32 kf = KF32::make(k.re, k.im);
    PairF32 pa, pb;
    double PAr, PAi, PBr, PBi;
    const int mode = max(mixed_pair_setup<CK>(x, ciA, dA, rhoA, k, kf, pa, PAr, PAi),
                         mixed_pair_setup<CK>(x, ciB, dB, rhoB, k, kf, pb, PBr, PBi));
    Moments<float> ma, mb;
    ma.zero();
    mb.zero();
#define BIELCC_BNODE2(MODE_)                                 \
    BIELCC_UNROLL(BIELCC_BATCH_U2) for (int i = 0; i < nn; i++) { \
        far_node_f32<CK, MODE_>(ma, pa, ndA[i], yyA[i], kf); \
        far_node_f32<CK, MODE_>(mb, pb, ndB[i], yyB[i], kf); \
    }
    switch (mode) {
        case 0: BIELCC_BNODE2(0) break;
        case 1: BIELCC_BNODE2(1) break;
        case 2: BIELCC_BNODE2(2) break;
        case 3: BIELCC_BNODE2(3) break;
        default: BIELCC_BNODE2(4) break;
    }
#undef BIELCC_BNODE2
    store_moments<CK, float>(ma, PAr, PAi, dA, momA);
    store_moments<CK, float>(mb, PBr, PBi, dB, momB);
}

// Phase B of one chunk: the right-hand sides s0 + sb + warp + 4 j (j < R) of the
// sp staged in s_j, contracted with the chunk's moments (s_mom[cc][20][32])
// and added into the job's partial sums (stored by the item's first chunk).
// A warp whose R right-hand sides are all staged runs the contraction without
// per-RHS tests; a warp with none skips the chunk.
// R: right-hand sides per thread; SP: right-hand sides per staged pass (the
// stride of s_j). Neither changes any sum: each RHS's chunk sum takes its
// cells in order, whatever the grouping.
template <bool MIXED, int R = BatchCfg<MIXED>::R, int SP = kSP>
BIELCC_D void batch_phase_b(const typename BatchCfg<MIXED>::F* s_mom, const typename BatchCfg<MIXED>::F* s_j, int nc,
                            int s0, int sp, int warp, int lane, bool live, const JobDev& jb, int range, int S, int P,
                            int p, bool first) {
    using C = BatchCfg<MIXED>;
    using F = typename C::F;
    static_assert(SP % (kBW * R) == 0, "a phase-B pass covers whole groups of kBW x R RHS");
    for (int sb = 0; sb < sp; sb += kBW * R) {
        const int sl0 = sb + warp;
        if (sl0 >= sp) break;  // warp-uniform: no staged RHS left for this warp
        if constexpr (MIXED) {
            float2 acc[R][6];
#pragma unroll
            for (int j = 0; j < R; j++)
#pragma unroll
                for (int q = 0; q < 6; q++) acc[j][q] = make_float2(0.f, 0.f);
            const float4* sj = reinterpret_cast<const float4*>(s_j);
            if (sl0 + kBW * (R - 1) < sp) {
                for (int cc = 0; cc < nc; cc++) {
                    float m[20];
                    load_cell_moments<float>(s_mom, cc, lane, m);
                    contract_packed_cell<R, true>(m, sj + (size_t)cc * SP * 3, sl0, kBW, sp, acc);
                }
            } else {
                for (int cc = 0; cc < nc; cc++) {
                    float m[20];
                    load_cell_moments<float>(s_mom, cc, lane, m);
                    contract_packed_cell<R, false>(m, sj + (size_t)cc * SP * 3, sl0, kBW, sp, acc);
                }
            }
            if (live) {
#pragma unroll
                for (int j = 0; j < R; j++) {
                    const int sl = sl0 + kBW * j;
                    if (sl >= sp) continue;
                    double* dst = jb.partial + (((size_t)range * S + (s0 + sl)) * 12) * (size_t)P + p;
                    // one writer per address (this thread), so the adds land in chunk
                    // order: the fire-and-forget reduction (no load to wait for) gives
                    // the same sums as a load-add-store
                    if (first) {
#pragma unroll
                        for (int q = 0; q < 6; q++) {
                            dst[(size_t)(2 * q) * P] = (double)acc[j][q].x;
                            dst[(size_t)(2 * q + 1) * P] = (double)acc[j][q].y;
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < 6; q++) {
                            atomicAdd(dst + (size_t)(2 * q) * P, (double)acc[j][q].x);
                            atomicAdd(dst + (size_t)(2 * q + 1) * P, (double)acc[j][q].y);
                        }
                    }
                }
            }
        } else {
            F acc[R][12];
#pragma unroll
            for (int j = 0; j < R; j++)
#pragma unroll
                for (int q = 0; q < 12; q++) acc[j][q] = 0;
            for (int cc = 0; cc < nc; cc++) {
                F m[20];
                load_cell_moments<F>(s_mom, cc, lane, m);
#pragma unroll
                for (int j = 0; j < R; j++) {
                    const int sl = sl0 + kBW * j;
                    if (sl < sp) {
                        const F* jj = s_j + (size_t)(cc * SP + sl) * 6;
                        const F jr[3] = {jj[0], jj[2], jj[4]}, ji[3] = {jj[1], jj[3], jj[5]};
                        contract12<F>(m, jr, ji, acc[j]);
                    }
                }
            }
            if (live) {
#pragma unroll
                for (int j = 0; j < R; j++) {
                    const int sl = sl0 + kBW * j;
                    if (sl >= sp) continue;
                    double* dst = jb.partial + (((size_t)range * S + (s0 + sl)) * 12) * (size_t)P + p;
                    if (first) {
#pragma unroll
                        for (int q = 0; q < 12; q++) dst[(size_t)q * P] = (double)acc[j][q];
                    } else {
#pragma unroll
                        for (int q = 0; q < 12; q++) atomicAdd(dst + (size_t)q * P, (double)acc[j][q]);
                    }
                }
            }
        }
    }
}

// Stages the currents of RHS s0 .. s0 + sp - 1 of cells c0 .. c0 + nc - 1
// (FP32 (re, im, im, re) for the packed contraction; FP64 (re, im)); SP: the
// staging stride in right-hand sides.
template <bool MIXED, int SP = kSP>
BIELCC_D void batch_stage_j(typename BatchCfg<MIXED>::F* s_j, const JobDev& jb, int c0, int nc, int s0, int sp,
                            int tid) {
    using C = BatchCfg<MIXED>;
    using F = typename C::F;
    const int N = jb.n_cells;
    for (int i = tid; i < nc * sp * 3; i += kBT) {
        const int cc = i / (sp * 3), rem = i - cc * sp * 3, sl = rem / 3, g = rem - sl * 3;
        const cplx v = jb.J[((size_t)(s0 + sl) * N + (c0 + cc)) * 3 + g];
        const size_t e = (size_t)(cc * SP + sl) * 3 + g;
        if constexpr (MIXED) {  // one 128-bit store: (re, im, im, re)
            const float re = (float)v.re, im = (float)v.im;
            reinterpret_cast<float4*>(s_j)[e] = make_float4(re, im, im, re);
        } else {
            reinterpret_cast<double2*>(s_j)[e] = make_double2(v.re, v.im);
        }
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(kBT, MIXED ? BIELCC_BATCH_MINB : BIELCC_BATCH64_MINB) batch_far_kernel(const JobDev* __restrict__ jobs,
                                                         const BatchItem* __restrict__ items, int n_items,
                                                         int* __restrict__ counter, double analytic_calc, int n_start,
                                                         int max_items) {
    using C = BatchCfg<MIXED>;
    using F = typename C::F;
    using NodeT = typename C::NodeT;
    extern __shared__ __align__(16) unsigned char smem[];
    NodeT* s_nodes = (NodeT*)smem;
    float* s_yy = (float*)(s_nodes + C::NODES);          // [NODES] (mixed form only)
    F* s_mom = (F*)(s_yy + C::YY);                       // [CH][20][kBP]
    F* s_j = s_mom + C::CH * 20 * kBP;                   // [CH][kSP][3][JW]
    double4* s_cell = (double4*)(s_j + C::CH * kSP * 3 * C::JW);  // centre, diam
    double* s_rho = (double*)(s_cell + C::CH);
    unsigned char* s_near = (unsigned char*)(s_rho + C::CH);  // [CH][kBP]
    __shared__ int s_item;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nn = n_start * n_start;
    const int ch = max(1, min(C::CH, C::NODES / nn));

    for (int taken = 0; taken < max_items; taken++) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const BatchItem bi = items[it];
        const JobDev& jb = jobs[bi.job];
        const int P = jb.n_pts, N = jb.n_cells, S = jb.n_rhs;
        const int p = bi.tile * kBP + lane;
        const bool live = p < P;
        double x[3] = {0., 0., 0.};
        if (live)
            for (int g = 0; g < 3; g++) x[g] = jb.pts[3 * (size_t)p + g];
        const int cb = bi.range * jb.cells_per_range;
        const int ce = min(N, cb + jb.cells_per_range);
        const cplx k = jb.k;
        const double k2r = k.re * k.re - k.im * k.im, k2i = 2.0 * k.re * k.im;
        unsigned nbits = 0;

        for (int c0 = cb; c0 < ce; c0 += ch) {
            const int nc = min(ch, ce - c0);
            // phase B: RHS s0 + sb + warp + 4 j (j < R) of the sp staged in s_j, contracted over
            // the chunk's cells and added into the job's partial sums
            auto phase_b = [&](int s0, int sp) {
                batch_phase_b<MIXED>(s_mom, s_j, nc, s0, sp, warp, lane, live, jb, bi.range, S, P, p, c0 == cb);
            };
            auto stage_j = [&](int s0, int sp) { batch_stage_j<MIXED>(s_j, jb, c0, nc, s0, sp, threadIdx.x); };
            __syncthreads();
            // stage node tables, cell rows and the first RHS pass's currents
            if constexpr (MIXED) {
                const float4* src = jb.nodes32 + (size_t)c0 * nn;
                for (int i = threadIdx.x; i < nc * nn; i += kBT) {
                    const float4 v = __ldg(src + i);
                    s_nodes[i] = v;
                    s_yy[i] = node_yy(v);
                }
            } else {
                const double2* src = reinterpret_cast<const double2*>(jb.nodes64 + (size_t)c0 * nn);
                double2* dst = reinterpret_cast<double2*>(s_nodes);
                for (int i = threadIdx.x; i < 2 * nc * nn; i += kBT) dst[i] = __ldg(src + i);
            }
            for (int i = threadIdx.x; i < nc; i += kBT) {
                const CellGeo& gg = jb.geo[c0 + i];
                s_cell[i] = make_double4(gg.c[0], gg.c[1], gg.c[2], gg.diam);
                s_rho[i] = (double)jb.rho32[c0 + i];
            }
            stage_j(0, min(kSP, S));
            __syncthreads();
            // phase A: moments of cells warp, warp+4, ... for this warp's 32 points; the
            // mixed form takes them two at a time (cells cc and cc + 4)
            if constexpr (MIXED && BIELCC_BATCH_TWO) {
                for (int cc = warp; cc < nc; cc += 2 * kBW) {
                    const int cb2 = cc + kBW;
                    const bool two = cb2 < nc;
                    const double4 ca = s_cell[cc], cbb = s_cell[two ? cb2 : cc];
                    const double cena[3] = {ca.x, ca.y, ca.z}, cenb[3] = {cbb.x, cbb.y, cbb.z};
                    double da, db;
                    const bool na = is_near(x, cena, ca.w, analytic_calc, &da);
                    const bool nb = is_near(x, cenb, cbb.w, analytic_calc, &db);
                    const bool fa = !na && live, fb = two && !nb && live;
                    s_near[cc * kBP + lane] = na ? 1 : 0;
                    if (two) s_near[cb2 * kBP + lane] = nb ? 1 : 0;
                    F moa[20], mob[20];
#pragma unroll
                    for (int q = 0; q < 20; q++) moa[q] = mob[q] = 0;
                    const NodeT *nda = s_nodes + cc * nn, *ndb = s_nodes + (two ? cb2 : cc) * nn;
                    const float *ya = s_yy + cc * nn, *yb = s_yy + (two ? cb2 : cc) * nn;
                    const bool ck = k.im != 0.0;
                    if (fa && fb) {
                        if (ck) batch_moments2<true>(nda, ya, ndb, yb, nn, x, ca, da, s_rho[cc], cbb, db,
                                                     s_rho[cb2], k, moa, mob);
                        else batch_moments2<false>(nda, ya, ndb, yb, nn, x, ca, da, s_rho[cc], cbb, db,
                                                   s_rho[cb2], k, moa, mob);
                    } else if (fa || fb) {
                        const NodeT* nd = fa ? nda : ndb;
                        const float* yy = fa ? ya : yb;
                        const double4 ci = fa ? ca : cbb;
                        const double d = fa ? da : db, rho = s_rho[fa ? cc : cb2];
                        F* mo = fa ? moa : mob;
                        if (ck) batch_moments<MIXED, true>(nd, yy, nn, x, ci, d, rho, k, k2r, k2i, mo);
                        else batch_moments<MIXED, false>(nd, yy, nn, x, ci, d, rho, k, k2r, k2i, mo);
                    }
#pragma unroll
                    for (int q = 0; q < 20; q++) s_mom[(cc * 20 + q) * kBP + lane] = moa[q];
                    if (two) {
#pragma unroll
                        for (int q = 0; q < 20; q++) s_mom[(cb2 * 20 + q) * kBP + lane] = mob[q];
                    }
                }
            } else {
                for (int cc = warp; cc < nc; cc += kBW) {
                    const double4 ci = s_cell[cc];
                    const double cen[3] = {ci.x, ci.y, ci.z};
                    double d;
                    const bool nr = is_near(x, cen, ci.w, analytic_calc, &d);
                    const bool far = !nr && live;
                    s_near[cc * kBP + lane] = nr ? 1 : 0;
                    F mom[20];
#pragma unroll
                    for (int q = 0; q < 20; q++) mom[q] = 0;
                    if (far) {
                        const NodeT* nd = s_nodes + cc * nn;
                        const float* yy = s_yy + (MIXED ? cc * nn : 0);
                        if (k.im != 0.0)
                            batch_moments<MIXED, true>(nd, yy, nn, x, ci, d, s_rho[cc], k, k2r, k2i, mom);
                        else
                            batch_moments<MIXED, false>(nd, yy, nn, x, ci, d, s_rho[cc], k, k2r, k2i, mom);
                    }
#pragma unroll
                    for (int q = 0; q < 20; q++) s_mom[(cc * 20 + q) * kBP + lane] = mom[q];
                }
            }
            __syncthreads();
            // near-cell mask: warp 0 owns the words of its points
            if (warp == 0) {
                for (int cc = 0; cc < nc; cc++) {
                    const int c = c0 + cc;
                    nbits |= (unsigned)s_near[cc * kBP + lane] << (c & 31);
                    if ((c & 31) == 31 || c == ce - 1) {
                        if (live) jb.mask[(size_t)(c >> 5) * P + p] = nbits;
                        nbits = 0;
                    }
                }
            }
            phase_b(0, min(kSP, S));
            // further RHS passes reuse the chunk's moments in shared memory
            for (int s0 = kSP; s0 < S; s0 += kSP) {
                __syncthreads();
                stage_j(s0, min(kSP, S - s0));
                __syncthreads();
                phase_b(s0, min(kSP, S - s0));
            }
        }
    }
}

// ---------------------------------------------------------------- split pipeline (mixed form)
// The same items as batch_far_kernel<true> in two kernels per wave of items:
// batch_moments_kernel evaluates the moments of every (point, cell) pair of
// an item and writes them to an HBM buffer laid out as the fused kernel's
// shared-memory chunk (cell, moment, point); batch_contract_kernel reads them
// back a 16-cell chunk at a time and runs phase B unchanged. The moments
// kernel holds no phase-B state, so it runs at more resident warps; the cell
// pairing of the two-cell node loop (cells c, c + 4 of each 8) and the 16-cell
// FP32 summation boundaries are the fused kernel's, so the results are
// bit-identical to it. Only for n_start <= 8.
#ifndef BIELCC_MOM_MINB
#define BIELCC_MOM_MINB 4
#endif
constexpr int kMomCells = 8;                     // cells per moments block
constexpr int kMomBlock = kMomCells * 20 * kBP;  // floats per block

__global__ void __launch_bounds__(kBT, BIELCC_MOM_MINB)
    batch_moments_kernel(const JobDev* __restrict__ jobs, const BatchItem* __restrict__ items, int n_items,
                         int* __restrict__ counter, double analytic_calc, int n_start, int max_items,
                         float* __restrict__ mom) {
    __shared__ __align__(16) float4 s_nodes[kMomCells * 64];
    __shared__ float s_yy[kMomCells * 64];
    __shared__ double4 s_cell[kMomCells];
    __shared__ double s_rho[kMomCells];
    __shared__ unsigned char s_near[kMomCells * kBP];
    __shared__ int s_item;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nn = n_start * n_start;

    for (int taken = 0; taken < max_items; taken++) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const BatchItem bi = items[it];
        const JobDev& jb = jobs[bi.job];
        const int P = jb.n_pts, N = jb.n_cells;
        const int p = bi.tile * kBP + lane;
        const bool live = p < P;
        double x[3] = {0., 0., 0.};
        if (live)
            for (int g = 0; g < 3; g++) x[g] = jb.pts[3 * (size_t)p + g];
        const int cb = bi.range * jb.cells_per_range;
        const int ce = min(N, cb + jb.cells_per_range);
        const cplx k = jb.k;
        const double k2r = k.re * k.re - k.im * k.im, k2i = 2.0 * k.re * k.im;
        const bool ck = k.im != 0.0;
        float* mo = mom + (size_t)bi.pad * kMomBlock;  // the item's blocks, in cell order
        unsigned nbits = 0;

        for (int c0 = cb; c0 < ce; c0 += kMomCells) {
            const int nc = min(kMomCells, ce - c0);
            __syncthreads();  // the previous chunk's reads of the staged nodes are done
            {
                const float4* src = jb.nodes32 + (size_t)c0 * nn;
                for (int i = threadIdx.x; i < nc * nn; i += kBT) {
                    const float4 v = __ldg(src + i);
                    s_nodes[i] = v;
                    s_yy[i] = node_yy(v);
                }
                for (int i = threadIdx.x; i < nc; i += kBT) {
                    const CellGeo& gg = jb.geo[c0 + i];
                    s_cell[i] = make_double4(gg.c[0], gg.c[1], gg.c[2], gg.diam);
                    s_rho[i] = (double)jb.rho32[c0 + i];
                }
            }
            __syncthreads();
            // cells warp and warp + 4 of the block, two at a time (batch_far_kernel's pairing)
            for (int cc = warp; cc < nc; cc += 2 * kBW) {
                const int cb2 = cc + kBW;
                const bool two = cb2 < nc;
                const double4 ca = s_cell[cc], cbb = s_cell[two ? cb2 : cc];
                const double cena[3] = {ca.x, ca.y, ca.z}, cenb[3] = {cbb.x, cbb.y, cbb.z};
                double da, db;
                const bool na = is_near(x, cena, ca.w, analytic_calc, &da);
                const bool nb = is_near(x, cenb, cbb.w, analytic_calc, &db);
                const bool fa = !na && live, fb = two && !nb && live;
                s_near[cc * kBP + lane] = na ? 1 : 0;
                if (two) s_near[cb2 * kBP + lane] = nb ? 1 : 0;
                float moa[20], mob[20];
#pragma unroll
                for (int q = 0; q < 20; q++) moa[q] = mob[q] = 0.f;
                const float4 *nda = s_nodes + cc * nn, *ndb = s_nodes + (two ? cb2 : cc) * nn;
                const float *ya = s_yy + cc * nn, *yb = s_yy + (two ? cb2 : cc) * nn;
                if (fa && fb) {
                    if (ck) batch_moments2<true>(nda, ya, ndb, yb, nn, x, ca, da, s_rho[cc], cbb, db, s_rho[cb2], k,
                                                 moa, mob);
                    else batch_moments2<false>(nda, ya, ndb, yb, nn, x, ca, da, s_rho[cc], cbb, db, s_rho[cb2], k,
                                               moa, mob);
                } else if (fa || fb) {
                    const float4* nd = fa ? nda : ndb;
                    const float* yy = fa ? ya : yb;
                    const double4 ci = fa ? ca : cbb;
                    const double d = fa ? da : db, rho = s_rho[fa ? cc : cb2];
                    float* mo1 = fa ? moa : mob;
                    if (ck) batch_moments<true, true>(nd, yy, nn, x, ci, d, rho, k, k2r, k2i, mo1);
                    else batch_moments<true, false>(nd, yy, nn, x, ci, d, rho, k, k2r, k2i, mo1);
                }
                float* da_ = mo + (size_t)(c0 - cb + cc) * 20 * kBP + lane;
#pragma unroll
                for (int q = 0; q < 20; q++) da_[q * kBP] = moa[q];
                if (two) {
                    float* db_ = mo + (size_t)(c0 - cb + cb2) * 20 * kBP + lane;
#pragma unroll
                    for (int q = 0; q < 20; q++) db_[q * kBP] = mob[q];
                }
            }
            __syncthreads();
            // near-cell mask: warp 0 owns the words of its points
            if (warp == 0) {
                for (int cc = 0; cc < nc; cc++) {
                    const int c = c0 + cc;
                    nbits |= (unsigned)s_near[cc * kBP + lane] << (c & 31);
                    if ((c & 31) == 31 || c == ce - 1) {
                        if (live) jb.mask[(size_t)(c >> 5) * P + p] = nbits;
                        nbits = 0;
                    }
                }
            }
        }
    }
}

// Bulk prefetch of [p, p + bytes) into L2 (p and bytes multiples of 16; a hint:
// no completion to wait for).
BIELCC_D void prefetch_l2_bulk(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Phase B of the split pipeline: per 16-cell chunk of an item, its moments
// (written by batch_moments_kernel) and the currents are staged and
// contracted exactly as in batch_far_kernel<true>.
// It holds no phase-A state, so it can afford more right-hand sides per thread
// (kConR, staged kConSP at a time) than the fused kernel: each cell's moments
// are loaded from shared memory once per kConR RHS.
constexpr int kConCells = 16;
#ifndef BIELCC_CON_R
#define BIELCC_CON_R 4
#endif
#ifndef BIELCC_CON_MINB
#define BIELCC_CON_MINB 4
#endif
constexpr int kConR = BIELCC_CON_R;
constexpr int kConSP = kBW * kConR * (kSP / (kBW * BatchCfg<true>::R) > 1 ? kSP / (kBW * BatchCfg<true>::R) : 1);
constexpr size_t kConSmem = sizeof(float) * kConCells * 20 * kBP + sizeof(float) * 4 * kConCells * kConSP * 3;

__global__ void __launch_bounds__(kBT, BIELCC_CON_MINB)
    batch_contract_kernel(const JobDev* __restrict__ jobs, const BatchItem* __restrict__ items, int n_items,
                          int* __restrict__ counter, int max_items, const float* __restrict__ mom) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* s_mom = (float*)smem;               // [16][20][kBP]
    float* s_j = s_mom + kConCells * 20 * kBP;  // [16][kConSP][3][4]
    __shared__ int s_item;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int taken = 0; taken < max_items; taken++) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const BatchItem bi = items[it];
        const JobDev& jb = jobs[bi.job];
        const int P = jb.n_pts, N = jb.n_cells, S = jb.n_rhs;
        const int p = bi.tile * kBP + lane;
        const bool live = p < P;
        const int cb = bi.range * jb.cells_per_range;
        const int ce = min(N, cb + jb.cells_per_range);
        const float* mo = mom + (size_t)bi.pad * kMomBlock;

        for (int c0 = cb; c0 < ce; c0 += kConCells) {
            const int nc = min(kConCells, ce - c0);
            __syncthreads();  // the previous chunk's phase B is done with s_mom and s_j
            {
                const float4* src = reinterpret_cast<const float4*>(mo + (size_t)(c0 - cb) * 20 * kBP);
                float4* dst = reinterpret_cast<float4*>(s_mom);
                for (int i = threadIdx.x; i < nc * 20 * kBP / 4; i += kBT) dst[i] = __ldcs(src + i);
            }
            batch_stage_j<true, kConSP>(s_j, jb, c0, nc, 0, min(kConSP, S), threadIdx.x);
            __syncthreads();
            // the next chunk of the item streams from HBM into L2 while this one is contracted
            if (threadIdx.x == 0 && c0 + kConCells < ce) {
                const int nc2 = min(kConCells, ce - c0 - kConCells);
                prefetch_l2_bulk(mo + (size_t)(c0 + kConCells - cb) * 20 * kBP, (unsigned)(nc2 * 20 * kBP * sizeof(float)));
            }
            batch_phase_b<true, kConR, kConSP>(s_mom, s_j, nc, 0, min(kConSP, S), warp, lane, live, jb, bi.range, S,
                                               P, p, c0 == cb);
            // further RHS passes reuse the chunk's moments in shared memory
            for (int s0 = kConSP; s0 < S; s0 += kConSP) {
                __syncthreads();
                batch_stage_j<true, kConSP>(s_j, jb, c0, nc, s0, min(kConSP, S - s0), threadIdx.x);
                __syncthreads();
                batch_phase_b<true, kConR, kConSP>(s_mom, s_j, nc, s0, min(kConSP, S - s0), warp, lane, live, jb,
                                                   bi.range, S, P, p, c0 == cb);
            }
        }
    }
}

// ---------------------------------------------------------------- tensor-core contraction (mixed form)
// batch_far_tc_kernel: the same items, phase A and summation boundaries as
// batch_far_kernel<true>, with the contraction of phase B on the 5th-generation
// tensor cores (tcgen05.mma kind::tf32, accumulators in tensor memory).
//
// Per item (job, 32-point tile, cell range) and chunk of 16 cells, in two
// rounds of 8 cells, warp w evaluates the moments of cell w of the round for
// the tile's 32 points (one point per lane) and writes them into the
// operand A of the round,
//     A[(a, p), (c, b, re|im)] = W_ab(p, c),   a = E x,y,z, H x,y,z;  b = x,y,z,
// with W = A1 I + T for E and the cross-product matrix of G for H
// (K_RotRot_Far = (A1 J + T J)/4pi, R_Rot_Colloc = (G x J)/4pi,
// electrodynamics/K.h:288-301, R.h:89-111). The currents of 16 right-hand
// sides at a time form the operand B, [[Jr, -Ji], [Ji, Jr]] per (cell, b), so
// that D[(a, p), (s, re|im)] = sum_(c, b) W_ab(p, c) J_b(c, s) is one real GEMM
// of M = 192 (two M = 128 MMAs, the second one's last 64 rows unused),
// K = 48 per round and N = 2 S. FP32 operands are split into TF32 hi + lo and
// each product is hi*hi + hi*lo + lo*hi (lo*lo is below the operands' own
// rounding: adding it left the measured error unchanged). D accumulates the chunk's 16 cells in tensor memory (FP32, as the
// CUDA-core form accumulates them in registers) and is then added into the
// job's FP64 partial sums. A chunk's MMAs run while the warps evaluate the next
// round.
//
// A CTA holds two such 8-warp groups, each with its own work item, shared
// memory, named barrier, mbarriers and half of the CTA's 512 tensor-memory
// columns: one CTA per SM, 16 warps, so that one group's barriers and loads
// overlap the other group's moments. (Two 8-warp CTAs of ~110 KB fit one SM
// by registers and shared memory, but measured only one of them was ever
// resident per SM.)
namespace tcb {
constexpr int kGroups = 2;                          // independent 8-warp groups per CTA
constexpr int kGroupThreads = 256;                  // 8 warps
constexpr int kThreads = kGroups * kGroupThreads;   // the CTA
constexpr int kRound = 8;      // cells per round: one per warp
constexpr int kK = 6 * kRound; // K of a round
constexpr int kRows = 192;     // (component, point)
constexpr int kSmax = 64;      // right-hand sides held in tensor memory
constexpr int kG = 16;         // right-hand sides per staged B group
constexpr bool kLoLo = false;  // the lo*lo product too (measured: no change of the error)
constexpr uint32_t kTmemCols = 256, kBlock2Col = 128;   // per group
constexpr uint32_t kTmemAlloc = kGroups * kTmemCols;    // per CTA (all 512 columns of the SM)
constexpr uint32_t kAbytes = kRows * kK * 4;     // one of A hi / A lo
constexpr uint32_t kBbytes = 2 * kG * kK * 4;    // one of B hi / B lo of one buffer
constexpr uint32_t kSbo = (kK / 4) * 128;        // byte distance of 8-row groups
constexpr int kNodes = kRound * 64;              // n_start <= 8
// per group: A hi, A lo, then B (2 buffers x hi, lo): the second M block of A
// lo reads its 64 unused rows from the B buffers, which are larger than that.
constexpr size_t kOffAl = kAbytes, kOffB = 2 * (size_t)kAbytes, kOffNodes = kOffB + 4 * (size_t)kBbytes;
constexpr size_t kOffYY = kOffNodes + 16 * (size_t)kNodes, kOffCell = kOffYY + 4 * (size_t)kNodes;
constexpr size_t kOffRho = kOffCell + 32 * kRound, kOffNear = kOffRho + 8 * kRound;
constexpr size_t kSmemGroup = kOffNear + kRound * 32;
constexpr size_t kGroupStride = (kSmemGroup + 1023) & ~(size_t)1023;
constexpr size_t kSmem = kGroups * kGroupStride;
static_assert(64 * kK * 4 <= 4 * kBbytes, "the unused rows of the second M block must stay inside shared memory");
static_assert(kSmem <= 232448 - 128, "two groups fit the opt-in shared memory of one CTA");
// longest wait for one group of MMAs before the kernel gives up: 2 s of the
// global timer, against microseconds of MMA work
constexpr uint64_t kWaitNs = 2000000000ull;
}  // namespace tcb

BIELCC_D void tc_put2(unsigned char* base, int row, int k, float v0, float v1) {
    *reinterpret_cast<float2*>(base + umma::kmajor_offset(row, k, tcb::kK)) = make_float2(v0, v1);
}

// Writes one (point, cell) block of A: rows a * 32 + lane, K columns
// 6 cl .. 6 cl + 5, hi and lo. m: the 20 moments times e^{ik r0}.
BIELCC_D void tc_write_a(unsigned char* Ah, unsigned char* Al, int lane, int cl, const float* m) {
    float tr[6], ti[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        tr[q] = m[2 + 2 * q];
        ti[q] = m[3 + 2 * q];
    }
    tr[0] += m[0];  // A1 onto the diagonal
    ti[0] += m[1];
    tr[3] += m[0];
    ti[3] += m[1];
    tr[5] += m[0];
    ti[5] += m[1];
    const float gr[3] = {m[14], m[16], m[18]}, gi[3] = {m[15], m[17], m[19]};
    const int ti_[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
    for (int a = 0; a < 6; a++) {
#pragma unroll
        for (int b = 0; b < 3; b++) {
            float wr, wi;
            if (a < 3) {
                wr = tr[ti_[a][b]];
                wi = ti[ti_[a][b]];
            } else {  // H_a = G_(a+1) J_(a+2) - G_(a+2) J_(a+1) (indices mod 3)
                const int h = a - 3, b1 = (h + 1) % 3, b2 = (h + 2) % 3;
                wr = b == b2 ? gr[b1] : (b == b1 ? -gr[b2] : 0.f);
                wi = b == b2 ? gi[b1] : (b == b1 ? -gi[b2] : 0.f);
            }
            float hr, lr, hi, li;
            umma::tf32_split(wr, hr, lr);
            umma::tf32_split(wi, hi, li);
            tc_put2(Ah, a * 32 + lane, 6 * cl + 2 * b, hr, hi);
            tc_put2(Al, a * 32 + lane, 6 * cl + 2 * b, lr, li);
        }
    }
}

// TF32 hi / lo of an FP64 value.
BIELCC_D void tc_split64(double v, float& hi, float& lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"((float)v));
    hi = __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"((float)(v - (double)hi)));
    lo = __uint_as_float(l);
}

// Stages B of right-hand sides s0 .. s0 + 15 for the round's cells (zeros for
// missing cells and right-hand sides): rows 2 s + (re|im of the output).
BIELCC_D void tc_stage_b(unsigned char* Bh, unsigned char* Bl, const JobDev& jb, int c0, int nc, int s0, int gt) {
    for (int i = gt; i < tcb::kRound * tcb::kG * 3; i += tcb::kGroupThreads) {
        const int cl = i / (tcb::kG * 3), rem = i - cl * (tcb::kG * 3), sl = rem / 3, b = rem - sl * 3;
        const int s = s0 + sl;
        cplx v = mk(0., 0.);
        if (cl < nc && s < jb.n_rhs) v = jb.J[((size_t)s * jb.n_cells + (c0 + cl)) * 3 + b];
        float rh, rl, ih, il;
        tc_split64(v.re, rh, rl);
        tc_split64(v.im, ih, il);
        const int k = 6 * cl + 2 * b;
        tc_put2(Bh, 2 * sl, k, rh, -ih);
        tc_put2(Bl, 2 * sl, k, rl, -il);
        tc_put2(Bh, 2 * sl + 1, k, ih, rh);
        tc_put2(Bl, 2 * sl + 1, k, il, rl);
    }
}

// MMAs of one B group into D columns [32 g, 32 g + N) of both M blocks.
BIELCC_D void tc_issue_group(uint32_t tmem, uint32_t sA, uint32_t sAl, uint32_t sBh, uint32_t sBl, int g, int n,
                             bool first_round) {
    const uint32_t id = umma::idesc_tf32(128, n);
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
        const uint32_t d = tmem + blk * tcb::kBlock2Col + 32 * g;
        const uint32_t ao = blk * 16 * tcb::kSbo;  // row 128
#pragma unroll
        for (int ks = 0; ks < tcb::kK / 8; ks++) {
            const uint64_t ah = umma::smem_desc(sA + ao + 256 * ks, 128, tcb::kSbo);
            const uint64_t al = umma::smem_desc(sAl + ao + 256 * ks, 128, tcb::kSbo);
            const uint64_t bh = umma::smem_desc(sBh + 256 * ks, 128, tcb::kSbo);
            const uint64_t bl = umma::smem_desc(sBl + 256 * ks, 128, tcb::kSbo);
            umma::mma_tf32(d, ah, bh, id, !(first_round && ks == 0));
            umma::mma_tf32(d, ah, bl, id, true);
            umma::mma_tf32(d, al, bh, id, true);
            if (tcb::kLoLo) umma::mma_tf32(d, al, bl, id, true);
        }
    }
}

// Barrier of one 8-warp group (named barrier `id`, kGroupThreads threads),
// and the same barrier reducing a predicate with OR over the group.
BIELCC_D void group_sync(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(tcb::kGroupThreads) : "memory");
}
BIELCC_D bool group_or(int id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t"
        ".reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t"
        "}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(tcb::kGroupThreads)
        : "memory");
    return r != 0;
}

// BUF = true: the contraction kernel of the split pipeline with this
// contraction: the moments of each round come from batch_moments_kernel's
// buffer `mom` (read once, streaming) instead of being evaluated here, and the
// near mask is already written.
template <bool BUF>
__global__ void __launch_bounds__(tcb::kThreads, 1)
    batch_far_tc_kernel(const JobDev* __restrict__ jobs, const BatchItem* __restrict__ items, int n_items,
                        int* __restrict__ counter, double analytic_calc, int n_start, int max_items,
                        long long* __restrict__ err, const float* __restrict__ mom) {
    extern __shared__ __align__(128) unsigned char smem_all[];
    const int grp = threadIdx.x / tcb::kGroupThreads;
    const int gt = threadIdx.x - grp * tcb::kGroupThreads;  // thread of the group
    const int bar_id = 1 + grp;                             // named barrier of the group (0: __syncthreads)
    unsigned char* smem = smem_all + grp * tcb::kGroupStride;
    unsigned char* sAh = smem;
    unsigned char* sAl = smem + tcb::kOffAl;
    unsigned char* sB = smem + tcb::kOffB;  // buffer q: hi at 2 q kBbytes, lo at (2 q + 1) kBbytes
    float4* s_nodes = reinterpret_cast<float4*>(smem + tcb::kOffNodes);
    float* s_yy = reinterpret_cast<float*>(smem + tcb::kOffYY);
    double4* s_cell = reinterpret_cast<double4*>(smem + tcb::kOffCell);
    double* s_rho = reinterpret_cast<double*>(smem + tcb::kOffRho);
    unsigned char* s_near = smem + tcb::kOffNear;
    __shared__ uint64_t bars[tcb::kGroups][2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_items[tcb::kGroups];
    uint64_t* bar = bars[grp];
    int& s_item = s_items[grp];

    const int warp = gt >> 5, lane = gt & 31;  // warp of the group; warp % 4 = the SM warp's % 4
    const int nn = n_start * n_start;
    if (threadIdx.x == 0) {
        for (int g = 0; g < tcb::kGroups; g++) {
            umma::mbar_init(&bars[g][0], 1);
            umma::mbar_init(&bars[g][1], 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) {
        umma::tmem_alloc(&s_tmem, tcb::kTmemAlloc);
        umma::tmem_relinquish();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = s_tmem + (uint32_t)grp * tcb::kTmemCols;
    const uint32_t uA = umma::smem_u32(sAh), uAl = umma::smem_u32(sAl), uB = umma::smem_u32(sB);
    // commits in flight per barrier (0 or 1) and the parity of the next phase to wait for
    int inflight[2] = {0, 0};
    uint32_t parity[2] = {0u, 0u};
    bool abort = false;
    // waits for every commit in flight; false on time-out (uniform over the CTA)
    // (a timed-out commit stays recorded as in flight for the final wait)
    auto wait_one_local = [&](int q) -> bool {
        if (!inflight[q]) return true;
        if (!umma::mbar_wait(&bar[q], parity[q], tcb::kWaitNs)) return false;
        parity[q] ^= 1u;
        inflight[q] = 0;
        return true;
    };
    auto wait_all = [&]() -> bool {
        const bool ok0 = wait_one_local(0);
        const bool ok1 = wait_one_local(1);
        return !group_or(bar_id, !(ok0 && ok1));
    };
    auto wait_one = [&](int q) -> bool { return !group_or(bar_id, !wait_one_local(q)); };

    // D of the last chunk, added to the partial sums once its MMAs completed
    bool pend = false, pend_first = false;
    int pend_range = 0;

    for (int taken = 0; taken < max_items && !abort; taken++) {
        group_sync(bar_id);
        if (gt == 0) s_item = atomicAdd(counter, 1);
        group_sync(bar_id);
        const int it = s_item;
        if (it >= n_items) break;
        const BatchItem bi = items[it];
        const JobDev& jb = jobs[bi.job];
        const int P = jb.n_pts, N = jb.n_cells, S = jb.n_rhs;
        const int p = bi.tile * kBP + lane;
        const bool live = p < P;
        double x[3] = {0., 0., 0.};
        if (!BUF && live)
            for (int g = 0; g < 3; g++) x[g] = jb.pts[3 * (size_t)p + g];
        const int cb = bi.range * jb.cells_per_range;
        const int ce = min(N, cb + jb.cells_per_range);
        const cplx k = jb.k;
        const double k2r = k.re * k.re - k.im * k.im, k2i = 2.0 * k.re * k.im;
        const bool ck = k.im != 0.0;
        const float* mo = BUF ? mom + (size_t)bi.pad * kMomBlock : nullptr;
        const int G = (S + tcb::kG - 1) / tcb::kG;
        const int Spad = (S + 7) & ~7;
        unsigned nbits = 0;

        // adds D (the chunk just finished) into the job's partial sums:
        // warps 0-3 hold E x,y,z and H x of their lane's point, warps 4-5 H y, H z
        auto drain = [&]() {
            if (warp < 6) {  // whole warps: tcgen05.ld is warp-collective
                const int a = warp, q = warp & 3;
                const uint32_t col0 = warp < 4 ? 0u : tcb::kBlock2Col;
                for (int g = 0; g < G; g++) {
                    float v[32];
                    umma::tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + col0 + 32 * g, v);
                    if (!live) continue;
                    const int ns = min(tcb::kG, S - g * tcb::kG);
#pragma unroll
                    for (int sl = 0; sl < tcb::kG; sl++) {
                        if (sl >= ns) break;
                        const int s = g * tcb::kG + sl;
                        double* dst = jb.partial + (((size_t)pend_range * S + s) * 12 + 2 * a) * (size_t)P + p;
                        if (pend_first) {
                            dst[0] = (double)v[2 * sl];
                            dst[P] = (double)v[2 * sl + 1];
                        } else {
                            atomicAdd(dst, (double)v[2 * sl]);
                            atomicAdd(dst + P, (double)v[2 * sl + 1]);
                        }
                    }
                }
            }
            umma::fence_before_sync();
            pend = false;
        };

        for (int c0 = cb; c0 < ce && !abort; c0 += 2 * tcb::kRound) {
            for (int r = 0; r < 2 && !abort; r++) {
                const int rc0 = c0 + r * tcb::kRound;
                const int nc = min(tcb::kRound, ce - rc0);
                if (nc <= 0) break;
                if constexpr (!BUF) {
                    group_sync(bar_id);  // the previous round's reads of the staged nodes are done
                    const float4* src = jb.nodes32 + (size_t)rc0 * nn;
                    for (int i = gt; i < nc * nn; i += tcb::kGroupThreads) {
                        const float4 v = __ldg(src + i);
                        s_nodes[i] = v;
                        s_yy[i] = node_yy(v);
                    }
                    for (int i = gt; i < nc; i += tcb::kGroupThreads) {
                        const CellGeo& gg = jb.geo[rc0 + i];
                        s_cell[i] = make_double4(gg.c[0], gg.c[1], gg.c[2], gg.diam);
                        s_rho[i] = (double)jb.rho32[rc0 + i];
                    }
                    group_sync(bar_id);
                }
                // phase A: the moments of cell `warp` of the round for this warp's 32 points
                float mom[20];
#pragma unroll
                for (int q = 0; q < 20; q++) mom[q] = 0.f;
                if constexpr (BUF) {
                    if (warp < nc) {
                        const float* src = mo + (size_t)(rc0 - cb + warp) * 20 * kBP + lane;
#pragma unroll
                        for (int q = 0; q < 20; q++) mom[q] = __ldcs(src + q * kBP);
                    }
                } else if (warp < nc) {
                    const double4 ci = s_cell[warp];
                    const double cen[3] = {ci.x, ci.y, ci.z};
                    double d;
                    const bool nr = is_near(x, cen, ci.w, analytic_calc, &d);
                    s_near[warp * 32 + lane] = nr ? 1 : 0;
                    if (!nr && live) {
                        const float4* nd = s_nodes + warp * nn;
                        const float* yy = s_yy + warp * nn;
                        if (ck) batch_moments<true, true>(nd, yy, nn, x, ci, d, s_rho[warp], k, k2r, k2i, mom);
                        else batch_moments<true, false>(nd, yy, nn, x, ci, d, s_rho[warp], k, k2r, k2i, mom);
                    }
                }
                // A and B are free once the previous round's MMAs completed; D of
                // the previous chunk is added to the partial sums before this
                // chunk's first MMA overwrites it
                if (!wait_all()) {
                    abort = true;
                    break;
                }
                umma::fence_after_sync();
                if (pend) drain();
                tc_write_a(sAh, sAl, lane, warp, mom);
                tc_stage_b(sB, sB + tcb::kBbytes, jb, rc0, nc, 0, gt);
                if (G > 1) tc_stage_b(sB + 2 * tcb::kBbytes, sB + 3 * tcb::kBbytes, jb, rc0, nc, tcb::kG, gt);
                umma::fence_async_smem();
                umma::fence_before_sync();
                group_sync(bar_id);
                umma::fence_after_sync();
                // near-cell mask: warp 0 owns the words of its points
                if (!BUF && warp == 0) {
                    for (int cc = 0; cc < nc; cc++) {
                        const int c = rc0 + cc;
                        nbits |= (unsigned)s_near[cc * 32 + lane] << (c & 31);
                        if ((c & 31) == 31 || c == ce - 1) {
                            if (live) jb.mask[(size_t)(c >> 5) * P + p] = nbits;
                            nbits = 0;
                        }
                    }
                }
                for (int g = 0; g < G && !abort; g++) {
                    const int q = g & 1;
                    if (g >= 2) {  // buffer q is free once group g - 2's MMAs completed
                        if (!wait_one(q)) {
                            abort = true;
                            break;
                        }
                        umma::fence_after_sync();
                        tc_stage_b(sB + 2 * q * tcb::kBbytes, sB + (2 * q + 1) * tcb::kBbytes, jb, rc0, nc,
                                   g * tcb::kG, gt);
                        umma::fence_async_smem();
                        umma::fence_before_sync();
                        group_sync(bar_id);
                        umma::fence_after_sync();
                    }
                    if (gt == 0) {
                        const int n = 2 * min(tcb::kG, Spad - g * tcb::kG);
                        tc_issue_group(tmem, uA, uAl, uB + 2 * q * tcb::kBbytes, uB + (2 * q + 1) * tcb::kBbytes, g, n,
                                       r == 0);
                        umma::mma_commit(&bar[q]);
                    }
                    inflight[q] = 1;
                }
            }
            pend = true;
            pend_first = c0 == cb;
            pend_range = bi.range;
        }
        // the item's last chunk: wait for its MMAs and add D
        if (!abort) {
            if (!wait_all()) abort = true;
            umma::fence_after_sync();
            if (!abort && pend) drain();
        }
    }
    if (abort) {
        if (gt == 0) atomicExch(reinterpret_cast<unsigned long long*>(err), 1ull);
        // MMAs still in flight: wait for them (bounded) before the tensor memory is released
        for (int q = 0; q < 2; q++)
            if (inflight[q]) umma::mbar_wait(&bar[q], parity[q], tcb::kWaitNs);
    }
    // both groups done: the first warp frees the CTA's tensor memory
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::fence_after_sync();
        umma::tmem_dealloc(s_tmem, tcb::kTmemAlloc);
    }
}

// ---------------------------------------------------------------- batched near path + finalize
__global__ void batch_near_count_kernel(const JobDev* __restrict__ jobs, const int* __restrict__ pt_job, int total,
                                        long long* __restrict__ counts) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const JobDev& jb = jobs[pt_job[g]];
    const int p = g - jb.pt_off;
    long long n = 0;
    for (int w = 0; w < jb.n_words; w++) n += __popc(jb.mask[(size_t)w * jb.n_pts + p]);
    counts[g] = n;
}

// Near list of a point in ascending cell order, one warp per point: lane l
// takes a contiguous run of the point's mask words and writes after the lanes
// before it (warp prefix sum of the bit counts).
__global__ void batch_near_fill_kernel(const JobDev* __restrict__ jobs, const int* __restrict__ pt_job, int total,
                                       const long long* __restrict__ offs, int* __restrict__ pair_cell,
                                       int* __restrict__ pair_gpt) {
    const long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= total) return;  // whole warps
    const long long o0 = offs[g];
    if (offs[g + 1] == o0) return;
    const JobDev& jb = jobs[pt_job[g]];
    const int p = (int)(g - jb.pt_off);
    const int run = (jb.n_words + 31) / 32, w0 = min(jb.n_words, lane * run), w1 = min(jb.n_words, w0 + run);
    int cnt = 0;
    for (int w = w0; w < w1; w++) cnt += __popc(jb.mask[(size_t)w * jb.n_pts + p]);
    int incl = cnt;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
    }
    long long o = o0 + (incl - cnt);
    for (int w = w0; w < w1; w++) {
        unsigned b = jb.mask[(size_t)w * jb.n_pts + p];
        while (b) {
            const int bit = __ffs(b) - 1;
            b &= b - 1;
            pair_cell[o] = w * 32 + bit;
            pair_gpt[o] = (int)g;
            o++;
        }
    }
}

__global__ void batch_near_pair_kernel(const JobDev* __restrict__ jobs, const int* __restrict__ pt_job,
                                       const int* __restrict__ pair_cell, const int* __restrict__ pair_gpt,
                                       long long n_pairs, DNP np, cplx* __restrict__ out) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_pairs) return;
    const int g = pair_gpt[q], c = pair_cell[q];
    const JobDev& jb = jobs[pt_job[g]];
    const int p = g - jb.pt_off;
    DCell cl;
    cl.nv = jb.nv;
    for (int v = 0; v < jb.nv; v++)
        for (int a = 0; a < 3; a++) cl.v[v][a] = jb.verts[((size_t)c * jb.nv + v) * 3 + a];
    double x[3] = {jb.pts[3 * (size_t)p], jb.pts[3 * (size_t)p + 1], jb.pts[3 * (size_t)p + 2]};
    near_pair_moments(x, cl, jb.k, np, out + q * 13);
}

// E and H of one (point, RHS): partial sums over the ranges in order, the
// near pairs in cell order, the multiplier and the incident field. Not
// inlined, so the arithmetic is compiled once and the complex64 and
// complex128 outputs round the very same FP64 values.
// Near pairs of a point contracted with its job's currents: one warp per
// point and RHS pass over the job's RHS. Lane l takes the point's pairs l,
// l + 32, ... (cell order) and sums them in order; a fixed xor butterfly
// combines the lanes, so the sum depends only on the point's own pair list.
// Written to the job's partial-sum slot after its cell ranges:
// partial[ranges][s][12][p], already / 4pi.
__global__ void batch_near_sum_kernel(const JobDev* __restrict__ jobs, const int* __restrict__ pt_job, int total,
                                      const long long* __restrict__ offs, const int* __restrict__ pair_cell,
                                      const cplx* __restrict__ moments) {
    const long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= total) return;  // whole warps
    const long long q0 = offs[g], q1 = offs[g + 1];
    if (q0 == q1) return;
    const JobDev& jb = jobs[pt_job[g]];
    const int p = (int)(g - jb.pt_off);
    const size_t P = jb.n_pts;
    for (int s = 0; s < jb.n_rhs; s++) {
        double v[12];
#pragma unroll
        for (int i = 0; i < 12; i++) v[i] = 0.;
        for (long long q = q0 + lane; q < q1; q += 32) {
            const int c = pair_cell[q];
            const cplx* o = moments + q * 13;
            const cplx* j = jb.J + ((size_t)s * jb.n_cells + c) * 3;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const cplx kv = o[0] * j[a] + o[1 + 3 * a] * j[0] + o[2 + 3 * a] * j[1] + o[3 + 3 * a] * j[2];
                v[2 * a] += kv.re;
                v[2 * a + 1] += kv.im;
            }
            cplx h[3];
            ccross_cc(o + 10, j, h);
#pragma unroll
            for (int a = 0; a < 3; a++) {
                v[6 + 2 * a] += h[a].re;
                v[7 + 2 * a] += h[a].im;
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
            jb.partial[(((size_t)jb.ranges * jb.n_rhs + s) * 12 + lane) * P + p] = x;
        }
    }
}

__device__ __noinline__ void finalize_values(const JobDev& jb, int p, int s, bool has_near, double cs, double sn,
                                             const double* kx0, cplx* E, cplx* H) {
    const size_t P = jb.n_pts;
    double v[12];
    for (int q = 0; q < 12; q++) v[q] = 0.;
    for (int r = 0; r < jb.ranges; r++) {
        const double* src = jb.partial + (((size_t)r * jb.n_rhs + s) * 12) * P + p;
        for (int q = 0; q < 12; q++) v[q] += src[(size_t)q * P];
    }
    for (int a = 0; a < 3; a++) {
        E[a] = mk(v[2 * a], v[2 * a + 1]) * kInvFourPi;
        H[a] = mk(v[6 + 2 * a], v[6 + 2 * a + 1]) * kInvFourPi;
    }
    if (has_near) {  // batch_near_sum_kernel's sums
        const double* nv = jb.partial + (((size_t)jb.ranges * jb.n_rhs + s) * 12) * P + p;
        for (int a = 0; a < 3; a++) {
            E[a] += mk(nv[(size_t)(2 * a) * P], nv[(size_t)(2 * a + 1) * P]);
            H[a] += mk(nv[(size_t)(6 + 2 * a) * P], nv[(size_t)(7 + 2 * a) * P]);
        }
    }
    for (int a = 0; a < 3; a++) E[a] = E[a] * jb.mult;
    if (jb.add_E)
        for (int a = 0; a < 3; a++) E[a] += mk(jb.e0[a] * cs, jb.e0[a] * sn);
    if (jb.add_H)
        for (int a = 0; a < 3; a++) H[a] += mk(kx0[a] * cs * jb.h_scale, kx0[a] * sn * jb.h_scale);
}

__global__ void batch_finalize_kernel(const JobDev* __restrict__ jobs, const int* __restrict__ pt_job, int total,
                                      const long long* __restrict__ offs, unsigned long long* nonfinite) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const JobDev& jb = jobs[pt_job[g]];
    const int p = g - jb.pt_off;
    const size_t P = jb.n_pts;
    const double* x = jb.pts + 3 * (size_t)p;
    double cs = 1., sn = 0.;
    if (jb.add_E || jb.add_H) sincos(jb.kvec[0] * x[0] + jb.kvec[1] * x[1] + jb.kvec[2] * x[2], &sn, &cs);
    double kx0[3];
    cross3(jb.kvec, jb.e0, kx0);
    const long long q0 = offs ? offs[g] : 0, q1 = offs ? offs[g + 1] : 0;
    bool bad = false;
    for (int s = 0; s < jb.n_rhs; s++) {
        cplx E[3], H[3];
        finalize_values(jb, p, s, q1 > q0, cs, sn, kx0, E, H);
        for (int a = 0; a < 3; a++) bad |= !isfinite(E[a].re) || !isfinite(E[a].im);
        if (jb.E32) {
            float2* eo = reinterpret_cast<float2*>(jb.E32) + ((size_t)s * P + p) * 3;
            for (int a = 0; a < 3; a++) eo[a] = make_float2((float)E[a].re, (float)E[a].im);
        } else {
            cplx* eo = reinterpret_cast<cplx*>(jb.E) + ((size_t)s * P + p) * 3;
            for (int a = 0; a < 3; a++) eo[a] = E[a];
        }
        if (jb.H || jb.H32) {
            for (int a = 0; a < 3; a++) bad |= !isfinite(H[a].re) || !isfinite(H[a].im);
            if (jb.H32) {
                float2* ho = reinterpret_cast<float2*>(jb.H32) + ((size_t)s * P + p) * 3;
                for (int a = 0; a < 3; a++) ho[a] = make_float2((float)H[a].re, (float)H[a].im);
            } else {
                cplx* ho = reinterpret_cast<cplx*>(jb.H) + ((size_t)s * P + p) * 3;
                for (int a = 0; a < 3; a++) ho[a] = H[a];
            }
        }
    }
    if (bad) {
        if (nonfinite) atomicAdd(nonfinite, 1ull);
        if (jb.nonfinite) atomicAdd(jb.nonfinite, 1ull);
    }
}

// ---------------------------------------------------------------- host side
static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }


int batch_grid(bool mixed, bool tc) {
    // resident CTAs of the persistent grid (dynamic shared memory opted in once)
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (tc) {
        for (const void* f : {(const void*)batch_far_tc_kernel<false>, (const void*)batch_far_tc_kernel<true>}) {
            cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tcb::kSmem);
            cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
        }
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_far_tc_kernel<false>, tcb::kThreads,
                                                          tcb::kSmem) != cudaSuccess) {
            cudaGetLastError();
            per = 1;
        }
        // the same bound from the kernel's registers and shared memory: the
        // occupancy query can assume a smaller carveout than the launch gets
        cudaFuncAttributes fa{};
        int regs_sm = 65536, smem_sm = 0, resv = 0;
        if (cudaFuncGetAttributes(&fa, batch_far_tc_kernel<false>) == cudaSuccess &&
            cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess) {
            const int by_regs = regs_sm / std::max(1, fa.numRegs * tcb::kThreads);
            const int by_smem = smem_sm / (int)(fa.sharedSizeBytes + tcb::kSmem + resv);
            per = std::max(per, std::min(by_regs, by_smem));
        }
        cudaGetLastError();
        // every resident CTA holds kTmemAlloc of the SM's 512 tensor-memory columns
        per = std::min(per, 512 / (int)tcb::kTmemAlloc);
        return sms * std::max(1, per);
    }
    size_t smem = mixed ? BatchCfg<true>::smem_bytes() : BatchCfg<false>::smem_bytes();
    if (mixed) {
        cudaFuncSetAttribute(batch_far_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_far_kernel<true>, kBT, smem);
    } else {
        cudaFuncSetAttribute(batch_far_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_far_kernel<false>, kBT, smem);
    }
    return sms * std::max(1, per);
}

size_t moments_block_bytes() { return (size_t)kMomBlock * sizeof(float); }

// Resident CTAs of the split pipeline's two kernels (dynamic shared memory
// opted in once).
void split_grids(int& grid_mom, int& grid_con) {
    int dev = 0, sms = 148, pm = 1, pc = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(batch_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConSmem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pm, batch_moments_kernel, kBT, 0) != cudaSuccess) pm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pc, batch_contract_kernel, kBT, kConSmem) != cudaSuccess) pc = 1;
    cudaGetLastError();
    grid_mom = sms * std::max(1, pm);
    grid_con = sms * std::max(1, pc);
}

// Cuts every job into items (32-point tile, range of cells). The range length
// depends only on the job itself and on `item_cost` (estimated node
// evaluations per item, a per-context autotuned constant), never on the other
// jobs of the batch, so a job's summation order - and its result - is the same
// alone and in any mix. Ranges are multiples of 32 cells (near-mask words).
int batch_cells_per_range(int n_cells, int n_rhs, int n_start, double item_cost) {
    const double per_cell = (double)kBP * ((double)n_start * n_start + 1.2 * n_rhs);
    // at most kMaxRanges ranges per job: bounds the partial sums to kMaxRanges x (S x 12 x P) doubles
    constexpr int kMaxRanges = 6;
    int cpr = (int)std::min<double>(n_cells, std::max(32.0, item_cost / per_cell));
    cpr = std::max(cpr, (n_cells + kMaxRanges - 1) / kMaxRanges);
    return (cpr + 31) / 32 * 32;
}

void plan_batch(BatchPlan& bp, const std::vector<JobDev>& jobs_in, int n_start, bool mixed, double item_cost,
                bool allow_tc, size_t split_cap) {
    bp.jobs = jobs_in;
    bp.mixed = mixed;
    bp.tc = mixed && allow_tc && n_start <= 8;
    for (const JobDev& j : jobs_in) bp.tc = bp.tc && j.n_rhs <= tcb::kSmax;
    bp.grid = batch_grid(mixed, bp.tc);
    bp.per_cta = bp.tc ? tcb::kGroups : 1;
    const double nodes = (double)n_start * n_start;
    bp.items.clear();
    bp.pt_job.clear();
    std::vector<double> cost;
    int pt_off = 0;
    for (size_t ji = 0; ji < bp.jobs.size(); ji++) {
        JobDev& j = bp.jobs[ji];
        j.pt_off = pt_off;
        pt_off += j.n_pts;
        for (int p = 0; p < j.n_pts; p++) bp.pt_job.push_back((int)ji);
        const double per_cell = (double)kBP * (nodes + 1.2 * j.n_rhs);
        const int cpr = batch_cells_per_range(j.n_cells, j.n_rhs, n_start, item_cost);
        j.cells_per_range = cpr;
        j.ranges = (j.n_cells + cpr - 1) / cpr;
        j.n_words = (j.n_cells + 31) / 32;
        const int tiles = (j.n_pts + kBP - 1) / kBP;
        for (int t = 0; t < tiles; t++)
            for (int r = 0; r < j.ranges; r++) {
                bp.items.push_back(BatchItem{(int)ji, t, r, 0});
                const int cells = std::min(cpr, j.n_cells - r * cpr);
                cost.push_back((double)cells * per_cell);
            }
        bp.ws_bytes += al256((size_t)(j.ranges + 1) * j.n_rhs * 12 * j.n_pts * sizeof(double)) +
                       al256((size_t)j.n_words * j.n_pts * sizeof(unsigned));
    }
    bp.total_pts = pt_off;
    std::vector<int> order(bp.items.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<BatchItem> sorted(bp.items.size());
    for (size_t i = 0; i < order.size(); i++) sorted[i] = bp.items[order[i]];
    bp.items.swap(sorted);
    const size_t T = bp.total_pts;
    bp.ws_bytes += al256(bp.jobs.size() * sizeof(JobDev)) + al256(bp.items.size() * sizeof(BatchItem)) +
                   al256(T * sizeof(int)) + 2 * al256((T + 1) * sizeof(long long)) + 3 * 256;
    // split pipeline: waves of consecutive (sorted) items whose moments fit the buffer
    bp.split = mixed && n_start <= 8 && split_cap > 0 && !bp.items.empty();
    bp.waves.clear();
    bp.mom_blocks = 0;
    if (bp.split) {
        const size_t cap = std::max<size_t>(1, split_cap / (kMomBlock * sizeof(float)));
        size_t used = 0;
        int w0 = 0;
        for (size_t i = 0; i < bp.items.size(); i++) {
            BatchItem& it = bp.items[i];
            const JobDev& j = bp.jobs[it.job];
            const int cells = std::min(j.cells_per_range, j.n_cells - it.range * j.cells_per_range);
            const size_t blocks = (size_t)(cells + kMomCells - 1) / kMomCells;
            if (used + blocks > cap && (int)i > w0) {
                bp.waves.emplace_back(w0, (int)i);
                w0 = (int)i;
                used = 0;
            }
            it.pad = (int)used;
            used += blocks;
            bp.mom_blocks = std::max(bp.mom_blocks, used);
        }
        bp.waves.emplace_back(w0, (int)bp.items.size());
        bp.ws_bytes += al256(bp.mom_blocks * kMomBlock * sizeof(float)) + al256(2 * bp.waves.size() * sizeof(int));
        split_grids(bp.grid_mom, bp.grid_con);
        if (bp.tc) bp.grid_con = bp.grid;  // the tensor-core contraction: one CTA of two groups per SM
        // the moments kernel sets the pace: planning counts its CTAs
        bp.grid = bp.grid_mom;
        bp.per_cta = 1;
    }
}

void batch_make_preemptible(BatchPlan& bp) {
    bp.max_items = 1;
    const size_t ctas = (bp.items.size() + bp.per_cta - 1) / bp.per_cta;
    bp.grid = std::max<int>(1, (int)std::min<size_t>(ctas, (size_t)INT32_MAX));
}

// The far-field launches of a planned batch: the fused kernel (or its
// tensor-core form), or per wave the moments kernel (when `moments`) and the
// contraction kernel. Resets the work counters first.
static cudaError_t launch_far(BatchPlan& bp, const BatchDevPtrs& d, double analytic_calc, int n_start, bool moments,
                       cudaStream_t s, int* launches) {
    *launches = 0;
    cudaError_t e = cudaMemsetAsync(d.counter, 0, sizeof(int), s);
    if (e == cudaSuccess && bp.split) e = cudaMemsetAsync(d.wave_counters, 0, 2 * bp.waves.size() * sizeof(int), s);
    if (e != cudaSuccess) return e;
    const int n_items = (int)bp.items.size();
    if (n_items == 0) return cudaSuccess;
    if (bp.split) {
        for (size_t w = 0; w < bp.waves.size(); w++) {
            const int b = bp.waves[w].first, n = bp.waves[w].second - bp.waves[w].first;
            const int gm = bp.max_items == 1 ? n : std::min(bp.grid_mom, n);
            const int gc = bp.max_items == 1 ? (bp.tc ? (n + tcb::kGroups - 1) / tcb::kGroups : n)
                                             : std::min(bp.grid_con, n);
            if (moments) {
                batch_moments_kernel<<<gm, kBT, 0, s>>>(d.jobs, d.items + b, n, d.wave_counters + 2 * w,
                                                        analytic_calc, n_start, bp.max_items, d.mom);
                *launches += 1;
            }
            if (bp.tc)
                batch_far_tc_kernel<true><<<gc, tcb::kThreads, tcb::kSmem, s>>>(
                    d.jobs, d.items + b, n, d.wave_counters + 2 * w + 1, analytic_calc, n_start, bp.max_items, d.err,
                    d.mom);
            else
                batch_contract_kernel<<<gc, kBT, kConSmem, s>>>(d.jobs, d.items + b, n, d.wave_counters + 2 * w + 1,
                                                                 bp.max_items, d.mom);
            *launches += 1;
        }
        return cudaGetLastError();
    }
    const size_t smem = bp.mixed ? BatchCfg<true>::smem_bytes() : BatchCfg<false>::smem_bytes();
    if (bp.tc)
        batch_far_tc_kernel<false><<<bp.grid, tcb::kThreads, tcb::kSmem, s>>>(
            d.jobs, d.items, n_items, d.counter, analytic_calc, n_start, bp.max_items, d.err, nullptr);
    else if (bp.mixed)
        batch_far_kernel<true><<<bp.grid, kBT, smem, s>>>(d.jobs, d.items, n_items, d.counter, analytic_calc, n_start,
                                                         bp.max_items);
    else
        batch_far_kernel<false><<<bp.grid, kBT, smem, s>>>(d.jobs, d.items, n_items, d.counter, analytic_calc,
                                                          n_start, bp.max_items);
    *launches = 1;
    return cudaGetLastError();
}

// Enqueues stage 1 (far kernel, near counting, scan) of a planned batch into
// `ws`; `host_tables` receive the device table pointers for stage 2.

cudaError_t batch_stage1(BatchPlan& bp, void* ws, double analytic_calc, int n_start, bool ck, cudaStream_t s,
                         BatchDevPtrs* out, int* launches) {
    char* w = (char*)ws;
    for (auto& j : bp.jobs) {
        j.partial = (double*)w;
        w += al256((size_t)(j.ranges + 1) * j.n_rhs * 12 * j.n_pts * sizeof(double));  // + the near sums
        j.mask = (unsigned*)w;
        w += al256((size_t)j.n_words * j.n_pts * sizeof(unsigned));
    }
    const size_t T = bp.total_pts;
    BatchDevPtrs d;
    d.jobs = (JobDev*)w;
    w += al256(bp.jobs.size() * sizeof(JobDev));
    d.items = (BatchItem*)w;
    w += al256(bp.items.size() * sizeof(BatchItem));
    d.pt_job = (int*)w;
    w += al256(T * sizeof(int));
    d.counts = (long long*)w;
    w += al256((T + 1) * sizeof(long long));
    d.offs = (long long*)w;
    w += al256((T + 1) * sizeof(long long));
    d.total = (long long*)w;
    d.err = d.total + 1;
    w += 256;
    d.counter = (int*)w;
    w += 256;
    if (bp.split) {
        d.mom = (float*)w;
        w += al256(bp.mom_blocks * kMomBlock * sizeof(float));
        d.wave_counters = (int*)w;
    }
    cudaError_t e = cudaMemcpyAsync(d.jobs, bp.jobs.data(), bp.jobs.size() * sizeof(JobDev), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !bp.items.empty())
        e = cudaMemcpyAsync(d.items, bp.items.data(), bp.items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && T) e = cudaMemcpyAsync(d.pt_job, bp.pt_job.data(), T * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.total, 0, 2 * sizeof(long long), s);
    if (e != cudaSuccess) return e;
    int lf = 0;
    e = launch_far(bp, d, analytic_calc, n_start, true, s, &lf);
    if (e != cudaSuccess) return e;
    const int tb = (int)((T + 127) / 128);
    if (T) batch_near_count_kernel<<<tb, 128, 0, s>>>(d.jobs, d.pt_job, (int)T, d.counts);
    scan_kernel<<<1, 1024, 0, s>>>(d.counts, (int)T, d.offs, d.total);
    *out = d;
    *launches = lf + (T ? 1 : 0) + 1;
    return cudaGetLastError();
}

cudaError_t batch_status_to_host(const BatchDevPtrs& d, long long* h, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(h, d.total, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h + 3, d.err, sizeof(long long), cudaMemcpyDeviceToHost, s);
    return e;
}

size_t batch_pair_ws_bytes(long long n_near) {
    return al256((size_t)n_near * 13 * sizeof(cplx)) + 2 * al256((size_t)n_near * sizeof(int));
}

cudaError_t batch_stage2(BatchPlan& bp, const BatchDevPtrs& d, long long n_near, void* pair_ws, const DNP& np,
                         unsigned long long* d_nonfinite, cudaStream_t s, int* launches) {
    const size_t T = bp.total_pts;
    const int tb = (int)((T + 127) / 128);
    cplx* moments = nullptr;
    int* pair_cell = nullptr;
    *launches = 0;
    if (n_near > 0) {
        char* pw = (char*)pair_ws;
        moments = (cplx*)pw;
        pw += al256((size_t)n_near * 13 * sizeof(cplx));
        pair_cell = (int*)pw;
        pw += al256((size_t)n_near * sizeof(int));
        int* pair_gpt = (int*)pw;
        batch_near_fill_kernel<<<(int)((T + 7) / 8), 256, 0, s>>>(d.jobs, d.pt_job, (int)T, d.offs, pair_cell,
                                                                  pair_gpt);
        batch_near_pair_kernel<<<(int)((n_near + 127) / 128), 128, 0, s>>>(d.jobs, d.pt_job, pair_cell, pair_gpt,
                                                                          n_near, np, moments);
        batch_near_sum_kernel<<<(int)((T + 7) / 8), 256, 0, s>>>(d.jobs, d.pt_job, (int)T, d.offs, pair_cell,
                                                                moments);
        *launches += 3;
    }
    if (T) {
        batch_finalize_kernel<<<tb, 128, 0, s>>>(d.jobs, d.pt_job, (int)T, n_near > 0 ? d.offs : nullptr,
                                                  d_nonfinite);
        *launches += 1;
    }
    return cudaGetLastError();
}

// The launch sequence of a repeated evaluation with fixed geometry: reset the
// work queue, far kernel, finalize with the near-pair list and FP64 near-pair
// moments that stage 2 left in pair_ws (they depend on geometry and k, not on
// the currents). Captured once into a CUDA graph by bielcc_batch_plan_create.
cudaError_t batch_replay(BatchPlan& bp, const BatchDevPtrs& d, long long n_near, void* pair_ws, double analytic_calc,
                         int n_start, cudaStream_t s) {
    const size_t T = bp.total_pts;
    // one wave: the moments left in the buffer by the first evaluation depend
    // on geometry, points and k only, so the replay contracts them again
    int lf = 0;
    cudaError_t e = launch_far(bp, d, analytic_calc, n_start, !(bp.split && bp.waves.size() == 1), s, &lf);
    if (e != cudaSuccess) return e;
    if (T) {
        const cplx* moments = nullptr;
        const int* pair_cell = nullptr;
        if (n_near > 0) {  // the near sums depend on the currents: recomputed every replay
            moments = (const cplx*)pair_ws;
            pair_cell = (const int*)((const char*)pair_ws + al256((size_t)n_near * 13 * sizeof(cplx)));
            batch_near_sum_kernel<<<(int)((T + 7) / 8), 256, 0, s>>>(d.jobs, d.pt_job, (int)T, d.offs, pair_cell,
                                                                    moments);
        }
        batch_finalize_kernel<<<(int)((T + 127) / 128), 128, 0, s>>>(d.jobs, d.pt_job, (int)T,
                                                                      n_near > 0 ? d.offs : nullptr, nullptr);
    }
    return cudaGetLastError();
}

}  // namespace bielcc_gpu
