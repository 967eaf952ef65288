// pairops.cu — batched per-pair kernels behind the drop-in operator calls:
// one thread evaluates one reference call (K_RotRot_*, R_Rot_*, K0,
// IntegralUniversalPnt, IntegralUniversalSegPnt, the analytic integrals) for
// one (cell, x[, j]) triple, FP64, with the reference's adaptive quadrature;
// the x-free IntegralUniversal / segment F(x) forms run through the same
// kernels with no point.
#include "internal.h"
#include "ops.cuh"

namespace bielcc_gpu {

BIELCC_D void load_cell(DCell& c, const double* cells, int nv, int q) {
    c.nv = nv;
    for (int v = 0; v < nv; v++)
        for (int g = 0; g < 3; g++) c.v[v][g] = cells[((size_t)q * nv + v) * 3 + g];
}

BIELCC_D void load_kp(DKP& p, const KParamDev& s) {
    p.smoothR = s.smoothR;
    p.smoothRMin = s.smoothRMin;
    p.k = mk(s.k_re, s.k_im);
    for (int i = 0; i < 3; i++) {
        p.current[i] = mk(s.current[i][0], s.current[i][1]);
        p.vec_dbl[i] = s.vec_dbl[i];
        p.n[i] = s.n[i];
        p.e0[i] = s.e0[i];
    }
}

__global__ void pair_op_kernel(int op, int nv, int n, const double* __restrict__ cells, const double* __restrict__ x,
                               const cplx* __restrict__ j, cplx k, DNP np, cplx* __restrict__ res) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    DCell c;
    load_cell(c, cells, nv, q);
    double xp[3] = {x[3 * (size_t)q], x[3 * (size_t)q + 1], x[3 * (size_t)q + 2]};
    cplx jj[3] = {j[3 * (size_t)q], j[3 * (size_t)q + 1], j[3 * (size_t)q + 2]};
    cplx r[3];
    run_pair_op(op, jj, xp, c, np, k, r);
    for (int g = 0; g < 3; g++) res[3 * (size_t)q + g] = r[g];
}

__global__ void integral_pnt_kernel(int id, int nv, int n, const double* __restrict__ cells,
                                    const double* __restrict__ x, KParamDev* __restrict__ kp, int n_start,
                                    int p_max, double eps, double* __restrict__ res) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    DCell c;
    load_cell(c, cells, nv, q);
    DKP p;
    load_kp(p, kp[q]);
    // x == nullptr: IntegralUniversal, the F(x) form (the integrand reads the node only)
    double xp[3] = {0., 0., 0.};
    if (x)
        for (int g = 0; g < 3; g++) xp[g] = x[3 * (size_t)q + g];
    int idim = integrand_dim(id);
    if (integrand_complex(id)) {
        cplx r[3];
        integral_cell<cplx>(id, xp, c, p, idim, n_start, p_max, eps, r);
        for (int g = 0; g < idim; g++) reinterpret_cast<cplx*>(res)[(size_t)idim * q + g] = r[g];
    } else {
        double r[3];
        integral_cell<double>(id, xp, c, p, idim, n_start, p_max, eps, r);
        for (int g = 0; g < idim; g++) res[(size_t)idim * q + g] = r[g];
    }
    kp[q].smoothR = p.smoothR;  // the reference mutates its KernelParam
}

__global__ void integral_seg_kernel(int id, int n, const double* __restrict__ a, const double* __restrict__ b,
                                    const double* __restrict__ x, KParamDev* __restrict__ kp, int n_start,
                                    int p_max, double eps, double* __restrict__ res) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    DKP p;
    load_kp(p, kp[q]);
    size_t o = 3 * (size_t)q;
    double A[3] = {a[o], a[o + 1], a[o + 2]}, B[3] = {b[o], b[o + 1], b[o + 2]}, X[3] = {0., 0., 0.};
    if (x)  // x == nullptr: the segment F(x) overload
        for (int g = 0; g < 3; g++) X[g] = x[o + g];
    int idim = integrand_dim(id);
    if (integrand_complex(id)) {
        cplx r[3];
        integral_seg<cplx>(id, A, B, X, p, idim, n_start, p_max, eps, r);
        for (int g = 0; g < idim; g++) reinterpret_cast<cplx*>(res)[(size_t)idim * q + g] = r[g];
    } else {
        double r[3];
        integral_seg<double>(id, A, B, X, p, idim, n_start, p_max, eps, r);
        for (int g = 0; g < idim; g++) res[(size_t)idim * q + g] = r[g];
    }
    kp[q].smoothR = p.smoothR;
}

__global__ void k0_kernel(int id, int common, int nv, int n, const double* __restrict__ cells,
                          const double* __restrict__ x, const cplx* __restrict__ j, KParamDev* __restrict__ kp,
                          int n_seg, int p_seg, double eps, cplx* __restrict__ res) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    DCell c;
    load_cell(c, cells, nv, q);
    DKP p;
    load_kp(p, kp[q]);
    double xp[3] = {x[3 * (size_t)q], x[3 * (size_t)q + 1], x[3 * (size_t)q + 2]};
    cplx r[3];
    if (common) {
        K0_common_dev(id, xp, c, p, n_seg, p_seg, eps, r);
    } else {
        cplx jj[3] = {j[3 * (size_t)q], j[3 * (size_t)q + 1], j[3 * (size_t)q + 2]};
        K0_dev(id, jj, xp, c, p, n_seg, p_seg, eps, r);
    }
    for (int g = 0; g < 3; g++) res[3 * (size_t)q + g] = r[g];
    kp[q].smoothR = p.smoothR;
}

// which: 0 integral1Divr, 1 integralGrad1DivrSeg, 2 IntegralSurf_SimplePot_H_HS,
//        3 IntegralSeg_GradSimplePot_H_HS
__global__ void analytic_kernel(int which, int nv, int n, const double* __restrict__ ca, const double* __restrict__ b,
                                const double* __restrict__ x, double analytic_r, int n_start, int p_max, double eps,
                                cplx k, double* __restrict__ res) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    size_t o = 3 * (size_t)q;
    double X[3] = {x[o], x[o + 1], x[o + 2]};
    if (which == 0 || which == 2) {
        DCell c;
        load_cell(c, ca, nv, q);
        if (which == 0) {
            res[q] = integral_1divr_dev(c, X);
        } else {
            reinterpret_cast<cplx*>(res)[q] = surf_simplepot_h_hs_dev(c, X, analytic_r, n_start, p_max, eps, k);
        }
    } else {
        double A[3] = {ca[o], ca[o + 1], ca[o + 2]}, B[3] = {b[o], b[o + 1], b[o + 2]};
        if (which == 1) {
            grad_1divr_seg_dev(A, B, X, res + o);
        } else {
            cplx r[3];
            seg_gradsimplepot_h_hs_dev(A, B, X, analytic_r, n_start, p_max, eps, k, r);
            for (int g = 0; g < 3; g++) reinterpret_cast<cplx*>(res)[o + g] = r[g];
        }
    }
}

static inline int blocks_for(int n) { return (n + 127) / 128; }

cudaError_t launch_pair_op(int op, int nv, int n, const double* cells, const double* x, const double* j, cplx k,
                           NumParamH np, double* res, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    DNP d{np.eps, np.rs, np.rs_seg, np.analytic_calc, np.n_start, np.n_start_seg, np.p_max, np.p_max_seg};
    pair_op_kernel<<<blocks_for(n), 128, 0, s>>>(op, nv, n, cells, x, reinterpret_cast<const cplx*>(j), k, d,
                                                 reinterpret_cast<cplx*>(res));
    return cudaGetLastError();
}

cudaError_t launch_integral_pnt(int integrand, int nv, int n, const double* cells, const double* x,
                                KParamDev* kp, int n_start, int p_max, double eps, double* res, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    integral_pnt_kernel<<<blocks_for(n), 128, 0, s>>>(integrand, nv, n, cells, x, kp, n_start, p_max, eps, res);
    return cudaGetLastError();
}

cudaError_t launch_integral_seg(int integrand, int n, const double* a, const double* b, const double* x,
                                KParamDev* kp, int n_start, int p_max, double eps, double* res, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    integral_seg_kernel<<<blocks_for(n), 128, 0, s>>>(integrand, n, a, b, x, kp, n_start, p_max, eps, res);
    return cudaGetLastError();
}

cudaError_t launch_k0(int integrand, int common, int nv, int n, const double* cells, const double* x, const double* j,
                      KParamDev* kp, int n_seg, int p_seg, double eps, double* res, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k0_kernel<<<blocks_for(n), 128, 0, s>>>(integrand, common, nv, n, cells, x, reinterpret_cast<const cplx*>(j), kp,
                                            n_seg, p_seg, eps, reinterpret_cast<cplx*>(res));
    return cudaGetLastError();
}

cudaError_t launch_analytic(int which, int nv, int n, const double* cells_or_a, const double* b, const double* x,
                            double analytic_r, int n_start, int p_max, double eps, cplx k, double* res, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    analytic_kernel<<<blocks_for(n), 128, 0, s>>>(which, nv, n, cells_or_a, b, x, analytic_r, n_start, p_max, eps, k,
                                                  res);
    return cudaGetLastError();
}

}  // namespace bielcc_gpu
