// solve.cu — the step after assembly: the collocation system of a perfectly
// conducting body, A x = b, and the currents it gives.
//   * A: the TAU2 matrix of bielcc_assemble_K (rows (i, a), columns (j, b),
//     A = tau_a(i) . K[tau_b(j)](c_i)); x: the coefficients of the currents in
//     the cells' tangent bases, J_j = x_{2j} tau1(j) + x_{2j+1} tau2(j)
//     (SurfaceCurrents_byBasis, electrodynamics/currents.h:22-33);
//   * b: the boundary condition n x (E_inc + multE K[J]) = 0 at the collocation
//     points in the tangent basis: b_(i,a) = -tau_a(i) . E_inc(c_i) / multE.
// The dense LU (getrf / getrs) is cuSOLVER's, loaded with dlopen at the first
// solve so that the library itself does not depend on it.
#include <dlfcn.h>

#include <cusolverDn.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/bielcc_gpu.h"
#include "internal.h"

namespace bielcc_gpu {

namespace {

struct Cusolver {
    bool tried = false, ok = false;
    std::string err;
    decltype(&cusolverDnCreate) create = nullptr;
    decltype(&cusolverDnDestroy) destroy = nullptr;
    decltype(&cusolverDnSetStream) set_stream = nullptr;
    decltype(&cusolverDnCgetrf_bufferSize) cbuf = nullptr;
    decltype(&cusolverDnCgetrf) cgetrf = nullptr;
    decltype(&cusolverDnCgetrs) cgetrs = nullptr;
    decltype(&cusolverDnZgetrf_bufferSize) zbuf = nullptr;
    decltype(&cusolverDnZgetrf) zgetrf = nullptr;
    decltype(&cusolverDnZgetrs) zgetrs = nullptr;
};

Cusolver& cusolver() {
    static Cusolver c;
    static std::mutex mu;
    std::lock_guard<std::mutex> g(mu);
    if (c.tried) return c;
    c.tried = true;
    void* h = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libcusolver.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        const char* e = dlerror();
        c.err = e ? e : "libcusolver not found";
        return c;
    }
#define BIELCC_SYM(field, name) c.field = reinterpret_cast<decltype(c.field)>(dlsym(h, #name))
    BIELCC_SYM(create, cusolverDnCreate);
    BIELCC_SYM(destroy, cusolverDnDestroy);
    BIELCC_SYM(set_stream, cusolverDnSetStream);
    BIELCC_SYM(cbuf, cusolverDnCgetrf_bufferSize);
    BIELCC_SYM(cgetrf, cusolverDnCgetrf);
    BIELCC_SYM(cgetrs, cusolverDnCgetrs);
    BIELCC_SYM(zbuf, cusolverDnZgetrf_bufferSize);
    BIELCC_SYM(zgetrf, cusolverDnZgetrf);
    BIELCC_SYM(zgetrs, cusolverDnZgetrs);
#undef BIELCC_SYM
    c.ok = c.create && c.destroy && c.set_stream && c.cbuf && c.cgetrf && c.cgetrs && c.zbuf && c.zgetrf && c.zgetrs;
    if (!c.ok) c.err = "libcusolver lacks a getrf / getrs entry point";
    return c;
}

template <typename T>
__global__ void efie_rhs_kernel(const CellGeo* __restrict__ geo, int n, double3 kvec, double3 e0, cplx scale,
                                T* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CellGeo& g = geo[i];
    double s, c;
    sincos(kvec.x * g.c[0] + kvec.y * g.c[1] + kvec.z * g.c[2], &s, &c);
    const double t1 = g.t1[0] * e0.x + g.t1[1] * e0.y + g.t1[2] * e0.z;
    const double t2 = g.t2[0] * e0.x + g.t2[1] * e0.y + g.t2[2] * e0.z;
    const cplx ph = mk(c, s) * scale;
    const cplx v1 = ph * t1, v2 = ph * t2;
    if constexpr (sizeof(T) == 8) {
        b[2 * i] = T{(float)v1.re, (float)v1.im};
        b[2 * i + 1] = T{(float)v2.re, (float)v2.im};
    } else {
        b[2 * i] = T{v1.re, v1.im};
        b[2 * i + 1] = T{v2.re, v2.im};
    }
}

template <typename T>
__global__ void basis_currents_kernel(const CellGeo* __restrict__ geo, int n, const T* __restrict__ x,
                                      cplx* __restrict__ J) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CellGeo& g = geo[i];
    const cplx x1 = mk((double)x[2 * i].x, (double)x[2 * i].y), x2 = mk((double)x[2 * i + 1].x, (double)x[2 * i + 1].y);
    for (int a = 0; a < 3; a++) J[3 * (size_t)i + a] = x1 * g.t1[a] + x2 * g.t2[a];
}

}  // namespace

cudaError_t launch_efie_rhs(const CellGeo* geo, int n, const double* kvec, const double* e0, cplx scale, int c64,
                            void* b, cudaStream_t s) {
    const double3 kv = make_double3(kvec[0], kvec[1], kvec[2]), ev = make_double3(e0[0], e0[1], e0[2]);
    if (n == 0) return cudaSuccess;
    if (c64) efie_rhs_kernel<float2><<<(n + 127) / 128, 128, 0, s>>>(geo, n, kv, ev, scale, (float2*)b);
    else efie_rhs_kernel<double2><<<(n + 127) / 128, 128, 0, s>>>(geo, n, kv, ev, scale, (double2*)b);
    return cudaGetLastError();
}

cudaError_t launch_basis_currents(const CellGeo* geo, int n, const void* x, int c64, double* J, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (c64) basis_currents_kernel<float2><<<(n + 127) / 128, 128, 0, s>>>(geo, n, (const float2*)x, (cplx*)J);
    else basis_currents_kernel<double2><<<(n + 127) / 128, 128, 0, s>>>(geo, n, (const double2*)x, (cplx*)J);
    return cudaGetLastError();
}

}  // namespace bielcc_gpu

using namespace bielcc_gpu;

extern "C" int bielcc_solve_dense(int n, int nrhs, int c64, void* A_dev, void* B_dev, void* stream, int* info) {
    if (n < 1 || nrhs < 1 || !A_dev || !B_dev) return set_api_error(BIELCC_ERR_ARG, "solve_dense: bad arguments");
    if ((long long)n * n >= (1ll << 31))
        return set_api_error(BIELCC_ERR_UNSUPPORTED, "solve_dense: n^2 must stay below 2^31 (32-bit LU interface)");
    Cusolver& cs = cusolver();
    if (!cs.ok) return set_api_error(BIELCC_ERR_UNSUPPORTED, ("cuSOLVER unavailable: " + cs.err).c_str());
    cudaStream_t s = (cudaStream_t)stream;
    cusolverDnHandle_t h = nullptr;
    if (cs.create(&h) != CUSOLVER_STATUS_SUCCESS) return set_api_error(BIELCC_ERR_CUDA, "cusolverDnCreate failed");
    int rc = BIELCC_OK;
    int lwork = 0;
    void* work = nullptr;
    int* ipiv = nullptr;
    int* dinfo = nullptr;
    // A is row-major: cuSOLVER (column-major) sees A^T. Factor A^T, then solve
    // with the transpose (not conjugate) operation to get A x = b.
    cusolverStatus_t st = cs.set_stream(h, s);
    if (st == CUSOLVER_STATUS_SUCCESS)
        st = c64 ? cs.cbuf(h, n, n, (cuComplex*)A_dev, n, &lwork) : cs.zbuf(h, n, n, (cuDoubleComplex*)A_dev, n, &lwork);
    if (st != CUSOLVER_STATUS_SUCCESS) rc = set_api_error(BIELCC_ERR_CUDA, "getrf workspace query failed");
    const size_t elt = c64 ? sizeof(cuComplex) : sizeof(cuDoubleComplex);
    if (rc == BIELCC_OK && (cudaMalloc(&work, (size_t)std::max(lwork, 1) * elt) != cudaSuccess ||
                            cudaMalloc((void**)&ipiv, (size_t)n * sizeof(int)) != cudaSuccess ||
                            cudaMalloc((void**)&dinfo, 2 * sizeof(int)) != cudaSuccess)) {
        cudaGetLastError();
        rc = set_api_error(BIELCC_ERR_OOM, "solve_dense: workspace allocation failed");
    }
    if (rc == BIELCC_OK) {
        if (c64) {
            st = cs.cgetrf(h, n, n, (cuComplex*)A_dev, n, (cuComplex*)work, ipiv, dinfo);
            if (st == CUSOLVER_STATUS_SUCCESS)
                st = cs.cgetrs(h, CUBLAS_OP_T, n, nrhs, (const cuComplex*)A_dev, n, ipiv, (cuComplex*)B_dev, n, dinfo + 1);
        } else {
            st = cs.zgetrf(h, n, n, (cuDoubleComplex*)A_dev, n, (cuDoubleComplex*)work, ipiv, dinfo);
            if (st == CUSOLVER_STATUS_SUCCESS)
                st = cs.zgetrs(h, CUBLAS_OP_T, n, nrhs, (const cuDoubleComplex*)A_dev, n, ipiv, (cuDoubleComplex*)B_dev,
                               n, dinfo + 1);
        }
        int hinfo[2] = {0, 0};
        if (st == CUSOLVER_STATUS_SUCCESS &&
            cudaMemcpyAsync(hinfo, dinfo, sizeof(hinfo), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
            cudaStreamSynchronize(s) == cudaSuccess) {
            if (info) *info = hinfo[0] ? hinfo[0] : hinfo[1];
            if (hinfo[0] > 0) rc = set_api_error(BIELCC_ERR_NAN, "solve_dense: the matrix is singular (U has a zero pivot)");
        } else {
            cudaGetLastError();
            rc = set_api_error(BIELCC_ERR_CUDA, "getrf / getrs failed");
        }
    }
    cudaStreamSynchronize(s);
    cudaFree(work);
    cudaFree(ipiv);
    cudaFree(dinfo);
    cs.destroy(h);
    return rc;
}
