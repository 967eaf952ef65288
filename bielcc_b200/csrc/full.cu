// full.cu — the full Stratton-Chu combination with electric and magnetic
// surface currents (bielcc_field_EH_full):
//     E = multE * sum K[j_E] - sum R[j_M] + E_inc,
//     H = multH * sum K[j_M] + sum R[j_E] + H_inc,
// as examples/field/main0_field_test.cpp:313-319 forms field_E_SCH and
// field_H_SCH from its four sums. The four sums come from one field
// evaluation over 2S right-hand sides [j_E(0..S-1), j_M(0..S-1)] with mult = 1
// and no incident field: its "E" output of a right-hand side is sum K[j], its
// "H" output sum R[j]; the J-independent moments make the extra right-hand
// sides a contraction each, not a second quadrature. This kernel combines them.
#include "../../include/bielcc_gpu.h"
#include "internal.h"

namespace bielcc_gpu {

__global__ void combine_full_kernel(const cplx* __restrict__ E2, const cplx* __restrict__ H2, int S, int P,
                                    cplx multE, cplx multH, const double* __restrict__ pts, FullInc inc,
                                    cplx* __restrict__ E, cplx* __restrict__ H,
                                    unsigned long long* __restrict__ nonfinite) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)S * P) return;
    const int s = (int)(i / P), p = (int)(i - (long long)s * P);
    double cs = 1., sn = 0.;
    if (inc.add_E || inc.add_H) {
        const double* x = pts + 3 * (size_t)p;
        sincos(inc.kvec[0] * x[0] + inc.kvec[1] * x[1] + inc.kvec[2] * x[2], &sn, &cs);
    }
    double kx0[3];
    cross3(inc.kvec, inc.e0, kx0);
    const size_t ie = ((size_t)s * P + p) * 3, im = ((size_t)(S + s) * P + p) * 3;
    bool bad = false;
    for (int a = 0; a < 3; a++) {
        cplx e = multE * E2[ie + a] - H2[im + a];  // multE K[j_E] - R[j_M]
        cplx h = multH * E2[im + a] + H2[ie + a];  // multH K[j_M] + R[j_E]
        if (inc.add_E) e += mk(inc.e0[a] * cs, inc.e0[a] * sn);
        if (inc.add_H) h += mk(kx0[a] * cs * inc.h_scale, kx0[a] * sn * inc.h_scale);
        E[ie + a] = e;
        H[ie + a] = h;
        bad |= !isfinite(e.re) || !isfinite(e.im) || !isfinite(h.re) || !isfinite(h.im);
    }
    if (bad && nonfinite) atomicAdd(nonfinite, 1ull);
}

cudaError_t launch_combine_full(const double* E2, const double* H2, int S, int P, cplx multE, cplx multH,
                                const double* pts, const FullInc& inc, double* E, double* H,
                                unsigned long long* nonfinite, cudaStream_t s) {
    const long long n = (long long)S * P;
    if (n == 0) return cudaSuccess;
    combine_full_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        reinterpret_cast<const cplx*>(E2), reinterpret_cast<const cplx*>(H2), S, P, multE, multH, pts, inc,
        reinterpret_cast<cplx*>(E), reinterpret_cast<cplx*>(H), nonfinite);
    return cudaGetLastError();
}

}  // namespace bielcc_gpu
