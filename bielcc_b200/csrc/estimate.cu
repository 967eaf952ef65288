// estimate.cu — the error report of a mixed-precision result: the relative L2
// difference between the mixed outputs and an FP64 evaluation of the same
// field at a sample of the points, computed on the device.
//
// Per evaluated job (a single-job call, or one job of a batch) the sample is
// Q points spread evenly over the job's point set (point q * P / Q) and its
// first Ss right-hand sides. The caller gathers the sample points
// (err_gather), evaluates them in FP64 (on a side stream, beside the main
// evaluation), then err_compare forms, per job,
//     num = sum |E_mixed - E_fp64|^2 + |H_mixed - H_fp64|^2,
//     den = sum |E_fp64|^2 + |H_fp64|^2
// over the sample's components (each thread sums a fixed stride, then a fixed
// tree: the value depends only on the job), writes sqrt(num / den) to the
// job's estimate address when it has one, and the sums over all jobs to
// `sums` (num, den).
#include "internal.h"

namespace bielcc_gpu {

namespace {
constexpr int kErrThreads = 256;
}

__global__ void err_gather_kernel(const ErrJob* __restrict__ jobs, double* __restrict__ spts) {
    const ErrJob& j = jobs[blockIdx.x];
    for (int q = threadIdx.x; q < j.Q; q += blockDim.x) {
        const long long p = (long long)q * j.P / j.Q;
        for (int g = 0; g < 3; g++) spts[3 * ((size_t)j.off + q) + g] = j.pts[3 * p + g];
    }
}

__device__ __forceinline__ double2 err_out(const double* d, const float* f, size_t i) {
    if (f) return make_double2((double)f[2 * i], (double)f[2 * i + 1]);
    return make_double2(d[2 * i], d[2 * i + 1]);
}

__global__ void err_compare_kernel(const ErrJob* __restrict__ jobs, double* __restrict__ nd) {
    const ErrJob& j = jobs[blockIdx.x];
    double num = 0., den = 0.;
    const int per = j.Q * 3;
    for (int e = threadIdx.x; e < j.Ss * per; e += blockDim.x) {
        const int s = e / per, r = e - s * per, q = r / 3, c = r - q * 3;
        const long long p = (long long)q * j.P / j.Q;
        const size_t im = ((size_t)s * j.P + p) * 3 + c, iq = ((size_t)s * j.Q + q) * 3 + c;
        const double2 a = err_out(j.E, j.E32, im);
        const double2 b = make_double2(j.Eq[2 * iq], j.Eq[2 * iq + 1]);
        num += (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y);
        den += b.x * b.x + b.y * b.y;
        if (j.Hq && (j.H || j.H32)) {
            const double2 ha = err_out(j.H, j.H32, im);
            const double2 hb = make_double2(j.Hq[2 * iq], j.Hq[2 * iq + 1]);
            num += (ha.x - hb.x) * (ha.x - hb.x) + (ha.y - hb.y) * (ha.y - hb.y);
            den += hb.x * hb.x + hb.y * hb.y;
        }
    }
    __shared__ double sn[kErrThreads], sd[kErrThreads];
    sn[threadIdx.x] = num;
    sd[threadIdx.x] = den;
    __syncthreads();
    for (int w = kErrThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sn[threadIdx.x] += sn[threadIdx.x + w];
            sd[threadIdx.x] += sd[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        nd[2 * blockIdx.x] = sn[0];
        nd[2 * blockIdx.x + 1] = sd[0];
        if (j.est_dev) *j.est_dev = sd[0] > 0. ? sqrt(sn[0] / sd[0]) : 0.;
    }
}

// sums over jobs in job order (one thread: a handful of jobs to a few thousand)
__global__ void err_sum_kernel(const double* __restrict__ nd, int n, double* __restrict__ sums) {
    double a = 0., b = 0.;
    for (int i = 0; i < n; i++) {
        a += nd[2 * i];
        b += nd[2 * i + 1];
    }
    sums[0] = a;
    sums[1] = b;
}

cudaError_t err_gather(const ErrJob* d_jobs, int n_jobs, double* spts, cudaStream_t s) {
    if (n_jobs <= 0) return cudaSuccess;
    err_gather_kernel<<<n_jobs, 128, 0, s>>>(d_jobs, spts);
    return cudaGetLastError();
}

cudaError_t err_compare(const ErrJob* d_jobs, int n_jobs, double* nd, double* sums, cudaStream_t s) {
    if (n_jobs <= 0) return cudaSuccess;
    err_compare_kernel<<<n_jobs, kErrThreads, 0, s>>>(d_jobs, nd);
    err_sum_kernel<<<1, 1, 0, s>>>(nd, n_jobs, sums);
    return cudaGetLastError();
}

}  // namespace bielcc_gpu
