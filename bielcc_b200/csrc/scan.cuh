// scan.cuh — single-CTA exclusive scan used to turn per-row near-pair counts
// into offsets (field and assembly near lists). Internal linkage per .cu file.
#pragma once
#include "common.cuh"

namespace bielcc_gpu {

// Exclusive scan of counts[0..n) into offs[0..n], one CTA of 1024 threads.
static __global__ void scan_kernel(const long long* __restrict__ counts, int n, long long* __restrict__ offs,
                            long long* __restrict__ total) {
    __shared__ long long s_part[1024];
    const int t = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int b = t * per, e = min(n, b + per);
    long long sum = 0;
    for (int i = b; i < e; i++) sum += counts[i];
    s_part[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        long long v = t >= off ? s_part[t - off] : 0;
        __syncthreads();
        s_part[t] += v;
        __syncthreads();
    }
    long long run = t ? s_part[t - 1] : 0;
    for (int i = b; i < e; i++) {
        offs[i] = run;
        run += counts[i];
    }
    if (t == 1023) {
        offs[n] = s_part[1023];
        *total = s_part[1023];
    }
}

}  // namespace bielcc_gpu
