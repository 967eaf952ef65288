// noalloc.cu — a field evaluation that allocates no memory.
//
// Who needs it: callers that must not call cudaMalloc once they are running.
// Typical cases are applications that reserve (nearly) all device memory up
// front in their own pool, where a library allocation can fail or fragment
// that pool, and latency-critical loops, where cudaMalloc / cudaFree stall
// the whole device while they synchronise. Such a caller owns every input and
// output buffer; this entry point takes only device pointers and keeps all of
// its scratch memory (cell rows, quadrature node tables, far partial sums,
// near-cell mask, near lists and near-pair moments) in one statically sized
// device array of this file.
//
// Properties of that array:
//   * its size is fixed at BIELCC_NOALLOC_SCRATCH_BYTES (64 MiB); every GPU on
//     which the library's device code is loaded holds it until the process
//     exits;
//   * every call uses the same array and leaves its contents behind; each
//     call rewrites every scratch word it later reads, so nothing has to be
//     cleared between calls;
//   * two calls whose work overlaps on the GPU (other streams, other host
//     threads) race on the array: callers must order them.
#include <cstdio>
#include <cstring>

#include "../../include/bielcc_gpu.h"
#include "internal.h"

namespace bielcc_gpu {

#define BIELCC_NOALLOC_SCRATCH_BYTES (64u << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[BIELCC_NOALLOC_SCRATCH_BYTES];

namespace {

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// The message is returned by bielcc_last_error() on this thread.
int fail(int code, const char* msg) { return set_api_error(code, msg); }

// Device address of the scratch array in the current context. The host symbol
// is only a stand-in and is never handed to a kernel. The address is looked up
// on every call rather than cached: after cudaDeviceReset, or under another
// context on the same device, the module is loaded again and the array can
// move, so a cached address could point at freed memory.
int scratch_address(void** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(BIELCC_ERR_CUDA, "cudaGetSymbolAddress of the static scratch array failed");
    }
    *out = p;
    return BIELCC_OK;
}

}  // namespace
}  // namespace bielcc_gpu

using namespace bielcc_gpu;

extern "C" int bielcc_field_EH_noalloc(int n_vert, int n_cells, const double* cells_dev, int n_rhs,
                                       const double* J_dev, double k_re, double k_im, double mult_re, double mult_im,
                                       const bielcc_planewave* inc, const bielcc_numparam* np, int n_pts,
                                       const double* pts_dev, double* E_dev, double* H_dev, int precision,
                                       void* stream, bielcc_report* report) {
    if (n_vert != 3 && n_vert != 4) return fail(BIELCC_ERR_ARG, "n_vert must be 3 or 4");
    if (n_cells < 1 || n_rhs < 1 || n_pts < 0 || !cells_dev || !J_dev || (n_pts > 0 && (!pts_dev || !E_dev)))
        return fail(BIELCC_ERR_ARG, "bad sizes or null buffers");
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return fail(BIELCC_ERR_ARG, "unknown precision");
    NumParamH n = np ? NumParamH{np->eps, np->rs, np->rs_seg, np->analytic_calc, np->n_start, np->n_start_seg,
                                 np->p_max, np->p_max_seg}
                     : NumParamH{1e-6, 2.0, 2.0, 3.0, 8, 10, 1, 1};
    if (n.n_start < 1 || n.n_start > 256 || n.n_start_seg < 1 || n.p_max < 1 || n.p_max > 20 || n.p_max_seg < 1 ||
        n.p_max_seg > 20)
        return fail(BIELCC_ERR_ARG, "numparam out of range");
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc != BIELCC_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;

    // carve the static array: cell rows, node tables, then the field workspace
    // node tables of the far pass's split (2 n_start when p_max = 2)
    const size_t N = n_cells, nn = (size_t)far_split_n(n) * far_split_n(n);
    MeshDev m;
    m.nv = n_vert;
    m.n_cells = n_cells;
    m.verts = const_cast<double*>(cells_dev);
    size_t off = 0;
    const size_t b_geo = al(N * sizeof(CellGeo)), b_n64 = al(N * nn * sizeof(double4)),
                 b_n32 = al(N * nn * sizeof(float4)), b_rho = al(N * sizeof(float));
    char* sp = (char*)base;
    m.geo = (CellGeo*)(sp + off);
    off += b_geo;
    m.nodes64 = (double4*)(sp + off);
    off += b_n64;
    m.nodes32 = (float4*)(sp + off);
    off += b_n32;
    m.rho32 = (float*)(sp + off);
    off += b_rho;
    m.table_n = far_split_n(n);
    if (far_adaptive(n)) {  // p_max >= 3: the FP64 table at n_start of the convergence test
        m.nodes64_lo = (double4*)(sp + off);
        off += al(N * (size_t)n.n_start * n.n_start * sizeof(double4));
        m.table_lo_n = n.n_start;
    }
    if (far_third_pass(n)) {  // p_max = 3: the tables at 4 n_start of the third pass
        const size_t nn3 = (size_t)16 * n.n_start * n.n_start;
        m.nodes64_hi = (double4*)(sp + off);
        off += al(N * nn3 * sizeof(double4));
        m.nodes32_hi = (float4*)(sp + off);
        off += al(N * nn3 * sizeof(float4));
        m.rho32_hi = (float*)(sp + off);
        off += al(N * sizeof(float));
        m.table_hi_n = 4 * n.n_start;
    }

    FieldLaunch f;
    f.mesh = &m;
    f.pts = pts_dev;
    f.n_pts = n_pts;
    f.J = J_dev;
    f.n_rhs = n_rhs;
    f.k = mk(k_re, k_im);
    f.mult = mk(mult_re, mult_im);
    f.np = n;
    f.precision = precision;
    for (int g = 0; g < 3; g++) {
        f.kvec[g] = inc ? inc->k_vec[g] : 0.;
        f.e0[g] = inc ? inc->e0[g] : 0.;
    }
    f.h_scale = inc ? inc->h_scale : 0.;
    f.add_E = inc ? inc->add_E : 0;
    f.add_H = inc ? inc->add_H : 0;
    f.E = E_dev;
    f.H = H_dev;
    // the far partial sums take at most half of the room left after the node
    // tables and the one-split workspace (more cell splits fill the GPU better;
    // the other half stays for the near pairs)
    int splits = 1;
    const size_t per_split = al((size_t)n_rhs * 12 * n_pts * sizeof(double));
    const size_t b_one = al(field_ws_base_bytes(f, &splits, 0));
    const size_t used = off + b_one + 256;
    const size_t room = used < BIELCC_NOALLOC_SCRATCH_BYTES ? BIELCC_NOALLOC_SCRATCH_BYTES - used : 0;
    const size_t b_ws = al(field_ws_base_bytes(f, &splits, per_split + room / 2));
    char* ws = sp + off;
    off += b_ws;
    long long* d_total = (long long*)(sp + off);
    off += 256;
    if (off > BIELCC_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof(msg), "needs %zu scratch bytes before near pairs; the static scratch holds %u",
                 off, BIELCC_NOALLOC_SCRATCH_BYTES);
        return fail(BIELCC_ERR_ARG, msg);
    }
    if (report) memset(report, 0, sizeof(*report));
    if (n_pts == 0) return BIELCC_OK;

    cudaError_t e = launch_cell_geometry(m.verts, n_vert, n_cells, m.geo, s);
    if (e == cudaSuccess)
        e = launch_node_tables(m.verts, m.geo, n_vert, n_cells, far_split_n(n), m.nodes64, m.nodes32, m.rho32, s);
    if (e == cudaSuccess && m.nodes64_lo)
        e = launch_node_tables(m.verts, m.geo, n_vert, n_cells, n.n_start, m.nodes64_lo, nullptr, nullptr, s);
    if (e == cudaSuccess && m.nodes64_hi)
        e = launch_node_tables(m.verts, m.geo, n_vert, n_cells, m.table_hi_n, m.nodes64_hi, m.nodes32_hi, m.rho32_hi,
                               s);
    int l1 = 0, lf = 0, l2 = 0;
    if (e == cudaSuccess) e = field_stage1(f, ws, splits, d_total, s, &l1, nullptr, nullptr, &lf);
    long long n_near = 0;  // pageable host copy: no pinned staging is allocated
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n_near, d_total, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(BIELCC_ERR_CUDA, cudaGetErrorString(e));
    }
    const size_t b_pairs = n_near > 0 ? field_pair_ws_bytes(n_near) : 0;
    if (off + b_pairs > BIELCC_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof(msg), "%lld near pairs need %zu scratch bytes in total; the static scratch holds %u",
                 n_near, off + b_pairs, BIELCC_NOALLOC_SCRATCH_BYTES);
        return fail(BIELCC_ERR_ARG, msg);
    }
    e = field_stage2(f, ws, splits, n_near, sp + off, nullptr, s, &l2);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(BIELCC_ERR_CUDA, cudaGetErrorString(e));
    }
    if (report) {
        report->n_pairs = (int64_t)n_pts * n_cells;
        report->n_near_pairs = n_near;
    }
    return BIELCC_OK;
}
