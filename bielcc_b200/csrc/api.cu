// api.cu — the C ABI of libbielcc_gpu.so (include/bielcc_gpu.h): contexts,
// resident meshes, workspaces, host<->device staging and kernel dispatch.
// No C++ exception crosses the boundary; every entry point returns a status.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/bielcc_gpu.h"
#include "internal.h"
#include "ops.cuh"

using namespace bielcc_gpu;

namespace {

thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_status(cudaError_t e, const char* what, int line) {
    if (e == cudaSuccess) return BIELCC_OK;
    int code = (e == cudaErrorMemoryAllocation) ? BIELCC_ERR_OOM : BIELCC_ERR_CUDA;
    cudaGetLastError();  // clear a non-sticky error
    return set_error(code, "%s (api.cu:%d): %s", what, line, cudaGetErrorString(e));
}
#define TRY_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_status(e_, #call, __LINE__); \
    } while (0)
#define TRY(call)                    \
    do {                             \
        int rc_ = (call);            \
        if (rc_ != BIELCC_OK) return rc_; \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return BIELCC_OK;
        if (p) {
            cudaDeviceSynchronize();  // the old buffer may still be in use on some stream
            cudaFree(p);
        }
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 4 + 256;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(BIELCC_ERR_OOM, "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
        }
        cap = want;
        return BIELCC_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

namespace bielcc_gpu {
int set_api_error(int code, const char* msg) { return set_error(code, "%s", msg); }
}  // namespace bielcc_gpu

struct bielcc_ctx_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ws_done = nullptr;  // last use of the shared workspaces
    std::mutex mu;
    std::map<int, MeshDev*> meshes;
    int next_mesh = 1;
    DevBuf ws, pair_ws, io, scratch_small;
    DevBuf full;  // [j_E; j_M] and the 2S-RHS outputs of bielcc_field_EH_full
    long long* h_total = nullptr;  // pinned
    // side stream and workspaces of the mixed form's FP64 error sample, which
    // runs beside the main evaluation (bielcc_field_EH)
    cudaStream_t side = nullptr;
    cudaEvent_t side_in = nullptr;
    cudaEvent_t side_out = nullptr;  // the side stream's error sample is complete
    DevBuf side_ws, side_pair_ws, side_io, side_scratch;
    bool batch_tc = false;              // mixed batches contract on the tensor cores when they qualify
    // moments-buffer cap of the split pipeline (0: never split). Batch plans
    // split when their moments fit one wave; every batch only with split_all.
    size_t batch_split = (size_t)16 << 30;
    bool batch_split_all = false;
    long long* h_side_total = nullptr;  // pinned
    unsigned long long* h_nonfinite = nullptr;
    // counters / timing (bielcc_ctx_stats)
    bool timing = false;
    cudaEvent_t far_begin = nullptr, far_end = nullptr;
    double batch_item_cost = 4.0e6;  // node evaluations per batched work item (bielcc_batch_autotune)
    bielcc_stats stats = {0, 0, 0, 0.0, 0};
};

namespace {

NumParamH to_np(const bielcc_numparam* p) {
    NumParamH n;
    if (!p) {
        n = {1e-6, 2.0, 2.0, 3.0, 8, 10, 1, 1};
        return n;
    }
    n.eps = p->eps;
    n.rs = p->rs;
    n.rs_seg = p->rs_seg;
    n.analytic_calc = p->analytic_calc;
    n.n_start = p->n_start;
    n.n_start_seg = p->n_start_seg;
    n.p_max = p->p_max;
    n.p_max_seg = p->p_max_seg;
    return n;
}

int check_np(const NumParamH& n) {
    if (n.n_start < 1 || n.n_start > 256 || n.n_start_seg < 1 || n.p_max < 1 || n.p_max > 20 || n.p_max_seg < 1 ||
        n.p_max_seg > 20)
        return set_error(BIELCC_ERR_ARG, "numparam out of range (n_start %d, n_start_seg %d, p_max %d, p_max_seg %d)",
                         n.n_start, n.n_start_seg, n.p_max, n.p_max_seg);
    return BIELCC_OK;
}

int enter(bielcc_ctx ctx) {
    if (!ctx) return set_error(BIELCC_ERR_ARG, "null context");
    TRY_CUDA(cudaSetDevice(ctx->device));
    return BIELCC_OK;
}

int get_mesh(bielcc_ctx ctx, bielcc_mesh id, MeshDev** out) {
    auto it = ctx->meshes.find(id);
    if (it == ctx->meshes.end()) return set_error(BIELCC_ERR_NOT_FOUND, "unknown mesh %d", id);
    *out = it->second;
    return BIELCC_OK;
}

void free_mesh(MeshDev* m) {
    cudaFree(m->verts);
    cudaFree(m->geo);
    cudaFree(m->nodes64);
    cudaFree(m->nodes32);
    cudaFree(m->rho32);
    cudaFree(m->nodes64_lo);
    cudaFree(m->nodes64_hi);
    cudaFree(m->nodes32_hi);
    cudaFree(m->rho32_hi);
    delete m;
}

// Node tables for split n, built on first use and cached on the mesh.
int ensure_tables(MeshDev* m, int n, cudaStream_t s) {
    if (m->table_n == n && m->nodes64) return BIELCC_OK;
    cudaFree(m->nodes64);
    cudaFree(m->nodes32);
    cudaFree(m->rho32);
    m->nodes64 = nullptr;
    m->nodes32 = nullptr;
    m->rho32 = nullptr;
    m->table_n = 0;
    size_t nn = (size_t)n * n * m->n_cells;
    TRY_CUDA(cudaMalloc(&m->nodes64, nn * sizeof(double4) + 16));
    TRY_CUDA(cudaMalloc(&m->nodes32, nn * sizeof(float4) + 16));
    TRY_CUDA(cudaMalloc(&m->rho32, (size_t)m->n_cells * sizeof(float) + 16));
    TRY_CUDA(launch_node_tables(m->verts, m->geo, m->nv, m->n_cells, n, m->nodes64, m->nodes32, m->rho32, s));
    m->table_n = n;
    return BIELCC_OK;
}

// The far pass's node tables (far_split_n) and, for p_max >= 3, the FP64
// table at n_start that the convergence test compares against and, for
// p_max = 3, the tables at 4 n_start of the third pass.
int ensure_far_tables(MeshDev* m, const NumParamH& np, cudaStream_t s) {
    TRY(ensure_tables(m, far_split_n(np), s));
    if (far_adaptive(np) && (m->table_lo_n != np.n_start || !m->nodes64_lo)) {
        cudaFree(m->nodes64_lo);
        m->nodes64_lo = nullptr;
        m->table_lo_n = 0;
        TRY_CUDA(cudaMalloc(&m->nodes64_lo, (size_t)np.n_start * np.n_start * m->n_cells * sizeof(double4) + 16));
        TRY_CUDA(launch_node_tables(m->verts, m->geo, m->nv, m->n_cells, np.n_start, m->nodes64_lo, nullptr, nullptr,
                                    s));
        m->table_lo_n = np.n_start;
    }
    const int n3 = 4 * np.n_start;
    if (far_third_pass(np) && (m->table_hi_n != n3 || !m->nodes64_hi)) {
        cudaFree(m->nodes64_hi);
        cudaFree(m->nodes32_hi);
        cudaFree(m->rho32_hi);
        m->nodes64_hi = nullptr;
        m->nodes32_hi = nullptr;
        m->rho32_hi = nullptr;
        m->table_hi_n = 0;
        const size_t nn = (size_t)n3 * n3 * m->n_cells;
        TRY_CUDA(cudaMalloc(&m->nodes64_hi, nn * sizeof(double4) + 16));
        TRY_CUDA(cudaMalloc(&m->nodes32_hi, nn * sizeof(float4) + 16));
        TRY_CUDA(cudaMalloc(&m->rho32_hi, (size_t)m->n_cells * sizeof(float) + 16));
        TRY_CUDA(launch_node_tables(m->verts, m->geo, m->nv, m->n_cells, n3, m->nodes64_hi, m->nodes32_hi,
                                    m->rho32_hi, s));
        m->table_hi_n = n3;
    }
    return BIELCC_OK;
}

// Orders `s` after the previous use of the shared workspaces.
int ws_acquire(bielcc_ctx ctx, cudaStream_t s) {
    TRY_CUDA(cudaStreamWaitEvent(s, ctx->ws_done, 0));
    return BIELCC_OK;
}
int ws_release(bielcc_ctx ctx, cudaStream_t s) {
    TRY_CUDA(cudaEventRecord(ctx->ws_done, s));
    return BIELCC_OK;
}

// The workspaces one field evaluation uses: the context's shared set, or the
// side set of the error sample.
struct WsSet {
    DevBuf* ws;
    DevBuf* pair_ws;
    DevBuf* scratch;
    long long* h_total;  // pinned near-pair count
    bool timed;          // far-kernel events into the context's stats
    bool sample;         // an FP64 error sample: its far work stays out of far_launches / far_pairs
};
}  // namespace

bool ctx_batch_tensor_cores(bielcc_ctx_s* ctx) { return ctx->batch_tc; }
size_t ctx_batch_split_cap(bielcc_ctx_s* ctx) { return ctx->batch_split_all ? ctx->batch_split : 0; }

namespace {

WsSet main_ws(bielcc_ctx ctx) {
    return {&ctx->ws, &ctx->pair_ws, &ctx->scratch_small, ctx->h_total, ctx->timing, false};
}
WsSet side_ws(bielcc_ctx ctx) {
    return {&ctx->side_ws, &ctx->side_pair_ws, &ctx->side_scratch, ctx->h_side_total, false, true};
}

struct FieldArgs {
    MeshDev* m;
    int n_rhs;
    const double* J;
    cplx k, mult;
    const bielcc_planewave* inc;
    NumParamH np;
    int n_pts;
    const double* pts;
    double* E;
    double* H;
    int precision;
};

// Several right-hand sides: the single-job far kernel takes 4, 2 or 1 per
// launch and repeats the quadrature in every launch (S = 3 is two launches,
// 2 + 1), and its 4-RHS variant holds 2 CTAs per SM; the batched kernel
// computes the J-independent moments once for all and contracts them with
// each. The job runs as a one-job batch when the single-job launches (about
// one quadrature each, 1.1 for a 4-RHS launch) outweigh the batched kernel's
// idle SMs on a small point set (its work items over its resident CTAs).
// Measured on 8192 cells x 20,000 points (mixed): S = 2 28.4 ms single-job
// against 31.6 batched, S = 3 53.8 against 31.9, S = 4 34.9 against 32.0.
// Returns false when the call is left to the single-job path.
int field_device_batched(bielcc_ctx ctx, const FieldArgs& a, cudaStream_t s, bielcc_report* rep,
                         unsigned long long* d_nonfinite, bool* done, const WsSet& w) {
    *done = false;
    if (a.n_rhs <= 2 || far_adaptive(a.np) || far_split_n(a.np) > kBatchMaxNStart || a.n_pts == 0) return BIELCC_OK;
    TRY(ensure_tables(a.m, far_split_n(a.np), s));
    JobDev d;
    memset(&d, 0, sizeof(d));
    d.geo = a.m->geo;
    d.nodes32 = a.m->nodes32;
    d.nodes64 = a.m->nodes64;
    d.rho32 = a.m->rho32;
    d.verts = a.m->verts;
    d.nv = a.m->nv;
    d.n_cells = a.m->n_cells;
    d.pts = a.pts;
    d.n_pts = a.n_pts;
    d.J = reinterpret_cast<const cplx*>(a.J);
    d.n_rhs = a.n_rhs;
    d.k = a.k;
    d.mult = a.mult;
    if (a.inc) {
        for (int g = 0; g < 3; g++) {
            d.kvec[g] = a.inc->k_vec[g];
            d.e0[g] = a.inc->e0[g];
        }
        d.h_scale = a.inc->h_scale;
        d.add_E = a.inc->add_E;
        d.add_H = a.inc->add_H;
    }
    d.E = a.E;
    d.H = a.H;
    BatchPlan bp;
    const bool mixed = a.precision == BIELCC_PREC_MIXED;
    const size_t split = ctx_batch_split_cap(ctx);
    plan_batch(bp, std::vector<JobDev>{d}, far_split_n(a.np), mixed, ctx->batch_item_cost, ctx->batch_tc, split);
    // The tuned item size suits batches of many jobs; one job alone is cut
    // finer (up to its range limit) when its items would leave resident CTAs idle.
    if ((int)bp.items.size() < 2 * bp.workers()) {
        const double finer = std::max(1.0e5, ctx->batch_item_cost * bp.items.size() / (2.0 * bp.workers()));
        if (finer < ctx->batch_item_cost)
            plan_batch(bp, std::vector<JobDev>{d}, far_split_n(a.np), mixed, finer, ctx->batch_tc, split);
    }
    const double busy = std::min(1.0, (double)bp.items.size() / std::max(1, bp.workers()));
    const int S = a.n_rhs;
    const double single = (S / 4) * 1.1 + (S % 4) / 2 + (S % 2);  // single-job launches, in quadratures
    if (single * busy <= 1.05) return BIELCC_OK;
    TRY(w.ws->ensure(bp.ws_bytes));
    BatchDevPtrs dp;
    int l1 = 0, l2 = 0;
    TRY_CUDA(batch_stage1(bp, w.ws->p, a.np.analytic_calc, far_split_n(a.np), a.k.im != 0., s, &dp, &l1));
    TRY_CUDA(batch_status_to_host(dp, w.h_total, s));
    TRY_CUDA(cudaStreamSynchronize(s));
    if (batch_timed_out(w.h_total)) return set_error(BIELCC_ERR_TIMEOUT, "batched far kernel: a bounded wait ran out");
    const long long n_near = *w.h_total;
    if (n_near > 0) TRY(w.pair_ws->ensure(batch_pair_ws_bytes(n_near)));
    DNP dn{a.np.eps, a.np.rs, a.np.rs_seg, a.np.analytic_calc, a.np.n_start, a.np.n_start_seg, a.np.p_max,
           a.np.p_max_seg};
    TRY_CUDA(batch_stage2(bp, dp, n_near, w.pair_ws->p, dn, d_nonfinite, s, &l2));
    ctx->stats.kernel_launches += l1 + l2;
    if (!w.sample) {
        ctx->stats.far_launches += 1;
        ctx->stats.far_pairs += ((long long)a.n_pts * a.m->n_cells - n_near) * a.n_rhs;
    }
    if (rep) {
        rep->n_pairs = (int64_t)a.n_pts * a.m->n_cells;
        rep->n_near_pairs = n_near;
    }
    *done = true;
    return BIELCC_OK;
}

// A single-job field evaluation between its two halves: stage 1 (far kernel,
// near counting) is enqueued and the near-pair count is on its way to the host.
struct FieldPending {
    FieldArgs a;
    FieldLaunch f;
    int splits = 1, l1 = 0, lf = 0;
    bool batched = false;  // ran whole as a one-job batch
};

// Enqueues stage 1 of a field evaluation on device buffers (or the whole
// evaluation, when it runs as a one-job batch).
int field_begin(bielcc_ctx ctx, const FieldArgs& a, cudaStream_t s, bielcc_report* rep,
                unsigned long long* d_nonfinite, const WsSet& w, FieldPending* p) {
    p->a = a;
    TRY(field_device_batched(ctx, a, s, rep, d_nonfinite, &p->batched, w));
    if (p->batched) return BIELCC_OK;
    TRY(ensure_far_tables(a.m, a.np, s));
    FieldLaunch& f = p->f;
    f.mesh = a.m;
    f.pts = a.pts;
    f.n_pts = a.n_pts;
    f.J = a.J;
    f.n_rhs = a.n_rhs;
    f.k = a.k;
    f.mult = a.mult;
    f.np = a.np;
    f.precision = a.precision;
    for (int g = 0; g < 3; g++) {
        f.kvec[g] = a.inc ? a.inc->k_vec[g] : 0.;
        f.e0[g] = a.inc ? a.inc->e0[g] : 0.;
    }
    f.h_scale = a.inc ? a.inc->h_scale : 0.;
    f.add_E = a.inc ? a.inc->add_E : 0;
    f.add_H = a.inc ? a.inc->add_H : 0;
    f.E = a.E;
    f.H = a.H;
    size_t base = field_ws_base_bytes(f, &p->splits);
    TRY(w.ws->ensure(base));
    TRY(w.scratch->ensure(256));
    long long* d_total = (long long*)w.scratch->p;
    TRY_CUDA(field_stage1(f, w.ws->p, p->splits, d_total, s, &p->l1, w.timed ? ctx->far_begin : nullptr,
                          w.timed ? ctx->far_end : nullptr, &p->lf));
    TRY_CUDA(cudaMemcpyAsync(w.h_total, d_total, sizeof(long long), cudaMemcpyDeviceToHost, s));
    return BIELCC_OK;
}

// Waits for the near-pair count (sizes the FP64 near workspace) and enqueues
// stage 2 (near pairs, finalize).
int field_finish(bielcc_ctx ctx, FieldPending& p, cudaStream_t s, bielcc_report* rep,
                 unsigned long long* d_nonfinite, const WsSet& w) {
    if (p.batched) return BIELCC_OK;
    const FieldArgs& a = p.a;
    TRY_CUDA(cudaStreamSynchronize(s));
    long long n_near = *w.h_total;
    if (w.timed && p.lf > 0) {
        float ms = 0.f;
        TRY_CUDA(cudaEventElapsedTime(&ms, ctx->far_begin, ctx->far_end));
        ctx->stats.far_ms += ms;
    }
    int l2 = 0;
    if (n_near > 0) TRY(w.pair_ws->ensure(field_pair_ws_bytes(n_near)));
    TRY_CUDA(field_stage2(p.f, w.ws->p, p.splits, n_near, w.pair_ws->p, d_nonfinite, s, &l2));
    ctx->stats.kernel_launches += p.l1 + l2;
    if (!w.sample) {
        ctx->stats.far_launches += p.lf;
        ctx->stats.far_pairs += ((long long)a.n_pts * a.m->n_cells - n_near) * a.n_rhs;
    }
    if (rep) {
        rep->n_pairs = (int64_t)a.n_pts * a.m->n_cells;
        rep->n_near_pairs = n_near;
    }
    return BIELCC_OK;
}

// Enqueues a field evaluation on device buffers; one short host wait for the
// near-pair count (sizes the FP64 near workspace).
int field_device(bielcc_ctx ctx, const FieldArgs& a, cudaStream_t s, bielcc_report* rep,
                 unsigned long long* d_nonfinite) {
    const WsSet w = main_ws(ctx);
    FieldPending p;
    TRY(field_begin(ctx, a, s, rep, d_nonfinite, w, &p));
    return field_finish(ctx, p, s, rep, d_nonfinite, w);
}

// Error sample of a single-job mixed evaluation: the FP64 field at
// Q = min(P, 256) points spread over the set (two full point tiles), all
// right-hand sides, evaluated on the side stream beside the main evaluation
// and compared with the mixed outputs on the device (estimate.cu). `full`:
// the outputs are the full Stratton-Chu combination of a 2S-RHS evaluation,
// so the sample is combined the same way before the comparison.
struct SingleEst {
    bool on = false;
    int Q = 0;
    ErrJob* d_job = nullptr;
    double *spts = nullptr, *Eq = nullptr, *Hq = nullptr, *Ec = nullptr, *Hc = nullptr, *nd = nullptr,
           *sums = nullptr;
    FieldPending ps;
    bool full = false;
    cplx multE, multH;
    const bielcc_planewave* inc = nullptr;
    int S_out = 0;
};

// a: the main evaluation's arguments (precision mixed); E_out / H_out: the
// outputs compared (a.E / a.H, or the full-field combination), S_out right-hand
// sides each.
int est_single_begin(bielcc_ctx ctx, const FieldArgs& a, cudaStream_t s, SingleEst& e, const double* E_out,
                     const double* H_out, int S_out) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    e.on = true;
    e.Q = std::min(a.n_pts, 256);
    e.S_out = S_out;
    const size_t Q = e.Q, Sa = a.n_rhs;
    const size_t bQ = Q * 24, bQo = Sa * Q * 48, bC = (size_t)S_out * Q * 48;
    TRY(ctx->side_io.ensure(3 * 256 + al(bQ) + 2 * al(bQo) + 2 * al(bC)));
    char* b = (char*)ctx->side_io.p;
    e.d_job = (ErrJob*)b;
    e.nd = (double*)(b + 256);
    e.sums = (double*)(b + 512);
    e.spts = (double*)(b + 768);
    e.Eq = (double*)(b + 768 + al(bQ));
    e.Hq = (double*)(b + 768 + al(bQ) + al(bQo));
    e.Ec = (double*)(b + 768 + al(bQ) + 2 * al(bQo));
    e.Hc = (double*)(b + 768 + al(bQ) + 2 * al(bQo) + al(bC));
    ErrJob j{};
    j.pts = a.pts;
    j.P = a.n_pts;
    j.Q = e.Q;
    j.S = S_out;
    j.Ss = S_out;
    j.off = 0;
    j.E = E_out;
    j.H = H_out;
    j.Eq = e.full ? e.Ec : e.Eq;
    j.Hq = H_out ? (e.full ? e.Hc : e.Hq) : nullptr;
    TRY(ensure_far_tables(a.m, a.np, s));
    TRY_CUDA(cudaEventRecord(ctx->side_in, s));  // inputs and node tables on the device
    TRY_CUDA(cudaStreamWaitEvent(ctx->side, ctx->side_in, 0));
    TRY_CUDA(cudaMemcpyAsync(e.d_job, &j, sizeof(j), cudaMemcpyHostToDevice, ctx->side));
    TRY_CUDA(err_gather(e.d_job, 1, e.spts, ctx->side));
    FieldArgs b64{a.m, a.n_rhs, a.J, a.k, a.mult, a.inc, a.np, e.Q, e.spts, e.Eq, (H_out || e.full) ? e.Hq : nullptr,
                  BIELCC_PREC_FP64};
    return field_begin(ctx, b64, ctx->side, nullptr, nullptr, side_ws(ctx), &e.ps);
}

// Completes the sample on the side stream and enqueues the comparison on s
// (after the main evaluation's outputs); the sums land in h_total[4], [5].
int est_single_finish(bielcc_ctx ctx, cudaStream_t s, SingleEst& e) {
    TRY(field_finish(ctx, e.ps, ctx->side, nullptr, nullptr, side_ws(ctx)));
    if (e.full) {
        FullInc fi;
        memset(&fi, 0, sizeof(fi));
        if (e.inc) {
            for (int g = 0; g < 3; g++) {
                fi.kvec[g] = e.inc->k_vec[g];
                fi.e0[g] = e.inc->e0[g];
            }
            fi.h_scale = e.inc->h_scale;
            fi.add_E = e.inc->add_E;
            fi.add_H = e.inc->add_H;
        }
        TRY_CUDA(launch_combine_full(e.Eq, e.Hq, e.S_out, e.Q, e.multE, e.multH, e.spts, fi, e.Ec, e.Hc, nullptr,
                                     ctx->side));
    }
    TRY_CUDA(cudaEventRecord(ctx->side_out, ctx->side));
    TRY_CUDA(cudaStreamWaitEvent(s, ctx->side_out, 0));
    TRY_CUDA(err_compare(e.d_job, 1, e.nd, e.sums, s));
    TRY_CUDA(cudaMemcpyAsync(ctx->h_total + 4, e.sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    ctx->stats.kernel_launches += 3 + (e.full ? 1 : 0);
    return BIELCC_OK;
}

// After the stream has been synchronised: the estimate into the report.
void est_single_report(bielcc_ctx ctx, const SingleEst& e, bielcc_report* rep) {
    if (!e.on || !rep) return;
    const double* v = reinterpret_cast<const double*>(ctx->h_total + 4);
    rep->est_rel_l2 = v[1] > 0. ? sqrt(v[0] / v[1]) : 0.;
    rep->est_sample = e.Q;
}

}  // namespace

extern "C" {

void bielcc_numparam_default(bielcc_numparam* np) {
    if (!np) return;
    np->eps = 1e-6;
    np->rs = 2.0;
    np->rs_seg = 2.0;
    np->analytic_calc = 3.0;
    np->n_start = 8;
    np->n_start_seg = 10;
    np->p_max = 1;
    np->p_max_seg = 1;
}

int bielcc_abi_version(void) { return BIELCC_ABI_VERSION; }

const char* bielcc_last_error(void) { return g_last_error.c_str(); }

int bielcc_ctx_create(int device, bielcc_ctx* out) {
    if (!out) return set_error(BIELCC_ERR_ARG, "null output pointer");
    *out = nullptr;
    int n = 0;
    TRY_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return set_error(BIELCC_ERR_ARG, "device %d of %d", device, n);
    TRY_CUDA(cudaSetDevice(device));
    bielcc_ctx c = new (std::nothrow) bielcc_ctx_s;
    if (!c) return set_error(BIELCC_ERR_OOM, "host allocation failed");
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ws_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_total, 64);
    if (e == cudaSuccess) e = cudaEventCreate(&c->far_begin);
    if (e == cudaSuccess) e = cudaEventCreate(&c->far_end);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->side_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->side_out, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_side_total, 64);
    if (e != cudaSuccess) {
        if (c->h_total) cudaFreeHost(c->h_total);
        if (c->h_side_total) cudaFreeHost(c->h_side_total);
        if (c->ws_done) cudaEventDestroy(c->ws_done);
        if (c->far_begin) cudaEventDestroy(c->far_begin);
        if (c->far_end) cudaEventDestroy(c->far_end);
        if (c->side_in) cudaEventDestroy(c->side_in);
        if (c->side_out) cudaEventDestroy(c->side_out);
        if (c->side) cudaStreamDestroy(c->side);
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return cuda_status(e, "context set-up", __LINE__);
    }
    c->h_nonfinite = reinterpret_cast<unsigned long long*>(c->h_total + 1);
    TRY_CUDA(cudaEventRecord(c->ws_done, c->stream));
    *out = c;
    return BIELCC_OK;
}

int bielcc_ctx_destroy(bielcc_ctx ctx) {
    if (!ctx) return BIELCC_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    for (auto& kv : ctx->meshes) free_mesh(kv.second);
    ctx->ws.release();
    ctx->pair_ws.release();
    ctx->io.release();
    ctx->scratch_small.release();
    ctx->full.release();
    ctx->side_ws.release();
    ctx->side_pair_ws.release();
    ctx->side_io.release();
    ctx->side_scratch.release();
    if (ctx->h_side_total) cudaFreeHost(ctx->h_side_total);
    if (ctx->side_in) cudaEventDestroy(ctx->side_in);
    if (ctx->side_out) cudaEventDestroy(ctx->side_out);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->h_total) cudaFreeHost(ctx->h_total);  // h_nonfinite lives in the same pinned block
    if (ctx->ws_done) cudaEventDestroy(ctx->ws_done);
    if (ctx->far_begin) cudaEventDestroy(ctx->far_begin);
    if (ctx->far_end) cudaEventDestroy(ctx->far_end);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    cudaGetLastError();  // leave no error of the clean-up behind for the next call on this thread
    return BIELCC_OK;
}

int bielcc_ctx_synchronize(bielcc_ctx ctx) {
    TRY(enter(ctx));
    TRY_CUDA(cudaDeviceSynchronize());
    return BIELCC_OK;
}

int bielcc_ctx_set_batch_tensor_cores(bielcc_ctx ctx, int on) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->batch_tc = on != 0;
    return BIELCC_OK;
}

int bielcc_ctx_set_batch_split(bielcc_ctx ctx, int64_t moments_bytes, int all_batches) {
    TRY(enter(ctx));
    if (moments_bytes < 0) return set_error(BIELCC_ERR_ARG, "negative moments buffer size");
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->batch_split = (size_t)moments_bytes;
    ctx->batch_split_all = all_batches != 0;
    return BIELCC_OK;
}

int bielcc_ctx_set_timing(bielcc_ctx ctx, int on) {
    if (!ctx) return set_error(BIELCC_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->timing = on != 0;
    return BIELCC_OK;
}

int bielcc_ctx_stats(bielcc_ctx ctx, bielcc_stats* out, int reset) {
    if (!ctx || !out) return set_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = ctx->stats;
    if (reset) ctx->stats = bielcc_stats{0, 0, 0, 0.0, 0};
    return BIELCC_OK;
}

int bielcc_ctx_mem_used(bielcc_ctx ctx, int64_t* bytes) {
    if (!ctx || !bytes) return set_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    int64_t b = ctx->ws.cap + ctx->pair_ws.cap + ctx->io.cap + ctx->scratch_small.cap;
    for (auto& kv : ctx->meshes) {
        const MeshDev* m = kv.second;
        b += (int64_t)m->n_cells * (m->nv * 3 * 8 + sizeof(CellGeo));
        if (m->table_n) b += (int64_t)m->n_cells * m->table_n * m->table_n * (32 + 16) + 4 * m->n_cells;
        if (m->table_lo_n) b += (int64_t)m->n_cells * m->table_lo_n * m->table_lo_n * 32;
        if (m->table_hi_n) b += (int64_t)m->n_cells * m->table_hi_n * m->table_hi_n * (32 + 16) + 4 * m->n_cells;
    }
    *bytes = b;
    return BIELCC_OK;
}

int bielcc_mesh_create(bielcc_ctx ctx, int n_vert, int n_cells, const double* cells, bielcc_mesh* out) {
    TRY(enter(ctx));
    if (!out || (!cells && n_cells > 0)) return set_error(BIELCC_ERR_ARG, "null argument");
    if (n_vert != 3 && n_vert != 4) return set_error(BIELCC_ERR_ARG, "n_vert must be 3 or 4, got %d", n_vert);
    if (n_cells < 1) return set_error(BIELCC_ERR_ARG, "n_cells must be positive, got %d", n_cells);
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m = new (std::nothrow) MeshDev;
    if (!m) return set_error(BIELCC_ERR_OOM, "host allocation failed");
    m->nv = n_vert;
    m->n_cells = n_cells;
    size_t vb = (size_t)n_cells * n_vert * 3 * sizeof(double);
    cudaError_t e = cudaMalloc(&m->verts, vb);
    if (e == cudaSuccess) e = cudaMalloc(&m->geo, (size_t)n_cells * sizeof(CellGeo));
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->verts, cells, vb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_cell_geometry(m->verts, n_vert, n_cells, m->geo, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        free_mesh(m);
        return cuda_status(e, "mesh upload", __LINE__);
    }
    int id = ctx->next_mesh++;
    ctx->meshes[id] = m;
    *out = id;
    return BIELCC_OK;
}

int bielcc_mesh_destroy(bielcc_ctx ctx, bielcc_mesh mesh) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    free_mesh(m);
    ctx->meshes.erase(mesh);
    return BIELCC_OK;
}

int bielcc_mesh_geometry(bielcc_ctx ctx, bielcc_mesh mesh, double* out) {
    TRY(enter(ctx));
    if (!out) return set_error(BIELCC_ERR_ARG, "null output");
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    std::vector<CellGeo> rows(m->n_cells);
    TRY_CUDA(cudaMemcpyAsync(rows.data(), m->geo, rows.size() * sizeof(CellGeo), cudaMemcpyDeviceToHost, ctx->stream));
    TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < m->n_cells; c++) {
        double* o = out + 14 * (size_t)c;
        const CellGeo& r = rows[c];
        for (int g2 = 0; g2 < 3; g2++) {
            o[g2] = r.c[g2];
            o[4 + g2] = r.n[g2];
            o[7 + g2] = r.t1[g2];
            o[10 + g2] = r.t2[g2];
        }
        o[3] = r.diam;
        o[13] = r.area;
    }
    return BIELCC_OK;
}

int bielcc_field_EH_device(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* J_dev, double k_re, double k_im,
                           double mult_re, double mult_im, const bielcc_planewave* inc, const bielcc_numparam* np,
                           int n_pts, const double* pts_dev, double* E_dev, double* H_dev, int precision, void* stream,
                           bielcc_report* report) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (n_rhs < 1 || n_pts < 0 || (n_pts > 0 && (!pts_dev || !E_dev)) || !J_dev)
        return set_error(BIELCC_ERR_ARG, "bad field arguments (n_rhs %d, n_pts %d)", n_rhs, n_pts);
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    TRY(ws_acquire(ctx, s));
    FieldArgs a{m, n_rhs, J_dev, mk(k_re, k_im), mk(mult_re, mult_im), inc, n, n_pts, pts_dev, E_dev, H_dev,
                precision};
    if (report) memset(report, 0, sizeof(*report));
    // mixed with a report: the error sample runs beside the evaluation and the
    // call waits for the stream to fill est_rel_l2
    const bool sample = report && precision == BIELCC_PREC_MIXED && n_pts > 0;
    SingleEst es;
    if (sample) TRY(est_single_begin(ctx, a, s, es, E_dev, H_dev, n_rhs));
    TRY(field_device(ctx, a, s, report, nullptr));
    if (sample) {
        TRY(est_single_finish(ctx, s, es));
        TRY_CUDA(cudaStreamSynchronize(s));
        est_single_report(ctx, es, report);
    }
    TRY(ws_release(ctx, s));
    return BIELCC_OK;
}

}  // extern "C"

namespace {

// Full Stratton-Chu on device buffers (caller holds ctx->mu and the shared
// workspaces): [j_E; j_M] into ctx->full, one field evaluation over 2S
// right-hand sides (mult 1, no incident field), then the combination.
int field_full_core(bielcc_ctx ctx, MeshDev* m, int S, const double* JE, const double* JM, cplx k, cplx multE,
                    cplx multH, const bielcc_planewave* inc, const NumParamH& n, int P, const double* pts, double* E,
                    double* H, int precision, cudaStream_t s, bielcc_report* rep, unsigned long long* d_nf,
                    SingleEst* es) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t N = m->n_cells, bJ = (size_t)S * N * 48, bO = (size_t)S * P * 48;
    TRY(ctx->full.ensure(al(2 * bJ) + 2 * al(2 * bO) + 256));
    char* b = (char*)ctx->full.p;
    double* J2 = (double*)b;
    double* E2 = (double*)(b + al(2 * bJ));
    double* H2 = (double*)(b + al(2 * bJ) + al(2 * bO));
    TRY_CUDA(cudaMemcpyAsync(J2, JE, bJ, cudaMemcpyDeviceToDevice, s));
    TRY_CUDA(cudaMemcpyAsync((char*)J2 + bJ, JM, bJ, cudaMemcpyDeviceToDevice, s));
    if (P == 0) return BIELCC_OK;
    FieldArgs a{m, 2 * S, J2, k, mk(1.0, 0.0), nullptr, n, P, pts, E2, H2, precision};
    if (es) {  // the error sample of the combined field (the caller reports it after its sync)
        es->full = true;
        es->multE = multE;
        es->multH = multH;
        es->inc = inc;
        TRY(est_single_begin(ctx, a, s, *es, E, H, S));
    }
    TRY(field_device(ctx, a, s, rep, nullptr));
    FullInc fi;
    memset(&fi, 0, sizeof(fi));
    if (inc) {
        for (int g = 0; g < 3; g++) {
            fi.kvec[g] = inc->k_vec[g];
            fi.e0[g] = inc->e0[g];
        }
        fi.h_scale = inc->h_scale;
        fi.add_E = inc->add_E;
        fi.add_H = inc->add_H;
    }
    TRY_CUDA(launch_combine_full(E2, H2, S, P, multE, multH, pts, fi, E, H, d_nf, s));
    ctx->stats.kernel_launches += 1;
    if (es) TRY(est_single_finish(ctx, s, *es));
    return BIELCC_OK;
}

}  // namespace

extern "C" {

int bielcc_field_EH_full_device(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* JE_dev,
                                const double* JM_dev, double k_re, double k_im, double multE_re, double multE_im,
                                double multH_re, double multH_im, const bielcc_planewave* inc,
                                const bielcc_numparam* np, int n_pts, const double* pts_dev, double* E_dev,
                                double* H_dev, int precision, void* stream, bielcc_report* report) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (n_rhs < 1 || n_pts < 0 || !JE_dev || !JM_dev || (n_pts > 0 && (!pts_dev || !E_dev || !H_dev)))
        return set_error(BIELCC_ERR_ARG, "bad full-field arguments (n_rhs %d, n_pts %d)", n_rhs, n_pts);
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    if (report) memset(report, 0, sizeof(*report));
    TRY(ws_acquire(ctx, s));
    const bool sample = report && precision == BIELCC_PREC_MIXED && n_pts > 0;
    SingleEst es;
    TRY(field_full_core(ctx, m, n_rhs, JE_dev, JM_dev, mk(k_re, k_im), mk(multE_re, multE_im),
                        mk(multH_re, multH_im), inc, n, n_pts, pts_dev, E_dev, H_dev, precision, s, report, nullptr,
                        sample ? &es : nullptr));
    if (sample) {
        TRY_CUDA(cudaStreamSynchronize(s));
        est_single_report(ctx, es, report);
    }
    TRY(ws_release(ctx, s));
    return BIELCC_OK;
}

int bielcc_field_EH_full(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* J_E, const double* J_M,
                         double k_re, double k_im, double multE_re, double multE_im, double multH_re,
                         double multH_im, const bielcc_planewave* inc, const bielcc_numparam* np, int n_pts,
                         const double* pts, double* E, double* H, int precision, bielcc_report* report) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (n_rhs < 1 || n_pts < 0 || !J_E || !J_M || (n_pts > 0 && (!pts || !E || !H)))
        return set_error(BIELCC_ERR_ARG, "bad full-field arguments (n_rhs %d, n_pts %d)", n_rhs, n_pts);
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    if (report) memset(report, 0, sizeof(*report));
    cudaStream_t s = ctx->stream;
    const size_t P = n_pts, N = m->n_cells, S = n_rhs;
    const size_t bJ = S * N * 48, bP = P * 24, bO = S * P * 48;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    TRY(ctx->io.ensure(2 * al(bJ) + al(bP) + 2 * al(bO) + 256));
    char* io = (char*)ctx->io.p;
    double* dJE = (double*)io;
    double* dJM = (double*)(io + al(bJ));
    double* dP = (double*)(io + 2 * al(bJ));
    double* dE = (double*)(io + 2 * al(bJ) + al(bP));
    double* dH = (double*)(io + 2 * al(bJ) + al(bP) + al(bO));
    unsigned long long* d_nf = (unsigned long long*)(io + 2 * al(bJ) + al(bP) + 2 * al(bO));
    TRY(ws_acquire(ctx, s));
    TRY_CUDA(cudaMemcpyAsync(dJE, J_E, bJ, cudaMemcpyHostToDevice, s));
    TRY_CUDA(cudaMemcpyAsync(dJM, J_M, bJ, cudaMemcpyHostToDevice, s));
    if (P) TRY_CUDA(cudaMemcpyAsync(dP, pts, bP, cudaMemcpyHostToDevice, s));
    TRY_CUDA(cudaMemsetAsync(d_nf, 0, sizeof(unsigned long long), s));
    const bool sample = report && precision == BIELCC_PREC_MIXED && n_pts > 0;
    SingleEst es;
    TRY(field_full_core(ctx, m, n_rhs, dJE, dJM, mk(k_re, k_im), mk(multE_re, multE_im), mk(multH_re, multH_im),
                        inc, n, n_pts, dP, dE, dH, precision, s, report, d_nf, sample ? &es : nullptr));
    if (P) {
        TRY_CUDA(cudaMemcpyAsync(E, dE, bO, cudaMemcpyDeviceToHost, s));
        TRY_CUDA(cudaMemcpyAsync(H, dH, bO, cudaMemcpyDeviceToHost, s));
    }
    TRY_CUDA(cudaMemcpyAsync(ctx->h_nonfinite, d_nf, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    TRY_CUDA(cudaStreamSynchronize(s));
    TRY(ws_release(ctx, s));
    const unsigned long long nf = *ctx->h_nonfinite;
    int rc = nf ? set_error(BIELCC_ERR_NAN, "%llu output points hold NaN/Inf", nf) : BIELCC_OK;
    if (report) {
        report->n_nonfinite = (int64_t)nf;
        report->status = rc;
    }
    est_single_report(ctx, es, report);
    return rc;
}

int bielcc_field_EH(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* J, double k_re, double k_im,
                    double mult_re, double mult_im, const bielcc_planewave* inc, const bielcc_numparam* np, int n_pts,
                    const double* pts, double* E, double* H, int precision, bielcc_report* report) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (n_rhs < 1 || n_pts < 0 || !J || (n_pts > 0 && (!pts || !E)))
        return set_error(BIELCC_ERR_ARG, "bad field arguments (n_rhs %d, n_pts %d)", n_rhs, n_pts);
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    if (report) memset(report, 0, sizeof(*report));
    cudaStream_t s = ctx->stream;
    const size_t P = n_pts, N = m->n_cells, S = n_rhs;
    const size_t bJ = S * N * 3 * 16, bP = P * 3 * 8, bO = S * P * 3 * 16;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    TRY(ctx->io.ensure(al(bJ) + al(bP) + 2 * al(bO) + 256));
    char* io = (char*)ctx->io.p;
    double* dJ = (double*)io;
    double* dP = (double*)(io + al(bJ));
    double* dE = (double*)(io + al(bJ) + al(bP));
    double* dH = H ? (double*)(io + al(bJ) + al(bP) + al(bO)) : nullptr;
    unsigned long long* d_nf = (unsigned long long*)(io + al(bJ) + al(bP) + 2 * al(bO));
    TRY(ws_acquire(ctx, s));
    TRY_CUDA(cudaMemcpyAsync(dJ, J, bJ, cudaMemcpyHostToDevice, s));
    if (P) TRY_CUDA(cudaMemcpyAsync(dP, pts, bP, cudaMemcpyHostToDevice, s));
    TRY_CUDA(cudaMemsetAsync(d_nf, 0, sizeof(unsigned long long), s));
    FieldArgs a{m, n_rhs, dJ, mk(k_re, k_im), mk(mult_re, mult_im), inc, n, n_pts, dP, dE, dH, precision};
    // Mixed form: its relative L2 error against the FP64 form on a sample of
    // min(P, 256) points, evaluated on the side stream beside the main one.
    const bool sample = report && precision == BIELCC_PREC_MIXED && P > 0;
    FieldPending pm;
    SingleEst es;
    const WsSet wm = main_ws(ctx);
    if (sample) TRY(est_single_begin(ctx, a, s, es, dE, dH, n_rhs));
    if (P) TRY(field_begin(ctx, a, s, report, d_nf, wm, &pm));
    if (P) TRY(field_finish(ctx, pm, s, report, d_nf, wm));
    if (sample) TRY(est_single_finish(ctx, s, es));
    if (P) TRY_CUDA(cudaMemcpyAsync(E, dE, bO, cudaMemcpyDeviceToHost, s));
    if (P && H) TRY_CUDA(cudaMemcpyAsync(H, dH, bO, cudaMemcpyDeviceToHost, s));
    TRY_CUDA(cudaMemcpyAsync(ctx->h_nonfinite, d_nf, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    TRY_CUDA(cudaStreamSynchronize(s));
    TRY(ws_release(ctx, s));
    int rc = BIELCC_OK;
    unsigned long long nf = *ctx->h_nonfinite;
    if (nf) rc = set_error(BIELCC_ERR_NAN, "%llu output points hold NaN/Inf", nf);
    if (report) {
        report->n_nonfinite = (int64_t)nf;
        report->status = rc;
    }
    est_single_report(ctx, es, report);
    return rc;
}

}  // extern "C"

namespace {

// bielcc_field_job records -> device job records (node tables built first).
int jobs_to_dev(int n_jobs, const bielcc_field_job* jobs, const std::vector<MeshDev*>& meshes, const NumParamH& n,
                cudaStream_t s, std::vector<JobDev>& jd, bool* ck, int64_t* pairs) {
    jd.assign(n_jobs, JobDev{});
    *ck = false;
    *pairs = 0;
    for (int i = 0; i < n_jobs; i++) {
        const bielcc_field_job& j = jobs[i];
        MeshDev* m = meshes[i];
        TRY(ensure_tables(m, far_split_n(n), s));
        JobDev& d = jd[i];
        memset(&d, 0, sizeof(d));
        d.geo = m->geo;
        d.nodes32 = m->nodes32;
        d.nodes64 = m->nodes64;
        d.rho32 = m->rho32;
        d.verts = m->verts;
        d.nv = m->nv;
        d.n_cells = m->n_cells;
        d.pts = j.pts_dev;
        d.n_pts = j.n_pts;
        d.J = reinterpret_cast<const cplx*>(j.J_dev);
        d.n_rhs = j.n_rhs;
        d.k = mk(j.k_re, j.k_im);
        d.mult = mk(j.mult_re, j.mult_im);
        for (int g = 0; g < 3; g++) {
            d.kvec[g] = j.inc.k_vec[g];
            d.e0[g] = j.inc.e0[g];
        }
        d.h_scale = j.inc.h_scale;
        d.add_E = j.inc.add_E;
        d.add_H = j.inc.add_H;
        d.E = j.E_dev;
        d.H = j.H_dev;
        *ck = *ck || j.k_im != 0.;
        *pairs += (int64_t)j.n_pts * m->n_cells * j.n_rhs;
    }
    return BIELCC_OK;
}

int check_jobs(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs, std::vector<MeshDev*>& meshes) {
    meshes.resize(n_jobs);
    for (int i = 0; i < n_jobs; i++) {
        const bielcc_field_job& j = jobs[i];
        TRY(get_mesh(ctx, j.mesh, &meshes[i]));
        if (j.n_rhs < 1 || j.n_pts < 0 || !j.J_dev || (j.n_pts > 0 && (!j.pts_dev || !j.E_dev)))
            return set_error(BIELCC_ERR_ARG, "job %d: bad sizes or null buffers", i);
    }
    return BIELCC_OK;
}

// Error sample of a mixed batch: per job min(P, 32) points spread over its set
// and its first min(S, 4) right-hand sides, evaluated as one FP64 batch on the
// side stream (side workspaces) beside the main batch, then compared with the
// main outputs on the device: each job's estimate to its est_dev, the sums
// over all jobs to h_total[4], [5].
struct BatchEst {
    bool on = false;
    int n_jobs = 0, total_q = 0;
    std::vector<ErrJob> ej;
    std::vector<JobDev> js;
    ErrJob* d_ej = nullptr;
    double *spts = nullptr, *nd = nullptr, *sums = nullptr;
    BatchPlan bp;
    BatchDevPtrs d{};
    int l1 = 0;
};

int batch_est_begin(bielcc_ctx ctx, const std::vector<JobDev>& jd, const bielcc_field_job* jobs, const NumParamH& n,
                    bool ck, double item_cost, cudaStream_t s, BatchEst& e) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    e.on = true;
    e.n_jobs = (int)jd.size();
    e.ej.assign(jd.size(), ErrJob{});
    size_t tq = 0, tout = 0;
    for (size_t i = 0; i < jd.size(); i++) {
        const int Q = std::min(jd[i].n_pts, 32), Ss = std::min(jd[i].n_rhs, 4);
        tq += Q;
        tout += (size_t)Ss * Q;
    }
    e.total_q = (int)tq;
    const size_t b_ej = al(jd.size() * sizeof(ErrJob)), b_nd = al(jd.size() * 16 + 16), b_p = al(tq * 24),
                 b_o = al(tout * 48);
    TRY(ctx->side_io.ensure(b_ej + b_nd + b_p + 2 * b_o + 256));
    char* b = (char*)ctx->side_io.p;
    e.d_ej = (ErrJob*)b;
    e.nd = (double*)(b + b_ej);
    e.sums = e.nd + 2 * jd.size();
    e.spts = (double*)(b + b_ej + b_nd);
    double* Eq = (double*)(b + b_ej + b_nd + b_p);
    double* Hq = (double*)(b + b_ej + b_nd + b_p + b_o);
    e.js.assign(jd.begin(), jd.end());
    size_t oq = 0, oo = 0;
    for (size_t i = 0; i < jd.size(); i++) {
        const JobDev& j = jd[i];
        const int Q = std::min(j.n_pts, 32), Ss = std::min(j.n_rhs, 4);
        ErrJob& r = e.ej[i];
        r.pts = j.pts;
        r.P = j.n_pts;
        r.Q = Q;
        r.S = j.n_rhs;
        r.Ss = Ss;
        r.off = (int)oq;
        r.E = j.E;
        r.H = j.H;
        r.E32 = j.E32;
        r.H32 = j.H32;
        r.Eq = Eq + 2 * 3 * oo;
        r.Hq = (j.H || j.H32) ? Hq + 2 * 3 * oo : nullptr;
        r.est_dev = jobs ? jobs[i].est_dev : nullptr;
        JobDev& q = e.js[i];
        q.pts = e.spts + 3 * oq;
        q.n_pts = Q;
        q.n_rhs = Ss;  // the first Ss right-hand sides: the leading part of J
        q.E = const_cast<double*>(r.Eq);
        q.H = const_cast<double*>(r.Hq);
        q.E32 = q.H32 = nullptr;
        q.nonfinite = nullptr;
        oq += Q;
        oo += (size_t)Ss * Q;
    }
    TRY_CUDA(cudaEventRecord(ctx->side_in, s));
    TRY_CUDA(cudaStreamWaitEvent(ctx->side, ctx->side_in, 0));
    TRY_CUDA(cudaMemcpyAsync(e.d_ej, e.ej.data(), jd.size() * sizeof(ErrJob), cudaMemcpyHostToDevice, ctx->side));
    TRY_CUDA(err_gather(e.d_ej, e.n_jobs, e.spts, ctx->side));
    plan_batch(e.bp, e.js, far_split_n(n), false, item_cost, false);
    TRY(ctx->side_ws.ensure(e.bp.ws_bytes));
    TRY_CUDA(batch_stage1(e.bp, ctx->side_ws.p, n.analytic_calc, far_split_n(n), ck, ctx->side, &e.d, &e.l1));
    TRY_CUDA(batch_status_to_host(e.d, ctx->h_side_total, ctx->side));
    return BIELCC_OK;
}

int batch_est_finish(bielcc_ctx ctx, const NumParamH& n, cudaStream_t s, BatchEst& e) {
    TRY_CUDA(cudaStreamSynchronize(ctx->side));
    if (batch_timed_out(ctx->h_side_total))
        return set_error(BIELCC_ERR_TIMEOUT, "batched far kernel: a bounded wait ran out");
    const long long n_near = *ctx->h_side_total;
    if (n_near > 0) TRY(ctx->side_pair_ws.ensure(batch_pair_ws_bytes(n_near)));
    DNP dn{n.eps, n.rs, n.rs_seg, n.analytic_calc, n.n_start, n.n_start_seg, n.p_max, n.p_max_seg};
    int l2 = 0;
    TRY_CUDA(batch_stage2(e.bp, e.d, n_near, ctx->side_pair_ws.p, dn, nullptr, ctx->side, &l2));
    TRY_CUDA(cudaEventRecord(ctx->side_out, ctx->side));
    TRY_CUDA(cudaStreamWaitEvent(s, ctx->side_out, 0));
    TRY_CUDA(err_compare(e.d_ej, e.n_jobs, e.nd, e.sums, s));
    TRY_CUDA(cudaMemcpyAsync(ctx->h_total + 4, e.sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    ctx->stats.kernel_launches += e.l1 + l2 + 3;
    return BIELCC_OK;
}

int field_batch_locked(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs, const NumParamH& n, int precision,
                       cudaStream_t s, bielcc_report* report, double item_cost) {
    std::vector<MeshDev*> meshes;
    TRY(check_jobs(ctx, n_jobs, jobs, meshes));
    if (report) memset(report, 0, sizeof(*report));
    TRY(ws_acquire(ctx, s));
    // p_max >= 3 (the convergence-test marks) and far splits beyond the batched
    // kernel's staging run outside it: one call per job
    if (far_adaptive(n) || far_split_n(n) > kBatchMaxNStart) {
        for (int i = 0; i < n_jobs; i++) {
            const bielcc_field_job& j = jobs[i];
            FieldArgs a{meshes[i], j.n_rhs, j.J_dev, mk(j.k_re, j.k_im), mk(j.mult_re, j.mult_im), &j.inc, n,
                        j.n_pts, j.pts_dev, j.E_dev, j.H_dev, precision};
            bielcc_report r{};
            TRY(field_device(ctx, a, s, &r, nullptr));
            if (report) {
                report->n_pairs += r.n_pairs * j.n_rhs;
                report->n_near_pairs += r.n_near_pairs;
            }
        }
        TRY(ws_release(ctx, s));
        return BIELCC_OK;
    }
    std::vector<JobDev> jd;
    bool ck = false;
    int64_t pairs = 0;
    TRY(jobs_to_dev(n_jobs, jobs, meshes, n, s, jd, &ck, &pairs));
    // mixed: the error sample, with a report or when a job asks for its estimate
    bool want_est = report != nullptr;
    for (int i = 0; i < n_jobs; i++) want_est = want_est || jobs[i].est_dev;
    BatchEst es;
    if (precision == BIELCC_PREC_MIXED && want_est && n_jobs > 0)
        TRY(batch_est_begin(ctx, jd, jobs, n, ck, item_cost, s, es));
    BatchPlan bp;
    plan_batch(bp, jd, far_split_n(n), precision == BIELCC_PREC_MIXED, item_cost, ctx->batch_tc,
               ctx_batch_split_cap(ctx));
    TRY(ctx->ws.ensure(bp.ws_bytes));
    TRY(ctx->scratch_small.ensure(256));
    BatchDevPtrs d;
    int l1 = 0, l2 = 0;
    TRY_CUDA(batch_stage1(bp, ctx->ws.p, n.analytic_calc, far_split_n(n), ck, s, &d, &l1));
    TRY_CUDA(batch_status_to_host(d, ctx->h_total, s));
    TRY_CUDA(cudaStreamSynchronize(s));
    if (batch_timed_out(ctx->h_total)) return set_error(BIELCC_ERR_TIMEOUT, "batched far kernel: a bounded wait ran out");
    const long long n_near = *ctx->h_total;
    if (n_near > 0) TRY(ctx->pair_ws.ensure(batch_pair_ws_bytes(n_near)));
    DNP dn{n.eps, n.rs, n.rs_seg, n.analytic_calc, n.n_start, n.n_start_seg, n.p_max, n.p_max_seg};
    TRY_CUDA(batch_stage2(bp, d, n_near, ctx->pair_ws.p, dn, nullptr, s, &l2));
    if (es.on) TRY(batch_est_finish(ctx, n, s, es));
    ctx->stats.kernel_launches += l1 + l2;
    ctx->stats.far_launches += 1;
    ctx->stats.far_pairs += pairs;
    ctx->stats.far_ctas = bp.grid;
    if (report) {
        report->n_pairs = pairs;
        report->n_near_pairs = n_near;
        if (es.on) {  // the estimate of the whole batch: wait for the stream
            TRY_CUDA(cudaStreamSynchronize(s));
            const double* v = reinterpret_cast<const double*>(ctx->h_total + 4);
            report->est_rel_l2 = v[1] > 0. ? sqrt(v[0] / v[1]) : 0.;
            report->est_sample = es.total_q;
        }
    }
    TRY(ws_release(ctx, s));
    return BIELCC_OK;
}

}  // namespace

extern "C" {

int bielcc_field_EH_batch(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs, const bielcc_numparam* np,
                          int precision, void* stream, bielcc_report* report) {
    TRY(enter(ctx));
    if (n_jobs < 0 || (n_jobs > 0 && !jobs)) return set_error(BIELCC_ERR_ARG, "bad job list");
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    NumParamH n = to_np(np);
    TRY(check_np(n));
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return field_batch_locked(ctx, n_jobs, jobs, n, precision, s, report, ctx->batch_item_cost);
}

}  // extern "C"

// A batch planned once for repeated evaluation (bielcc_batch_plan_*): its
// own workspaces (never shared with the context's), the near-pair list and
// FP64 near moments of the first evaluation, and the CUDA graph of the
// replay sequence.
struct bielcc_batch_plan_s {
    bielcc_ctx ctx = nullptr;
    BatchPlan bp;
    BatchDevPtrs d{};
    void* ws = nullptr;
    void* pair_ws = nullptr;
    long long n_near = 0;
    double analytic_calc = 3.0;
    int n_start = 8;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t pairs = 0;
};

namespace {

void free_plan(bielcc_batch_plan p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    cudaFree(p->ws);
    cudaFree(p->pair_ws);
    delete p;
}

}  // namespace

extern "C" {

int bielcc_batch_plan_create(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs, const bielcc_numparam* np,
                             int precision, void* stream, bielcc_batch_plan* out, bielcc_report* report) {
    TRY(enter(ctx));
    if (n_jobs < 1 || !jobs || !out) return set_error(BIELCC_ERR_ARG, "bad job list");
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (far_adaptive(n) || far_split_n(n) > kBatchMaxNStart)
        return set_error(BIELCC_ERR_UNSUPPORTED,
                         "batch plans run the batched kernel: p_max <= 2 and a far split (n_start, 2 n_start "
                         "for p_max = 2) of at most 22");
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    std::vector<MeshDev*> meshes;
    TRY(check_jobs(ctx, n_jobs, jobs, meshes));
    bielcc_batch_plan p = new (std::nothrow) bielcc_batch_plan_s;
    if (!p) return set_error(BIELCC_ERR_OOM, "out of host memory");
    p->ctx = ctx;
    p->analytic_calc = n.analytic_calc;
    p->n_start = n.n_start;
    std::vector<JobDev> jd;
    bool ck = false;
    int rc = jobs_to_dev(n_jobs, jobs, meshes, n, s, jd, &ck, &p->pairs);
    cudaError_t e = cudaSuccess;
    int l1 = 0, l2 = 0;
    if (rc == BIELCC_OK) {
        // A plan keeps the moments only when they fit one wave of the buffer:
        // its replays then run the contraction alone. Over several waves a
        // replay would evaluate every moment again, so it runs the fused kernel
        // (unless every batch is set to split).
        const bool mixed = precision == BIELCC_PREC_MIXED;
        plan_batch(p->bp, jd, far_split_n(n), mixed, ctx->batch_item_cost, ctx->batch_tc, ctx->batch_split);
        if (p->bp.split && p->bp.waves.size() > 1 && !ctx->batch_split_all)
            plan_batch(p->bp, jd, far_split_n(n), mixed, ctx->batch_item_cost, ctx->batch_tc, 0);
        e = cudaMalloc(&p->ws, p->bp.ws_bytes);
        if (e == cudaSuccess) e = batch_stage1(p->bp, p->ws, n.analytic_calc, far_split_n(n), ck, s, &p->d, &l1);
        if (e == cudaSuccess) e = batch_status_to_host(p->d, ctx->h_total, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && batch_timed_out(ctx->h_total))
            rc = set_error(BIELCC_ERR_TIMEOUT, "batched far kernel: a bounded wait ran out");
    }
    if (rc == BIELCC_OK && e == cudaSuccess) {
        p->n_near = *ctx->h_total;
        if (p->n_near > 0) e = cudaMalloc(&p->pair_ws, batch_pair_ws_bytes(p->n_near));
        DNP dn{n.eps, n.rs, n.rs_seg, n.analytic_calc, n.n_start, n.n_start_seg, n.p_max, n.p_max_seg};
        if (e == cudaSuccess) e = batch_stage2(p->bp, p->d, p->n_near, p->pair_ws, dn, nullptr, s, &l2);
    }
    // capture the replay sequence on a private stream (capture needs a stream
    // other than the legacy default one), then instantiate it
    cudaStream_t cs = nullptr;
    if (rc == BIELCC_OK && e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (rc == BIELCC_OK && e == cudaSuccess) {
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e1 = batch_replay(p->bp, p->d, p->n_near, p->pair_ws, n.analytic_calc, far_split_n(n), cs);
            cudaError_t e2 = cudaStreamEndCapture(cs, &p->graph);
            e = e1 != cudaSuccess ? e1 : e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    }
    if (cs) cudaStreamDestroy(cs);
    if (rc == BIELCC_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (rc != BIELCC_OK || e != cudaSuccess) {
        cudaGetLastError();
        cudaStreamSynchronize(s);
        free_plan(p);
        return rc != BIELCC_OK ? rc : set_error(BIELCC_ERR_CUDA, "batch plan: %s", cudaGetErrorString(e));
    }
    ctx->stats.kernel_launches += l1 + l2;
    if (report) {
        memset(report, 0, sizeof(*report));
        report->n_pairs = p->pairs;
        report->n_near_pairs = p->n_near;
    }
    *out = p;
    return BIELCC_OK;
}

int bielcc_batch_plan_launch(bielcc_batch_plan p, void* stream) {
    if (!p) return set_error(BIELCC_ERR_ARG, "null plan");
    TRY(enter(p->ctx));
    cudaStream_t s = stream ? (cudaStream_t)stream : p->ctx->stream;
    TRY_CUDA(cudaGraphLaunch(p->exec, s));
    return BIELCC_OK;
}

int bielcc_batch_plan_destroy(bielcc_batch_plan p) {
    if (!p) return BIELCC_OK;
    TRY(enter(p->ctx));
    TRY_CUDA(cudaDeviceSynchronize());
    free_plan(p);
    return BIELCC_OK;
}

int bielcc_batch_autotune(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs, const bielcc_numparam* np,
                          int precision, void* stream, double* item_cost) {
    TRY(enter(ctx));
    if (n_jobs < 1 || !jobs) return set_error(BIELCC_ERR_ARG, "autotuning needs a non-empty batch");
    NumParamH n = to_np(np);
    TRY(check_np(n));
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    cudaEvent_t e0, e1;
    TRY_CUDA(cudaEventCreate(&e0));
    TRY_CUDA(cudaEventCreate(&e1));
    const double candidates[] = {0.5e6, 1e6, 2e6, 4e6, 8e6, 16e6};
    double best = ctx->batch_item_cost, best_ms = 1e30;
    int rc = BIELCC_OK;
    for (int rep = 0; rep < 2 && rc == BIELCC_OK; rep++) {  // first sweep warms up
        for (double c : candidates) {
            cudaEventRecord(e0, s);
            rc = field_batch_locked(ctx, n_jobs, jobs, n, precision, s, nullptr, c);
            if (rc != BIELCC_OK) break;
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep == 1 && ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != BIELCC_OK) return rc;
    ctx->batch_item_cost = best;
    if (item_cost) *item_cost = best;
    return BIELCC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- per-pair entry points
namespace {

// Host-buffer batch helper: copies `ins` to the device, runs `launch` with
// their device pointers, copies `out_bytes` back into `out`.
// `back` (optional): input index whose device copy is written back to
// `back_host` after the launch (in/out records such as kernel parameters).
template <typename L>
int run_batch(bielcc_ctx ctx, std::initializer_list<std::pair<const void*, size_t>> ins, void* out, size_t out_bytes,
              L launch, int back = -1, void* back_host = nullptr) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tot = al(out_bytes);
    for (auto& in : ins) tot += al(in.second);
    TRY(ctx->io.ensure(tot + 256));
    cudaStream_t s = ctx->stream;
    TRY(ws_acquire(ctx, s));
    char* p = (char*)ctx->io.p;
    std::vector<const void*> dptrs;
    for (auto& in : ins) {
        if (in.first && in.second) TRY_CUDA(cudaMemcpyAsync(p, in.first, in.second, cudaMemcpyHostToDevice, s));
        dptrs.push_back(in.first ? p : nullptr);
        p += al(in.second);
    }
    TRY_CUDA(launch(dptrs, (void*)p, s));
    if (out_bytes) TRY_CUDA(cudaMemcpyAsync(out, p, out_bytes, cudaMemcpyDeviceToHost, s));
    if (back >= 0 && back_host) {
        size_t b = (ins.begin() + back)->second;
        TRY_CUDA(cudaMemcpyAsync(back_host, dptrs[back], b, cudaMemcpyDeviceToHost, s));
    }
    TRY_CUDA(cudaStreamSynchronize(s));
    TRY(ws_release(ctx, s));
    return BIELCC_OK;
}

int check_nv(int nv) {
    if (nv != 3 && nv != 4) return set_error(BIELCC_ERR_ARG, "n_vert must be 3 or 4, got %d", nv);
    return BIELCC_OK;
}

int check_quad_params(int n_start, int p_max) {
    if (n_start < 1 || n_start > 4096 || p_max < 1 || p_max > 20)
        return set_error(BIELCC_ERR_ARG, "n_start %d / p_max %d out of range", n_start, p_max);
    return BIELCC_OK;
}

}  // namespace

extern "C" {

int bielcc_pair_op(bielcc_ctx ctx, int op, int n_vert, int n_pairs, const double* cells, const double* x,
                   const double* j, double k_re, double k_im, const bielcc_numparam* np, double* res) {
    TRY(enter(ctx));
    TRY(check_nv(n_vert));
    if (op < 0 || op >= BIELCC_OP_COUNT) return set_error(BIELCC_ERR_ARG, "unknown operator %d", op);
    if (n_pairs < 0 || (n_pairs > 0 && (!cells || !x || !j || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    return run_batch(ctx, {{cells, N * n_vert * 24}, {x, N * 24}, {j, N * 48}}, res, N * 48,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_pair_op(op, n_vert, n_pairs, (const double*)d[0], (const double*)d[1],
                                               (const double*)d[2], mk(k_re, k_im), n, (double*)o, s);
                     });
}

int bielcc_integrand_info(int integrand, int* idim, int* is_complex) {
    if (integrand < 0 || integrand >= BIELCC_F_COUNT) return set_error(BIELCC_ERR_ARG, "unknown integrand %d", integrand);
    if (idim) *idim = integrand_dim(integrand);
    if (is_complex) *is_complex = integrand_complex(integrand) ? 1 : 0;
    return BIELCC_OK;
}

// Pair integrands F(x, y), and F = 1, for the *_pnt forms.
static int check_pair_integrand(int integrand) {
    if (integrand < 0 || integrand >= BIELCC_F_COUNT) return set_error(BIELCC_ERR_ARG, "unknown integrand %d", integrand);
    if (integrand_one_point(integrand) && integrand != BIELCC_F_ONE)
        return set_error(BIELCC_ERR_ARG, "integrand %d is a function of one point: use bielcc_integral", integrand);
    return BIELCC_OK;
}

// One-point integrands F(x) for IntegralUniversal and the segment F(x) overload.
static int check_one_point_integrand(int integrand) {
    if (integrand < 0 || integrand >= BIELCC_F_COUNT || !integrand_one_point(integrand))
        return set_error(BIELCC_ERR_ARG, "integrand %d is not a function of one point F(x)", integrand);
    return BIELCC_OK;
}

int bielcc_integral(bielcc_ctx ctx, int integrand, int n_vert, int n_cells, const double* cells,
                    bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    TRY(enter(ctx));
    TRY(check_nv(n_vert));
    TRY(check_quad_params(n_start, p_max));
    TRY(check_one_point_integrand(integrand));
    if (n_cells < 0 || (n_cells > 0 && (!cells || !kp || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_cells == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_cells;
    int idim = integrand_dim(integrand);
    size_t ob = N * idim * (integrand_complex(integrand) ? 16 : 8);
    return run_batch(ctx, {{cells, N * n_vert * 24}, {kp, N * sizeof(KParamDev)}}, res, ob,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_integral_pnt(integrand, n_vert, n_cells, (const double*)d[0], nullptr,
                                                    (KParamDev*)d[1], n_start, p_max, eps, (double*)o, s);
                     },
                     1, kp);
}

int bielcc_integral_seg(bielcc_ctx ctx, int integrand, int n_segs, const double* a, const double* b,
                        bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    TRY(enter(ctx));
    TRY(check_quad_params(n_start, p_max));
    TRY(check_one_point_integrand(integrand));
    if (n_segs < 0 || (n_segs > 0 && (!a || !b || !kp || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_segs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_segs;
    int idim = integrand_dim(integrand);
    size_t ob = N * idim * (integrand_complex(integrand) ? 16 : 8);
    return run_batch(ctx, {{a, N * 24}, {b, N * 24}, {kp, N * sizeof(KParamDev)}}, res, ob,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_integral_seg(integrand, n_segs, (const double*)d[0], (const double*)d[1],
                                                    nullptr, (KParamDev*)d[2], n_start, p_max, eps, (double*)o, s);
                     },
                     2, kp);
}

int bielcc_integral_pnt(bielcc_ctx ctx, int integrand, int n_vert, int n_pairs, const double* cells, const double* x,
                        bielcc_kernelparam* kp, int n_start, int p_max, double eps, double* res) {
    TRY(enter(ctx));
    TRY(check_nv(n_vert));
    TRY(check_quad_params(n_start, p_max));
    TRY(check_pair_integrand(integrand));
    if (n_pairs < 0 || (n_pairs > 0 && (!cells || !x || !kp || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    static_assert(sizeof(bielcc_kernelparam) == sizeof(KParamDev), "kernel-parameter layouts differ");
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    int idim = integrand_dim(integrand);
    size_t ob = N * idim * (integrand_complex(integrand) ? 16 : 8);
    return run_batch(ctx, {{cells, N * n_vert * 24}, {x, N * 24}, {kp, N * sizeof(KParamDev)}}, res, ob,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_integral_pnt(integrand, n_vert, n_pairs, (const double*)d[0],
                                                    (const double*)d[1], (KParamDev*)d[2], n_start, p_max, eps,
                                                    (double*)o, s);
                     },
                     2, kp);
}

int bielcc_integral_seg_pnt(bielcc_ctx ctx, int integrand, int n_pairs, const double* a, const double* b,
                            const double* x, bielcc_kernelparam* kp, int n_start, int p_max, double eps,
                            double* res) {
    TRY(enter(ctx));
    TRY(check_quad_params(n_start, p_max));
    TRY(check_pair_integrand(integrand));
    if (n_pairs < 0 || (n_pairs > 0 && (!a || !b || !x || !kp || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    int idim = integrand_dim(integrand);
    size_t ob = N * idim * (integrand_complex(integrand) ? 16 : 8);
    return run_batch(ctx, {{a, N * 24}, {b, N * 24}, {x, N * 24}, {kp, N * sizeof(KParamDev)}}, res, ob,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_integral_seg(integrand, n_pairs, (const double*)d[0], (const double*)d[1],
                                                    (const double*)d[2], (KParamDev*)d[3], n_start, p_max, eps,
                                                    (double*)o, s);
                     },
                     3, kp);
}

int bielcc_k0(bielcc_ctx ctx, int integrand, int common, int n_vert, int n_pairs, const double* cells,
              const double* x, const double* j, bielcc_kernelparam* kp, int n_start_seg, int p_max_seg,
              double eps, double* res) {
    TRY(enter(ctx));
    TRY(check_nv(n_vert));
    TRY(check_quad_params(n_start_seg, p_max_seg));
    if (integrand < 0 || integrand >= BIELCC_F_COUNT || integrand_one_point(integrand) ||
        !integrand_complex(integrand) || integrand_dim(integrand) != 3)
        return set_error(BIELCC_ERR_ARG, "K0 needs a complex 3-vector integrand, got %d", integrand);
    if (n_pairs < 0 || (n_pairs > 0 && (!cells || !x || !kp || !res || (!common && !j))))
        return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    return run_batch(ctx, {{cells, N * n_vert * 24}, {x, N * 24}, {common ? nullptr : j, N * 48},
                           {kp, N * sizeof(KParamDev)}},
                     res, N * 48, [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_k0(integrand, common, n_vert, n_pairs, (const double*)d[0],
                                          (const double*)d[1], (const double*)d[2], (KParamDev*)d[3],
                                          n_start_seg, p_max_seg, eps, (double*)o, s);
                     },
                     3, kp);
}

int bielcc_integral_1divr(bielcc_ctx ctx, int n_vert, int n_pairs, const double* cells, const double* x,
                          double* res) {
    TRY(enter(ctx));
    TRY(check_nv(n_vert));
    if (n_pairs < 0 || (n_pairs > 0 && (!cells || !x || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    return run_batch(ctx, {{cells, N * n_vert * 24}, {x, N * 24}}, res, N * 8,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_analytic(0, n_vert, n_pairs, (const double*)d[0], nullptr, (const double*)d[1],
                                                0., 1, 1, 0., mk(0, 0), (double*)o, s);
                     });
}

int bielcc_integral_grad1divr_seg(bielcc_ctx ctx, int n_pairs, const double* a, const double* b, const double* x,
                                  double* res) {
    TRY(enter(ctx));
    if (n_pairs < 0 || (n_pairs > 0 && (!a || !b || !x || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    return run_batch(ctx, {{a, N * 24}, {b, N * 24}, {x, N * 24}}, res, N * 24,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_analytic(1, 3, n_pairs, (const double*)d[0], (const double*)d[1],
                                                (const double*)d[2], 0., 1, 1, 0., mk(0, 0), (double*)o, s);
                     });
}

int bielcc_integral_surf_simplepot_h_hs(bielcc_ctx ctx, int n_vert, int n_pairs, const double* cells,
                                        const double* x, double analytic_r, int n_start, int p_max, double eps,
                                        double k_re, double k_im, double* res) {
    TRY(enter(ctx));
    TRY(check_nv(n_vert));
    TRY(check_quad_params(n_start, p_max));
    if (n_pairs < 0 || (n_pairs > 0 && (!cells || !x || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    return run_batch(ctx, {{cells, N * n_vert * 24}, {x, N * 24}}, res, N * 16,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_analytic(2, n_vert, n_pairs, (const double*)d[0], nullptr, (const double*)d[1],
                                                analytic_r, n_start, p_max, eps, mk(k_re, k_im), (double*)o, s);
                     });
}

int bielcc_integral_seg_gradsimplepot_h_hs(bielcc_ctx ctx, int n_pairs, const double* a, const double* b,
                                           const double* x, double analytic_r, int n_start, int p_max, double eps,
                                           double k_re, double k_im, double* res) {
    TRY(enter(ctx));
    TRY(check_quad_params(n_start, p_max));
    if (n_pairs < 0 || (n_pairs > 0 && (!a || !b || !x || !res))) return set_error(BIELCC_ERR_ARG, "null buffer");
    if (n_pairs == 0) return BIELCC_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    size_t N = n_pairs;
    return run_batch(ctx, {{a, N * 24}, {b, N * 24}, {x, N * 24}}, res, N * 48,
                     [&](std::vector<const void*>& d, void* o, cudaStream_t s) {
                         return launch_analytic(3, 3, n_pairs, (const double*)d[0], (const double*)d[1],
                                                (const double*)d[2], analytic_r, n_start, p_max, eps, mk(k_re, k_im),
                                                (double*)o, s);
                     });
}

// Collocation assembly: implemented in assemble.cu's stages, driven here.
int bielcc_assemble_K_device(bielcc_ctx ctx, bielcc_mesh mesh, double k_re, double k_im, const bielcc_numparam* np,
                             int layout, int out_c64, int precision, void* A_dev, void* stream,
                             bielcc_report* report) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, mesh, &m));
    NumParamH n = to_np(np);
    TRY(check_np(n));
    if (layout != BIELCC_LAYOUT_TAU2 && layout != BIELCC_LAYOUT_FULL3)
        return set_error(BIELCC_ERR_ARG, "unknown layout %d", layout);
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    if (!A_dev) return set_error(BIELCC_ERR_ARG, "null matrix");
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    TRY(ws_acquire(ctx, s));
    TRY(ensure_far_tables(m, n, s));
    AssembleLaunch a{m, mk(k_re, k_im), n, layout, out_c64 ? 1 : 0, precision, A_dev};
    TRY(ctx->ws.ensure(assemble_ws_base_bytes(a)));
    TRY(ctx->scratch_small.ensure(256));
    long long* d_total = (long long*)ctx->scratch_small.p;
    TRY_CUDA(assemble_stage1(a, ctx->ws.p, d_total, s));
    TRY_CUDA(cudaMemcpyAsync(ctx->h_total, d_total, sizeof(long long), cudaMemcpyDeviceToHost, s));
    TRY_CUDA(cudaStreamSynchronize(s));
    long long n_near = *ctx->h_total;
    if (n_near > 0) TRY(ctx->pair_ws.ensure((size_t)n_near * (2 * sizeof(int)) + 1024));
    TRY_CUDA(assemble_stage2(a, ctx->ws.p, n_near, ctx->pair_ws.p, s));
    ctx->stats.kernel_launches += 3 + (n_near > 0 ? 2 : 0);
    // mixed with a report: min(N, 16) sampled rows in FP64 against the stored
    // matrix, and the call waits for the stream to fill est_rel_l2
    const int R = (report && precision == BIELCC_PREC_MIXED) ? std::min(m->n_cells, 16) : 0;
    if (R > 0) {
        TRY(ctx->side_io.ensure(assemble_error_ws_bytes(a, R) + 256));
        double* sums = (double*)((char*)ctx->side_io.p + assemble_error_ws_bytes(a, R));
        TRY_CUDA(assemble_error_sample(a, R, ctx->side_io.p, sums, s));
        TRY_CUDA(cudaMemcpyAsync(ctx->h_total + 4, sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        TRY_CUDA(cudaStreamSynchronize(s));
        ctx->stats.kernel_launches += 2;
    }
    TRY(ws_release(ctx, s));
    if (report) {
        memset(report, 0, sizeof(*report));
        report->n_pairs = (int64_t)m->n_cells * m->n_cells;
        report->n_near_pairs = n_near;
        if (R > 0) {
            const double* v = reinterpret_cast<const double*>(ctx->h_total + 4);
            report->est_rel_l2 = v[1] > 0. ? sqrt(v[0] / v[1]) : 0.;
            report->est_sample = R;
        }
    }
    return BIELCC_OK;
}

int bielcc_solve_pec(bielcc_ctx ctx, bielcc_mesh mesh, double k_re, double k_im, double multE_re, double multE_im,
                     const bielcc_planewave* inc, const bielcc_numparam* np, int precision, double* J_host,
                     bielcc_report* report) {
    TRY(enter(ctx));
    if (!inc || !J_host) return set_error(BIELCC_ERR_ARG, "solve_pec: incident wave and J required");
    if (multE_re == 0. && multE_im == 0.) return set_error(BIELCC_ERR_ARG, "solve_pec: multE must not be 0");
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_error(BIELCC_ERR_ARG, "unknown precision %d", precision);
    MeshDev* m;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        TRY(get_mesh(ctx, mesh, &m));
    }
    const int N = m->n_cells, dim = 2 * N;
    const int c64 = precision == BIELCC_PREC_MIXED ? 1 : 0;
    const size_t elt = c64 ? 8 : 16;
    void* A = nullptr;
    void* b = nullptr;
    double* dJ = nullptr;
    if (cudaMalloc(&A, (size_t)dim * dim * elt) != cudaSuccess || cudaMalloc(&b, (size_t)dim * elt) != cudaSuccess ||
        cudaMalloc((void**)&dJ, (size_t)N * 48) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(A);
        cudaFree(b);
        return set_error(BIELCC_ERR_OOM, "solve_pec: device allocation of the %d x %d system failed", dim, dim);
    }
    int rc = bielcc_assemble_K_device(ctx, mesh, k_re, k_im, np, BIELCC_LAYOUT_TAU2, c64, precision, A, nullptr,
                                      report);
    int info = 0;
    if (rc == BIELCC_OK) {
        // b_(i,a) = -tau_a(i) . E_inc(c_i) / multE
        const double m2 = multE_re * multE_re + multE_im * multE_im;
        const cplx scale = mk(-multE_re / m2, multE_im / m2);  // -1 / multE
        cudaError_t e = launch_efie_rhs(m->geo, N, inc->k_vec, inc->e0, scale, c64, b, ctx->stream);
        if (e != cudaSuccess) rc = cuda_status(e, "efie rhs", __LINE__);
    }
    if (rc == BIELCC_OK) rc = bielcc_solve_dense(dim, 1, c64, A, b, ctx->stream, &info);
    if (rc == BIELCC_OK) {
        cudaError_t e = launch_basis_currents(m->geo, N, b, c64, dJ, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(J_host, dJ, (size_t)N * 48, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_status(e, "solve_pec currents", __LINE__);
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(A);
    cudaFree(b);
    cudaFree(dJ);
    if (report) report->status = rc;
    return rc;
}

int bielcc_assemble_K(bielcc_ctx ctx, bielcc_mesh mesh, double k_re, double k_im, const bielcc_numparam* np,
                      int layout, int out_c64, int precision, void* A_host, bielcc_report* report) {
    TRY(enter(ctx));
    MeshDev* m;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        TRY(get_mesh(ctx, mesh, &m));
    }
    if (!A_host) return set_error(BIELCC_ERR_ARG, "null matrix");
    size_t dim = (size_t)(layout == BIELCC_LAYOUT_FULL3 ? 3 : 2) * m->n_cells;
    size_t bytes = dim * dim * (out_c64 ? 8 : 16);
    void* dA = nullptr;
    TRY_CUDA(cudaMalloc(&dA, bytes));
    int rc = bielcc_assemble_K_device(ctx, mesh, k_re, k_im, np, layout, out_c64, precision, dA, nullptr, report);
    if (rc == BIELCC_OK) {
        // the download runs on the context's (non-blocking) stream, after the kernels
        cudaError_t e = cudaMemcpyAsync(A_host, dA, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_status(e, "matrix download", __LINE__);
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(dA);
    return rc;
}

}  // extern "C"

namespace bielcc_gpu {

// The server's view of a context's mesh: node tables built for `n_start`
// (and finished) before the mesh joins a batch on another stream.
int server_mesh(bielcc_ctx ctx, bielcc_mesh id, int n_start, MeshDev** out) {
    TRY(enter(ctx));
    std::lock_guard<std::mutex> g(ctx->mu);
    MeshDev* m;
    TRY(get_mesh(ctx, id, &m));
    if (m->table_n != n_start || !m->nodes64) {
        TRY(ensure_tables(m, n_start, ctx->stream));
        TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    *out = m;
    return BIELCC_OK;
}

int server_device(bielcc_ctx ctx) { return ctx ? ctx->device : 0; }

}  // namespace bielcc_gpu
