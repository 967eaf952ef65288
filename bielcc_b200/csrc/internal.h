// internal.h — host-side declarations shared by the .cu files of
// libbielcc_gpu.so (kernel launchers and workspace records). Not installed.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

struct bielcc_ctx_s;  // the C ABI's context (api.cu)
// Whether the context's mixed batches may use the tensor-core contraction (api.cu).
bool ctx_batch_tensor_cores(bielcc_ctx_s* ctx);
// moments-buffer cap of the split pipeline for one-shot and served batches
// (0: the fused kernel; nonzero only when the context sets every batch to split)
size_t ctx_batch_split_cap(bielcc_ctx_s* ctx);

namespace bielcc_gpu {

struct NumParamH {
    double eps, rs, rs_seg, analytic_calc;
    int n_start, n_start_seg, p_max, p_max_seg;
};

// Node split of the far pass. The reference's adaptive quadrature
// (IntegralUniversalPnt, integral_universal.h:58-119 quads, :160-219
// triangles) stops at the first pass after the first whose squared L2 change
// is below eps^2, and returns the last pass it computed once p_max passes are
// spent; the far operators run it with the smoothing radius at its floor
// (K_RotRot_Far, K.h:293-295; R_Rot_Colloc, R.h:101-102), so it never halves.
// So a far pair's result is the pass at 2 n_start when p_max = 2 (whatever the
// test decides), and also when p_max >= 3 and the test passes at that pass.
// The table-driven far kernels evaluate that pass. With p_max >= 3 a first
// kernel runs the test for every far pair (passes at n_start and 2 n_start);
// the pairs that fail it (far_adaptive) take the full loop in a kernel of their
// own. Near pairs always take the full schedule.
inline int far_split_n(const NumParamH& np) { return np.p_max >= 2 ? 2 * np.n_start : np.n_start; }
inline bool far_adaptive(const NumParamH& np) { return np.p_max > 2; }
// p_max = 3: the pairs that fail the test return the third pass (4 n_start)
// with no further test, so they too run the table-driven far kernels.
inline bool far_third_pass(const NumParamH& np) { return np.p_max == 3; }

// Device-resident mesh with its per-cell geometry and cached node tables.
struct MeshDev {
    int nv = 0, n_cells = 0;
    double* verts = nullptr;  // [N][nv][3]
    CellGeo* geo = nullptr;   // [N]
    // node tables for one split n (n^2 nodes per cell): FP64 absolute
    // (x, y, z, weight) and FP32 relative to the centre (dx, dy, dz, weight)
    int table_n = 0;
    double4* nodes64 = nullptr;  // [N][n*n]
    float4* nodes32 = nullptr;   // [N][n*n]
    float* rho32 = nullptr;      // [N] max |node - centre|
    // p_max >= 3: the FP64 table at n_start (table_lo_n) of the convergence test
    int table_lo_n = 0;
    double4* nodes64_lo = nullptr;  // [N][n_start^2]
    // p_max = 3: the tables at 4 n_start (table_hi_n), the last pass, which
    // the pairs that fail the test take
    int table_hi_n = 0;
    double4* nodes64_hi = nullptr;
    float4* nodes32_hi = nullptr;
    float* rho32_hi = nullptr;
    size_t bytes = 0;
};

// ---- api.cu: records `msg` as this thread's bielcc_last_error() and returns code
int set_api_error(int code, const char* msg);
// a context's mesh with node tables ready for n_start; the context's device
int server_mesh(::bielcc_ctx_s* ctx, int32_t id, int n_start, MeshDev** out);
int server_device(::bielcc_ctx_s* ctx);

// ---- mesh.cu
cudaError_t launch_cell_geometry(const double* verts, int nv, int n_cells, CellGeo* geo, cudaStream_t s);
cudaError_t launch_node_tables(const double* verts, const CellGeo* geo, int nv, int n_cells, int n, double4* nodes64,
                               float4* nodes32, float* rho32, cudaStream_t s);

// ---- field.cu
struct FieldLaunch {
    const MeshDev* mesh;
    const double* pts;  // [P][3] device
    int n_pts;
    const double* J;  // [S][N][3] complex device
    int n_rhs;
    cplx k;
    cplx mult;
    NumParamH np;
    int precision;
    // incident plane wave (add flags 0/1)
    double kvec[3], e0[3], h_scale;
    int add_E, add_H;
    double* E;  // [S][P][3] complex device
    double* H;  // may be null
};
// Workspace bytes a field call needs before the near-pair count is known
// (partials, counts, offsets) and the per-near-pair bytes.
// partial_cap bounds the far partial sums (the split count), at least one split.
size_t field_ws_base_bytes(const FieldLaunch& f, int* splits_out, size_t partial_cap = (size_t)256 << 20);
size_t field_pair_ws_bytes(long long n_near);
// Stage 1: far kernel + near counting + scan; writes total near pairs to
// *d_total (device). Stage 2 (after the host knows the total): near fill,
// near pair kernel, finalize.
cudaError_t field_stage1(const FieldLaunch& f, void* ws, int splits, long long* d_total, cudaStream_t s,
                         int* launches, cudaEvent_t far_begin, cudaEvent_t far_end, int* far_launches);
cudaError_t field_stage2(const FieldLaunch& f, void* ws, int splits, long long n_near, void* pair_ws,
                         unsigned long long* d_nonfinite, cudaStream_t s, int* launches);

// ---- full.cu: E = multE K[j_E] - R[j_M] + E_inc, H = multH K[j_M] + R[j_E] + H_inc
// from a field evaluation over [j_E, j_M] (2S right-hand sides, mult 1, no
// incident field): E2 / H2 are its [2S][P][3] complex outputs.
struct FullInc {
    double kvec[3], e0[3], h_scale;
    int add_E, add_H;
};
cudaError_t launch_combine_full(const double* E2, const double* H2, int S, int P, cplx multE, cplx multH,
                                const double* pts, const FullInc& inc, double* E, double* H,
                                unsigned long long* nonfinite, cudaStream_t s);

// ---- solve.cu: right-hand side of the perfect-conductor collocation system and
// the currents from its solution (TAU2 layout; c64 selects complex64 vectors)
cudaError_t launch_efie_rhs(const CellGeo* geo, int n, const double* kvec, const double* e0, cplx scale, int c64,
                            void* b, cudaStream_t s);
cudaError_t launch_basis_currents(const CellGeo* geo, int n, const void* x, int c64, double* J, cudaStream_t s);

// ---- pairops.cu
cudaError_t launch_pair_op(int op, int nv, int n, const double* cells, const double* x, const double* j, cplx k,
                           NumParamH np, double* res, cudaStream_t s);
struct KParamDev {
    double smoothR, smoothRMin, k_re, k_im;
    double current[3][2];
    double vec_dbl[3];
    double n[3];
    double e0[3];
};
cudaError_t launch_integral_pnt(int integrand, int nv, int n, const double* cells, const double* x,
                                KParamDev* kp, int n_start, int p_max, double eps, double* res, cudaStream_t s);
cudaError_t launch_integral_seg(int integrand, int n, const double* a, const double* b, const double* x,
                                KParamDev* kp, int n_start, int p_max, double eps, double* res, cudaStream_t s);
// x-free forms: x == nullptr (IntegralUniversal / the segment F(x) overload)
cudaError_t launch_k0(int integrand, int common, int nv, int n, const double* cells, const double* x, const double* j,
                      KParamDev* kp, int n_seg, int p_seg, double eps, double* res, cudaStream_t s);
cudaError_t launch_analytic(int which, int nv, int n, const double* cells_or_a, const double* b, const double* x,
                            double analytic_r, int n_start, int p_max, double eps, cplx k, double* res, cudaStream_t s);

// ---- assemble.cu
struct AssembleLaunch {
    const MeshDev* mesh;
    cplx k;
    NumParamH np;
    int layout;     // 0 tau2, 1 full3
    int out_c64;    // complex64 storage
    int precision;  // fp64 / mixed far entries
    void* A;        // device
};
size_t assemble_ws_base_bytes(const AssembleLaunch& a);
cudaError_t assemble_stage1(const AssembleLaunch& a, void* ws, long long* d_total, cudaStream_t s);
cudaError_t assemble_stage2(const AssembleLaunch& a, void* ws, long long n_near, void* pair_ws, cudaStream_t s);
// Error sample of a mixed assembly: R rows (cells r N / R) recomputed in FP64
// and compared with the stored matrix; sums[0] = sum |stored - FP64|^2,
// sums[1] = sum |FP64|^2 (device), on stream s after the assembly.
size_t assemble_error_ws_bytes(const AssembleLaunch& a, int R);
cudaError_t assemble_error_sample(const AssembleLaunch& a, int R, void* ws, double* sums, cudaStream_t s);


// ---- estimate.cu: error report of a mixed result against an FP64 sample
struct ErrJob {
    const double* pts;  // the job's points (device) [P][3]
    int P, Q;           // points, sample points (point q * P / Q)
    int S, Ss;          // right-hand sides of the outputs, sampled right-hand sides (the first Ss)
    int off;            // first sample point of this job in the gathered array
    const double* E;    // mixed outputs [S][P][3] complex128 (or E32 / H32 complex64)
    const double* H;
    const float* E32;
    const float* H32;
    const double* Eq;   // FP64 sample outputs [Ss][Q][3] complex128
    const double* Hq;   // may be null
    double* est_dev;    // receives sqrt(num / den) of this job (may be null)
};
cudaError_t err_gather(const ErrJob* d_jobs, int n_jobs, double* spts, cudaStream_t s);
// per-job (num, den) into nd[2 n_jobs], their sums into sums[2]
cudaError_t err_compare(const ErrJob* d_jobs, int n_jobs, double* nd, double* sums, cudaStream_t s);

// ---- batch.cu: many field jobs in one persistent launch
struct JobDev {
    const CellGeo* geo;
    const float4* nodes32;
    const double4* nodes64;
    const float* rho32;
    const double* verts;
    int nv, n_cells;
    const double* pts;
    int n_pts, pt_off;
    const cplx* J;
    int n_rhs;
    cplx k, mult;
    double kvec[3], e0[3], h_scale;
    int add_E, add_H;
    double* E;
    double* H;
    float* E32;                     // complex64 outputs instead of E / H when set
    float* H32;
    unsigned long long* nonfinite;  // per-job count of points with a non-finite output (may be null)
    double* partial;  // [ranges][S][12][P]
    unsigned* mask;   // [words][P]
    int n_words, ranges, cells_per_range;
};

struct BatchItem {
    int job, tile, range, pad;
};

struct BatchPlan {
    std::vector<JobDev> jobs;
    std::vector<BatchItem> items;
    std::vector<int> pt_job;
    size_t ws_bytes = 0;  // per-job partials + masks + global tables
    int total_pts = 0;
    int grid = 0;
    // items a CTA takes before it exits: unbounded = persistent grid of
    // resident CTAs; 1 with grid = items = every CTA retires after one item,
    // so batches on higher-priority streams get SMs within one item's time
    int max_items = 1 << 30;
    bool mixed = true, ck = false;
    // mixed batches whose jobs have at most 64 right-hand sides (n_start <= 8)
    // contract their moments on the tensor cores (batch_far_tc_kernel)
    bool tc = false;
    int per_cta = 1;  // items a CTA works on at once (the tensor-core kernel's CTA holds two groups)
    int workers() const { return grid * per_cta; }
    // split pipeline (mixed, n_start <= 8): per wave [first, last) of the
    // sorted items, batch_moments_kernel then batch_contract_kernel, through a
    // moments buffer of mom_blocks blocks (BatchItem::pad = the item's first block)
    bool split = false;
    std::vector<std::pair<int, int>> waves;
    size_t mom_blocks = 0;
    int grid_mom = 0, grid_con = 0;
};
// Turns a planned batch into one CTA per item (see BatchPlan::max_items).
void batch_make_preemptible(BatchPlan& bp);

struct BatchDevPtrs {
    JobDev* jobs;
    BatchItem* items;
    int* pt_job;
    long long* counts;
    long long* offs;
    long long* total;
    long long* err;  // nonzero: a bounded wait in the far kernel ran out (next to total)
    int* counter;
    float* mom = nullptr;           // split pipeline: the moments buffer
    int* wave_counters = nullptr;   // split pipeline: two work counters per wave
};
// Copies the near-pair count into h[0] and the far kernel's status into h[3]
// (a 64-byte pinned block; h[1] may hold another count).
cudaError_t batch_status_to_host(const BatchDevPtrs& d, long long* h, cudaStream_t s);
inline bool batch_timed_out(const long long* h) { return h[3] != 0; }

// Cells per item of one job (a multiple of 32; at most 6 ranges per job);
// depends on the job and item_cost only.
int batch_cells_per_range(int n_cells, int n_rhs, int n_start, double item_cost);
// allow_tc: mixed batches that qualify run the tensor-core contraction
// (bielcc_ctx_set_batch_tensor_cores); otherwise the CUDA-core kernel.
// split_cap > 0: mixed batches with n_start <= 8 run the split pipeline with
// a moments buffer of at most split_cap bytes (waves of items); 0: the fused
// kernel.
void plan_batch(BatchPlan& bp, const std::vector<JobDev>& jobs, int n_start, bool mixed, double item_cost,
                bool allow_tc = true, size_t split_cap = 0);
// bytes of one moments block of the split pipeline (8 cells x 20 moments x 32 points, FP32)
size_t moments_block_bytes();
cudaError_t batch_stage1(BatchPlan& bp, void* ws, double analytic_calc, int n_start, bool ck, cudaStream_t s,
                         BatchDevPtrs* out, int* launches);
size_t batch_pair_ws_bytes(long long n_near);
struct DNP;
cudaError_t batch_stage2(BatchPlan& bp, const BatchDevPtrs& d, long long n_near, void* pair_ws, const DNP& np,
                         unsigned long long* d_nonfinite, cudaStream_t s, int* launches);
cudaError_t batch_replay(BatchPlan& bp, const BatchDevPtrs& d, long long n_near, void* pair_ws, double analytic_calc,
                         int n_start, cudaStream_t s);
// largest n_start the batched kernel stages (node tile capacity)
constexpr int kBatchMaxNStart = 22;

}  // namespace bielcc_gpu
