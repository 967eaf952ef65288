/*
 * bielcc_gpu.h — C ABI of the B200 (sm_100a) implementation of BIELcc's
 * Stratton-Chu hot path: the K, K0 and R operators, the cell/segment midpoint
 * quadrature of the kernel_lib integrands, the analytic singular integrals,
 * E/H field evaluation over every observation-point x cell pair
 * (GetFieldE_Ideal and its H counterpart) and collocation-matrix assembly.
 *
 * Conventions (every entry point):
 *   - plain C types only; complex numbers are interleaved (re, im) doubles,
 *     i.e. the memory layout of std::complex<double>;
 *   - cells are `double[n_cells][n_vert][3]` with n_vert = 4 (CellQuad) or
 *     3 (CellTriangle), the layout of CellType::GetCellCoords();
 *   - return value: BIELCC_OK (0) or a negative BIELCC_ERR_* code; the
 *     message of the last failure on the calling thread is returned by
 *     bielcc_last_error(); no C++ exception crosses this boundary;
 *   - a context owns one CUDA device, one stream and the resident meshes;
 *     calls on one context are serialised by an internal mutex.
 *
 * Reference interfaces each entry point replaces are cited as
 * path:line inside AlenaSetukha/BIELcc.
 */
#ifndef BIELCC_GPU_H_
#define BIELCC_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exported with default visibility even when the library is built with
 * -fvisibility=hidden. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define BIELCC_ABI_VERSION 4

/* ---- status codes ---------------------------------------------------- */
#define BIELCC_OK                 0
#define BIELCC_ERR_ARG           -1  /* bad argument (null pointer, size, enum) */
#define BIELCC_ERR_CUDA          -2  /* a CUDA runtime call failed */
#define BIELCC_ERR_OOM           -3  /* device allocation failed / over budget */
#define BIELCC_ERR_NAN           -4  /* result written, but holds NaN/Inf */
#define BIELCC_ERR_TIMEOUT       -5  /* a bounded device wait gave up */
#define BIELCC_ERR_UNSUPPORTED   -6  /* valid input outside what the GPU path covers */
#define BIELCC_ERR_NOT_FOUND     -7  /* unknown mesh / request handle */
#define BIELCC_ERR_BUSY          -8  /* admission refused (serving queue full) */
#define BIELCC_ERR_CANCELLED     -9  /* serving request cancelled before it ran */
#define BIELCC_ERR_IO           -10  /* a mesh / current file is missing or malformed */

/* ---- numerical parameters -------------------------------------------- */
/* Mirrors NumParam (electrodynamics/num_param.h:28-55); defaults are the
 * library's Calculation_Constants (electrodynamics/constants.h:17-27):
 * eps=1e-6, rs=2, rs_seg=2, analytic_calc=3, n_start=8, n_start_seg=10,
 * p_max=1, p_max_seg=1. */
typedef struct bielcc_numparam {
    double eps;            /* integral accuracy; also smoothRMin of K near  */
    double rs;             /* surface smoothing radius, relative to diam/n_start */
    double rs_seg;         /* segment smoothing radius, relative to diam/n_start_seg */
    double analytic_calc;  /* near-zone radius, relative to cell diameter */
    int32_t n_start;       /* initial n of the n x n cell split */
    int32_t n_start_seg;   /* initial segment split */
    int32_t p_max;         /* refinement levels of the cell quadrature */
    int32_t p_max_seg;     /* refinement levels of the segment quadrature */
} bielcc_numparam;

/* Fills *np with the Calculation_Constants defaults. */
void bielcc_numparam_default(bielcc_numparam* np);

/* Plane-wave incident field, restating PlaneWaveFieldE / PlaneWaveFieldH
 * (electrodynamics/incident_field.h:20-59):
 *   E_inc(x) = e0 exp(i k_vec.x),  H_inc(x) = h_scale (k_vec x e0) exp(i k_vec.x).
 * add_E / add_H select whether the incident field is added to the output. */
typedef struct bielcc_planewave {
    double k_vec[3];
    double e0[3];
    double h_scale;
    int32_t add_E;
    int32_t add_H;
} bielcc_planewave;

/* Integrand parameters: the fields of KernelParam<KType>
 * (integrators/kernel_param.h:25-57) that the kernel_lib integrands read. */
typedef struct bielcc_kernelparam {
    double smoothR;
    double smoothRMin;
    double k_re, k_im;
    double current[3][2];  /* KernelParam::current (complex) */
    double vec_dbl[3];     /* KernelParam::vec_dbl */
    double n[3];           /* KernelParam::n */
    double e0[3];          /* KernelParam::e0 (read by PlaneWaveFieldE) */
} bielcc_kernelparam;

/* Precision of the field / assembly path. */
#define BIELCC_PREC_FP64   0  /* complex FP64 everywhere (parity form) */
#define BIELCC_PREC_MIXED  1  /* complex FP32 far cells, FP64 near / singular cells */

/* Result report of a field / assembly call. Every mixed-precision call given
 * a report estimates its error against the FP64 form on a sample evaluated in
 * FP64 beside it (and then waits for its stream to fill the estimate):
 * single-job calls min(n_pts, 256) points spread over the set and all RHS;
 * batches min(n_pts, 32) points and the first min(n_rhs, 4) RHS of every job
 * (each job's own estimate also goes to its est_dev); assembly min(N, 16)
 * rows spread over the matrix. FP64 calls report 0. */
typedef struct bielcc_report {
    int64_t n_pairs;        /* point x cell pairs evaluated (per RHS) */
    int64_t n_near_pairs;   /* pairs that took the FP64 near path */
    int64_t n_nonfinite;    /* non-finite output components */
    double  est_rel_l2;     /* mixed: relative L2 difference from FP64 over the sample; FP64: 0 */
    int32_t est_sample;     /* points (rows for assembly) in that sample */
    int32_t status;         /* same as the return value */
} bielcc_report;

typedef struct bielcc_ctx_s* bielcc_ctx;
typedef int32_t bielcc_mesh;

/* ---- context ----------------------------------------------------------- */
int bielcc_abi_version(void);
const char* bielcc_last_error(void);
int bielcc_ctx_create(int device, bielcc_ctx* out);
int bielcc_ctx_destroy(bielcc_ctx ctx);
int bielcc_ctx_synchronize(bielcc_ctx ctx);
/* Device bytes currently held by the context (meshes + workspaces). */
int bielcc_ctx_mem_used(bielcc_ctx ctx, int64_t* bytes);

/* Counters of the kernels a context enqueued. With timing on, the far-field
 * kernels of each field call are bracketed by CUDA events on the stream they
 * run on and their elapsed time accumulates in far_ms (read back at the call's
 * own synchronisation point). No counterpart in the reference (it has no
 * device code); used by bench.py for the roofline figures. */
typedef struct bielcc_stats {
    int64_t kernel_launches;  /* all kernels enqueued by this context */
    int64_t far_launches;     /* far-field kernel launches */
    int64_t far_pairs;        /* far (point, cell, RHS) pairs those launches evaluated */
    double  far_ms;           /* summed CUDA-event time of the far-field kernels */
    int64_t far_ctas;         /* CTAs of the last batched far launch (the persistent grid) */
} bielcc_stats;
int bielcc_ctx_set_timing(bielcc_ctx ctx, int on);
/* Mixed-precision batches (bielcc_field_EH_batch, batch plans, served
 * batches, single-job calls routed as one-job batches) whose jobs have at most
 * 64 right-hand sides and n_start <= 8 contract their far moments with the
 * currents on the tensor cores (tcgen05, TF32 split into hi + lo, FP32
 * accumulation over 16 cells, FP64 across) when on = 1; on = 0 (the default)
 * keeps that contraction on the CUDA cores, which measured faster and more
 * accurate on the batched workloads (the moments, not the contraction, bound
 * both forms). No counterpart in the reference. */
int bielcc_ctx_set_batch_tensor_cores(bielcc_ctx ctx, int on);
/* The split pipeline of mixed-precision batches (n_start <= 8): two kernels
 * per wave of work items, the far moments of every (point, cell) pair into a
 * device buffer of at most moments_bytes, then their contraction with the
 * currents (on the CUDA cores, or on the tensor cores when
 * bielcc_ctx_set_batch_tensor_cores is on).
 *   - Batch plans (bielcc_batch_plan_create) use it when their moments fit
 *     one wave of moments_bytes (default 16 GiB, held by the plan): the
 *     moments depend on geometry and k only, so a replay with new currents
 *     runs the contraction alone. Other plans run the fused kernel.
 *   - all_batches = 1 also splits one-shot batches (bielcc_field_EH_batch,
 *     single-job calls routed as one-job batches, served batches) and plans
 *     of several waves; measured no faster than the fused kernel there
 *     (0.99-1.04x), so the default is 0.
 *   - moments_bytes = 0 never splits.
 * With the CUDA-core contraction the results are bit-identical to the fused
 * kernel; with the tensor-core contraction they agree with the fused
 * tensor-core kernel within the mixed-precision tolerance (the moments kernel
 * pairs cells in its node loop). No counterpart in the reference. */
int bielcc_ctx_set_batch_split(bielcc_ctx ctx, int64_t moments_bytes, int all_batches);
int bielcc_ctx_stats(bielcc_ctx ctx, bielcc_stats* out, int reset);

/* Measured FMA throughput (TFLOP/s, 2 flops per FMA) of the current device's
 * CUDA-core pipes: kind 0 = scalar FP32 FMA, 1 = FP64 FMA, 2 = packed FP32
 * pairs (fma.rn.f32x2, 4 flops per instruction): the roofline denominators of
 * the field kernels. No counterpart in the reference. */
int bielcc_measure_fma_peak(int kind, double* tflops);

/* ---- resident meshes -------------------------------------------------- */
/* Uploads cells and precomputes per-cell geometry on the device: centre
 * (get_center_mass, geometry/element_geom.cpp:320-342), diameter (get_diam,
 * element_geom.cpp:275-317), normal (norm_func, element_geom.cpp:130-156),
 * tangent basis tau1/tau2 (CellQuad/CellTriangle::CellFill, mesh/cell.cpp:8-51,
 * 60-99). Replaces SurfMesh<CellType> (mesh/surf_mesh.h:47-302) as the input of
 * the field driver; mesh parsing stays with the caller. */
int bielcc_mesh_create(bielcc_ctx ctx, int n_vert, int n_cells, const double* cells,
                       bielcc_mesh* out);
int bielcc_mesh_destroy(bielcc_ctx ctx, bielcc_mesh mesh);
/* Per-cell geometry rows computed on the device, 14 doubles per cell:
 * centre(3), diam, normal(3), tau1(3), tau2(3), area — the collocation points,
 * normals and surface basis of SurfMesh::FormCollocPoints /
 * FormNormalVectors / FormSurfaceBasis (mesh/surf_mesh.h:205-268) and
 * get_diam, and the cell area of CellFill; out: [n_cells][14]. */
int bielcc_mesh_geometry(bielcc_ctx ctx, bielcc_mesh mesh, double* out);

/* ---- media ---------------------------------------------------------------
 * Constants of a field evaluation inside a material at one frequency, from
 * the reference's material description: MaterialParam::Calc
 * (electrodynamics/material.cpp:60-128), RadiationSource::CalcK
 * (electrodynamics/radiation_source.cpp:159-180) and the Stratton-Chu
 * multipliers of examples/field/main0_field_test.cpp:185-199. Host only.
 * For a lossy material (complex eps) k is the complex omega sqrt(eps mu)
 * with Im k > 0, which bielcc_field_EH_full takes as (k_re, k_im); the
 * reference's CalcK throws there (it reads its real mu as complex). */
#define BIELCC_DISPERSION_NONE     0  /* NonDispersive / Dispersive: eps_r, mu_r, sigma */
#define BIELCC_DISPERSION_REFRACT  1  /* DispersiveByRefractIndex: table of (freq, n, k_absorb) */
typedef struct bielcc_material {
    int32_t dispersion;
    int32_t n_table;        /* rows of table (BIELCC_DISPERSION_REFRACT) */
    double eps_r, mu_r;     /* relative permittivity / permeability */
    double sigma;           /* conductivity, S/m (0: lossless) */
    const double* table;    /* [n_table][3]: frequency, refractive index n, absorption index
                               (0: CalcEpsN, else CalcEpsNK); the frequency must be listed */
} bielcc_material;
typedef struct bielcc_medium {
    double eps[2];          /* absolute permittivity, complex (F/m) */
    double mu[2];           /* absolute permeability (H/m); real, as CalcMu */
    double k[2];            /* omega sqrt(eps mu), Im >= 0 */
    double k_source;        /* RadiationSource's real wave number, Re k */
    double multE[2];        /* i / (omega eps) */
    double multH[2];        /* i / (omega mu) */
    double tand;            /* electric loss tangent, as Calc leaves it */
    double skin_depth;      /* sqrt(2 / (omega mu sigma)); 0 without sigma */
} bielcc_medium;
int bielcc_medium_at(const bielcc_material* mat, double freq, bielcc_medium* out);
/* Plane wave of RadiationSource in that medium, PlaneWaveFieldE / H
 * (incident_field.h:20-59): k_vec = k_source * direction / |direction|,
 * h_scale = 1 / (2 pi f mu). */
int bielcc_planewave_in_medium(const bielcc_medium* md, double freq, const double* direction,
                               const double* e0, int add_E, int add_H, bielcc_planewave* out);

/* ---- field evaluation ------------------------------------------------- */
/* E(x_i) = mult * sum_j K[cell_j, J_j](x_i) + E_inc(x_i)
 * H(x_i) =        sum_j R[cell_j, J_j](x_i) + H_inc(x_i)
 * with the near/far split of GetFieldE_Ideal (electrodynamics/get_field.h:35-78):
 * near iff |x - centre_j| < analytic_calc * diam_j; near K = K_RotRot_Near_Smooth
 * (electrodynamics/K.h:47-79), far K = K_RotRot_Far (K.h:288-301); near R =
 * R_Rot_Smooth (electrodynamics/R.h:46-61), far R = R_Rot_Colloc (R.h:89-111),
 * the operator pairing of examples/field/main0_field_test.cpp:237-311.
 *   J : [n_rhs][n_cells][3] complex   (the j_E argument, one set per RHS)
 *   pts: [n_pts][3]                    (the points argument)
 *   E, H: [n_rhs][n_pts][3] complex    (field_E and its H counterpart; H may be NULL)
 * Host buffers; the copies are part of the call. */
int bielcc_field_EH(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* J,
                    double k_re, double k_im, double mult_re, double mult_im,
                    const bielcc_planewave* inc, const bielcc_numparam* np,
                    int n_pts, const double* pts, double* E, double* H,
                    int precision, bielcc_report* report);

/* Same computation on device buffers, enqueued on `stream` (a cudaStream_t,
 * NULL = the context's own non-blocking stream; pass cudaStreamLegacy for the
 * legacy default stream); returns once enqueued. The report's
 * n_nonfinite / est_rel_l2 are not filled (no host synchronisation). */
int bielcc_field_EH_device(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* J_dev,
                           double k_re, double k_im, double mult_re, double mult_im,
                           const bielcc_planewave* inc, const bielcc_numparam* np,
                           int n_pts, const double* pts_dev, double* E_dev, double* H_dev,
                           int precision, void* stream, bielcc_report* report);

/* The full Stratton-Chu field of electric and magnetic surface currents, as
 * examples/field/main0_field_test.cpp:237-319 forms it (field_E_SCH,
 * field_H_SCH), with get_field.h:58's per-cell near test:
 *   E = multE * sum_j K[j_E](x) - sum_j R[j_M](x) + E_inc(x),
 *   H = multH * sum_j K[j_M](x) + sum_j R[j_E](x) + H_inc(x),
 * K far = K_RotRot_Far, near = K_RotRot_Near_Smooth; R far = R_Rot_Colloc,
 * near = R_Rot_Smooth. J_E, J_M: [n_rhs][n_cells][3] complex; E, H (both
 * required): [n_rhs][n_pts][3] complex. For a dielectric body, multE / multH
 * carry the medium's constants (the example's multE, multH). The four sums come
 * from one evaluation over 2 n_rhs right-hand sides (the moments are shared),
 * so the cost is that of bielcc_field_EH with twice the RHS. The host form
 * fills report->n_nonfinite but no est_rel_l2. No library counterpart in the
 * reference (only the example's loop). */
int bielcc_field_EH_full(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs, const double* J_E,
                         const double* J_M, double k_re, double k_im, double multE_re,
                         double multE_im, double multH_re, double multH_im,
                         const bielcc_planewave* inc, const bielcc_numparam* np, int n_pts,
                         const double* pts, double* E, double* H, int precision,
                         bielcc_report* report);
int bielcc_field_EH_full_device(bielcc_ctx ctx, bielcc_mesh mesh, int n_rhs,
                                const double* J_E_dev, const double* J_M_dev, double k_re,
                                double k_im, double multE_re, double multE_im, double multH_re,
                                double multH_im, const bielcc_planewave* inc,
                                const bielcc_numparam* np, int n_pts, const double* pts_dev,
                                double* E_dev, double* H_dev, int precision, void* stream,
                                bielcc_report* report);

/* Field evaluation that allocates nothing. No counterpart in the reference.
 * For callers that must not call cudaMalloc while they run: applications that
 * reserve (nearly) all device memory in their own pool up front, where a
 * library allocation can fail or fragment that pool, and latency-critical
 * loops, where cudaMalloc / cudaFree would stall the device. Same computation
 * as bielcc_field_EH_device without a context or resident mesh: the caller
 * passes device pointers for the cells ([n_cells][n_vert][3]), J, points and
 * outputs, and the call's scratch memory (cell rows, node tables, partial
 * sums, near lists) lives in one static device array of 64 MiB that every GPU
 * loading the library holds until exit. Sizes whose scratch exceeds 64 MiB are
 * rejected with BIELCC_ERR_ARG and a message giving the bytes needed. The
 * scratch is, in bytes (each term rounded up to 256):
 *   per cell:  128 + 48 n^2 + 4              (3204 B = 3.1 KiB at n = 8; n is
 *                                             n_start for p_max = 1, else
 *                                             2 n_start)
 *              + 32 n_start^2                (p_max >= 3)
 *              + 48 (4 n_start)^2 + 4        (p_max = 3)
 *   per point: 96 n_rhs per cell split + 96 n_rhs (near sums) + 16
 *              + 4 ceil(n_cells / 32)        (near-cell mask: 1 KiB per point
 *                                             at 8192 cells)
 *              + 4 ceil(n_cells / 32) (1 + n_rhs) (p_max >= 3: test marks)
 *              and the cell splits again (p_max = 3), or
 *              min(8, ceil(n_cells / 32)) more (p_max > 3)
 *   per near pair: 216
 * The far partial sums take at most half of what is left after the cells and
 * a one-split workspace; the cell-split count is capped to fit. Every call
 * looks up the array's device address in the current context
 * (cudaGetSymbolAddress). All calls share the array and leave its contents
 * behind; each call rewrites what it reads, and calls that overlap on the GPU
 * race on it. `stream` may be NULL (legacy default stream); like the _device
 * call it waits once for the near-pair count. The report carries n_pairs and
 * n_near_pairs only. */
int bielcc_field_EH_noalloc(int n_vert, int n_cells, const double* cells_dev, int n_rhs,
                            const double* J_dev, double k_re, double k_im, double mult_re,
                            double mult_im, const bielcc_planewave* inc,
                            const bielcc_numparam* np, int n_pts, const double* pts_dev,
                            double* E_dev, double* H_dev, int precision, void* stream,
                            bielcc_report* report);

/* ---- batched field evaluation ---------------------------------------- */
/* One field evaluation of a batch: a resident mesh, its right-hand sides and
 * points (device buffers, same layouts as bielcc_field_EH_device). */
typedef struct bielcc_field_job {
    bielcc_mesh mesh;
    int32_t n_rhs;
    int32_t n_pts;
    const double* J_dev;    /* [n_rhs][n_cells][3] complex */
    const double* pts_dev;  /* [n_pts][3] */
    double* E_dev;          /* [n_rhs][n_pts][3] complex */
    double* H_dev;          /* may be NULL */
    double k_re, k_im, mult_re, mult_im;
    bielcc_planewave inc;   /* add_E = add_H = 0 for no incident field */
    double* est_dev;        /* mixed precision: device address that receives this job's estimated
                               relative L2 error against FP64 (may be NULL) */
} bielcc_field_job;

/* Many field evaluations (meshes of uneven sizes, their own k, 1..n RHS) in
 * one persistent launch: the far field of every job in one kernel that pulls
 * (job, 32-point tile, cell range) items from a device queue, largest first;
 * per cell chunk the 20 far moments of each (point, cell) are staged in shared
 * memory and contracted with every RHS, so extra RHS cost a contraction, not
 * the quadrature. Near pairs take the FP64 path of bielcc_field_EH. Each
 * job's result depends only on the job (never on the rest of the batch).
 * Same per-job results as GetFieldE_Ideal + H (electrodynamics/get_field.h:35-78)
 * within the precision's tolerance. p_max > 1 or n_start > 22 fall back to one
 * bielcc_field_EH_device per job. report->n_pairs counts (point, cell, RHS). */
int bielcc_field_EH_batch(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs,
                          const bielcc_numparam* np, int precision, void* stream,
                          bielcc_report* report);
/* Times bielcc_field_EH_batch on the given batch for a set of item sizes
 * (estimated node evaluations per work item) and keeps the fastest on the
 * context for later batched calls; *item_cost receives it. The jobs' outputs
 * are overwritten. No counterpart in the reference. */
int bielcc_batch_autotune(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs,
                          const bielcc_numparam* np, int precision, void* stream,
                          double* item_cost);

/* A batch planned once for repeated evaluation with fixed geometry: meshes,
 * points, k, mult and incident field are fixed when the plan is made; the
 * currents J (new contents at the same device addresses) may change between
 * launches, as in an iterative solve or a sweep over incident fields.
 * bielcc_batch_plan_create runs the full batch once (outputs valid when the
 * stream reaches that point) and keeps its work items, workspaces, near-pair
 * list and FP64 near-pair moments (they depend on geometry and k only); the
 * sequence of every later evaluation (reset of the work queue, the
 * persistent far kernel, finalize) is captured once in a CUDA graph, which
 * bielcc_batch_plan_launch replays on a stream: no host planning, no host
 * round trip, 3 graph nodes. Results are identical to bielcc_field_EH_batch
 * with the same J. p_max must be 1 or 2 and the far pass's split (n_start,
 * or 2 n_start when p_max = 2) at most 22. The plan owns its
 * device memory; the jobs' buffers must outlive it. No counterpart in the
 * reference. */
typedef struct bielcc_batch_plan_s* bielcc_batch_plan;
int bielcc_batch_plan_create(bielcc_ctx ctx, int n_jobs, const bielcc_field_job* jobs,
                             const bielcc_numparam* np, int precision, void* stream,
                             bielcc_batch_plan* out, bielcc_report* report);
int bielcc_batch_plan_launch(bielcc_batch_plan plan, void* stream);
int bielcc_batch_plan_destroy(bielcc_batch_plan plan);

/* ---- per-pair operators ----------------------------------------------- */
/* One operator applied to n_pairs independent (cell, x, j) triples, each as
 * the reference call op(j, x, cell, num_param, k, res):
 *   cells: [n_pairs][n_vert][3], x: [n_pairs][3], j: [n_pairs][3] complex,
 *   res:   [n_pairs][3] complex. Host buffers. */
#define BIELCC_OP_K_NEAR_SMOOTH   0  /* K_RotRot_Near_Smooth  electrodynamics/K.h:47-79   */
#define BIELCC_OP_K_HS            1  /* K_RotRot_HS           electrodynamics/K.h:119-145 */
#define BIELCC_OP_K_HS_COLLOC     2  /* K_RotRot_HS_Colloc    electrodynamics/K.h:179-204 */
#define BIELCC_OP_K_HS2_COLLOC    3  /* K_RotRot_HS2_Colloc   electrodynamics/K.h:230-252 */
#define BIELCC_OP_K_FAR           4  /* K_RotRot_Far          electrodynamics/K.h:288-301 */
#define BIELCC_OP_R_SMOOTH        5  /* R_Rot_Smooth          electrodynamics/R.h:46-61   */
#define BIELCC_OP_R_COLLOC        6  /* R_Rot_Colloc          electrodynamics/R.h:89-111  */
#define BIELCC_OP_R_NEAR          7  /* R_Rot_Near            electrodynamics/R.h:140-175 */
#define BIELCC_OP_COUNT           8
int bielcc_pair_op(bielcc_ctx ctx, int op, int n_vert, int n_pairs, const double* cells,
                   const double* x, const double* j, double k_re, double k_im,
                   const bielcc_numparam* np, double* res);

/* ---- kernel_lib integrands under the universal quadratures ------------ */
/* Integrand ids (electrodynamics/kernel_lib.h). Real-valued ones write
 * doubles, complex ones interleaved complex. */
#define BIELCC_F_SIMPLEPOT_L        0  /* F_SimplePot_L        kernel_lib.h:62-69   idim 1 real */
#define BIELCC_F_GRADSIMPLEPOT_L    1  /* F_GradSimplePot_L    kernel_lib.h:87-98   idim 3 real */
#define BIELCC_F_DOUBLEPOT_L        2  /* F_DoublePot_L        kernel_lib.h:117-129 idim 1 real */
#define BIELCC_F_VECTORPOT_L        3  /* F_VectorPot_L        kernel_lib.h:149-177 idim 3 real */
#define BIELCC_F_SIMPLEPOT_H        4  /* F_SimplePot_H        kernel_lib.h:209-217 idim 1 cplx */
#define BIELCC_F_NU_SIMPLEPOT_H     5  /* nuF_SimplePot_H      kernel_lib.h:235-245 idim 3 cplx */
#define BIELCC_F_SIMPLEPOT_HM1      6  /* F_SimplePot_Hm1      kernel_lib.h:262-278 idim 1 cplx */
#define BIELCC_F_GRADSIMPLEPOT_H    7  /* F_GradSimplePot_H    kernel_lib.h:295-313 idim 3 cplx */
#define BIELCC_F_GRADSIMPLEPOT_HM1  8  /* F_GradSimplePot_Hm1  kernel_lib.h:332-356 idim 3 cplx */
#define BIELCC_F_DOUBLEPOT_H        9  /* F_DoublePot_H        kernel_lib.h:375-390 idim 1 cplx */
#define BIELCC_F_N_DOUBLEPOT_H     10  /* nF_DoublePot_H       kernel_lib.h:409-419 idim 3 cplx */
#define BIELCC_F_ROTROTSIMPLEPOT_H 11  /* F_RotRotSimplePot_H  kernel_lib.h:453-492 idim 3 cplx */
#define BIELCC_F_ONE               12  /* F(x) = 1: IntegralUniversal area check   idim 1 real */
#define BIELCC_F_PLANEWAVE_E       13  /* PlaneWaveFieldE electrodynamics/incident_field.h:20-29:
                                          F(x) = e0 exp(i vec_dbl . x)           idim 3 cplx */
#define BIELCC_F_COUNT             14
/* F_ONE and F_PLANEWAVE_E are functions of one point (the F(x) form); the
 * others of a pair (x, y). The *_pnt and K0 entries take the pair form (and
 * F_ONE), bielcc_integral / bielcc_integral_seg the F(x) form. */

/* Returns the value dimension (1 or 3) and whether it is complex. */
int bielcc_integrand_info(int integrand, int* idim, int* is_complex);

/* IntegralUniversalPnt (integrators/integral_universal.h:38-120 quad,
 * :136-220 triangle) of one integrand over n_pairs (cell, x) pairs with the
 * adaptive n -> 2n refinement and smoothing-radius halving of the reference.
 * kp is per pair ([n_pairs]) so each pair has its own smoothR / current / n;
 * on return each record's smoothR holds the value the reference leaves in its
 * KernelParam (halved after every pass while above smoothRMin).
 * res: [n_pairs][idim] (complex interleaved when the integrand is complex). */
int bielcc_integral_pnt(bielcc_ctx ctx, int integrand, int n_vert, int n_pairs,
                        const double* cells, const double* x,
                        bielcc_kernelparam* kp, int n_start, int p_max,
                        double eps, double* res);

/* IntegralUniversalSegPnt (integrators/integral_universal_seg.h:38-98):
 * a, b, x: [n_pairs][3]; kp in/out as for bielcc_integral_pnt. */
int bielcc_integral_seg_pnt(bielcc_ctx ctx, int integrand, int n_pairs,
                            const double* a, const double* b, const double* x,
                            bielcc_kernelparam* kp, int n_start, int p_max,
                            double eps, double* res);

/* IntegralUniversal, the F(x) form (integrators/integral_universal.h:252-334
 * quad, :347-431 triangle): the same adaptive sub-cell rule as
 * bielcc_integral_pnt over n_cells cells, with an integrand of one point
 * (BIELCC_F_ONE or BIELCC_F_PLANEWAVE_E); kp per cell, in/out as above.
 * res: [n_cells][idim]. */
int bielcc_integral(bielcc_ctx ctx, int integrand, int n_vert, int n_cells,
                    const double* cells, bielcc_kernelparam* kp, int n_start, int p_max,
                    double eps, double* res);

/* IntegralUniversalSegPnt, the F(x) overload (integral_universal_seg.h:120-179):
 * a, b: [n_segs][3]; integrand and kp as for bielcc_integral. */
int bielcc_integral_seg(bielcc_ctx ctx, int integrand, int n_segs, const double* a,
                        const double* b, bielcc_kernelparam* kp, int n_start, int p_max,
                        double eps, double* res);

/* K0 / K0_Common (electrodynamics/K0.h:36-86 / :112-166): contour integral
 * of one integrand over the cell edges. common = 0: -sum_e (j.nu_e) int_e F;
 * common = 1: sum_e int_e F nu_e (vec_dbl set to nu_e per edge). The
 * kernel-parameter record is shared by the edges of a pair exactly as in the
 * reference (its smoothR shrinks from edge to edge); kp in/out. */
int bielcc_k0(bielcc_ctx ctx, int integrand, int common, int n_vert, int n_pairs,
              const double* cells, const double* x, const double* j,
              bielcc_kernelparam* kp, int n_start_seg, int p_max_seg,
              double eps, double* res);

/* ---- analytic singular integrals -------------------------------------- */
/* integral1Divr (integrators/integrals_analytic.cpp:218-235): exact
 * integral of 1/|x-y| over a triangle, a quad = triangles (0,1,2)+(2,3,0). */
int bielcc_integral_1divr(bielcc_ctx ctx, int n_vert, int n_pairs, const double* cells,
                          const double* x, double* res);
/* integralGrad1DivrSeg (integrals_analytic.cpp:240-257): closed-form
 * integral over [A,B] of grad_x 1/|x-y|; res: [n_pairs][3]. */
int bielcc_integral_grad1divr_seg(bielcc_ctx ctx, int n_pairs, const double* a,
                                  const double* b, const double* x, double* res);
/* IntegralSurf_SimplePot_H_HS (integrators/integrals_analytic.h:136-164):
 * res [n_pairs] complex. */
int bielcc_integral_surf_simplepot_h_hs(bielcc_ctx ctx, int n_vert, int n_pairs,
                                        const double* cells, const double* x,
                                        double analytic_r, int n_start, int p_max,
                                        double eps, double k_re, double k_im, double* res);
/* IntegralSeg_GradSimplePot_H_HS (integrals_analytic.h:193-221):
 * res [n_pairs][3] complex. */
int bielcc_integral_seg_gradsimplepot_h_hs(bielcc_ctx ctx, int n_pairs, const double* a,
                                           const double* b, const double* x,
                                           double analytic_r, int n_start, int p_max,
                                           double eps, double k_re, double k_im, double* res);

/* ---- collocation-matrix assembly -------------------------------------- */
/* A[(i,a),(j,b)] = tau_a(i) . K[cell_j, tau_b(j)](c_i), c_i = centre of cell i
 * (collocation points as SurfMesh::FormCollocPoints, mesh/surf_mesh.h:688-700),
 * tau from CellFill (mesh/cell.cpp). Near (|c_i - c_j| < analytic_calc*diam_j)
 * entries use K_RotRot_HS_Colloc (electrodynamics/K.h:179-204) in FP64, far
 * entries K_RotRot_Far (K.h:288-301). The reference has no assembly loop,
 * only the operator "for matrix assembly" (examples/ED_Operators/main0_K.cpp:60-69).
 * layout BIELCC_LAYOUT_TAU2: A is (2N x 2N) row-major, row 2i+a, column 2j+b;
 * layout BIELCC_LAYOUT_FULL3: A is (3N x 3N), the 3x3 block K_ij (x, y, z).
 * out_c64 = 1: complex64 storage, 0: complex128. */
#define BIELCC_LAYOUT_TAU2  0
#define BIELCC_LAYOUT_FULL3 1
int bielcc_assemble_K(bielcc_ctx ctx, bielcc_mesh mesh, double k_re, double k_im,
                      const bielcc_numparam* np, int layout, int out_c64, int precision,
                      void* A_host, bielcc_report* report);
int bielcc_assemble_K_device(bielcc_ctx ctx, bielcc_mesh mesh, double k_re, double k_im,
                             const bielcc_numparam* np, int layout, int out_c64,
                             int precision, void* A_dev, void* stream,
                             bielcc_report* report);

/* ---- mesh and current files --------------------------------------------
 * Host-side readers of the reference's files, so that meshes and currents go
 * from disk into bielcc_mesh_create / the field calls without the reference's
 * SurfMesh classes. No GPU work. Each reader counts when its output pointer is
 * NULL (first call: size the buffer), and fills a buffer of the counted size
 * otherwise (on input *n_cells / *n is the buffer's capacity). File errors
 * return BIELCC_ERR_IO, where the reference throws std::runtime_error.
 *   bielcc_read_mesh_dat: geodat .dat, SurfMesh::ReadFromDatFile
 *     (mesh/surf_mesh.cpp:18-175); n_vert 3 (CellTriangle) or 4 (CellQuad).
 *   bielcc_read_mesh_vtk: legacy ASCII VTK, SurfMesh::ReadFromVtkFile +
 *     FillMeshFromVTK (mesh/surf_mesh.h:382-560, surf_mesh.cpp:195-290):
 *     POLYGONS or CELLS with exactly n_vert vertices, others skipped.
 *   bielcc_read_currents: SurfaceCurrentsC_fromFiles
 *     (electrodynamics/currents.cpp:74-109): J as interleaved complex [n][3].
 * cells: [n_cells][n_vert][3] doubles, the layout bielcc_mesh_create takes. */
int bielcc_read_mesh_dat(const char* path, int n_vert, int* n_cells, double* cells);
int bielcc_read_mesh_vtk(const char* path, int n_vert, int* n_cells, double* cells, int* n_skipped);
int bielcc_read_currents(const char* path_re, const char* path_im, int* n, double* J);

/* ---- serving: continuous batching ---------------------------------------
 * A server runs field and assembly requests submitted at any time, from any
 * thread, against meshes resident in its context. It owns n_slots slots (a
 * CUDA stream, device workspaces and pinned staging each) and a scheduler
 * thread. Whenever a slot is idle the scheduler admits queued requests in
 * arrival order while their device bytes fit the HBM budget: every field
 * request admitted together runs as ONE bielcc_field_EH_batch launch, an
 * assembly request runs alone. Requests that arrive while batches are on the
 * GPU are admitted as soon as a slot and memory free up, and their work
 * overlaps the running batches on the other slots' streams; a batch smaller
 * than one already running goes to a high-priority stream and takes SMs as
 * soon as the running batch's CTAs retire (each far-kernel CTA of a served
 * batch handles one work item). A request's
 * result depends only on the request (never on the rest of its batch), so it
 * is the same alone and in any mix. No counterpart in the reference (it has
 * no request loop). Meshes a server uses must stay alive, and must not be
 * evaluated through the context with another n_start, while the server holds
 * requests on them. */
typedef struct bielcc_server_s* bielcc_server;

typedef struct bielcc_field_request {
    bielcc_mesh mesh;
    int32_t n_rhs;
    int32_t n_pts;
    int32_t out_c64;        /* 1: E/H written as complex64, 0: complex128 */
    const double* J;        /* host [n_rhs][n_cells][3] complex; or NULL and: */
    const double* J_dev;    /* device-resident currents, same layout */
    const double* pts;      /* host [n_pts][3] */
    void* E;                /* host [n_rhs][n_pts][3] complex, written on completion */
    void* H;                /* host, may be NULL */
    double k_re, k_im, mult_re, mult_im;
    bielcc_planewave inc;   /* add_E = add_H = 0 for no incident field */
    double* est;            /* mixed server: host address that receives the request's estimated
                               relative L2 error against FP64 on completion (may be NULL) */
} bielcc_field_request;

typedef struct bielcc_assemble_request {
    bielcc_mesh mesh;
    int32_t layout;         /* BIELCC_LAYOUT_TAU2 / BIELCC_LAYOUT_FULL3 */
    int32_t out_c64;
    void* A;                /* host matrix, written on completion; or NULL and: */
    void* A_dev;            /* device matrix owned by the caller */
    double k_re, k_im;
} bielcc_assemble_request;

typedef struct bielcc_server_stats {
    int64_t submitted, completed, failed, cancelled, rejected, queued, running;
    int64_t batches;              /* GPU batches launched */
    int64_t priority_batches;     /* of which: launched at high priority to overtake a larger running batch */
    int64_t max_batch;            /* most requests in one batch */
    int64_t bytes_reserved;       /* device bytes held by admitted requests now */
    int64_t peak_bytes_reserved;
    int64_t bytes_allocated;      /* device bytes the slots hold now */
    int64_t budget;
    int64_t pairs_done;           /* (point, cell, RHS) pairs of completed field requests */
    int64_t pool_mapped_bytes;    /* device memory the server's pool holds mapped */
    int64_t pinned_bytes;         /* pinned host staging the server holds */
    double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> result in the caller's buffer */
    double wall_s;                /* first submit -> last completion */
    double pairs_per_s;           /* pairs_done / wall_s */
    double stage_in_s;            /* host time slots spent staging inputs and launching stage 1 */
    double copy_out_s;            /* host time slots spent copying results into the callers' buffers */
    double gpu_busy_s;            /* union of the batches' spans on the GPU (first copy in to last copy out) */
    double stage_alloc_s, stage_copy_s, stage_plan_s, stage_launch_s;  /* parts of stage_in_s (field batches):
                                     buffer acquisition, host copies into pinned staging, planning, launches */
} bielcc_server_stats;

/* hbm_budget <= 0 selects 150 GiB. np: NULL for the defaults; the server runs
 * the batched kernel, so np->p_max must be 1 or 2 and the far pass's split
 * (np->n_start, or 2 np->n_start when p_max = 2) at most 22. The
 * server maps a quarter of its budget (at most half the free device memory)
 * into its memory pool at creation. */
int bielcc_server_create(bielcc_ctx ctx, int64_t hbm_budget, int n_slots, const bielcc_numparam* np,
                         int precision, bielcc_server* out);
/* Drains the server (bounded wait), then frees it. */
int bielcc_server_destroy(bielcc_server sv);
/* Node evaluations per batched work item (bielcc_batch_autotune's result). */
int bielcc_server_set_item_cost(bielcc_server sv, double item_cost);
/* Maps device_bytes of the server's memory pool and pins pinned_bytes of
 * host staging up front, so that the first batches do not pay for mapping
 * and pinning (the memory counts against nothing but the GPU / host; the
 * HBM budget still bounds what admitted requests use). */
int bielcc_server_reserve(bielcc_server sv, int64_t device_bytes, int64_t pinned_bytes);
/* on = 1 (default): every far-kernel CTA of a served batch handles one work
 * item and retires, so a batch on a higher-priority stream gets SMs at once;
 * 0: persistent CTAs (no overtaking inside a running batch). */
int bielcc_server_set_preemptible(bielcc_server sv, int on);
/* on = 1 (default): a batch smaller (in pairs) than one running on another
 * slot is launched on its slot's high-priority stream and overtakes it;
 * 0: every batch on the same priority, so the GPU serves the batches' CTAs in
 * launch order. */
int bielcc_server_set_overtake(bielcc_server sv, int on);
/* A batch of at most `pairs` (point, cell, RHS) pairs (N^2 for an assembly)
 * runs on its slot's high-priority stream whatever the overtake setting, so
 * small requests get SMs within one work item's time (0 = off, the default). */
int bielcc_server_set_priority_pairs(bielcc_server sv, int64_t pairs);
/* Most requests one batch admits (default 64). */
int bielcc_server_set_max_batch(bielcc_server sv, int max_batch);
/* Most (point, cell, RHS) pairs one batch admits (0 = no cap, the default):
 * a batch's length bounds the latency of every request in it, so a cap keeps
 * large requests from lengthening the batches of small ones. With a cap, a
 * request above a quarter of it (and every assembly request) runs in a batch
 * of its own, and smaller field requests queued behind it are admitted past
 * it into other slots' batches; the queue's first request always goes into
 * the next batch. Without a cap, requests are admitted in arrival order. */
int bielcc_server_set_max_batch_pairs(bielcc_server sv, int64_t pairs);
/* paused = 1: queue requests without admitting any (running batches finish);
 * 0: resume. Lets a caller release a burst of requests as one batch. */
int bielcc_server_pause(bielcc_server sv, int paused);
/* Queue a request; returns at once with a ticket. The host input buffers are
 * read when the request is admitted, the output buffers written when it
 * completes: keep them alive until bielcc_server_poll reports done.
 * BIELCC_ERR_BUSY: the request alone exceeds the budget. */
int bielcc_server_submit_field(bielcc_server sv, const bielcc_field_request* req, int64_t* ticket);
int bielcc_server_submit_assemble(bielcc_server sv, const bielcc_assemble_request* req, int64_t* ticket);
/* *done = 1 once the request finished; then *status is its result code and
 * *latency_ms its submit-to-completion time, and the ticket is released. */
int bielcc_server_poll(bielcc_server sv, int64_t ticket, int* done, int* status, double* latency_ms);
/* Blocks (at most timeout_s) until the ticket's request finished; same outputs. */
int bielcc_server_wait(bielcc_server sv, int64_t ticket, double timeout_s, int* status, double* latency_ms);
/* Removes a request that is still queued (its status becomes
 * BIELCC_ERR_CANCELLED); BIELCC_ERR_BUSY once it was admitted. */
int bielcc_server_cancel(bielcc_server sv, int64_t ticket);
/* Blocks (at most timeout_s) until nothing is queued or running. */
int bielcc_server_drain(bielcc_server sv, double timeout_s);
int bielcc_server_get_stats(bielcc_server sv, bielcc_server_stats* out, int reset);
/* Trace of the last batches the server ran (up to 4096, oldest first; reset
 * with the statistics). Times are ms from the first submission since the
 * last reset: when a slot admitted the batch, when its stage 1 (far kernel,
 * near-pair count) and stage 2 had completed on the GPU, and when its results
 * were in the callers' buffers. No counterpart in the reference. */
typedef struct bielcc_batch_trace {
    int32_t slot;
    int32_t n_requests;
    int32_t assembly;       /* 1: an assembly request */
    int32_t high_priority;  /* launched on the slot's high-priority stream */
    int64_t pairs;          /* (point, cell, RHS) pairs; N^2 for an assembly */
    int64_t first_ticket;
    double admit_ms, stage1_ms, done_ms, complete_ms;
    double oldest_wait_ms;  /* longest time one of its requests had queued when the batch was admitted */
} bielcc_batch_trace;
/* Copies at most `capacity` records into out; *n_out = the number copied. */
int bielcc_server_trace(bielcc_server sv, bielcc_batch_trace* out, int capacity, int* n_out);

/* ---- solving the collocation system ------------------------------------
 * No counterpart in the reference (it assembles operators but has no solver).
 * bielcc_solve_dense: A X = B for a dense complex n x n matrix in row-major
 * order (the layout bielcc_assemble_K writes), B the nrhs right-hand sides,
 * each contiguous ([nrhs][n]); LU with partial pivoting from cuSOLVER
 * (getrf / getrs, loaded on first use; BIELCC_ERR_UNSUPPORTED without it).
 * c64 = 1: complex64, 0: complex128. A is overwritten by its factors, B by X;
 * *info is cuSOLVER's (0 = success); n^2 < 2^31. Device pointers, `stream` as
 * in the _device calls (NULL = legacy default stream); returns after the
 * solve has finished.
 * bielcc_solve_pec: the perfectly conducting body under a plane wave. Builds
 * the TAU2 matrix (bielcc_assemble_K), the right-hand side
 * b_(i,a) = -tau_a(i) . E_inc(c_i) / multE (the tangential boundary condition
 * E_inc + multE K[J] = 0 at the collocation points), solves, and writes the
 * currents J_j = x_(j,1) tau1(j) + x_(j,2) tau2(j) (SurfaceCurrents_byBasis,
 * electrodynamics/currents.h:22-33) as complex128 [n_cells][3] to J_host.
 * MIXED: complex64 matrix and LU; FP64: complex128. The (2N)^2 matrix is
 * allocated for the call (13.4 GB complex64 at N = 20,480). */
int bielcc_solve_dense(int n, int nrhs, int c64, void* A_dev, void* B_dev, void* stream, int* info);
int bielcc_solve_pec(bielcc_ctx ctx, bielcc_mesh mesh, double k_re, double k_im, double multE_re,
                     double multE_im, const bielcc_planewave* inc, const bielcc_numparam* np,
                     int precision, double* J_host, bielcc_report* report);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}  /* extern "C" */
#endif
#endif  /* BIELCC_GPU_H_ */
