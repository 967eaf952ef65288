// server.cu — request serving with continuous batching (bielcc_server_* in
// include/bielcc_gpu.h).
//
// A server owns S slots; each slot is a worker thread with a high- and a
// low-priority CUDA stream, device workspaces and pinned staging. An idle
// slot admits queued requests in arrival order while their device bytes fit
// the HBM budget: all field requests admitted together run as one batched
// launch (batch.cu), an assembly request runs alone (assemble.cu). The slot
// then stages the inputs, runs stage 1 (far kernel, near counting), waits for
// the near-pair count, passes the memory gate (the reservation becomes exact),
// runs stage 2 (FP64 near pairs, finalize), copies the results to pinned
// memory and from there into the callers' buffers. A request that arrives
// while batches run is admitted by the next idle slot, and its batch overlaps
// the running ones on that slot's stream; a batch smaller than one already
// running goes to the high-priority stream, and since every far-kernel CTA of
// a served batch handles a single work item, it takes SMs as soon as the
// running batch's CTAs retire. batch.cu plans every job from the job alone
// (cell ranges, item sizes, reduction order), so a field request's result is
// bit-identical alone and in any mix. The device kernels have no waits; host
// waits on the caller side (wait / drain / destroy) take timeouts.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bielcc_gpu.h"
#include "internal.h"
#include "ops.cuh"

using namespace bielcc_gpu;
using Clock = std::chrono::steady_clock;

namespace {

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// Device buffer of one batch, allocated stream-ordered from the server's
// memory pool and returned to it when the batch's stream reaches its end. The
// pool keeps its memory mapped (release threshold = unlimited), so a batch's
// allocations reuse memory instead of mapping new pages, and memory freed by
// one slot is reused by the others.
struct SBuf {
    void* p = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaError_t ensure(size_t b, cudaStream_t s) {
        release(s);
        if (!b) return cudaSuccess;
        cudaError_t e = cudaMallocFromPoolAsync(&p, b, pool, s);
        if (e != cudaSuccess) p = nullptr;
        return e;
    }
    void release(cudaStream_t s) {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
    }
};

// Pinned host staging shared by the slots: large pinned regions (pinned once,
// kept until the server is destroyed: pinning is slow and freeing pinned
// memory synchronises the device), sub-allocated first-fit in 4 KiB units; a
// slot holds one range per batch and returns it when the results are in the
// callers' buffers. Free ranges are coalesced within their region.
struct PinRef {
    void* p = nullptr;
    size_t cap = 0;
};
struct PinPool {
    static constexpr size_t kMinRegion = (size_t)256 << 20;
    std::mutex mu;
    std::vector<std::pair<char*, size_t>> regions;
    std::map<char*, size_t> free_;  // start -> bytes
    size_t pinned = 0;
    double alloc_s = 0;

    bool same_region(const char* a, const char* b) const {
        for (const auto& r : regions)
            if (a >= r.first && a < r.first + r.second) return b >= r.first && b < r.first + r.second;
        return false;
    }
    cudaError_t add_region(size_t bytes) {  // caller holds mu
        char* p = nullptr;
        const auto t0 = Clock::now();
        cudaError_t e = cudaMallocHost((void**)&p, bytes);
        alloc_s += std::chrono::duration<double>(Clock::now() - t0).count();
        if (e != cudaSuccess) return e;
        regions.emplace_back(p, bytes);
        free_[p] = bytes;
        pinned += bytes;
        return cudaSuccess;
    }
    cudaError_t acquire(size_t b, PinRef& out) {
        b = (std::max<size_t>(b, 1) + 4095) & ~(size_t)4095;
        std::lock_guard<std::mutex> g(mu);
        for (int pass = 0; pass < 2; pass++) {
            for (auto it = free_.begin(); it != free_.end(); ++it) {
                if (it->second < b) continue;
                out.p = it->first;
                out.cap = b;
                if (it->second > b) free_[it->first + b] = it->second - b;
                free_.erase(it);
                return cudaSuccess;
            }
            if (pass == 0) {
                cudaError_t e = add_region(std::max(b, kMinRegion));
                if (e != cudaSuccess) return e;
            }
        }
        return cudaErrorMemoryAllocation;
    }
    void release(PinRef& r) {
        if (!r.p) return;
        std::lock_guard<std::mutex> g(mu);
        char* p = (char*)r.p;
        size_t n = r.cap;
        auto next = free_.lower_bound(p);
        if (next != free_.end() && p + n == next->first && same_region(p, next->first)) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == p && same_region(prev->first, p)) {
                prev->second += n;
                r.p = nullptr;
                r.cap = 0;
                return;
            }
        }
        free_[p] = n;
        r.p = nullptr;
        r.cap = 0;
    }
    void destroy() {
        for (auto& r : regions) cudaFreeHost(r.first);
        regions.clear();
        free_.clear();
        pinned = 0;
    }
};

enum { kQueued = 0, kRunning = 1, kDone = 2 };
enum { kField = 0, kAssemble = 1 };
enum { kIdle = 0, kStage1 = 1, kStage2 = 2, kCompleting = 3 };

struct Req {
    int64_t ticket = 0;
    int type = kField;
    bielcc_field_request f{};
    bielcc_assemble_request a{};
    MeshDev* mesh = nullptr;
    int64_t bytes = 0;         // reserved device bytes
    int64_t near_est = 0;      // of which: estimated near-pair workspace
    int64_t pairs = 0;
    int state = kQueued;
    int status = BIELCC_OK;
    Clock::time_point t_submit, t_done;
    // placement in the slot's device buffer and its pinned mirror
    size_t in_J = 0, in_P = 0;  // inputs
    size_t out_off = 0, out_bytes = 0, e_bytes = 0;
};

struct Slot {
    // a batch runs on s_hi when it is smaller than a batch already running on
    // another slot (so that it overtakes it: every far-kernel CTA retires
    // after one item), else on s_lo; s = the stream of the current batch
    cudaStream_t s_hi = nullptr, s_lo = nullptr, s = nullptr;
    int64_t work = 0;  // pairs of the current batch
    cudaEvent_t ev_stage1 = nullptr, ev_done = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;  // timed: the batch's span on the GPU
    std::atomic<int> state{kIdle};  // written by the scheduler and the completion thread
    std::vector<Req*> reqs;
    SBuf ws, pair_ws, io;
    PinRef pin;  // pinned staging block of the current batch
    long long* h_total = nullptr;  // pinned
    long long* d_total = nullptr;  // assembly near count
    BatchPlan bp;
    BatchDevPtrs d{};
    AssembleLaunch asl{};
    size_t out_base = 0, out_total = 0, nan_off = 0;
    int64_t extra = 0;  // reservation correction once the near count is known
    // error sample of a mixed field batch (estimate.cu): per request min(P, 32)
    // points and min(S, 4) right-hand sides in FP64, after the main stage 1
    bool samp_on = false;
    size_t est_off = 0, samp_off = 0;  // per-request estimates (copied back), sample scratch (device only)
    SBuf samp_ws, samp_pair_ws;
    BatchPlan samp_bp;
    BatchDevPtrs samp_d{};
    ErrJob* samp_ej = nullptr;
    double *samp_nd = nullptr, *samp_sums = nullptr;
};

}  // namespace

struct bielcc_server_s {
    bielcc_ctx ctx = nullptr;
    int device = 0;
    NumParamH np{};
    int precision = BIELCC_PREC_MIXED;
    int64_t budget = 0, reserved = 0, peak_reserved = 0;
    std::unique_ptr<Slot[]> slot_mem;  // slots hold atomics: not movable
    int n_slots = 0;
    std::deque<Req*> queue;
    std::unordered_map<int64_t, Req*> reqs;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<std::thread> workers;  // one per slot
    cudaMemPool_t pool = nullptr;      // device memory of the batches
    PinPool pins;
    std::atomic<bool> stop{false};
    int64_t next_ticket = 1;
    int max_batch = 64;
    int64_t max_batch_pairs = 0;  // 0: no cap on a batch's (point, cell, RHS) pairs
    bool paused = false;
    bool preemptible = true;
    bool overtake = true;  // a batch smaller than a running one goes to the high-priority stream
    int64_t priority_pairs = 0;  // a batch of at most this many pairs goes to the high-priority stream (0: off)
    cudaEvent_t ev_ref = nullptr;              // time origin of the batch spans
    std::vector<std::pair<double, double>> spans;  // [begin, end] ms of every batch on the GPU
    double item_cost = 4.0e6;
    int running = 0;
    std::vector<double> lat_ms;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, rejected = 0, batches = 0, max_in_batch = 0,
            pairs_done = 0, priority_batches = 0;
    double stage_in_s = 0, copy_out_s = 0;  // host time of input staging / result copies, summed over batches
    double st_alloc = 0, st_copy = 0, st_plan = 0, st_launch = 0;  // parts of stage_in_s
    Clock::time_point t_first, t_last;
    bool any = false;
    std::deque<bielcc_batch_trace> trace;  // the last kTraceCap batches
};

constexpr size_t kTraceCap = 4096;
// largest moments buffer of one served batch (split pipeline): larger batches run in waves
constexpr size_t kServeMomCap = (size_t)1 << 30;

namespace {

struct SlotRange {
    Slot *b, *e;
    Slot* begin() const { return b; }
    Slot* end() const { return e; }
};
SlotRange slots_of(bielcc_server_s* sv) { return SlotRange{sv->slot_mem.get(), sv->slot_mem.get() + sv->n_slots}; }

int64_t near_estimate(int64_t pts, int64_t cells) {
    // room for 8 near cells per point; corrected to the actual count after stage 1
    return (int64_t)batch_pair_ws_bytes(std::min<int64_t>(pts * 8, pts * cells));
}

// Device bytes of a field request inside a batch: inputs, outputs, the
// job's partial sums and near mask (as plan_batch lays them out), the
// near-pair estimate and, for the split pipeline (mom_cap > 0), its share of
// the batch's moments buffer (at most the buffer's cap, so the batch's buffer
// never exceeds its requests' sum). The item size is read under the server lock.
int64_t field_bytes(const Req& r, int n_start, double item_cost, int64_t mom_cap) {
    const int64_t S = r.f.n_rhs, P = r.f.n_pts, N = r.mesh->n_cells;
    const int64_t in = (r.f.J_dev ? 0 : al(S * N * 48)) + al(P * 24);
    const int64_t out = al(S * P * 3 * (r.f.out_c64 ? 8 : 16) * (r.f.H ? 2 : 1)) + 8;
    const int64_t cpr = batch_cells_per_range((int)N, (int)S, n_start, item_cost);
    const int64_t ranges = (N + cpr - 1) / cpr, words = (N + 31) / 32;
    const int64_t ws = al((ranges + 1) * S * 12 * P * 8) + al(words * P * 4) + P * 24 + 4096;
    // the mixed form's error sample: its points, FP64 outputs, partial sums and near mask
    const int64_t Q = std::min<int64_t>(P, 32), Ss = std::min<int64_t>(S, 4);
    const int64_t samp = 3 * al(Q * 24 + Ss * Q * 96) + al((ranges + 1) * Ss * 12 * Q * 8) + al(words * Q * 4) +
                         al(Q * 8 * 216) + 1024;
    int64_t mom = 0;
    if (mom_cap > 0) {
        const int64_t blocks = (P + 31) / 32 * ((N + 7) / 8 + ranges);
        mom = std::min<int64_t>(mom_cap, blocks * (int64_t)moments_block_bytes());
    }
    return in + out + ws + samp + r.near_est + mom;
}

int64_t assemble_bytes(const Req& r) {
    const int64_t N = r.mesh->n_cells, m = r.a.layout == BIELCC_LAYOUT_FULL3 ? 3 : 2;
    const int64_t mat = r.a.A_dev ? 0 : al(m * N * m * N * (r.a.out_c64 ? 8 : 16));
    return mat + 2 * al((N + 1) * 8) + al((N + 31) / 32 * N * 4) + 256 + r.near_est;
}

// Marks a slot's requests done with `code` (caller holds the lock).
void fail_slot_locked(bielcc_server_s* sv, Slot& sl, int code) {
    const auto now = Clock::now();
    for (Req* r : sl.reqs) {
        r->status = code;
        r->state = kDone;
        r->t_done = now;
        sv->reserved -= r->bytes;
        sv->failed++;
    }
    sv->reserved -= sl.extra;
    sl.extra = 0;
    sv->running -= (int)sl.reqs.size();
    sl.reqs.clear();
    sl.state = kIdle;
    sv->cv_done.notify_all();
}

cudaError_t start_field_batch(bielcc_server_s* sv, Slot& sl) {
    size_t off = 0;
    for (Req* r : sl.reqs) {
        const size_t S = r->f.n_rhs, P = r->f.n_pts, N = r->mesh->n_cells;
        if (!r->f.J_dev) {
            r->in_J = off;
            off += al(S * N * 48);
        }
        r->in_P = off;
        off += al(P * 24);
    }
    const size_t in_bytes = off;
    sl.out_base = off;
    for (Req* r : sl.reqs) {
        const size_t S = r->f.n_rhs, P = r->f.n_pts;
        r->e_bytes = S * P * 3 * (r->f.out_c64 ? 8 : 16);
        r->out_off = off;
        r->out_bytes = r->e_bytes * (r->f.H ? 2 : 1);
        off += al(r->out_bytes);
    }
    sl.nan_off = off;
    off += al(sl.reqs.size() * 8);
    sl.samp_on = sv->precision == BIELCC_PREC_MIXED;
    sl.est_off = off;
    if (sl.samp_on) off += al(sl.reqs.size() * 8);
    sl.out_total = off - sl.out_base;
    // sample scratch (device only): ErrJob records, per-job sums, points, FP64 outputs
    sl.samp_off = off;
    size_t samp_q = 0, samp_o = 0;
    for (Req* r : sl.reqs) {
        samp_q += std::min(r->f.n_pts, 32);
        samp_o += (size_t)std::min(r->f.n_pts, 32) * std::min(r->f.n_rhs, 4);
    }
    if (sl.samp_on)
        off += al(sl.reqs.size() * sizeof(ErrJob)) + al(sl.reqs.size() * 16 + 16) + al(samp_q * 24) +
               2 * al(samp_o * 48);
    auto t0 = Clock::now();
    cudaError_t e = sl.io.ensure(off, sl.s);
    if (e == cudaSuccess) e = sv->pins.acquire(off, sl.pin);
    if (e != cudaSuccess) return e;
    auto t1 = Clock::now();
    char* dev = (char*)sl.io.p;
    char* pin = (char*)sl.pin.p;
    for (Req* r : sl.reqs) {
        const size_t S = r->f.n_rhs, P = r->f.n_pts, N = r->mesh->n_cells;
        if (!r->f.J_dev) memcpy(pin + r->in_J, r->f.J, S * N * 48);
        memcpy(pin + r->in_P, r->f.pts, P * 24);
    }
    auto t2 = Clock::now();
    e = cudaEventRecord(sl.ev_begin, sl.s);  // the batch's GPU span starts with its input copy
    if (e == cudaSuccess && in_bytes) e = cudaMemcpyAsync(dev, pin, in_bytes, cudaMemcpyHostToDevice, sl.s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dev + sl.nan_off, 0, sl.reqs.size() * 8, sl.s);
    if (e != cudaSuccess) return e;
    std::vector<JobDev> jd(sl.reqs.size());
    for (size_t i = 0; i < sl.reqs.size(); i++) {
        const Req* r = sl.reqs[i];
        const MeshDev* m = r->mesh;
        JobDev& d = jd[i];
        memset(&d, 0, sizeof(d));
        d.geo = m->geo;
        d.nodes32 = m->nodes32;
        d.nodes64 = m->nodes64;
        d.rho32 = m->rho32;
        d.verts = m->verts;
        d.nv = m->nv;
        d.n_cells = m->n_cells;
        d.pts = (const double*)(dev + r->in_P);
        d.n_pts = r->f.n_pts;
        d.J = reinterpret_cast<const cplx*>(r->f.J_dev ? r->f.J_dev : (const double*)(dev + r->in_J));
        d.n_rhs = r->f.n_rhs;
        d.k = mk(r->f.k_re, r->f.k_im);
        d.mult = mk(r->f.mult_re, r->f.mult_im);
        for (int g = 0; g < 3; g++) {
            d.kvec[g] = r->f.inc.k_vec[g];
            d.e0[g] = r->f.inc.e0[g];
        }
        d.h_scale = r->f.inc.h_scale;
        d.add_E = r->f.inc.add_E;
        d.add_H = r->f.inc.add_H;
        char* o = dev + r->out_off;
        if (r->f.out_c64) {
            d.E32 = (float*)o;
            d.H32 = r->f.H ? (float*)(o + r->e_bytes) : nullptr;
        } else {
            d.E = (double*)o;
            d.H = r->f.H ? (double*)(o + r->e_bytes) : nullptr;
        }
        d.nonfinite = (unsigned long long*)(dev + sl.nan_off) + i;
    }
    auto t3 = Clock::now();
    plan_batch(sl.bp, jd, far_split_n(sv->np), sv->precision == BIELCC_PREC_MIXED, sv->item_cost,
               ctx_batch_tensor_cores(sv->ctx), std::min<size_t>(ctx_batch_split_cap(sv->ctx), kServeMomCap));
    if (sv->preemptible) batch_make_preemptible(sl.bp);

    auto t4 = Clock::now();
    e = sl.ws.ensure(sl.bp.ws_bytes, sl.s);
    if (e != cudaSuccess) return e;
    auto t5 = Clock::now();
    int launches = 0;
    e = batch_stage1(sl.bp, sl.ws.p, sv->np.analytic_calc, far_split_n(sv->np), false, sl.s, &sl.d, &launches);
    if (e == cudaSuccess) e = batch_status_to_host(sl.d, sl.h_total, sl.s);
    if (e == cudaSuccess && sl.samp_on) {  // the error sample: gather, FP64 stage 1 (status in h_total[4], [7])
        char* sb = dev + sl.samp_off;
        const size_t n = sl.reqs.size();
        sl.samp_ej = (ErrJob*)sb;
        sb += al(n * sizeof(ErrJob));
        sl.samp_nd = (double*)sb;
        sl.samp_sums = sl.samp_nd + 2 * n;
        sb += al(n * 16 + 16);
        double* spts = (double*)sb;
        size_t tq = 0, to = 0;
        for (const JobDev& j : jd) {
            tq += std::min(j.n_pts, 32);
            to += (size_t)std::min(j.n_pts, 32) * std::min(j.n_rhs, 4);
        }
        sb += al(tq * 24);
        double* Eq = (double*)sb;
        double* Hq = (double*)(sb + al(to * 48));
        std::vector<ErrJob> ej(n);
        std::vector<JobDev> js(jd);
        size_t oq = 0, oo = 0;
        for (size_t i = 0; i < n; i++) {
            const JobDev& j = jd[i];
            const int Q = std::min(j.n_pts, 32), Ss = std::min(j.n_rhs, 4);
            ej[i] = ErrJob{j.pts, j.n_pts, Q, j.n_rhs, Ss, (int)oq, j.E, j.H, j.E32, j.H32, Eq + 6 * oo,
                           (j.H || j.H32) ? Hq + 6 * oo : nullptr, (double*)(dev + sl.est_off) + i};
            js[i].pts = spts + 3 * oq;
            js[i].n_pts = Q;
            js[i].n_rhs = Ss;
            js[i].E = Eq + 6 * oo;
            js[i].H = (j.H || j.H32) ? Hq + 6 * oo : nullptr;
            js[i].E32 = js[i].H32 = nullptr;
            js[i].nonfinite = nullptr;
            oq += Q;
            oo += (size_t)Ss * Q;
        }
        e = cudaMemcpyAsync(sl.samp_ej, ej.data(), n * sizeof(ErrJob), cudaMemcpyHostToDevice, sl.s);
        if (e == cudaSuccess) e = err_gather(sl.samp_ej, (int)n, spts, sl.s);
        if (e == cudaSuccess) {
            plan_batch(sl.samp_bp, js, far_split_n(sv->np), false, sv->item_cost, false);
            e = sl.samp_ws.ensure(sl.samp_bp.ws_bytes, sl.s);
        }
        int l = 0;
        if (e == cudaSuccess)
            e = batch_stage1(sl.samp_bp, sl.samp_ws.p, sv->np.analytic_calc, far_split_n(sv->np), false, sl.s, &sl.samp_d,
                             &l);
        if (e == cudaSuccess) e = batch_status_to_host(sl.samp_d, sl.h_total + 4, sl.s);
    }
    auto t6 = Clock::now();
    auto sec = [](Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    std::lock_guard<std::mutex> g(sv->mu);
    sv->st_alloc += sec(t0, t1) + sec(t4, t5);
    sv->st_copy += sec(t1, t2);
    sv->st_plan += sec(t2, t4);
    sv->st_launch += sec(t5, t6);
    return e;
}

cudaError_t start_assemble(bielcc_server_s* sv, Slot& sl) {
    Req* r = sl.reqs[0];
    sl.samp_on = false;
    const size_t N = r->mesh->n_cells, m = r->a.layout == BIELCC_LAYOUT_FULL3 ? 3 : 2;
    r->out_bytes = m * N * m * N * (r->a.out_c64 ? 8 : 16);
    r->out_off = 0;
    sl.out_base = 0;
    sl.out_total = r->a.A_dev ? 0 : r->out_bytes;
    void* target = r->a.A_dev;
    cudaError_t e = cudaEventRecord(sl.ev_begin, sl.s);
    if (!target) {
        e = sl.io.ensure(r->out_bytes, sl.s);
        if (e == cudaSuccess) e = sv->pins.acquire(r->out_bytes, sl.pin);
        target = sl.io.p;
    }
    if (e != cudaSuccess) return e;
    sl.asl = AssembleLaunch{r->mesh, mk(r->a.k_re, r->a.k_im), sv->np, r->a.layout, r->a.out_c64 ? 1 : 0,
                            sv->precision, target};
    e = sl.ws.ensure(assemble_ws_base_bytes(sl.asl), sl.s);
    if (e == cudaSuccess) e = assemble_stage1(sl.asl, sl.ws.p, sl.d_total, sl.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_total, sl.d_total, sizeof(long long), cudaMemcpyDeviceToHost, sl.s);
    return e;
}

size_t pair_ws_bytes(const Slot& sl, long long n_near) {
    if (n_near <= 0) return 0;
    return sl.reqs[0]->type == kField ? batch_pair_ws_bytes(n_near) : (size_t)n_near * 8 + 1024;
}

// Memory gate of stage 2: once the near-pair count is known the batch's
// reservation becomes exact (its estimate replaced by the real near-pair
// workspace). If that no longer fits the budget, the batch waits until
// batches in stage 2 free memory; with none in stage 2 the first waiting
// batch proceeds, so the gate cannot deadlock. Returns whether to proceed.
bool stage2_gate(bielcc_server_s* sv, Slot& sl, size_t pair_bytes) {
    int64_t est = 0;
    for (const Req* r : sl.reqs) est += r->near_est;
    const int64_t extra = (int64_t)pair_bytes - est;
    std::lock_guard<std::mutex> g(sv->mu);
    bool others_freeing = false;
    for (const Slot& o : slots_of(sv))
        if (&o != &sl && (o.state == kStage2 || o.state == kCompleting)) others_freeing = true;
    if (sv->reserved + extra > sv->budget && others_freeing) return false;
    sl.extra = extra;
    sv->reserved += extra;
    sv->peak_reserved = std::max(sv->peak_reserved, sv->reserved);
    return true;
}

cudaError_t finish_batch(bielcc_server_s* sv, Slot& sl, long long n_near, size_t pair_bytes) {
    cudaError_t e = cudaSuccess;
    if (sl.reqs[0]->type == kField) {
        if (pair_bytes) e = sl.pair_ws.ensure(pair_bytes, sl.s);
        DNP dn{sv->np.eps, sv->np.rs, sv->np.rs_seg, sv->np.analytic_calc, sv->np.n_start, sv->np.n_start_seg,
               sv->np.p_max, sv->np.p_max_seg};
        int launches = 0;
        if (e == cudaSuccess) e = batch_stage2(sl.bp, sl.d, n_near, sl.pair_ws.p, dn, nullptr, sl.s, &launches);
        if (e == cudaSuccess && sl.samp_on) {  // the error sample's stage 2, then the comparison
            const long long sn = sl.h_total[4];
            if (sn > 0) e = sl.samp_pair_ws.ensure(batch_pair_ws_bytes(sn), sl.s);
            if (e == cudaSuccess)
                e = batch_stage2(sl.samp_bp, sl.samp_d, sn, sl.samp_pair_ws.p, dn, nullptr, sl.s, &launches);
            if (e == cudaSuccess) e = err_compare(sl.samp_ej, (int)sl.reqs.size(), sl.samp_nd, sl.samp_sums, sl.s);
        }
    } else {
        if (pair_bytes) e = sl.pair_ws.ensure(pair_bytes, sl.s);
        if (e == cudaSuccess) e = assemble_stage2(sl.asl, sl.ws.p, n_near, sl.pair_ws.p, sl.s);
    }
    if (e == cudaSuccess && sl.out_total)
        e = cudaMemcpyAsync((char*)sl.pin.p + sl.out_base, (char*)sl.io.p + sl.out_base, sl.out_total,
                            cudaMemcpyDeviceToHost, sl.s);
    // the batch's device memory goes back to the pool when the stream gets here
    sl.ws.release(sl.s);
    sl.pair_ws.release(sl.s);
    sl.io.release(sl.s);
    sl.samp_ws.release(sl.s);
    sl.samp_pair_ws.release(sl.s);
    if (e == cudaSuccess) e = cudaEventRecord(sl.ev_end, sl.s);
    if (e == cudaSuccess) e = cudaEventRecord(sl.ev_done, sl.s);
    return e;
}

// Copies a finished slot's results into the callers' buffers and retires it.
void complete_slot(bielcc_server_s* sv, Slot& sl) {
    const auto t_out = Clock::now();
    const char* pin = (const char*)sl.pin.p;
    std::vector<int> status(sl.reqs.size(), BIELCC_OK);
    for (size_t i = 0; i < sl.reqs.size(); i++) {
        Req* r = sl.reqs[i];
        if (r->type == kField) {
            memcpy(r->f.E, pin + r->out_off, r->e_bytes);
            if (r->f.H) memcpy(r->f.H, pin + r->out_off + r->e_bytes, r->e_bytes);
            const unsigned long long bad = ((const unsigned long long*)(pin + sl.nan_off))[i];
            if (bad) status[i] = BIELCC_ERR_NAN;
            if (r->f.est) *r->f.est = sl.samp_on ? ((const double*)(pin + sl.est_off))[i] : 0.;
        } else if (!r->a.A_dev) {
            memcpy(r->a.A, pin, r->out_bytes);
        }
    }
    sv->pins.release(sl.pin);
    const auto now = Clock::now();
    std::lock_guard<std::mutex> g(sv->mu);
    sv->copy_out_s += std::chrono::duration<double>(now - t_out).count();
    for (size_t i = 0; i < sl.reqs.size(); i++) {
        Req* r = sl.reqs[i];
        r->status = status[i];
        r->state = kDone;
        r->t_done = now;
        sv->reserved -= r->bytes;
        sv->completed++;
        if (r->type == kField) sv->pairs_done += r->pairs;
        sv->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
    }
    sv->reserved -= sl.extra;
    sl.extra = 0;
    sv->t_last = now;
    sv->running -= (int)sl.reqs.size();
    sl.reqs.clear();
    sl.state = kIdle;
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
}

// Takes queued requests for one idle slot (caller holds the lock): a run of
// field requests in arrival order, or one assembly request, within budget.
std::vector<Req*> admit_locked(bielcc_server_s* sv) {
    std::vector<Req*> take;
    int64_t work = 0;
    // With a cap on a batch's work, a request above a quarter of the cap is
    // "large": it runs in a batch of its own, and small requests queued behind
    // it (or behind an assembly) go ahead into the next batch instead of
    // waiting for it (every request of a batch completes with the whole batch).
    // The queue's head always goes into the batch, so nothing waits forever.
    const int64_t large = sv->max_batch_pairs > 0 ? sv->max_batch_pairs / 4 : INT64_MAX;
    for (auto it = sv->queue.begin(); !sv->paused && it != sv->queue.end();) {
        Req* r = *it;
        const bool alone = r->type == kAssemble || r->pairs > large;
        if (alone && !take.empty()) {
            if (sv->max_batch_pairs > 0) {
                ++it;  // it waits for the next idle slot; smaller requests behind it go on
                continue;
            }
            break;  // no cap: arrival order
        }
        // a batch's length bounds the latency of every request in it: past the
        // cap, the rest waits for the next idle slot (an empty batch takes any one)
        if (sv->max_batch_pairs > 0 && !take.empty() && work + r->pairs > sv->max_batch_pairs) break;
        const bool fits = sv->reserved + r->bytes <= sv->budget;
        if (!fits && !(sv->reserved == 0 && take.empty())) break;  // the first in line waits for memory
        it = sv->queue.erase(it);
        sv->reserved += r->bytes;
        r->state = kRunning;
        work += r->pairs;
        take.push_back(r);
        if (alone || (int)take.size() >= sv->max_batch) break;
    }
    if (!take.empty()) {
        sv->peak_reserved = std::max(sv->peak_reserved, sv->reserved);
        sv->running += (int)take.size();
        sv->batches++;
        sv->max_in_batch = std::max<int64_t>(sv->max_in_batch, (int64_t)take.size());
    }
    return take;
}

// Whether an idle slot can take work now (caller holds the lock).
bool admissible_locked(bielcc_server_s* sv) {
    if (sv->paused || sv->queue.empty()) return false;
    const Req* r = sv->queue.front();
    return sv->reserved + r->bytes <= sv->budget || sv->reserved == 0;
}

// One slot's worker: admit a batch, stage its inputs, launch stage 1, wait
// for the near-pair count, pass the memory gate, launch stage 2, wait, copy
// the results to the callers, repeat. Slots run their host work (staging
// copies, planning, result copies) in parallel, one thread each; the waits
// are blocking-sync events (the thread sleeps, no polling).
void slot_loop(bielcc_server_s* sv, Slot* slp) {
    Slot& sl = *slp;
    cudaSetDevice(sv->device);
    bielcc_batch_trace tr{};
    Clock::time_point t_admit, t_stage1, t_done;
    for (;;) {
        std::vector<Req*> take;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv_work.wait(lk, [&] { return sv->stop.load() || admissible_locked(sv); });
            if (sv->stop.load()) return;
            take = admit_locked(sv);
            if (take.empty()) continue;
            sl.reqs = take;
            sl.state = kStage1;
            sl.work = 0;
            for (const Req* r : take) sl.work += r->pairs;
            bool overtake = sv->priority_pairs > 0 && sl.work <= sv->priority_pairs;
            for (const Slot& o : slots_of(sv))
                if (sv->overtake && &o != &sl && o.state != kIdle && o.work > sl.work) overtake = true;
            sl.s = overtake ? sl.s_hi : sl.s_lo;
            if (overtake) sv->priority_batches++;
            tr = bielcc_batch_trace{};
            tr.slot = (int32_t)(slp - sv->slot_mem.get());
            tr.n_requests = (int32_t)take.size();
            tr.assembly = take[0]->type == kAssemble ? 1 : 0;
            tr.high_priority = overtake ? 1 : 0;
            tr.pairs = sl.work;
            tr.first_ticket = take[0]->ticket;
            t_admit = Clock::now();
            for (const Req* r : take) {
                const double w = std::chrono::duration<double, std::milli>(t_admit - r->t_submit).count();
                tr.oldest_wait_ms = std::max(tr.oldest_wait_ms, w);
            }
        }
        const auto t_in = Clock::now();
        cudaError_t e = take[0]->type == kField ? start_field_batch(sv, sl) : start_assemble(sv, sl);
        if (e == cudaSuccess) e = cudaEventRecord(sl.ev_stage1, sl.s);
        const double in_s = std::chrono::duration<double>(Clock::now() - t_in).count();
        {
            std::lock_guard<std::mutex> g(sv->mu);
            sv->stage_in_s += in_s;
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(sl.ev_stage1);
        t_stage1 = Clock::now();
        if (e == cudaSuccess && take[0]->type == kField &&
            (batch_timed_out(sl.h_total) || (sl.samp_on && batch_timed_out(sl.h_total + 4))))
            e = cudaErrorTimeout;  // a bounded wait in the far kernel ran out: the batch fails
        if (e == cudaSuccess) {
            const long long n_near = *sl.h_total;
            const size_t pb = pair_ws_bytes(sl, n_near);
            while (!stage2_gate(sv, sl, pb)) {  // memory gate: wait for batches in stage 2 to finish
                std::unique_lock<std::mutex> lk(sv->mu);
                sv->cv_done.wait_for(lk, std::chrono::milliseconds(1));
            }
            sl.state = kStage2;
            e = finish_batch(sv, sl, n_near, pb);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(sl.ev_done);
        t_done = Clock::now();
        if (e == cudaSuccess) {
            float b = 0.f, t = 0.f;
            if (cudaEventElapsedTime(&b, sv->ev_ref, sl.ev_begin) == cudaSuccess &&
                cudaEventElapsedTime(&t, sv->ev_ref, sl.ev_end) == cudaSuccess) {
                std::lock_guard<std::mutex> g(sv->mu);
                sv->spans.emplace_back(b, t);
            }
            cudaGetLastError();
            sl.state = kCompleting;
            complete_slot(sv, sl);
            const auto t_complete = Clock::now();
            std::lock_guard<std::mutex> g(sv->mu);
            auto ms = [&](Clock::time_point t) {
                return std::chrono::duration<double, std::milli>(t - sv->t_first).count();
            };
            tr.admit_ms = ms(t_admit);
            tr.stage1_ms = ms(t_stage1);
            tr.done_ms = ms(t_done);
            tr.complete_ms = ms(t_complete);
            if (sv->trace.size() >= kTraceCap) sv->trace.pop_front();
            sv->trace.push_back(tr);
        } else {
            cudaGetLastError();
            cudaStreamSynchronize(sl.s);  // nothing of this batch may still write the pinned block
            cudaGetLastError();
            sv->pins.release(sl.pin);
            std::lock_guard<std::mutex> g(sv->mu);
            fail_slot_locked(sv, sl, e == cudaErrorMemoryAllocation ? BIELCC_ERR_OOM : BIELCC_ERR_CUDA);
            sv->cv_work.notify_all();
        }
    }
}

bool idle_locked(bielcc_server_s* sv) { return sv->queue.empty() && sv->running == 0; }

int submit(bielcc_server_s* sv, Req* r, int64_t* ticket) {
    std::lock_guard<std::mutex> g(sv->mu);
    if (r->bytes > sv->budget) {
        sv->rejected++;
        delete r;
        return set_api_error(BIELCC_ERR_BUSY, "request needs more device memory than the server's HBM budget");
    }
    r->ticket = sv->next_ticket++;
    r->t_submit = Clock::now();
    if (!sv->any) {
        sv->t_first = r->t_submit;
        sv->any = true;
    }
    sv->reqs[r->ticket] = r;
    sv->queue.push_back(r);
    sv->submitted++;
    *ticket = r->ticket;
    sv->cv_work.notify_all();
    return BIELCC_OK;
}

// Releases a finished ticket and reports it (caller holds the lock).
void report_locked(bielcc_server_s* sv, std::unordered_map<int64_t, Req*>::iterator it, int* status,
                   double* latency_ms) {
    Req* r = it->second;
    if (status) *status = r->status;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    sv->reqs.erase(it);
    delete r;
}

}  // namespace

extern "C" {

int bielcc_server_create(bielcc_ctx ctx, int64_t hbm_budget, int n_slots, const bielcc_numparam* np, int precision,
                         bielcc_server* out) {
    if (!ctx || !out) return set_api_error(BIELCC_ERR_ARG, "null argument");
    if (n_slots < 1 || n_slots > 16) return set_api_error(BIELCC_ERR_ARG, "n_slots must be 1..16");
    if (precision != BIELCC_PREC_FP64 && precision != BIELCC_PREC_MIXED)
        return set_api_error(BIELCC_ERR_ARG, "unknown precision");
    NumParamH n{1e-6, 2.0, 2.0, 3.0, 8, 10, 1, 1};
    if (np) n = NumParamH{np->eps, np->rs, np->rs_seg, np->analytic_calc, np->n_start, np->n_start_seg, np->p_max,
                          np->p_max_seg};
    if (n.p_max < 1 || far_adaptive(n) || n.n_start < 1 || far_split_n(n) > kBatchMaxNStart || n.n_start_seg < 1 ||
        n.p_max_seg < 1 || n.p_max_seg > 20)
        return set_api_error(BIELCC_ERR_UNSUPPORTED,
                             "the server runs the batched kernel: p_max <= 2, far split (n_start, 2 n_start for "
                             "p_max = 2) of at most 22");
    bielcc_server_s* sv = new (std::nothrow) bielcc_server_s;
    if (!sv) return set_api_error(BIELCC_ERR_OOM, "out of host memory");
    sv->ctx = ctx;
    sv->device = server_device(ctx);
    sv->np = n;
    sv->precision = precision;
    sv->budget = hbm_budget > 0 ? hbm_budget : ((int64_t)150 << 30);
    sv->slot_mem.reset(new Slot[n_slots]);
    sv->n_slots = n_slots;
    {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = sv->device;
        uint64_t keep = UINT64_MAX;  // never trim: batches reuse mapped memory
        if (cudaSetDevice(sv->device) != cudaSuccess || cudaMemPoolCreate(&sv->pool, &props) != cudaSuccess ||
            cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
            cudaGetLastError();
            if (sv->pool) cudaMemPoolDestroy(sv->pool);
            delete sv;
            return set_api_error(BIELCC_ERR_CUDA, "server memory pool set-up failed");
        }
    }
    for (Slot& sl : slots_of(sv)) sl.ws.pool = sl.pair_ws.pool = sl.io.pool = sl.samp_ws.pool = sl.samp_pair_ws.pool =
        sv->pool;
    for (Slot& sl : slots_of(sv)) {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        cudaError_t e = cudaStreamCreateWithPriority(&sl.s_lo, cudaStreamNonBlocking, least);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&sl.s_hi, cudaStreamNonBlocking, greatest);
        sl.s = sl.s_lo;
        const unsigned ef = cudaEventDisableTiming | cudaEventBlockingSync;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_stage1, ef);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_done, ef);
        if (e == cudaSuccess) e = cudaEventCreate(&sl.ev_begin);
        if (e == cudaSuccess) e = cudaEventCreate(&sl.ev_end);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_total, 64);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_total, 256);
        if (e != cudaSuccess) {
            cudaGetLastError();
            for (Slot& t : slots_of(sv)) {
                if (t.s_lo) cudaStreamDestroy(t.s_lo);
                if (t.s_hi) cudaStreamDestroy(t.s_hi);
                if (t.ev_stage1) cudaEventDestroy(t.ev_stage1);
                if (t.ev_done) cudaEventDestroy(t.ev_done);
                if (t.ev_begin) cudaEventDestroy(t.ev_begin);
                if (t.ev_end) cudaEventDestroy(t.ev_end);
                if (t.h_total) cudaFreeHost(t.h_total);
                if (t.d_total) cudaFree(t.d_total);
            }
            cudaMemPoolDestroy(sv->pool);
            delete sv;
            return set_api_error(BIELCC_ERR_CUDA, "server slot set-up failed");
        }
    }
    if (cudaEventCreate(&sv->ev_ref) != cudaSuccess || cudaEventRecord(sv->ev_ref, 0) != cudaSuccess ||
        cudaEventSynchronize(sv->ev_ref) != cudaSuccess) {
        cudaGetLastError();
        sv->ev_ref = nullptr;
    }
    // Map a quarter of the budget (at most half the free device memory) into the
    // pool up front: growing the pool while other slots' kernels run can block a
    // slot's thread for seconds. Best effort; bielcc_server_reserve adds more.
    {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const int64_t want = std::min<int64_t>(sv->budget / 4, (int64_t)(free_b / 2)) & ~((int64_t)(2 << 20) - 1);
            cudaStream_t s0 = slots_of(sv).begin()->s_lo;
            void* p = nullptr;
            if (want > 0 && cudaMallocFromPoolAsync(&p, (size_t)want, sv->pool, s0) == cudaSuccess) {
                cudaFreeAsync(p, s0);
                cudaStreamSynchronize(s0);
            }
            cudaGetLastError();
        }
    }
    for (Slot& sl : slots_of(sv)) sv->workers.emplace_back(slot_loop, sv, &sl);
    *out = sv;
    return BIELCC_OK;
}

int bielcc_server_set_item_cost(bielcc_server sv, double item_cost) {
    if (!sv || !(item_cost > 0)) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->item_cost = item_cost;
    return BIELCC_OK;
}

int bielcc_server_reserve(bielcc_server sv, int64_t device_bytes, int64_t pinned_bytes) {
    if (!sv || device_bytes < 0 || pinned_bytes < 0) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    if (cudaSetDevice(sv->device) != cudaSuccess) return set_api_error(BIELCC_ERR_CUDA, "cudaSetDevice failed");
    if (device_bytes > 0) {
        // allocate and free once: the pool never trims, so the memory stays mapped for the batches
        cudaStream_t s = slots_of(sv).begin()->s_lo;
        void* p = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&p, (size_t)device_bytes, sv->pool, s);
        if (e == cudaSuccess) e = cudaFreeAsync(p, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_api_error(e == cudaErrorMemoryAllocation ? BIELCC_ERR_OOM : BIELCC_ERR_CUDA,
                                 "device reservation failed");
        }
    }
    if (pinned_bytes > 0) {
        std::lock_guard<std::mutex> g(sv->pins.mu);
        if (sv->pins.add_region((size_t)pinned_bytes) != cudaSuccess) {
            cudaGetLastError();
            return set_api_error(BIELCC_ERR_OOM, "pinned host reservation failed");
        }
    }
    return BIELCC_OK;
}

int bielcc_server_set_preemptible(bielcc_server sv, int on) {
    if (!sv) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->preemptible = on != 0;
    return BIELCC_OK;
}

int bielcc_server_set_overtake(bielcc_server sv, int on) {
    if (!sv) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->overtake = on != 0;
    return BIELCC_OK;
}

int bielcc_server_set_priority_pairs(bielcc_server sv, int64_t pairs) {
    if (!sv || pairs < 0) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->priority_pairs = pairs;
    return BIELCC_OK;
}

int bielcc_server_set_max_batch(bielcc_server sv, int max_batch) {
    if (!sv || max_batch < 1) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->max_batch = max_batch;
    return BIELCC_OK;
}

int bielcc_server_set_max_batch_pairs(bielcc_server sv, int64_t pairs) {
    if (!sv || pairs < 0) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->max_batch_pairs = pairs;
    return BIELCC_OK;
}

int bielcc_server_pause(bielcc_server sv, int paused) {
    if (!sv) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->paused = paused != 0;
    sv->cv_work.notify_all();
    return BIELCC_OK;
}

int bielcc_server_submit_field(bielcc_server sv, const bielcc_field_request* req, int64_t* ticket) {
    if (!sv || !req || !ticket) return set_api_error(BIELCC_ERR_ARG, "null argument");
    if (req->n_rhs < 1 || req->n_pts < 1 || (!req->J && !req->J_dev) || !req->pts || !req->E)
        return set_api_error(BIELCC_ERR_ARG, "field request: n_rhs, n_pts >= 1 and J (or J_dev), pts, E required");
    Req* r = new (std::nothrow) Req;
    if (!r) return set_api_error(BIELCC_ERR_OOM, "out of host memory");
    r->type = kField;
    r->f = *req;
    int rc = server_mesh(sv->ctx, req->mesh, far_split_n(sv->np), &r->mesh);
    if (rc != BIELCC_OK) {
        delete r;
        return rc;
    }
    r->near_est = near_estimate(req->n_pts, r->mesh->n_cells);
    double item_cost;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        item_cost = sv->item_cost;
    }
    // served batches split only when the context sets every batch to split
    const int64_t mom_cap = sv->precision == BIELCC_PREC_MIXED && far_split_n(sv->np) <= 8
                                ? (int64_t)std::min<size_t>(ctx_batch_split_cap(sv->ctx), kServeMomCap)
                                : 0;
    r->bytes = field_bytes(*r, far_split_n(sv->np), item_cost, mom_cap);
    r->pairs = (int64_t)req->n_pts * r->mesh->n_cells * req->n_rhs;
    return submit(sv, r, ticket);
}

int bielcc_server_submit_assemble(bielcc_server sv, const bielcc_assemble_request* req, int64_t* ticket) {
    if (!sv || !req || !ticket) return set_api_error(BIELCC_ERR_ARG, "null argument");
    if (!req->A && !req->A_dev) return set_api_error(BIELCC_ERR_ARG, "assembly request: A or A_dev required");
    if (req->layout != BIELCC_LAYOUT_TAU2 && req->layout != BIELCC_LAYOUT_FULL3)
        return set_api_error(BIELCC_ERR_ARG, "unknown layout");
    Req* r = new (std::nothrow) Req;
    if (!r) return set_api_error(BIELCC_ERR_OOM, "out of host memory");
    r->type = kAssemble;
    r->a = *req;
    int rc = server_mesh(sv->ctx, req->mesh, far_split_n(sv->np), &r->mesh);
    if (rc != BIELCC_OK) {
        delete r;
        return rc;
    }
    r->near_est = (int64_t)r->mesh->n_cells * 16 * 8;
    r->bytes = assemble_bytes(*r);
    r->pairs = (int64_t)r->mesh->n_cells * r->mesh->n_cells;
    return submit(sv, r, ticket);
}

int bielcc_server_poll(bielcc_server sv, int64_t ticket, int* done, int* status, double* latency_ms) {
    if (!sv || !done) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return set_api_error(BIELCC_ERR_NOT_FOUND, "unknown or released ticket");
    *done = it->second->state == kDone ? 1 : 0;
    if (*done) report_locked(sv, it, status, latency_ms);
    return BIELCC_OK;
}

int bielcc_server_wait(bielcc_server sv, int64_t ticket, double timeout_s, int* status, double* latency_ms) {
    if (!sv) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return set_api_error(BIELCC_ERR_NOT_FOUND, "unknown or released ticket");
    const bool done = sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        it = sv->reqs.find(ticket);  // another thread may have released the ticket meanwhile
        return it == sv->reqs.end() || it->second->state == kDone;
    });
    if (!done) return set_api_error(BIELCC_ERR_TIMEOUT, "request did not finish in time");
    if (it == sv->reqs.end()) return set_api_error(BIELCC_ERR_NOT_FOUND, "ticket released by another caller");
    report_locked(sv, it, status, latency_ms);
    return BIELCC_OK;
}

int bielcc_server_cancel(bielcc_server sv, int64_t ticket) {
    if (!sv) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return set_api_error(BIELCC_ERR_NOT_FOUND, "unknown or released ticket");
    Req* r = it->second;
    if (r->state != kQueued) return set_api_error(BIELCC_ERR_BUSY, "request already admitted");
    sv->queue.erase(std::find(sv->queue.begin(), sv->queue.end(), r));
    r->state = kDone;
    r->status = BIELCC_ERR_CANCELLED;
    r->t_done = Clock::now();
    sv->cancelled++;
    sv->cv_done.notify_all();
    return BIELCC_OK;
}

int bielcc_server_drain(bielcc_server sv, double timeout_s) {
    if (!sv) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return idle_locked(sv); }))
        return set_api_error(BIELCC_ERR_TIMEOUT, "server did not drain in time");
    return BIELCC_OK;
}

int bielcc_server_get_stats(bielcc_server sv, bielcc_server_stats* st, int reset) {
    if (!sv || !st) return set_api_error(BIELCC_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = sv->submitted;
    st->completed = sv->completed;
    st->failed = sv->failed;
    st->cancelled = sv->cancelled;
    st->rejected = sv->rejected;
    st->queued = (int64_t)sv->queue.size();
    st->running = sv->running;
    st->batches = sv->batches;
    st->priority_batches = sv->priority_batches;
    st->stage_in_s = sv->stage_in_s;
    st->stage_alloc_s = sv->st_alloc;
    {
        std::lock_guard<std::mutex> gp(sv->pins.mu);
        st->pinned_bytes = (int64_t)sv->pins.pinned;
    }
    uint64_t mapped = 0;
    if (cudaMemPoolGetAttribute(sv->pool, cudaMemPoolAttrReservedMemCurrent, &mapped) == cudaSuccess)
        st->pool_mapped_bytes = (int64_t)mapped;
    st->stage_copy_s = sv->st_copy;
    st->stage_plan_s = sv->st_plan;
    st->stage_launch_s = sv->st_launch;
    {
        // union of the batch spans: time the GPU had at least one batch
        std::vector<std::pair<double, double>> v = sv->spans;
        std::sort(v.begin(), v.end());
        double busy = 0, cb = 0, ce = -1e300;
        for (const auto& iv : v) {
            if (iv.first > ce) {
                if (ce > cb) busy += ce - cb;
                cb = iv.first;
                ce = iv.second;
            } else {
                ce = std::max(ce, iv.second);
            }
        }
        if (ce > cb) busy += ce - cb;
        st->gpu_busy_s = busy * 1e-3;
    }
    st->copy_out_s = sv->copy_out_s;
    st->max_batch = sv->max_in_batch;
    st->bytes_reserved = sv->reserved;
    st->peak_bytes_reserved = sv->peak_reserved;
    uint64_t used = 0;
    if (cudaMemPoolGetAttribute(sv->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess)
        st->bytes_allocated = (int64_t)used;
    st->budget = sv->budget;
    st->pairs_done = sv->pairs_done;
    std::vector<double> l = sv->lat_ms;
    std::sort(l.begin(), l.end());
    if (!l.empty()) {
        // nearest-rank percentiles
        auto q = [&](double f) {
            size_t i = (size_t)std::ceil(f * (double)l.size());
            return l[std::min(l.size() - 1, i > 0 ? i - 1 : 0)];
        };
        st->p50_ms = q(0.50);
        st->p99_ms = q(0.99);
        st->max_ms = l.back();
        double s = 0;
        for (double v : l) s += v;
        st->mean_ms = s / (double)l.size();
    }
    if (sv->any && sv->completed) {
        st->wall_s = std::chrono::duration<double>(sv->t_last - sv->t_first).count();
        st->pairs_per_s = st->wall_s > 0 ? (double)sv->pairs_done / st->wall_s : 0.;
    }
    if (reset) {
        sv->lat_ms.clear();
        sv->submitted = sv->completed = sv->failed = sv->cancelled = sv->rejected = 0;
        sv->batches = sv->max_in_batch = sv->pairs_done = sv->priority_batches = 0;
        sv->stage_in_s = sv->copy_out_s = 0;
        sv->st_alloc = sv->st_copy = sv->st_plan = sv->st_launch = 0;
        sv->spans.clear();
        sv->trace.clear();
        sv->peak_reserved = sv->reserved;
        sv->any = false;
    }
    return BIELCC_OK;
}

int bielcc_server_trace(bielcc_server sv, bielcc_batch_trace* out, int capacity, int* n_out) {
    if (!sv || !n_out || capacity < 0 || (capacity > 0 && !out)) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    const int n = std::min<int>(capacity, (int)sv->trace.size());
    for (int i = 0; i < n; i++) out[i] = sv->trace[i];
    *n_out = n;
    return BIELCC_OK;
}

int bielcc_server_destroy(bielcc_server sv) {
    if (!sv) return BIELCC_OK;
    int rc = bielcc_server_drain(sv, 600.0);
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stop.store(true);
        sv->cv_work.notify_all();
    }
    for (std::thread& t : sv->workers)
        if (t.joinable()) t.join();
    cudaSetDevice(sv->device);
    for (Slot& sl : slots_of(sv)) {
        cudaStreamSynchronize(sl.s_hi);
        cudaStreamSynchronize(sl.s_lo);
        sl.ws.release(sl.s_lo);
        sl.pair_ws.release(sl.s_lo);
        sl.io.release(sl.s_lo);
        sv->pins.release(sl.pin);
        cudaStreamSynchronize(sl.s_lo);
        cudaFreeHost(sl.h_total);
        cudaFree(sl.d_total);
        cudaEventDestroy(sl.ev_stage1);
        cudaEventDestroy(sl.ev_done);
        cudaEventDestroy(sl.ev_begin);
        cudaEventDestroy(sl.ev_end);
        cudaStreamDestroy(sl.s_lo);
        cudaStreamDestroy(sl.s_hi);
    }
    sv->pins.destroy();
    cudaMemPoolDestroy(sv->pool);
    cudaEventDestroy(sv->ev_ref);
    for (auto& kv : sv->reqs) delete kv.second;
    delete sv;
    return rc;
}

}  // extern "C"
