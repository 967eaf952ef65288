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

// Stream-ordered device buffer: growing it never stalls the other slots.
// Shrinks when a batch needs under a quarter of a large buffer, so an idle
// slot does not hoard HBM that the budget has handed to other requests.
struct SBuf {
    void* p = nullptr;
    std::atomic<size_t> cap{0};  // read by bielcc_server_stats from other threads
    cudaError_t ensure(size_t b, cudaStream_t s) {
        const size_t c = cap.load();
        if (b <= c && !(c > 4 * b && c > ((size_t)256 << 20))) return cudaSuccess;
        release(s);
        const size_t want = b + b / 4 + 4096;
        cudaError_t e = cudaMallocAsync(&p, want, s);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        cap = want;
        return cudaSuccess;
    }
    void release(cudaStream_t s) {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        cap = 0;
    }
};

// Pinned host staging; grow-only (pinning pages is slow).
struct PinBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t b) {
        if (b <= cap) return cudaSuccess;
        release();
        const size_t want = b + b / 4 + 4096;
        cudaError_t e = cudaMallocHost(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        cap = want;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
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
    std::atomic<int> state{kIdle};  // written by the scheduler and the completion thread
    std::vector<Req*> reqs;
    SBuf ws, pair_ws, io;
    PinBuf pin;
    long long* h_total = nullptr;  // pinned
    long long* d_total = nullptr;  // assembly near count
    BatchPlan bp;
    BatchDevPtrs d{};
    AssembleLaunch asl{};
    size_t out_base = 0, out_total = 0, nan_off = 0;
    int64_t extra = 0;  // reservation correction once the near count is known
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
    std::atomic<bool> stop{false};
    int64_t next_ticket = 1;
    int max_batch = 64;
    bool paused = false;
    double item_cost = 4.0e6;
    int running = 0;
    std::vector<double> lat_ms;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, rejected = 0, batches = 0, max_in_batch = 0,
            pairs_done = 0, priority_batches = 0;
    double stage_in_s = 0, copy_out_s = 0;  // host time of input staging / result copies, summed over batches
    Clock::time_point t_first, t_last;
    bool any = false;
};

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
// job's partial sums and near mask (as plan_batch lays them out) and the
// near-pair estimate. The item size is read under the server lock.
int64_t field_bytes(const Req& r, int n_start, double item_cost) {
    const int64_t S = r.f.n_rhs, P = r.f.n_pts, N = r.mesh->n_cells;
    const int64_t in = (r.f.J_dev ? 0 : al(S * N * 48)) + al(P * 24);
    const int64_t out = al(S * P * 3 * (r.f.out_c64 ? 8 : 16) * (r.f.H ? 2 : 1)) + 8;
    const int64_t cpr = batch_cells_per_range((int)N, (int)S, n_start, item_cost);
    const int64_t ranges = (N + cpr - 1) / cpr, words = (N + 31) / 32;
    const int64_t ws = al(ranges * S * 12 * P * 8) + al(words * P * 4) + P * 24 + 4096;
    return in + out + ws + r.near_est;
}

int64_t assemble_bytes(const Req& r) {
    const int64_t N = r.mesh->n_cells, m = r.a.layout == BIELCC_LAYOUT_FULL3 ? 3 : 2;
    const int64_t mat = r.a.A_dev ? 0 : al(m * N * m * N * (r.a.out_c64 ? 8 : 16));
    return mat + 2 * al((N + 1) * 8) + 256 + r.near_est;
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
    sl.out_total = off - sl.out_base;
    cudaError_t e = sl.io.ensure(off, sl.s);
    if (e == cudaSuccess) e = sl.pin.ensure(off);
    if (e != cudaSuccess) return e;
    char* dev = (char*)sl.io.p;
    char* pin = (char*)sl.pin.p;
    for (Req* r : sl.reqs) {
        const size_t S = r->f.n_rhs, P = r->f.n_pts, N = r->mesh->n_cells;
        if (!r->f.J_dev) memcpy(pin + r->in_J, r->f.J, S * N * 48);
        memcpy(pin + r->in_P, r->f.pts, P * 24);
    }
    if (in_bytes) e = cudaMemcpyAsync(dev, pin, in_bytes, cudaMemcpyHostToDevice, sl.s);
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
    plan_batch(sl.bp, jd, sv->np.n_start, sv->precision == BIELCC_PREC_MIXED, sv->item_cost);
    batch_make_preemptible(sl.bp);
    e = sl.ws.ensure(sl.bp.ws_bytes, sl.s);
    if (e != cudaSuccess) return e;
    int launches = 0;
    e = batch_stage1(sl.bp, sl.ws.p, sv->np.analytic_calc, sv->np.n_start, false, sl.s, &sl.d, &launches);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_total, sl.d.total, sizeof(long long), cudaMemcpyDeviceToHost, sl.s);
    return e;
}

cudaError_t start_assemble(bielcc_server_s* sv, Slot& sl) {
    Req* r = sl.reqs[0];
    const size_t N = r->mesh->n_cells, m = r->a.layout == BIELCC_LAYOUT_FULL3 ? 3 : 2;
    r->out_bytes = m * N * m * N * (r->a.out_c64 ? 8 : 16);
    r->out_off = 0;
    sl.out_base = 0;
    sl.out_total = r->a.A_dev ? 0 : r->out_bytes;
    void* target = r->a.A_dev;
    cudaError_t e = cudaSuccess;
    if (!target) {
        e = sl.io.ensure(r->out_bytes, sl.s);
        if (e == cudaSuccess) e = sl.pin.ensure(r->out_bytes);
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
    } else {
        if (pair_bytes) e = sl.pair_ws.ensure(pair_bytes, sl.s);
        if (e == cudaSuccess) e = assemble_stage2(sl.asl, sl.ws.p, n_near, sl.pair_ws.p, sl.s);
    }
    if (e == cudaSuccess && sl.out_total)
        e = cudaMemcpyAsync((char*)sl.pin.p + sl.out_base, (char*)sl.io.p + sl.out_base, sl.out_total,
                            cudaMemcpyDeviceToHost, sl.s);
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
        } else if (!r->a.A_dev) {
            memcpy(r->a.A, pin, r->out_bytes);
        }
    }
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
    while (!sv->paused && !sv->queue.empty()) {
        Req* r = sv->queue.front();
        if (r->type == kAssemble && !take.empty()) break;
        const bool fits = sv->reserved + r->bytes <= sv->budget;
        if (!fits && !(sv->reserved == 0 && take.empty())) break;  // head of line waits for memory
        sv->queue.pop_front();
        sv->reserved += r->bytes;
        r->state = kRunning;
        take.push_back(r);
        if (r->type == kAssemble || (int)take.size() >= sv->max_batch) break;
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
            bool overtake = false;
            for (const Slot& o : slots_of(sv))
                if (&o != &sl && o.state != kIdle && o.work > sl.work) overtake = true;
            sl.s = overtake ? sl.s_hi : sl.s_lo;
            if (overtake) sv->priority_batches++;
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
        if (e == cudaSuccess) {
            sl.state = kCompleting;
            complete_slot(sv, sl);
        } else {
            cudaGetLastError();
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
    if (n.p_max != 1 || n.n_start < 1 || n.n_start > kBatchMaxNStart || n.n_start_seg < 1 || n.p_max_seg < 1 ||
        n.p_max_seg > 20)
        return set_api_error(BIELCC_ERR_UNSUPPORTED, "the server runs the batched kernel: p_max = 1, 1 <= n_start <= 22");
    bielcc_server_s* sv = new (std::nothrow) bielcc_server_s;
    if (!sv) return set_api_error(BIELCC_ERR_OOM, "out of host memory");
    sv->ctx = ctx;
    sv->device = server_device(ctx);
    sv->np = n;
    sv->precision = precision;
    sv->budget = hbm_budget > 0 ? hbm_budget : ((int64_t)150 << 30);
    sv->slot_mem.reset(new Slot[n_slots]);
    sv->n_slots = n_slots;
    if (cudaSetDevice(sv->device) != cudaSuccess) {
        delete sv;
        return set_api_error(BIELCC_ERR_CUDA, "cudaSetDevice failed");
    }
    for (Slot& sl : slots_of(sv)) {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        cudaError_t e = cudaStreamCreateWithPriority(&sl.s_lo, cudaStreamNonBlocking, least);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&sl.s_hi, cudaStreamNonBlocking, greatest);
        sl.s = sl.s_lo;
        const unsigned ef = cudaEventDisableTiming | cudaEventBlockingSync;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_stage1, ef);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_done, ef);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_total, 64);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_total, 256);
        if (e != cudaSuccess) {
            cudaGetLastError();
            for (Slot& t : slots_of(sv)) {
                if (t.s_lo) cudaStreamDestroy(t.s_lo);
                if (t.s_hi) cudaStreamDestroy(t.s_hi);
                if (t.ev_stage1) cudaEventDestroy(t.ev_stage1);
                if (t.ev_done) cudaEventDestroy(t.ev_done);
                if (t.h_total) cudaFreeHost(t.h_total);
                if (t.d_total) cudaFree(t.d_total);
            }
            delete sv;
            return set_api_error(BIELCC_ERR_CUDA, "server slot set-up failed");
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

int bielcc_server_set_max_batch(bielcc_server sv, int max_batch) {
    if (!sv || max_batch < 1) return set_api_error(BIELCC_ERR_ARG, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->max_batch = max_batch;
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
    int rc = server_mesh(sv->ctx, req->mesh, sv->np.n_start, &r->mesh);
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
    r->bytes = field_bytes(*r, sv->np.n_start, item_cost);
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
    int rc = server_mesh(sv->ctx, req->mesh, sv->np.n_start, &r->mesh);
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
    st->copy_out_s = sv->copy_out_s;
    st->max_batch = sv->max_in_batch;
    st->bytes_reserved = sv->reserved;
    st->peak_bytes_reserved = sv->peak_reserved;
    for (const Slot& sl : slots_of(sv)) st->bytes_allocated += (int64_t)(sl.ws.cap + sl.pair_ws.cap + sl.io.cap);
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
        sv->peak_reserved = sv->reserved;
        sv->any = false;
    }
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
        cudaStreamSynchronize(sl.s_lo);
        sl.pin.release();
        cudaFreeHost(sl.h_total);
        cudaFree(sl.d_total);
        cudaEventDestroy(sl.ev_stage1);
        cudaEventDestroy(sl.ev_done);
        cudaStreamDestroy(sl.s_lo);
        cudaStreamDestroy(sl.s_hi);
    }
    for (auto& kv : sv->reqs) delete kv.second;
    delete sv;
    return rc;
}

}  // extern "C"
