// Serving loop with continuous batching (pk_server_*).
//
// Requests (volume, PSF id, method, iterations) are copied at submit and queued.  A scheduler
// thread admits them while their device buffers fit the HBM budget, keeps their iterates resident
// in HBM, and runs rounds: each round is one launch program with four pass slots (y, x, z, x);
// every active request contributes its next pending pass to the slot of that kind, so requests
// at different iterations and of different methods share launches, and a new request joins at
// the next round.  The per-request arithmetic is the same as the single-volume call's (each CTA
// works on one volume, lambda sums are per request), so a result does not depend on the mix.
// Request volumes are staged in pinned memory at submit and uploaded on a copy stream; the client
// that waits for a request copies its result out and releases the request's device memory.
// All waits are host-side with timeouts; no kernel waits on another.
//
// With device_loop set the request loop is device-resident instead: admission, allocation and the
// uploads stay on the host, but each admitted request's whole pass program becomes a graph that a
// dispatcher kernel (dloop_rdc.cu) takes from a ring in page-locked memory and launches from the
// device as soon as its input is on the GPU; requests then overlap as independent graphs rather
// than sharing launches.  The last node of a request's graph sets its done flag in page-locked
// memory, which the scheduler thread polls.  The dispatcher's waits are bounded (stop flag, launch
// budget, idle time, the scheduler's heartbeat); the host starts a new dispatcher instance when the
// last one has returned and requests are pending.  Nothing on the scheduler's path synchronises the
// whole device (page-locked staging buffers are pooled, not freed, and device memory is freed
// stream-ordered), so the host side never waits on a running dispatcher.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pk_internal.h"

void set_post(VolDesc& d, const pk_decon_params* p, int mask_mode, void* d_out);

namespace {

using clk = std::chrono::steady_clock;

struct PsfEntry {
    std::vector<float> f, b;
    int64_t dims[3];
    bool has_b = false;
    // the OTF cache's copies these (immutable) PSFs were found equal to: later lookups at other
    // data sizes compare pointers instead of the whole PSF
    std::shared_ptr<const std::vector<float>> seen_f, seen_b;
};

struct Step {
    int kind, mode;
    VolDesc d;
};

enum ReqState { RQ_QUEUED, RQ_ACTIVE, RQ_DONE, RQ_FAILED, RQ_CANCELLED };

struct Request {
    int64_t id;
    uint16_t* vol = nullptr;         // pinned staging copy of the input (copy mode)
    size_t vol_cap = 0;              // its capacity (pooled buffers can be larger)
    const uint16_t* src = nullptr;   // the bytes the upload reads (staging copy or the caller's buffer)
    size_t vol_bytes = 0;
    int64_t dims[3];
    int psf_id, method, numit;
    pk_decon_params params;
    ReqState state = RQ_QUEUED;
    pk_status err = PK_OK;
    std::string msg;
    clk::time_point t_submit, t_done;
    // device state
    void* dev = nullptr;             // one allocation: raw | out | work arena
    size_t dev_bytes = 0;
    void* d_out = nullptr;
    size_t out_bytes = 0;
    std::deque<Step> steps;
    cudaEvent_t ev_up = nullptr;     // upload finished
    cudaEvent_t ev_done = nullptr;   // last pass finished
    bool last_queued = false;
    bool uploading = false;          // input still on its way to the device
    bool collected = false;          // the waiter took the result
    // device loop: the request's graph, its descriptor blob and done flag, its ring entry
    cudaGraphExec_t gexec = nullptr;
    void* gblob_d = nullptr;
    void* gblob_h = nullptr;
    size_t gblob_cap = 0;
    int done_slot = -1;
    long long ring_idx = -1;
};

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

struct pk_server {
    pk_ctx* ctx = nullptr;
    pk_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<int32_t, PsfEntry> psfs;
    std::map<int64_t, std::shared_ptr<Request>> reqs;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::shared_ptr<Request>> active;
    std::atomic<bool> stop{false};
    std::thread th;
    int64_t next_id = 0;
    int64_t completed = 0, rejected = 0, rounds = 0;
    size_t inflight = 0, peak_inflight = 0;
    cudaStream_t up = nullptr, down = nullptr;
    // device loop
    static constexpr int kInstances = 64;
    static constexpr int kDoneSlots = 4096;
    DlRing* ring = nullptr;           // page-locked, mapped
    DlRing* d_ring = nullptr;
    int* done_h = nullptr;            // page-locked, mapped: one flag per slot
    int* done_d = nullptr;
    std::vector<int> free_done;
    cudaStream_t dl_st[kInstances] = {};
    cudaGraphExec_t dl_exec[kInstances] = {};
    cudaEvent_t dl_ev[kInstances] = {};
    long long dl_epoch_of[kInstances] = {};   // the instance each stream ran last (0: none)
    int dl_next = 0;
    std::atomic<bool> hb_paused{false};
    // graphs and blobs of finished requests, freed once the dispatcher instance that launched them
    // has completed (its completion includes every graph it launched)
    struct Retired { long long epoch; cudaGraphExec_t g; void* d; void* h; size_t cap; };
    std::vector<Retired> retired;
    std::multimap<size_t, void*> blob_pool;   // page-locked descriptor staging buffers by capacity
    std::multimap<size_t, void*> stage_pool;  // page-locked input staging buffers (copy mode) by capacity
    int64_t instances = 0;

    void loop();
    void loop_device();
    pk_status setup_device_loop();
    void retire(const std::shared_ptr<Request>& r);
    void free_retired(bool all);
    pk_status admit(const std::shared_ptr<Request>& r);
    void build_steps(Request& r, const VolDesc& base, const float2* otf_f, const float2* otf_b);
    void finish(const std::shared_ptr<Request>& r, pk_status st, const std::string& msg);
    void release(const std::shared_ptr<Request>& r);
    void stage_return(void* p, size_t cap);
};

void pk_server::stage_return(void* p, size_t cap) {
    if (stage_pool.size() < 256) stage_pool.emplace(cap, p);
    else cudaFreeHost(p);   // pool full (rare: hundreds of distinct sizes in flight)
}

void pk_server::release(const std::shared_ptr<Request>& r) {
    if (r->dev) {
        cudaFreeAsync(r->dev, ctx->stream);
        inflight -= r->dev_bytes;
        r->dev = nullptr;
    }
    if (r->vol) {   // back to the staging pool: freeing page-locked memory would synchronise the device
        stage_return(r->vol, r->vol_cap);
        r->vol = nullptr;
    }
    if (r->ev_up) { cudaEventDestroy(r->ev_up); r->ev_up = nullptr; }
    if (r->ev_done) { cudaEventDestroy(r->ev_done); r->ev_done = nullptr; }
}

// Mark a request finished; on success its device result stays until the waiter collects it.
void pk_server::finish(const std::shared_ptr<Request>& r, pk_status st, const std::string& msg) {
    r->err = st;
    r->msg = msg;
    if (st != PK_OK) release(r);
    else if (r->vol) {
        stage_return(r->vol, r->vol_cap);
        r->vol = nullptr;
    }
    if (r->state != RQ_CANCELLED) r->state = st == PK_OK ? RQ_DONE : RQ_FAILED;
    r->t_done = clk::now();
    if (st == PK_OK) completed++;
    cv_done.notify_all();
}

// The request's pass sequence (the single-volume program of decon.cu, step by step).
void pk_server::build_steps(Request& r, const VolDesc& b, const float2* otf_f, const float2* otf_b) {
    auto push = [&](int kind, int mode, const VolDesc& d) { r.steps.push_back(Step{kind, mode, d}); };
    char* arena = (char*)r.dev + al256((size_t)b.nrows * b.ny * 2) + al256(r.out_bytes);
    DeconJob j;
    for (int k = 0; k < 3; k++) j.dims[k] = j.rdims[k] = (int)r.dims[k];
    pk_job_carve(j, r.method, false, b.blocksY, arena);
    VolDesc base = b;
    base.I = j.I;
    base.S = j.S;
    base.partials = j.part;
    VolDesc pre = base;
    pre.raw = r.dev;
    pre.raw_type = PK_U16;
    for (int k = 0; k < 3; k++) pre.rdims[k] = (int)r.dims[k];
    pre.bg_f = (float)r.params.background;
    double b16 = std::floor(std::fabs(r.params.background) + 0.5);
    if (r.params.background < 0 || !(b16 == b16)) b16 = 0;
    pre.bg16 = (int)std::min(b16, 65535.0);
    push(PK_STEP_Y, Y_PRE, pre);
    auto conv = [&](int which) {
        VolDesc z = base;
        if (r.method == 1) { z.otf = which ? otf_b : otf_f; z.conj = 0; }
        else { z.otf = otf_f; z.conj = which; }
        push(PK_STEP_X, XZ_FWD, base);
        push(PK_STEP_Z, XZ_CONV, z);
        push(PK_STEP_X, XZ_INV, base);
    };
    if (r.method == 1) {
        for (int it = 1; it <= r.numit; it++) {
            conv(0);
            push(PK_STEP_Y, Y_RATIO, base);
            conv(1);
            VolDesc u = base;
            u.Jo = it == 1 ? j.I : j.J;
            u.Jn = j.J;
            if (it < r.numit) push(PK_STEP_Y, Y_UPDATE, u);
            else {
                set_post(u, &r.params, 0, r.d_out);
                push(PK_STEP_Y, Y_FINAL, u);
            }
        }
    } else {
        float* Jb[2] = {j.J, j.JB};
        for (int k = 1; k <= r.numit; k++) {
            if (k >= 2) {
                VolDesc q = base;
                q.J2 = Jb[k % 2];
                q.J3 = k == 2 ? j.I : Jb[(k - 1) % 2];
                q.Yb = j.Yb;
                q.lam_on = k >= 3 ? 1 : 0;
                push(PK_STEP_Y, Y_RLPRE, q);
            }
            conv(0);
            push(PK_STEP_Y, Y_RATIO, base);
            conv(1);
            VolDesc u = base;
            u.Yb = k == 1 ? j.I : j.Yb;
            if (k < r.numit) {
                u.J4 = j.J4;
                u.rl_first = k == 1 ? 1 : 0;
                u.J2n = Jb[(k + 1) % 2];
                push(PK_STEP_Y, Y_RLUPD, u);
                push(PK_STEP_LAMBDA, 0, u);
            } else {
                set_post(u, &r.params, 0, r.d_out);
                push(PK_STEP_Y, Y_RLFINAL, u);
            }
        }
    }
}

pk_status pk_server::admit(const std::shared_ptr<Request>& r) {
    pk_ctx* c = ctx;
    VolDesc b;
    pk_status s = pk_init_desc(c, (int)r->dims[0], (int)r->dims[1], (int)r->dims[2], &b);
    if (s != PK_OK) return s;
    PsfEntry& pe = psfs[r->psf_id];
    const float2 *of = nullptr, *ob = nullptr;
    if ((s = pk_get_otf(c, pe.f.data(), pe.dims, b.ny, b.nx, b.nz, &of, c->stream, &pe.seen_f)) != PK_OK) return s;
    if (r->method == 1 &&
        (s = pk_get_otf(c, pe.b.data(), pe.dims, b.ny, b.nx, b.nz, &ob, c->stream, &pe.seen_b)) != PK_OK)
        return s;
    const size_t raw_b = (size_t)b.nrows * b.ny * 2;
    int64_t od[3];
    pk_output_dims(r->dims, &r->params, od);
    r->out_bytes = (size_t)od[0] * od[1] * od[2] * (r->params.save16bit ? 2 : 4);
    const int dims[3] = {b.ny, b.nx, b.nz};
    r->dev_bytes = al256(raw_b) + al256(r->out_bytes) + pk_job_bytes(r->method, dims, false, b.blocksY);
    if (!r->ev_up) PK_CUDA(cudaEventCreateWithFlags(&r->ev_up, cudaEventDisableTiming));
    if (!r->ev_done) PK_CUDA(cudaEventCreateWithFlags(&r->ev_done, cudaEventDisableTiming));
    cudaError_t e = cudaMallocAsync(&r->dev, r->dev_bytes, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        r->dev = nullptr;
        return pk_fail(PK_ERR_NOMEM, "request allocation failed");
    }
    inflight += r->dev_bytes;
    peak_inflight = std::max(peak_inflight, inflight);
    r->d_out = (char*)r->dev + al256(raw_b);
    // upload on the copy stream (pinned source); the request joins rounds once the upload has
    // completed, so a large upload never holds back the other requests' passes
    PK_CUDA(cudaEventRecord(r->ev_up, c->stream));          // the allocation is ordered on the compute stream
    PK_CUDA(cudaStreamWaitEvent(up, r->ev_up, 0));
    PK_CUDA(cudaMemcpyAsync(r->dev, r->src, raw_b, cudaMemcpyHostToDevice, up));
    PK_CUDA(cudaEventRecord(r->ev_up, up));
    r->uploading = true;
    build_steps(*r, b, of, ob);
    if (cfg.device_loop) {
        // the whole pass program as one device-launchable graph, ready once its input has landed
        if (free_done.empty()) return pk_fail(PK_ERR_BUSY, "no free completion flag");
        PkProgram prog;
        for (const Step& st : r->steps) pk_program_add(prog, st.kind, st.mode, {st.d});
        r->steps.clear();
        r->done_slot = free_done.back();
        free_done.pop_back();
        done_h[r->done_slot] = 0;
        auto host_blob = [&](size_t need) -> void* {
            auto it = blob_pool.lower_bound(need);
            if (it != blob_pool.end()) {
                r->gblob_h = it->second;
                r->gblob_cap = it->first;
                blob_pool.erase(it);
                return r->gblob_h;
            }
            const size_t cap = std::max<size_t>(4096, need);
            if (cudaMallocHost(&r->gblob_h, cap) != cudaSuccess) {
                cudaGetLastError();
                r->gblob_h = nullptr;
                return nullptr;
            }
            r->gblob_cap = cap;
            return r->gblob_h;
        };
        s = pk_program_device_graph(c, prog, up, done_d + r->done_slot, host_blob, &r->gblob_d, &r->gexec);
        if (s != PK_OK) {
            retire(r);
            return s;
        }
        PK_CUDA(cudaEventRecord(r->ev_up, up));   // input, descriptors and graph are on the device
    }
    r->state = RQ_ACTIVE;
    return PK_OK;
}

void pk_server::retire(const std::shared_ptr<Request>& r) {
    if (r->done_slot >= 0) {
        free_done.push_back(r->done_slot);
        r->done_slot = -1;
    }
    if (r->gexec || r->gblob_d || r->gblob_h) {
        long long ep = 0;   // never launched: free at once
        if (r->ring_idx >= 0 && ring->head > r->ring_idx) ep = ring->epoch[r->ring_idx % kDlRingCap];
        retired.push_back(Retired{ep, r->gexec, r->gblob_d, r->gblob_h, r->gblob_cap});
        r->gexec = nullptr;
        r->gblob_d = r->gblob_h = nullptr;
    }
}

// Frees retired request graphs whose dispatcher instance has completed (an instance's execution
// completes only after every graph it launched); `all` after the dispatcher streams are drained.
void pk_server::free_retired(bool all) {
    for (auto it = retired.begin(); it != retired.end();) {
        bool ok = all || it->epoch == 0;
        if (!ok) {
            ok = true;   // a stream that has moved on to a later instance finished this one first
            for (int j = 0; j < kInstances; j++)
                if (dl_epoch_of[j] == it->epoch) {
                    ok = cudaEventQuery(dl_ev[j]) == cudaSuccess;
                    if (!ok) cudaGetLastError();
                    break;
                }
        }
        if (!ok) {
            ++it;
            continue;
        }
        if (it->g) cudaGraphExecDestroy(it->g);
        if (it->d) cudaFreeAsync(it->d, up);
        if (it->h) blob_pool.emplace(it->cap, it->h);
        it = retired.erase(it);
    }
}

pk_status pk_server::setup_device_loop() {
    PK_CUDA(cudaHostAlloc((void**)&ring, sizeof(DlRing), cudaHostAllocMapped));
    memset((void*)ring, 0, sizeof(DlRing));
    ring->heartbeat_ns = (long long)cfg.heartbeat_ms * 1000000LL;
    ring->idle_ns = (long long)cfg.idle_us * 1000LL;
    PK_CUDA(cudaHostGetDevicePointer((void**)&d_ring, (void*)ring, 0));
    PK_CUDA(cudaHostAlloc((void**)&done_h, sizeof(int) * kDoneSlots, cudaHostAllocMapped));
    memset(done_h, 0, sizeof(int) * kDoneSlots);
    PK_CUDA(cudaHostGetDevicePointer((void**)&done_d, done_h, 0));
    for (int i = kDoneSlots - 1; i >= 0; i--) free_done.push_back(i);
    for (int k = 0; k < kInstances; k++) {
        PK_CUDA(cudaStreamCreateWithFlags(&dl_st[k], cudaStreamNonBlocking));
        PK_CUDA(cudaEventCreateWithFlags(&dl_ev[k], cudaEventDisableTiming));
        pk_status s = pk_dloop_instance(d_ring, dl_st[k], &dl_exec[k]);
        if (s != PK_OK) return s;
    }
    return PK_OK;
}

// The device-resident loop's host side: admission and uploads as in loop(), then ready requests go
// to the ring, a dispatcher instance is started when the last one has returned and entries wait,
// and finished requests are found by their done flags.
void pk_server::loop_device() {
    cudaSetDevice(ctx->device);
    while (!stop.load()) {
        std::unique_lock<std::mutex> lk(mu);
        if (!hb_paused.load()) ring->heartbeat = ring->heartbeat + 1;
        const long long head = ring->head;
        for (auto it = active.begin(); it != active.end();) {
            auto& r = *it;
            bool gone = false;
            if (r->ring_idx >= 0) {
                const int i = (int)(r->ring_idx % kDlRingCap);
                const int launch = head > r->ring_idx ? ring->status[i] : 0;
                if (launch > 1) {
                    finish(r, PK_ERR_CUDA, std::string("device launch of the request's graph failed: ") +
                                               cudaGetErrorString((cudaError_t)(launch - 1)));
                    gone = true;
                } else if (launch == 1 && done_h[r->done_slot]) {
                    // a bounded device wait that ran out (context status word) fails the request
                    const pk_status ws = pk_check_device_waits(ctx);
                    if (r->state == RQ_CANCELLED) finish(r, PK_ERR_CANCELLED, "cancelled");
                    else finish(r, ws, ws == PK_OK ? "" : pk_last_error());
                    gone = true;
                }
            } else if (r->state == RQ_CANCELLED) {   // not handed to the device yet
                cudaStreamSynchronize(up);
                finish(r, PK_ERR_CANCELLED, "cancelled");
                gone = true;
            }
            if (gone) {
                retire(r);
                it = active.erase(it);
            } else {
                ++it;
            }
        }
        while (!queue.empty() && (int)active.size() < cfg.max_batch) {
            auto r = queue.front();
            if (r->state == RQ_CANCELLED) {
                queue.pop_front();
                finish(r, PK_ERR_CANCELLED, "cancelled");
                continue;
            }
            VolDesc tmp;
            size_t need = 0;
            {
                std::lock_guard<std::recursive_mutex> cl(ctx->mu);
                if (pk_init_desc(ctx, (int)r->dims[0], (int)r->dims[1], (int)r->dims[2], &tmp) == PK_OK) {
                    const int dims[3] = {tmp.ny, tmp.nx, tmp.nz};
                    need = pk_job_bytes(r->method, dims, false, tmp.blocksY) + 4 * (size_t)tmp.nrows * tmp.ny;
                }
            }
            if (inflight + need > (size_t)cfg.budget_bytes && !active.empty()) break;   // wait for memory
            queue.pop_front();
            pk_status s;
            {
                std::lock_guard<std::recursive_mutex> cl(ctx->mu);
                s = admit(r);
            }
            if (s != PK_OK) {
                finish(r, s, pk_last_error());
                retire(r);
                continue;
            }
            active.push_back(r);
        }
        // requests whose input, descriptors and graph are on the device join the ring
        for (auto& r : active) {
            if (r->ring_idx >= 0 || r->state == RQ_CANCELLED) continue;
            const cudaError_t q = cudaEventQuery(r->ev_up);
            if (q == cudaErrorNotReady) {
                cudaGetLastError();
                continue;
            }
            if (ring->tail - ring->head >= kDlRingCap) break;
            const long long t = ring->tail;
            ring->graph[t % kDlRingCap] = r->gexec;
            ring->status[t % kDlRingCap] = 0;
            std::atomic_thread_fence(std::memory_order_seq_cst);
            ring->tail = t + 1;
            r->ring_idx = t;
        }
        // a dispatcher instance for waiting entries, once the previous one has returned
        if (ring->tail > ring->head && ring->epoch_ended == ring->epoch_launched) {
            for (int k = 0; k < kInstances; k++) {
                const int j = (dl_next + k) % kInstances;
                if (dl_epoch_of[j] && cudaEventQuery(dl_ev[j]) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                const long long ep = ring->epoch_launched + 1;
                ring->epoch_launched = ep;
                std::atomic_thread_fence(std::memory_order_seq_cst);
                if (cudaGraphLaunch(dl_exec[j], dl_st[j]) != cudaSuccess || cudaEventRecord(dl_ev[j], dl_st[j]) != cudaSuccess) {
                    cudaGetLastError();
                    ring->epoch_launched = ep - 1;
                    break;
                }
                dl_epoch_of[j] = ep;
                dl_next = (j + 1) % kInstances;
                instances++;
                rounds++;
                break;
            }
        }
        free_retired(false);
        cv_work.wait_for(lk, std::chrono::microseconds(200));
    }
}

void pk_server::loop() {
    cudaSetDevice(ctx->device);
    const int kinds[4] = {PK_STEP_Y, PK_STEP_X, PK_STEP_Z, PK_STEP_X};
    while (!stop.load()) {
        std::unique_lock<std::mutex> lk(mu);
        // finished requests (last pass complete)
        for (auto it = active.begin(); it != active.end();) {
            auto& r = *it;
            if (r->state == RQ_CANCELLED) {       // cancelled requests leave at a round boundary
                cudaStreamSynchronize(ctx->stream);
                finish(r, PK_ERR_CANCELLED, "cancelled");
                it = active.erase(it);
            } else if (r->last_queued && cudaEventQuery(r->ev_done) == cudaSuccess) {
                finish(r, PK_OK, "");
                it = active.erase(it);
            } else {
                ++it;
            }
        }
        // admission against the budget, at most kAdmitPerRound a round (PK_ADMIT_PER_ROUND overrides
        // it, diagnostics): requests admitted together run their rounds in step, so a burst admitted
        // at once finishes at once and leaves the GPU idle while the next burst uploads; staggered
        // cohorts keep uploads, rounds and downloads of different requests overlapping
        static const int kAdmitPerRound =
            getenv("PK_ADMIT_PER_ROUND") && atoi(getenv("PK_ADMIT_PER_ROUND")) > 0 ? atoi(getenv("PK_ADMIT_PER_ROUND")) : 16;
        int admitted = 0;
        while (!queue.empty() && (int)active.size() < cfg.max_batch && admitted < kAdmitPerRound) {
            auto r = queue.front();
            if (r->state == RQ_CANCELLED) {
                queue.pop_front();
                finish(r, PK_ERR_CANCELLED, "cancelled");
                continue;
            }
            VolDesc tmp;
            size_t need = 0;
            {
                std::lock_guard<std::recursive_mutex> cl(ctx->mu);
                if (pk_init_desc(ctx, (int)r->dims[0], (int)r->dims[1], (int)r->dims[2], &tmp) == PK_OK) {
                    const int dims[3] = {tmp.ny, tmp.nx, tmp.nz};
                    need = pk_job_bytes(r->method, dims, false, tmp.blocksY) + 4 * (size_t)tmp.nrows * tmp.ny;
                }
            }
            if (inflight + need > (size_t)cfg.budget_bytes && !active.empty()) break;  // wait for memory
            queue.pop_front();
            pk_status s;
            {
                std::lock_guard<std::recursive_mutex> cl(ctx->mu);
                s = admit(r);
            }
            if (s != PK_OK) {
                finish(r, s, pk_last_error());
                continue;
            }
            active.push_back(r);
            admitted++;
        }
        bool work = false;
        for (auto& r : active) {
            if (r->uploading && cudaEventQuery(r->ev_up) == cudaSuccess) r->uploading = false;
            if (!r->steps.empty() && !r->uploading) work = true;
        }
        if (!work) {
            cv_work.wait_for(lk, std::chrono::milliseconds(1));
            continue;
        }
        // one round: slots y, x, z, x; lambda steps ride with their y slot
        std::vector<std::shared_ptr<Request>> batch;
        for (auto& r : active)
            if (!r->uploading) batch.push_back(r);
        lk.unlock();
        {
            std::lock_guard<std::recursive_mutex> cl(ctx->mu);
            PkProgram prog;
            for (int slot = 0; slot < 4; slot++) {
                std::map<int, std::vector<VolDesc>> by_mode;
                std::vector<VolDesc> lam;
                for (auto& r : batch) {
                    if (r->steps.empty() || r->steps.front().kind != kinds[slot]) continue;
                    Step st = r->steps.front();
                    r->steps.pop_front();
                    by_mode[st.mode].push_back(st.d);
                    if (!r->steps.empty() && r->steps.front().kind == PK_STEP_LAMBDA) {
                        lam.push_back(r->steps.front().d);
                        r->steps.pop_front();
                    }
                }
                for (auto& kv : by_mode) pk_program_add(prog, kinds[slot], kv.first, kv.second);
                if (!lam.empty()) pk_program_add(prog, PK_STEP_LAMBDA, 0, lam);
            }
            pk_status s = pk_program_upload(ctx, prog, ctx->stream);
            if (s == PK_OK) s = pk_program_launch(ctx, prog, ctx->stream);
            if (s != PK_OK) {
                std::lock_guard<std::mutex> l2(mu);
                for (auto& r : batch) finish(r, s, pk_last_error());
                active.clear();
                continue;
            }
            // requests whose last pass is queued: mark the point their result is complete
            for (auto& r : batch) {
                if (!r->steps.empty() || r->last_queued) continue;
                cudaEventRecord(r->ev_done, ctx->stream);
                r->last_queued = true;
            }
        }
        lk.lock();
        rounds++;
    }
}

extern "C" {

pk_server* pk_server_create(pk_ctx* ctx, const pk_server_config* cfg) {
    if (!ctx) {
        pk_set_error("null pk_ctx");
        return nullptr;
    }
    pk_server* s = new pk_server();
    s->ctx = ctx;
    s->cfg.budget_bytes = cfg && cfg->budget_bytes > 0 ? cfg->budget_bytes : (int64_t)150e9;
    s->cfg.max_batch = cfg && cfg->max_batch > 0 ? cfg->max_batch : 64;
    s->cfg.queue_capacity = cfg && cfg->queue_capacity > 0 ? cfg->queue_capacity : 1024;
    s->cfg.borrow_inputs = cfg ? cfg->borrow_inputs : 0;
    s->cfg.device_loop = cfg ? cfg->device_loop : 0;
    s->cfg.heartbeat_ms = cfg && cfg->heartbeat_ms > 0 ? cfg->heartbeat_ms : 2000;
    s->cfg.idle_us = cfg && cfg->idle_us > 0 ? cfg->idle_us : 2000;
    cudaSetDevice(ctx->device);
    {
        // request buffers come from the device's stream-ordered pool; keep freed blocks in the pool
        // instead of returning them to the driver at every synchronisation (this process only)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        cudaGetLastError();
    }
    if (cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking) != cudaSuccess) {
        pk_set_error("stream creation failed");
        delete s;
        return nullptr;
    }
    if (s->cfg.device_loop && s->setup_device_loop() != PK_OK) {
        const std::string m = pk_last_error();
        pk_server_destroy(s);
        pk_set_error(m);
        return nullptr;
    }
    if (s->cfg.device_loop) s->th = std::thread([s] { s->loop_device(); });
    else s->th = std::thread([s] { s->loop(); });
    return s;
}

pk_status pk_server_add_psf(pk_server* s, int32_t psf_id, const float* psf_f, const float* psf_b,
                            const int64_t psf_dims[3]) {
    if (!s || !psf_f || !psf_dims) return pk_fail(PK_ERR_INVALID, "bad arguments");
    const int64_t n = psf_dims[0] * psf_dims[1] * psf_dims[2];
    if (n < 1) return pk_fail(PK_ERR_INVALID, "empty PSF");
    std::lock_guard<std::mutex> lk(s->mu);
    PsfEntry e;
    e.f.assign(psf_f, psf_f + n);
    if (psf_b) {
        e.b.assign(psf_b, psf_b + n);
        e.has_b = true;
    }
    for (int i = 0; i < 3; i++) e.dims[i] = psf_dims[i];
    s->psfs[psf_id] = std::move(e);
    return PK_OK;
}

int64_t pk_server_submit(pk_server* s, const uint16_t* vol, const int64_t dims[3], int32_t psf_id, int32_t method,
                         int32_t numit, const pk_decon_params* params) {
    if (!s || !vol || !dims) return -(int64_t)pk_fail(PK_ERR_INVALID, "bad arguments");
    if (method != 0 && method != 1) return -(int64_t)pk_fail(PK_ERR_INVALID, "method must be 0 (RL) or 1 (OMW)");
    if (numit < 1) return -(int64_t)pk_fail(PK_ERR_INVALID, "NUMIT must be >= 1 for served requests");
    pk_decon_params p;
    if (params) p = *params;
    else pk_params_default(&p);
    if (p.decon_offset != 0.0 || p.edge_erosion > 0)
        return -(int64_t)pk_fail(PK_ERR_UNSUPPORTED, "served requests do not take deconOffset/EdgeErosion");
    pk_status st = pk_check_params(dims, &p);
    if (st != PK_OK) return -(int64_t)st;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->psfs.find(psf_id);
    if (it == s->psfs.end()) return -(int64_t)pk_fail(PK_ERR_INVALID, "unknown psf_id");
    if (method == 1 && !it->second.has_b) return -(int64_t)pk_fail(PK_ERR_INVALID, "psf_id has no backprojector");
    if ((int)s->queue.size() >= s->cfg.queue_capacity) {
        s->rejected++;
        return -(int64_t)pk_fail(PK_ERR_BUSY, "queue full");
    }
    lk.unlock();
    auto r = std::make_shared<Request>();
    const int64_t n = dims[0] * dims[1] * dims[2];
    r->vol_bytes = (size_t)n * 2;
    if (s->cfg.borrow_inputs) {
        r->src = vol;
    } else {
        {   // a pooled page-locked staging buffer, else a new one
            std::lock_guard<std::mutex> pl(s->mu);
            auto it = s->stage_pool.lower_bound(r->vol_bytes);
            if (it != s->stage_pool.end() && it->first <= 2 * r->vol_bytes) {
                r->vol = (uint16_t*)it->second;
                r->vol_cap = it->first;
                s->stage_pool.erase(it);
            }
        }
        if (!r->vol) {
            cudaSetDevice(s->ctx->device);
            if (cudaMallocHost(&r->vol, r->vol_bytes) != cudaSuccess) {
                cudaGetLastError();
                r->vol = nullptr;
                return -(int64_t)pk_fail(PK_ERR_NOMEM, "pinned staging allocation failed");
            }
            r->vol_cap = r->vol_bytes;
        }
        memcpy(r->vol, vol, r->vol_bytes);
        r->src = r->vol;
    }
    lk.lock();
    r->id = s->next_id++;
    for (int i = 0; i < 3; i++) r->dims[i] = dims[i];
    r->psf_id = psf_id;
    r->method = method;
    r->numit = numit;
    r->params = p;
    r->t_submit = clk::now();
    s->reqs[r->id] = r;
    s->queue.push_back(r);
    s->cv_work.notify_all();
    return r->id;
}

pk_status pk_server_wait(pk_server* s, int64_t id, void* out, int32_t timeout_ms, double* latency_ms) {
    if (!s) return pk_fail(PK_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return pk_fail(PK_ERR_INVALID, "unknown request id");
    auto r = it->second;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(0, timeout_ms)), [&] {
        return r->state == RQ_DONE || r->state == RQ_FAILED || (r->state == RQ_CANCELLED && r->t_done != clk::time_point());
    });
    if (!ok) return pk_fail(PK_ERR_TIMEOUT, "request not finished within the timeout");
    if (r->state == RQ_CANCELLED) {
        s->reqs.erase(id);
        return pk_fail(PK_ERR_CANCELLED, "request cancelled");
    }
    if (r->state == RQ_FAILED) {
        const pk_status e = r->err;
        const std::string m = r->msg;
        s->reqs.erase(id);
        return pk_fail(e, m);
    }
    s->reqs.erase(id);
    lk.unlock();
    // the result is complete on the device: copy it out on a stream of this thread, then free
    cudaSetDevice(s->ctx->device);
    cudaError_t e = cudaSuccess;
    if (out) e = cudaMemcpyAsync(out, r->d_out, r->out_bytes, cudaMemcpyDeviceToHost, s->down);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->down);
    const auto t_out = clk::now();
    lk.lock();
    s->release(r);
    lk.unlock();
    if (e != cudaSuccess) return pk_fail(PK_ERR_CUDA, std::string("result copy: ") + cudaGetErrorString(e));
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(t_out - r->t_submit).count();
    return PK_OK;
}

pk_status pk_server_cancel(pk_server* s, int64_t id) {
    if (!s) return pk_fail(PK_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return pk_fail(PK_ERR_INVALID, "unknown request id");
    if (it->second->state == RQ_QUEUED || it->second->state == RQ_ACTIVE) it->second->state = RQ_CANCELLED;
    s->cv_work.notify_all();
    return PK_OK;
}

pk_status pk_server_stats(pk_server* s, int64_t stats[4]) {
    if (!s || !stats) return pk_fail(PK_ERR_INVALID, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    stats[0] = s->completed;
    stats[1] = s->rejected;
    stats[2] = (int64_t)s->peak_inflight;
    stats[3] = s->rounds;
    return PK_OK;
}

pk_status pk_server_loop_status(pk_server* s, int32_t* running, int32_t* exit_code, int64_t* instances) {
    if (!s) return pk_fail(PK_ERR_INVALID, "null server");
    if (!s->ring) return pk_fail(PK_ERR_UNSUPPORTED, "the server runs the host scheduler (device_loop = 0)");
    std::lock_guard<std::mutex> lk(s->mu);
    if (running) *running = s->ring->epoch_ended != s->ring->epoch_launched ? 1 : 0;
    if (exit_code) *exit_code = s->ring->exit_code;
    if (instances) *instances = s->instances;
    return PK_OK;
}

pk_status pk_server_pause_heartbeat(pk_server* s, int32_t pause) {
    if (!s) return pk_fail(PK_ERR_INVALID, "null server");
    if (!s->ring) return pk_fail(PK_ERR_UNSUPPORTED, "the server runs the host scheduler (device_loop = 0)");
    s->hb_paused.store(pause != 0);
    return PK_OK;
}

void pk_server_destroy(pk_server* s) {
    if (!s) return;
    s->stop.store(true);
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    if (s->ring) {
        // dispatchers return at their next poll; then their streams drain every graph they launched
        cudaSetDevice(s->ctx->device);
        s->ring->stop = 1;
        const auto t0 = clk::now();
        while (s->ring->epoch_ended != s->ring->epoch_launched &&
               clk::now() - t0 < std::chrono::milliseconds(s->cfg.heartbeat_ms + 2000))
            std::this_thread::sleep_for(std::chrono::microseconds(200));
        for (int k = 0; k < pk_server::kInstances; k++)
            if (s->dl_st[k]) cudaStreamSynchronize(s->dl_st[k]);
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& r : s->active) s->retire(r);
        s->free_retired(true);
        if (s->up) cudaStreamSynchronize(s->up);
        for (auto& kv : s->blob_pool) cudaFreeHost(kv.second);
        s->blob_pool.clear();
        for (int k = 0; k < pk_server::kInstances; k++) {
            if (s->dl_exec[k]) cudaGraphExecDestroy(s->dl_exec[k]);
            if (s->dl_ev[k]) cudaEventDestroy(s->dl_ev[k]);
            if (s->dl_st[k]) cudaStreamDestroy(s->dl_st[k]);
        }
        cudaFreeHost((void*)s->ring);
        s->ring = nullptr;
        if (s->done_h) cudaFreeHost(s->done_h);
        s->done_h = nullptr;
    }
    {
        std::lock_guard<std::recursive_mutex> cl(s->ctx->mu);
        cudaSetDevice(s->ctx->device);
        cudaStreamSynchronize(s->ctx->stream);
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& kv : s->reqs) s->release(kv.second);
        for (auto& r : s->queue) s->release(r);
        for (auto& r : s->active) s->release(r);
        cudaStreamSynchronize(s->ctx->stream);
        for (auto& kv : s->stage_pool) cudaFreeHost(kv.second);
        s->stage_pool.clear();
        cudaStreamDestroy(s->up);
        cudaStreamDestroy(s->down);
    }
    delete s;
}

}  // extern "C"
