// extern "C" entry points of libpkdecon.so (declared in include/pkdecon.h).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <thread>
#include <string>
#include <vector>

#include "pk_internal.h"

static thread_local std::string g_err;

void pk_set_error(const std::string& msg) { g_err = msg; }
pk_status pk_fail(pk_status st, const std::string& msg) {
    g_err = msg;
    return st;
}

pk_status pk_make_otf(pk_ctx* ctx, const float* h_psf, const int64_t pd[3], int ny, int nx, int nz, double scale,
                      float2* d_otf, cudaStream_t st);

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

size_t dtype_size(pk_dtype t) { return t == PK_U16 ? 2 : t == PK_F32 ? 4 : 8; }

pk_status check_ctx(pk_ctx* ctx) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    return PK_OK;
}

pk_status check_dims(const int64_t d[3], const char* what) {
    if (!d) return pk_fail(PK_ERR_INVALID, std::string(what) + " dims must not be NULL");
    for (int i = 0; i < 3; i++)
        if (d[i] < 1) return pk_fail(PK_ERR_INVALID, std::string(what) + " is empty");
    return PK_OK;
}

pk_status check_psf(const float* psf, const int64_t d[3], const char* what) {
    pk_status s = check_dims(d, what);
    if (s != PK_OK) return s;
    if (!psf) return pk_fail(PK_ERR_INVALID, std::string(what) + " must not be NULL");
    return PK_OK;
}

cudaStream_t pick_stream(pk_ctx* ctx, void* stream) { return stream ? (cudaStream_t)stream : ctx->stream; }

}  // namespace

extern "C" {

void pk_params_default(pk_decon_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->background = 0.0;
    p->damp_factor = 1.0;
    p->scale_factor = 1.0;
    p->decon_offset = 0.0;
    p->edge_erosion = 0;
    p->save16bit = 1;
    p->has_bbox = 0;
}

const char* pk_last_error(void) { return g_err.c_str(); }
const char* pk_version(void) { return "pkdecon 0.1 (sm_100a)"; }

pk_ctx* pk_ctx_create(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        pk_set_error("no CUDA device " + std::to_string(device));
        return nullptr;
    }
    DeviceGuard g(device);
    pk_ctx* ctx = new pk_ctx();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        pk_set_error("cudaStreamCreate failed");
        delete ctx;
        return nullptr;
    }
    // the device-wait status word: page-locked, written by the kernels only when a wait runs out
    if (cudaHostAlloc((void**)&ctx->h_err, 64, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&ctx->d_err, ctx->h_err, 0) != cudaSuccess) {
        cudaGetLastError();
        if (ctx->h_err) cudaFreeHost(ctx->h_err);
        cudaStreamDestroy(ctx->stream);
        pk_set_error("page-locked status word: cudaHostAlloc failed");
        delete ctx;
        return nullptr;
    }
    for (int i = 0; i < 16; i++) ((volatile int*)ctx->h_err)[i] = 0;   // page-locked memory is not zeroed
    return ctx;
}

static void release_all(pk_ctx* ctx) {
    cudaStreamSynchronize(ctx->stream);
    if (ctx->h2d) { cudaStreamSynchronize(ctx->h2d); cudaStreamDestroy(ctx->h2d); ctx->h2d = nullptr; }
    if (ctx->d2h) { cudaStreamSynchronize(ctx->d2h); cudaStreamDestroy(ctx->d2h); ctx->d2h = nullptr; }
    for (auto& a : ctx->aslot) {
        if (a.d_in) cudaFree(a.d_in);
        if (a.d_out) cudaFree(a.d_out);
        for (cudaEvent_t e : {a.up, a.comp, a.down})
            if (e) cudaEventDestroy(e);
        a = pk_ctx::AsyncSlot();
    }
    for (auto& kv : ctx->tickets) cudaEventDestroy(kv.second);
    ctx->tickets.clear();
    for (auto& kv : ctx->dev_tables) cudaFree(kv.second);
    ctx->dev_tables.clear();
    for (auto e : ctx->io_ev) cudaEventDestroy(e);
    ctx->io_ev.clear();
    pk_release_graphs(ctx);
    ctx->graph_seen.clear();
    for (auto& kv : ctx->otf) cudaFree(kv.second.d);
    ctx->otf.clear();
    for (auto& s : ctx->scratch)
        if (s.first) cudaFree(s.first);
    ctx->scratch.clear();
    for (auto& sl : ctx->slots) {
        if (sl.d) cudaFree(sl.d);
        if (sl.h) cudaFreeHost(sl.h);
        if (sl.ev) cudaEventDestroy(sl.ev);
        sl = pk_ctx::ProgSlot();
    }
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    ctx->d_counter = nullptr;
}

void pk_ctx_destroy(pk_ctx* ctx) {
    if (!ctx) return;
    {
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        DeviceGuard g(ctx->device);
        release_all(ctx);
        for (auto& kv : ctx->tw) cudaFree(kv.second.d);
        ctx->tw.clear();
        for (void* p : ctx->host_pinned) cudaFreeHost(p);
    for (auto& r : ctx->prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : ctx->ev_pool) cudaEventDestroy(e);
        ctx->host_pinned.clear();
        cudaStreamDestroy(ctx->stream);
        if (ctx->h_err) cudaFreeHost(ctx->h_err);
    }
    delete ctx;
}

pk_status pk_ctx_reset(pk_ctx* ctx) {
    pk_status s = check_ctx(ctx);
    if (s != PK_OK) return s;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    release_all(ctx);
    return PK_OK;
}

void* pk_ctx_stream(pk_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t pk_ctx_kernel_launches(pk_ctx* ctx) { return ctx ? ctx->launches : 0; }

pk_status pk_ctx_profile(pk_ctx* ctx, int32_t enable) {
    pk_status s = check_ctx(ctx);
    if (s != PK_OK) return s;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    ctx->prof_on = enable != 0;
    return PK_OK;
}

int32_t pk_ctx_profile_read(pk_ctx* ctx, char* buf, int32_t cap) {
    if (!ctx) return -1;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    std::map<std::string, std::tuple<long long, double, double>> agg;
    for (auto& r : ctx->prof) {
        cudaEventSynchronize(r.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        auto& t = agg[r.kind];
        std::get<0>(t) += 1;
        std::get<1>(t) += ms;
        std::get<2>(t) = r.bytes;
        ctx->ev_pool.push_back(r.a);
        ctx->ev_pool.push_back(r.b);
    }
    ctx->prof.clear();
    std::string js = "{";
    bool first = true;
    for (auto& kv : agg) {
        char tmp[256];
        snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f, \"bytes\": %.0f}", first ? "" : ", ",
                 kv.first.c_str(), std::get<0>(kv.second), std::get<1>(kv.second), std::get<2>(kv.second));
        js += tmp;
        first = false;
    }
    js += "}";
    if (buf && cap > 0) {
        const int n = std::min((int)js.size(), cap - 1);
        memcpy(buf, js.data(), n);
        buf[n] = 0;
    }
    return (int32_t)js.size();
}

pk_status pk_output_dims(const int64_t dims[3], const pk_decon_params* p, int64_t out[3]) {
    if (!dims || !out) return pk_fail(PK_ERR_INVALID, "NULL dims");
    for (int i = 0; i < 3; i++) out[i] = dims[i];
    if (p && p->has_bbox)
        for (int i = 0; i < 3; i++) out[i] = p->bbox[i + 3] - p->bbox[i] + 1;
    return PK_OK;
}

static pk_status decon_device(pk_ctx* ctx, int method, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                              const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                              const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params,
                              void* d_out, cudaStream_t st, HostStreamIO* io = nullptr) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    if ((s = check_dims(dims, "input volume")) != PK_OK) return s;
    if ((s = check_psf(psf_f, psf_f_dims, "PSF")) != PK_OK) return s;
    if (method == 1 && (s = check_psf(psf_b, psf_b_dims, "PSF_b")) != PK_OK) return s;
    if (!d_in || !d_out) return pk_fail(PK_ERR_INVALID, "NULL input/output buffer");
    if (in_type != PK_U16 && in_type != PK_F32 && in_type != PK_F64) return pk_fail(PK_ERR_INVALID, "bad input dtype");
    pk_decon_params def;
    if (!params) {
        pk_params_default(&def);
        params = &def;
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    return pk_decon_run(ctx, method, d_in, in_type, dims, psf_f, psf_f_dims, psf_b, psf_b_dims, numit, params,
                        d_out, st, io);
}

static pk_status decon_host(pk_ctx* ctx, int method, const void* in, pk_dtype in_type, const int64_t dims[3],
                            const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                            const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params, void* out) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    if ((s = check_dims(dims, "input volume")) != PK_OK) return s;
    if (!in || !out) return pk_fail(PK_ERR_INVALID, "NULL input/output buffer");
    if (in_type != PK_U16 && in_type != PK_F32 && in_type != PK_F64) return pk_fail(PK_ERR_INVALID, "bad input dtype");
    pk_decon_params def;
    if (!params) {
        pk_params_default(&def);
        params = &def;
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    const size_t N = (size_t)dims[0] * dims[1] * dims[2];
    int64_t od[3];
    pk_output_dims(dims, params, od);
    const size_t outb = (size_t)od[0] * od[1] * od[2] * (params->save16bit ? 2 : 4);
    void *d_in, *d_out;
    if ((s = pk_scratch(ctx, 9, N * dtype_size(in_type), &d_in)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 10, outb, &d_out)) != PK_OK) return s;
    cudaStream_t st = ctx->stream;
    // the driver uploads the input (by z-slab where it can, overlapping the first passes) and, when it
    // streams, downloads the result slab by slab on its copy stream as the last passes finish
    HostStreamIO io;
    io.h_in = in;
    io.h_out = out;
    io.in_esize = dtype_size(in_type);
    io.out_esize = params->save16bit ? 2 : 4;
    s = decon_device(ctx, method, d_in, in_type, dims, psf_f, psf_f_dims, psf_b, psf_b_dims, numit, params, d_out, st,
                     &io);
    if (s != PK_OK) {
        cudaStreamSynchronize(st);
        if (ctx->h2d) cudaStreamSynchronize(ctx->h2d);
        if (ctx->d2h) cudaStreamSynchronize(ctx->d2h);
        return s;
    }
    if (io.active) {
        PK_CUDA(cudaStreamSynchronize(ctx->d2h));
        PK_CUDA(cudaStreamSynchronize(st));
    } else {
        PK_CUDA(cudaMemcpyAsync(out, d_out, outb, cudaMemcpyDeviceToHost, st));
        PK_CUDA(cudaStreamSynchronize(st));
    }
    return pk_check_device_waits(ctx);   // a device wait of this call that ran out
}

// ---- asynchronous host-buffer calls
static pk_status grow(void** p, size_t* cap, size_t need, cudaEvent_t in_use) {
    if (*cap >= need && *p) return PK_OK;
    if (in_use) PK_CUDA(cudaEventSynchronize(in_use));
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, std::max<size_t>(need, 256)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return pk_fail(PK_ERR_NOMEM, "staging buffer allocation failed");
    }
    *cap = need;
    return PK_OK;
}

pk_status pk_decon_submit(pk_ctx* ctx, int32_t method, const void* in, pk_dtype in_type, const int64_t dims[3],
                          const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                          const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params, void* out,
                          int64_t* ticket) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    if (!ticket) return pk_fail(PK_ERR_INVALID, "NULL ticket");
    if (method != 0 && method != 1) return pk_fail(PK_ERR_INVALID, "method must be 0 (RL) or 1 (OMW)");
    if ((s = check_dims(dims, "input volume")) != PK_OK) return s;
    if (!in || !out) return pk_fail(PK_ERR_INVALID, "NULL input/output buffer");
    if (in_type != PK_U16 && in_type != PK_F32 && in_type != PK_F64) return pk_fail(PK_ERR_INVALID, "bad input dtype");
    pk_decon_params def;
    if (!params) {
        pk_params_default(&def);
        params = &def;
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    if (!ctx->h2d) PK_CUDA(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
    if (!ctx->d2h) PK_CUDA(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
    pk_ctx::AsyncSlot& a = ctx->aslot[ctx->next_ticket & 1];
    for (cudaEvent_t* e : {&a.up, &a.comp, &a.down})
        if (!*e) PK_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    const size_t inb = (size_t)dims[0] * dims[1] * dims[2] * dtype_size(in_type);
    int64_t od[3];
    pk_output_dims(dims, params, od);
    const size_t outb = (size_t)od[0] * od[1] * od[2] * (params->save16bit ? 2 : 4);
    if ((s = grow(&a.d_in, &a.in_cap, inb, a.used ? a.comp : nullptr)) != PK_OK) return s;
    if ((s = grow(&a.d_out, &a.out_cap, outb, a.used ? a.down : nullptr)) != PK_OK) return s;
    cudaStream_t st = ctx->stream;
    // upload once the slot's previous call has read its input; compute once the upload has landed and
    // the slot's previous result has been downloaded; download once the compute is done
    if (a.used) PK_CUDA(cudaStreamWaitEvent(ctx->h2d, a.comp, 0));
    PK_CUDA(cudaMemcpyAsync(a.d_in, in, inb, cudaMemcpyHostToDevice, ctx->h2d));
    PK_CUDA(cudaEventRecord(a.up, ctx->h2d));
    PK_CUDA(cudaStreamWaitEvent(st, a.up, 0));
    if (a.used) PK_CUDA(cudaStreamWaitEvent(st, a.down, 0));
    if ((s = decon_device(ctx, method, a.d_in, in_type, dims, psf_f, psf_f_dims, psf_b, psf_b_dims, numit, params,
                          a.d_out, st)) != PK_OK)
        return s;
    PK_CUDA(cudaEventRecord(a.comp, st));
    PK_CUDA(cudaStreamWaitEvent(ctx->d2h, a.comp, 0));
    PK_CUDA(cudaMemcpyAsync(out, a.d_out, outb, cudaMemcpyDeviceToHost, ctx->d2h));
    PK_CUDA(cudaEventRecord(a.down, ctx->d2h));
    cudaEvent_t done;
    PK_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    PK_CUDA(cudaEventRecord(done, ctx->d2h));
    a.used = true;
    *ticket = ctx->next_ticket++;
    ctx->tickets[*ticket] = done;
    return PK_OK;
}

pk_status pk_decon_wait(pk_ctx* ctx, int64_t ticket, int32_t timeout_ms) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    cudaEvent_t ev;
    {
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        auto it = ctx->tickets.find(ticket);
        if (it == ctx->tickets.end()) return pk_fail(PK_ERR_INVALID, "unknown or already collected ticket");
        ev = it->second;
    }
    DeviceGuard g(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e;
    while ((e = cudaEventQuery(ev)) == cudaErrorNotReady) {
        if (timeout_ms >= 0 &&
            std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
            return pk_fail(PK_ERR_TIMEOUT, "pk_decon_wait: the call has not finished");
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    ctx->tickets.erase(ticket);
    cudaEventDestroy(ev);
    if (e != cudaSuccess) return pk_fail(PK_ERR_CUDA, std::string("pk_decon_wait: ") + cudaGetErrorString(e));
    return PK_OK;
}

pk_status pk_ctx_join(pk_ctx* ctx) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    for (cudaStream_t c : {ctx->h2d, ctx->d2h}) {
        if (!c) continue;
        cudaEvent_t e;
        PK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        PK_CUDA(cudaEventRecord(e, c));
        PK_CUDA(cudaStreamWaitEvent(ctx->stream, e, 0));
        cudaEventDestroy(e);
    }
    return PK_OK;
}

// err_mat of the reference's debug branch from the per-iteration MSEs (1-based rows as in MATLAB;
// decon_lucy_omw_function.m:113-127 and decon_lucy_function.m:144-158, including their use of the
// step index istp as a row index).  Returns the number of rows kept, or -1 where the reference's
// trim would fail (RL without any step index).
static int err_mat_rows(int method, int numit, int estep, const std::vector<double>& mse, std::vector<double>& e) {
    e.assign((size_t)(numit + 1) * 4, 0.0);   // e[k * 4 + c], k = 1..numit, c = 0..3
    auto E = [&](int k, int c) -> double& { return e[(size_t)k * 4 + c]; };
    int istp = -1;
    for (int k = 1; k <= numit; k++) {
        E(k, 0) = k;
        E(k, 1) = mse[k - 1];
        E(k, 2) = E(k, 1) / E(1, 1);
        if (k % estep == 0 && k > estep * 2) {
            istp = k / estep;
            E(k, 3) = std::min(std::fabs(E(istp, 2) - E(istp - 1, 2)) / 10,
                               std::fabs(E(istp, 2) + E(istp - 2, 2) - 2 * E(istp - 1, 2)) / 2);
        } else if (k < 3 * estep) {
            E(k, 3) = 1;
        } else {
            E(k, 3) = E(istp * estep, 3);
        }
    }
    if (method == 1) return numit / estep;
    return istp;
}

pk_status pk_decon_debug(pk_ctx* ctx, int32_t method, const void* in, pk_dtype in_type, const int64_t dims[3],
                         const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                         const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params,
                         int32_t save_step, void* out, double* err_mat, int32_t* err_rows, uint16_t* snapshots) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    if ((s = check_dims(dims, "input volume")) != PK_OK) return s;
    if ((s = check_psf(psf_f, psf_f_dims, "PSF")) != PK_OK) return s;
    if (method != 0 && method != 1) return pk_fail(PK_ERR_INVALID, "method must be 0 (RL) or 1 (OMW)");
    if (method == 1 && (s = check_psf(psf_b, psf_b_dims, "PSF_b")) != PK_OK) return s;
    if (!in || !out || !err_mat || !err_rows) return pk_fail(PK_ERR_INVALID, "NULL buffer");
    if (in_type != PK_U16 && in_type != PK_F32 && in_type != PK_F64) return pk_fail(PK_ERR_INVALID, "bad input dtype");
    if (numit < 1) return pk_fail(PK_ERR_INVALID, "a debug run needs NUMIT >= 1");
    if (save_step < 1) return pk_fail(PK_ERR_INVALID, "saveStep must be >= 1");
    if (method == 0 && numit < 3 * save_step)
        return pk_fail(PK_ERR_INVALID, "debug with NUMIT < 3*saveStep: the reference's err_mat trim has no step "
                                       "index then (decon_lucy_function.m:173-175)");
    pk_decon_params def;
    if (!params) {
        pk_params_default(&def);
        params = &def;
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    const size_t N = (size_t)dims[0] * dims[1] * dims[2];
    int64_t od[3];
    pk_output_dims(dims, params, od);
    const size_t outb = (size_t)od[0] * od[1] * od[2] * (params->save16bit ? 2 : 4);
    void *d_in, *d_out, *d_err, *d_snap = nullptr;
    if ((s = pk_scratch(ctx, 9, N * dtype_size(in_type), &d_in)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 10, outb, &d_out)) != PK_OK) return s;
    constexpr int kSq = 64;   // partial blocks of the error sum
    if ((s = pk_scratch(ctx, 15, sizeof(double) * ((size_t)numit + kSq), &d_err)) != PK_OK) return s;
    if (snapshots && (s = pk_scratch(ctx, 16, sizeof(uint16_t) * N, &d_snap)) != PK_OK) return s;
    cudaStream_t st = ctx->stream;
    PK_CUDA(cudaMemcpyAsync(d_in, in, N * dtype_size(in_type), cudaMemcpyHostToDevice, st));
    DebugHook hook;
    hook.after_iter = [&](int k, const float* J, const float* I) -> pk_status {
        pk_status r;
        if ((r = pk_debug_error(J, I, (long long)N, (double*)d_err + numit, kSq, (double*)d_err + (k - 1), st)) != PK_OK)
            return r;
        if (snapshots && k % save_step == 0) {
            if ((r = pk_debug_u16(J, (long long)N, (uint16_t*)d_snap, st)) != PK_OK) return r;
            PK_CUDA(cudaMemcpyAsync(snapshots + (size_t)(k / save_step - 1) * N, d_snap, sizeof(uint16_t) * N,
                                    cudaMemcpyDeviceToHost, st));
        }
        return PK_OK;
    };
    s = pk_decon_run(ctx, method, d_in, in_type, dims, psf_f, psf_f_dims, psf_b, psf_b_dims, numit, params, d_out,
                     st, nullptr, &hook);
    if (s != PK_OK) {
        cudaStreamSynchronize(st);
        return s;
    }
    std::vector<double> mse(numit);
    PK_CUDA(cudaMemcpyAsync(out, d_out, outb, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaMemcpyAsync(mse.data(), d_err, sizeof(double) * numit, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    std::vector<double> e;
    const int rows = err_mat_rows(method, numit, save_step, mse, e);
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < rows; r++) err_mat[(size_t)c * rows + r] = e[(size_t)(r + 1) * 4 + c];
    *err_rows = rows;
    return PK_OK;
}

pk_status pk_decon_lucy(pk_ctx* ctx, const void* in, pk_dtype in_type, const int64_t dims[3], const float* psf,
                        const int64_t psf_dims[3], int32_t numit, const pk_decon_params* params, void* out,
                        int32_t* iters_run) {
    pk_status s = decon_host(ctx, 0, in, in_type, dims, psf, psf_dims, nullptr, nullptr, numit, params, out);
    if (s == PK_OK && iters_run) *iters_run = numit;
    return s;
}

pk_status pk_decon_lucy_omw(pk_ctx* ctx, const void* in, pk_dtype in_type, const int64_t dims[3],
                            const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                            const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params, void* out) {
    return decon_host(ctx, 1, in, in_type, dims, psf_f, psf_f_dims, psf_b, psf_b_dims, numit, params, out);
}

pk_status pk_decon_lucy_device(pk_ctx* ctx, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                               const float* psf, const int64_t psf_dims[3], int32_t numit,
                               const pk_decon_params* params, void* d_out, void* stream) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    return decon_device(ctx, 0, d_in, in_type, dims, psf, psf_dims, nullptr, nullptr, numit, params, d_out,
                        pick_stream(ctx, stream));
}

pk_status pk_decon_lucy_omw_device(pk_ctx* ctx, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                                   const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                                   const int64_t psf_b_dims[3], int32_t numit, const pk_decon_params* params,
                                   void* d_out, void* stream) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    return decon_device(ctx, 1, d_in, in_type, dims, psf_f, psf_f_dims, psf_b, psf_b_dims, numit, params, d_out,
                        pick_stream(ctx, stream));
}

pk_status pk_psf2otf(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], const int64_t dims[3],
                     float* otf_half) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    if ((s = check_psf(psf, psf_dims, "PSF")) != PK_OK) return s;
    if ((s = check_dims(dims, "output size")) != PK_OK) return s;
    if (!otf_half) return pk_fail(PK_ERR_INVALID, "NULL output");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    const int ny = (int)dims[0], nx = (int)dims[1], nz = (int)dims[2];
    const int Py = ny / 2 + 1, Pp = Py + (Py & 1);
    const size_t nb = sizeof(float2) * (size_t)Pp * nx * nz;
    void* d;
    if ((s = pk_scratch(ctx, 10, nb, &d)) != PK_OK) return s;
    if ((s = pk_make_otf(ctx, psf, psf_dims, ny, nx, nz, 1.0, (float2*)d, ctx->stream)) != PK_OK) return s;
    PK_CUDA(cudaMemcpy2DAsync(otf_half, sizeof(float2) * Py, d, sizeof(float2) * Pp, sizeof(float2) * Py,
                              (size_t)nx * nz, cudaMemcpyDeviceToHost, ctx->stream));
    PK_CUDA(cudaStreamSynchronize(ctx->stream));
    return PK_OK;
}

static pk_status fft3(pk_ctx* ctx, int inverse, const float* d_a, const int64_t dims[3], float* d_b, void* stream) {
    pk_status s;
    if ((s = check_ctx(ctx)) != PK_OK) return s;
    if ((s = check_dims(dims, "volume")) != PK_OK) return s;
    if (!d_a || !d_b) return pk_fail(PK_ERR_INVALID, "NULL buffer");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard g(ctx->device);
    VolDesc d;
    if ((s = pk_init_desc(ctx, (int)dims[0], (int)dims[1], (int)dims[2], &d)) != PK_OK) return s;
    cudaStream_t st = pick_stream(ctx, stream);
    PkProgram prog;
    // the transforms run on a pitched work spectrum; the caller's spectrum is dense [Py nx nz]
    void* w;
    if ((s = pk_scratch(ctx, 5, sizeof(float2) * pk_spec_elems(d), &w)) != PK_OK) return s;
    const size_t rows = (size_t)d.nrows, wb = sizeof(float2) * d.Py, pb = sizeof(float2) * d.Pp;
    d.S = (float2*)w;
    if (!inverse) {
        d.src = d_a;
        pk_program_add(prog, PK_STEP_Y, Y_R2C, {d});
        pk_program_add(prog, PK_STEP_X, XZ_FWD, {d});
        pk_program_add(prog, PK_STEP_Z, XZ_FWD, {d});
    } else {
        PK_CUDA(cudaMemcpy2DAsync(w, pb, d_a, wb, wb, rows, cudaMemcpyDeviceToDevice, st));
        d.dst = d_b;
        pk_program_add(prog, PK_STEP_Z, XZ_INV, {d});
        pk_program_add(prog, PK_STEP_X, XZ_INV, {d});
        pk_program_add(prog, PK_STEP_Y, Y_C2R, {d});
    }
    if ((s = pk_program_upload(ctx, prog, st)) != PK_OK) return s;
    if ((s = pk_program_launch(ctx, prog, st)) != PK_OK) return s;
    if (!inverse) PK_CUDA(cudaMemcpy2DAsync(d_b, wb, w, pb, wb, rows, cudaMemcpyDeviceToDevice, st));
    return PK_OK;
}

pk_status pk_fft3_r2c_device(pk_ctx* ctx, const float* d_in, const int64_t dims[3], float* d_spec, void* stream) {
    return fft3(ctx, 0, d_in, dims, d_spec, stream);
}

pk_status pk_fft3_c2r_device(pk_ctx* ctx, const float* d_spec, const int64_t dims[3], float* d_out, void* stream) {
    return fft3(ctx, 1, d_spec, dims, d_out, stream);
}

// ------------------------------------------------------------------ chunking helpers
static void factorize(int64_t n, std::vector<int64_t>& f) {
    f.clear();
    for (int64_t p = 2; p * p <= n; p++)
        while (n % p == 0) {
            f.push_back(p);
            n /= p;
        }
    if (n > 1 || f.empty()) f.push_back(n);
}

int64_t pk_find_good_factor_number(int64_t n, int32_t direction, int32_t allow_odd_seven) {
    if (n < 1) return n;
    if (direction == 0) direction = 1;
    std::vector<int64_t> f;
    int64_t g = n;
    factorize(g, f);
    while (f.back() > 7 || (!allow_odd_seven && f.front() > 2 && f.back() == 7)) {
        g += direction;
        if (g < 1) return -1;
        factorize(g, f);
    }
    return g;
}

int64_t pk_chunk_coordinates(const int64_t vol[3], const int64_t batch_size[3], const int64_t block_size[3],
                             const int64_t* bbox, int32_t same_batch_size, const int64_t border[3],
                             int64_t* batch_bb, int64_t* region_bb, int64_t* local_bb) {
    if (!vol || !batch_size || !block_size || !border) return -1;
    int64_t ws[3], we[3], wsz[3], bs[3], blk[3], nsub[3];
    for (int i = 0; i < 3; i++) {
        ws[i] = bbox ? bbox[i] : 1;
        we[i] = bbox ? bbox[i + 3] : vol[i];
        wsz[i] = we[i] - ws[i] + 1;
        if (wsz[i] < 1 || batch_size[i] < 1 || block_size[i] < 1) return -1;
        bs[i] = std::min(wsz[i], batch_size[i]);
        blk[i] = std::min(wsz[i], block_size[i]);
        bs[i] = (bs[i] + blk[i] - 1) / blk[i] * blk[i];
        nsub[i] = (wsz[i] + bs[i] - 1) / bs[i];
    }
    const int64_t n = nsub[0] * nsub[1] * nsub[2];
    if (!batch_bb || !region_bb || !local_bb) return n;
    int64_t c = 0;
    for (int64_t z = 0; z < nsub[2]; z++)
        for (int64_t x = 0; x < nsub[1]; x++)
            for (int64_t y = 0; y < nsub[0]; y++, c++) {
                const int64_t sub[3] = {y, x, z};
                int64_t r[6], b[6], l[6];
                for (int i = 0; i < 3; i++) {
                    r[i] = sub[i] * bs[i] + ws[i];
                    r[i + 3] = std::min(r[i] + bs[i] - 1, we[i]);
                    b[i] = r[i];
                    b[i + 3] = r[i + 3];
                    if (same_batch_size) b[i] = b[i + 3] - bs[i] + 1;
                    b[i] = std::max<int64_t>(1, b[i] - border[i]);
                    b[i + 3] = std::min(vol[i], b[i + 3] + border[i]);
                }
                for (int i = 0; i < 3; i++) {
                    l[i] = r[i] - b[i] + 1;
                    l[i + 3] = l[i] + (r[i + 3] - r[i]);
                }
                for (int i = 0; i < 6; i++) {
                    batch_bb[c * 6 + i] = b[i];
                    local_bb[c * 6 + i] = l[i];
                    region_bb[c * 6 + i] = r[i] - ws[i % 3] + 1;
                }
            }
    return n;
}

}  // extern "C"
