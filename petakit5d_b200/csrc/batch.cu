// Batched chunk deconvolution (pk_batch_decon): many uneven chunks, each with its own PSF pair and
// output crop (RLdecon_for_zarr_block.m:101-171, RLdecon_large_in_memory.m:177-260 run them one
// RLdecon call at a time).  Here the chunks of a wave share every launch: one launch per pass and
// transform plan covers all of them through per-chunk descriptors.  Waves are pipelined: while
// wave w computes, wave w+1 uploads and wave w-1 downloads on separate streams (host chunks
// should be in pinned memory for the copies to overlap).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

size_t dsize(pk_dtype t) { return t == PK_U16 ? 2 : t == PK_F32 ? 4 : 8; }
size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

struct Plan {
    int idx;                 // chunk index
    int rdims[3], dims[3];
    size_t in_b, out_b, work_b;
    int blocksY;
    int64_t od[3];
};

}  // namespace

extern "C" pk_status pk_batch_decon(pk_ctx* ctx, int32_t method, int32_t n, const pk_chunk* chunks, pk_dtype in_type,
                                    int32_t npsf, const float* const* psf_f, const float* const* psf_b,
                                    const int64_t* psf_dims, int32_t numit, const pk_decon_params* params,
                                    int32_t pad_good, int32_t device) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (n < 0 || (n > 0 && !chunks)) return pk_fail(PK_ERR_INVALID, "bad chunk list");
    if (method != 0 && method != 1) return pk_fail(PK_ERR_INVALID, "method must be 0 (RL) or 1 (OMW)");
    if (npsf < 1 || !psf_f || !psf_dims || (method == 1 && !psf_b)) return pk_fail(PK_ERR_INVALID, "bad PSF list");
    if (in_type != PK_U16 && in_type != PK_F32 && in_type != PK_F64) return pk_fail(PK_ERR_INVALID, "bad input dtype");
    if (numit < 0) return pk_fail(PK_ERR_INVALID, "NUMIT must be non-negative");
    pk_decon_params def;
    if (!params) {
        pk_params_default(&def);
        params = &def;
    }
    if (n == 0) return PK_OK;
    PkRange range("pk_batch_decon");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool need_mask = params->decon_offset != 0.0 || params->edge_erosion > 0;
    pk_status s;

    // ---- per-chunk plans and OTFs
    std::vector<Plan> plans(n);
    std::vector<const float2*> otf_f(n), otf_b(n, nullptr);
    // each PSF is compared with the cache once per call; its other data sizes reuse that result
    std::vector<std::shared_ptr<const std::vector<float>>> seen_f(npsf), seen_b(npsf);
    for (int i = 0; i < n; i++) {
        const pk_chunk& c = chunks[i];
        Plan& P = plans[i];
        P.idx = i;
        if (!c.in || !c.out) return pk_fail(PK_ERR_INVALID, "chunk " + std::to_string(i) + ": NULL buffer");
        if (c.psf_id < 0 || c.psf_id >= npsf) return pk_fail(PK_ERR_INVALID, "chunk " + std::to_string(i) + ": bad psf_id");
        pk_decon_params q = *params;
        q.has_bbox = c.has_bbox;
        for (int k = 0; k < 6; k++) q.bbox[k] = c.bbox[k];
        if ((s = pk_check_params(c.dims, &q)) != PK_OK) return s;
        for (int k = 0; k < 3; k++) {
            P.rdims[k] = (int)c.dims[k];
            P.dims[k] = pad_good ? (int)pk_find_good_factor_number(c.dims[k], 1, 0) : (int)c.dims[k];
        }
        if (pad_good && params->edge_erosion > 0)
            return pk_fail(PK_ERR_UNSUPPORTED, "EdgeErosion with padded chunks is not supported (the raw mask would include the padding)");
        pk_output_dims(c.dims, &q, P.od);
        P.in_b = (size_t)c.dims[0] * c.dims[1] * c.dims[2] * dsize(in_type);
        P.out_b = (size_t)P.od[0] * P.od[1] * P.od[2] * (params->save16bit ? 2 : 4);
        VolDesc d;
        if ((s = pk_init_desc(ctx, P.dims[0], P.dims[1], P.dims[2], &d)) != PK_OK) return s;
        P.blocksY = d.blocksY;
        P.work_b = pk_job_bytes(method, P.dims, need_mask, P.blocksY) + (device ? 0 : al256(P.in_b) + al256(P.out_b));
        const int64_t* pd = psf_dims + 3 * c.psf_id;
        if ((s = pk_get_otf(ctx, psf_f[c.psf_id], pd, P.dims[0], P.dims[1], P.dims[2], &otf_f[i], st,
                            &seen_f[c.psf_id])) != PK_OK)
            return s;
        if (method == 1 && (s = pk_get_otf(ctx, psf_b[c.psf_id], pd, P.dims[0], P.dims[1], P.dims[2], &otf_b[i], st,
                                           &seen_b[c.psf_id])) != PK_OK)
            return s;
    }

    // ---- waves under a memory budget (two wave slots in flight)
    size_t freeb = 0, totalb = 0;
    PK_CUDA(cudaMemGetInfo(&freeb, &totalb));
    const size_t budget = std::max<size_t>((size_t)(freeb * 0.40), 1ull << 28);
    const int max_per_wave = device ? n : std::max(2, (n + 11) / 12);  // host mode: ~12 waves so copies overlap compute
    // chunks ordered by transform size, so a wave holds few distinct plans (each pass launches once per
    // plan in the wave, and fewer, larger launches fill the GPU better); in host mode the first wave
    // is half size, so the compute starts after a shorter first upload (8 to 16 waves measured the
    // same on 96 chunks; 24 waves, whose launches fill the GPU less, measured slower)
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const Plan& A = plans[a];
        const Plan& Bp = plans[b];
        if (A.dims[0] != Bp.dims[0]) return A.dims[0] < Bp.dims[0];
        if (A.dims[1] != Bp.dims[1]) return A.dims[1] < Bp.dims[1];
        return A.dims[2] < Bp.dims[2];
    });
    if (!device && n >= 4 * max_per_wave) {
        // host mode: the first wave's upload and the last wave's download are not hidden behind any
        // compute, so both waves take the smallest chunks (the smallest half-wave first, the next
        // smallest half-wave last); the waves between stay ordered by size
        const int h = std::max(1, max_per_wave / 2);
        std::vector<int> o2(order.begin(), order.begin() + h);
        o2.insert(o2.end(), order.begin() + 2 * h, order.end());
        o2.insert(o2.end(), order.begin() + h, order.begin() + 2 * h);
        order.swap(o2);
    }
    std::vector<std::vector<int>> waves;
    {
        std::vector<int> cur;
        size_t cb = 0;
        for (int oi = 0; oi < n; oi++) {
            const int i = order[oi];
            const bool last_h = !device && n >= 4 * max_per_wave && oi == n - std::max(1, max_per_wave / 2);
            const int cap = (!device && waves.empty()) ? std::max(1, max_per_wave / 2) : max_per_wave;
            if (last_h && !cur.empty()) {   // the smallest chunks' second half-wave is a wave of its own
                waves.push_back(cur);
                cur.clear();
                cb = 0;
            }
            if (!cur.empty() && (cb + plans[i].work_b > budget || (int)cur.size() >= cap)) {
                waves.push_back(cur);
                cur.clear();
                cb = 0;
            }
            cur.push_back(i);
            cb += plans[i].work_b;
        }
        if (!cur.empty()) waves.push_back(cur);
    }
    size_t slot_b[2] = {0, 0};
    for (size_t w = 0; w < waves.size(); w++) {
        size_t b = 0;
        for (int i : waves[w]) b += plans[i].work_b;
        slot_b[w % 2] = std::max(slot_b[w % 2], b);
    }
    if (getenv("PK_BATCH_LOG") && getenv("PK_BATCH_LOG")[0] == '1')
        fprintf(stderr, "pk_batch_decon: %d chunks, %zu waves, budget %.1f GB of %.1f GB free, slots %.1f / %.1f GB\n", n,
                waves.size(), budget / 1e9, freeb / 1e9, slot_b[0] / 1e9, slot_b[1] / 1e9);
    void* arena[2] = {nullptr, nullptr};
    for (int k = 0; k < 2 && k < (int)waves.size(); k++)
        if ((s = pk_scratch(ctx, 20 + k, slot_b[k], &arena[k])) != PK_OK) return s;

    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    auto cleanup = [&]() {
        if (h2d) { cudaStreamSynchronize(h2d); cudaStreamDestroy(h2d); }
        if (d2h) { cudaStreamSynchronize(d2h); cudaStreamDestroy(d2h); }
        cudaStreamSynchronize(st);
        for (int k = 0; k < 2; k++) {
            if (ev_in[k]) cudaEventDestroy(ev_in[k]);
            if (ev_comp[k]) cudaEventDestroy(ev_comp[k]);
            if (ev_free[k]) cudaEventDestroy(ev_free[k]);
        }
    };
    if (!device) {
        PK_CUDA(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
        PK_CUDA(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
        for (int k = 0; k < 2; k++) {
            PK_CUDA(cudaEventCreateWithFlags(&ev_in[k], cudaEventDisableTiming));
            PK_CUDA(cudaEventCreateWithFlags(&ev_comp[k], cudaEventDisableTiming));
            PK_CUDA(cudaEventCreateWithFlags(&ev_free[k], cudaEventDisableTiming));
        }
    }
    for (size_t w = 0; w < waves.size(); w++) {
        const int slot = (int)(w % 2);
        char* base = (char*)arena[slot];
        std::vector<DeconJob> jobs;
        size_t off = 0;
        if (!device) {
            if (w >= 2) cudaStreamWaitEvent(h2d, ev_free[slot], 0);   // downloads of wave w-2 have finished
        } else if (w >= 1) {
            // device mode runs waves back to back on one stream; the arena slot is reused in order
        }
        for (int i : waves[w]) {
            const Plan& P = plans[i];
            DeconJob j;
            for (int k = 0; k < 3; k++) {
                j.rdims[k] = P.rdims[k];
                j.dims[k] = P.dims[k];
            }
            j.otf_f = otf_f[i];
            j.otf_b = otf_b[i];
            j.has_bbox = chunks[i].has_bbox;
            for (int k = 0; k < 6; k++) j.bbox[k] = chunks[i].bbox[k];
            char* mine = base + off;
            pk_job_carve(j, method, need_mask, P.blocksY, mine);
            size_t o2 = pk_job_bytes(method, P.dims, need_mask, P.blocksY);
            if (device) {
                j.d_raw = chunks[i].in;
                j.d_out = chunks[i].out;
            } else {
                void* din = mine + o2;
                void* dout = mine + o2 + al256(P.in_b);
                if (cudaMemcpyAsync(din, chunks[i].in, P.in_b, cudaMemcpyHostToDevice, h2d) != cudaSuccess) {
                    cleanup();
                    return pk_fail(PK_ERR_CUDA, "chunk upload failed");
                }
                j.d_raw = din;
                j.d_out = dout;
                o2 += al256(P.in_b) + al256(P.out_b);
            }
            off += o2;
            jobs.push_back(j);
        }
        if (!device) {
            cudaEventRecord(ev_in[slot], h2d);
            cudaStreamWaitEvent(st, ev_in[slot], 0);
        }
        if ((s = pk_decon_multi(ctx, method, jobs, in_type, numit, params, st)) != PK_OK) {
            cleanup();
            return s;
        }
        if (!device) {
            cudaEventRecord(ev_comp[slot], st);
            cudaStreamWaitEvent(d2h, ev_comp[slot], 0);
            for (size_t q = 0; q < jobs.size(); q++) {
                const Plan& P = plans[waves[w][q]];
                if (cudaMemcpyAsync(chunks[P.idx].out, jobs[q].d_out, P.out_b, cudaMemcpyDeviceToHost, d2h) != cudaSuccess) {
                    cleanup();
                    return pk_fail(PK_ERR_CUDA, "chunk download failed");
                }
            }
            cudaEventRecord(ev_free[slot], d2h);
        }
    }
    cudaError_t e = device ? cudaStreamSynchronize(st) : cudaStreamSynchronize(d2h);
    cleanup();
    if (e != cudaSuccess) return pk_fail(PK_ERR_CUDA, std::string("batch: ") + cudaGetErrorString(e));
    return PK_OK;
}
