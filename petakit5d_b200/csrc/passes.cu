// Host side of the pass kernels: transform plans, twiddle tables, per-volume descriptors and the
// launch programs (pass_kernels.cuh holds the kernels; kern_[a-i].cu instantiate them per plan).
//
// y pass   (k_y<plan>): one CTA = Ly consecutive rows (contiguous in HBM).  Forward: real row ->
//          length-ny/2 complex FFT -> split into the ny/2+1 half-spectrum bins.  Inverse: the
//          reverse, then the mode's per-voxel epilogue; modes that continue into the next
//          convolution transform the epilogue's output straight back, so a row makes one HBM
//          round trip between the two convolutions of an iteration.
// x/z pass (k_xz<plan>): one CTA = T adjacent spectrum columns k along a full x (or z) line;
//          XZ_CONV runs forward FFT, OTF multiply and inverse FFT on the tile in shared memory.
// Every launch covers a list of volumes (descriptors + block prefix), so the batched and served
// paths reuse the same kernels as the single-volume call.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "fft_engine.cuh"
#include "pass_kernels.cuh"
#include "pass_tma.cuh"
#include "pass_conv3.cuh"
#include "pass_yreg.cuh"
#include "pk_internal.h"
#include "plans.h"

using namespace pkfft;

void pk_fill_kernels_a(pkpass::KernelTable& t);
void pk_fill_kernels_b(pkpass::KernelTable& t);
void pk_fill_kernels_c(pkpass::KernelTable& t);
void pk_fill_kernels_d(pkpass::KernelTable& t);
void pk_fill_kernels_e(pkpass::KernelTable& t);
void pk_fill_kernels_f(pkpass::KernelTable& t);
void pk_fill_kernels_g(pkpass::KernelTable& t);
void pk_fill_kernels_h(pkpass::KernelTable& t);
void pk_fill_kernels_i(pkpass::KernelTable& t);
void pk_fill_tma_0(pkpass::TmaTable& t);
void pk_fill_tma_1(pkpass::TmaTable& t);
void pk_fill_tma_2(pkpass::TmaTable& t);
void pk_fill_tma_3(pkpass::TmaTable& t);
void pk_fill_conv3(std::vector<pkpass::Conv3Entry>& v);
void pk_fill_yreg(pkpass::YregTable& t);

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 148;
        }
    }
    return n;
}

// Every plan's kernels, with their shared-memory limits raised on the current device.
void pk_fill_all_kernels(pkpass::KernelTable& t) {
    memset(&t, 0, sizeof(t));
    pk_fill_kernels_a(t);
    pk_fill_kernels_b(t);
    pk_fill_kernels_c(t);
    pk_fill_kernels_d(t);
    pk_fill_kernels_e(t);
    pk_fill_kernels_f(t);
    pk_fill_kernels_g(t);
    pk_fill_kernels_h(t);
    pk_fill_kernels_i(t);
}

static size_t step_smem(int kind, int mode, const VolDesc& v) {
    if (kind == PK_STEP_Y)
        return sizeof(float2) * (tw_slots(v.M) + (v.odd ? 0 : v.M + 1) + padded_size(v.Ly * v.M) + v.Ly +
                                 (size_t)pkpass::y_aux_arrays(mode) * v.Ly * v.M);
    const bool conv = mode == XZ_CONV;
    if (kind == PK_STEP_X)
        return sizeof(float2) * (tw_slots(v.ax.n) + padded_size2(v.Tx * v.ax.n) + (conv ? v.Tx * v.ax.n : 0));
    if (kind == PK_STEP_Z)
        return sizeof(float2) * (tw_slots(v.az.n) + padded_size2(v.Tz * v.az.n) + (conv ? v.Tz * v.az.n : 0));
    return 0;
}

// Descriptor blobs reach the device through this kernel, which reads the page-locked host copy
// directly (zero-copy): a cudaMemcpyAsync would go through a copy engine, where it can queue behind
// a large volume upload of another stream and hold back the compute stream for the whole upload.
__global__ void k_blob_copy(uint4* __restrict__ dst, const uint4* __restrict__ src, long long n16) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

namespace {

const pkpass::KernelTable& kernels() {
    static pkpass::KernelTable t;
    static std::once_flag once;
    std::call_once(once, [] { pk_fill_all_kernels(t); });
    return t;
}

// The persistent TMA x / z kernels (pass_tma.cuh); PK_NO_TMA=1 keeps every x / z pass on the
// register-IO kernels (diagnostics and A/B timing).
const pkpass::TmaTable* tma_kernels() {
    static pkpass::TmaTable t;
    static bool on = false;
    static std::once_flag once;
    std::call_once(once, [] {
        memset(&t, 0, sizeof(t));
        const char* e = getenv("PK_NO_TMA");
        if (e && e[0] == '1') return;
        pk_fill_tma_0(t);
        pk_fill_tma_1(t);
        pk_fill_tma_2(t);
        pk_fill_tma_3(t);
        on = true;
    });
    return on ? &t : nullptr;
}

// The fused x-z-x convolution kernels (pass_conv3.cuh), by (x plan, z plan); used with PK_CONV3=1
// (otherwise the three separate passes run).
const std::vector<pkpass::Conv3Entry>& conv3_kernels() {
    static std::vector<pkpass::Conv3Entry> v;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* e = getenv("PK_CONV3");
        if (!(e && e[0] == '1')) return;
        pk_fill_conv3(v);
    });
    return v;
}

// The register-packing y kernels (pass_yreg.cuh); PK_NO_YREG=1 keeps every y pass on the rolled
// kernels (diagnostics and A/B timing).
const pkpass::YregTable* yreg_kernels() {
    static pkpass::YregTable t;
    static bool on = false;
    static std::once_flag once;
    std::call_once(once, [] {
        memset(&t, 0, sizeof(t));
        const char* e = getenv("PK_NO_YREG");
        if (e && e[0] == '1') return;
        pk_fill_yreg(t);
        on = true;
    });
    return on ? &t : nullptr;
}

// A y step's descriptor the register-packing kernel can take: 512-voxel rows on the 4096-point
// tiles, per-voxel inputs 16-byte aligned (bulk copies), the rolled kernel's fused-path conditions
// (no padded / float64 raw input, no damping, scaling, mask or crop in the final pass).
bool yreg_ok(const VolDesc& d, int mode) {
    auto al = [](const void* p) { return p && (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    if (d.odd || d.ny != 512 || d.M != 256 || d.tiles_small || !d.tw_rc) return false;
    switch (mode) {
        case Y_PRE: return !d.padded && (d.raw_type == PK_U16 || d.raw_type == PK_F32) && al(d.raw);
        case Y_R2C: return al(d.src);
        case Y_RATIO: return al(d.I);
        case Y_UPDATE: return al(d.Jo);
        case Y_FINAL: return al(d.Jo) && !(d.damp > 1.f || d.scale_mode != 0 || d.need_xz);
        case Y_RLPRE: return al(d.J2) && al(d.J3);
        case Y_RLUPD: return al(d.Yb) && (d.rl_first || al(d.J4));
        case Y_RLFINAL: return al(d.Yb) && !(d.damp > 1.f || d.scale_mode != 0 || d.need_xz);
        case Y_C2R: return true;
        default: return false;
    }
}

// cuTensorMapEncodeTiled from the driver, found through the runtime (no link against libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn f = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f = (EncodeTiledFn)p;
        else
            cudaGetLastError();
    });
    return f;
}

// Tensor map of a half spectrum (S or an OTF) laid out [z][x][k] with row pitch Pp, as
// {2 Py floats, nx, nz}, with the column-tile box of an x (axis 1) or z (axis 2) pass of plan p.
bool encode_spec_map(CUtensorMap* m, const void* base, const VolDesc& d, int axis, int p, int T) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc || !base || (reinterpret_cast<uintptr_t>(base) & 15)) return false;
    const int n = kPlans[p].n;
    const int rows = pkpass::tma_box_rows(n);
    const cuuint64_t dims[3] = {(cuuint64_t)2 * d.Py, (cuuint64_t)d.nx, (cuuint64_t)d.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)d.Pp * 8, (cuuint64_t)d.Pp * 8 * (cuuint64_t)d.nx};
    const cuuint32_t box[3] = {(cuuint32_t)(2 * T), (cuuint32_t)(axis == 1 ? rows : 1), (cuuint32_t)(axis == 2 ? rows : 1)};
    const cuuint32_t es[3] = {1, 1, 1};
    // L2 promotion of the TMA's DRAM fetches (PK_TMA_L2 = 0 none, 1 64 B, 2 128 B, 3 256 B: diagnostics)
    static const CUtensorMapL2promotion promo = [] {
        const char* e = getenv("PK_TMA_L2");
        const int v = e ? atoi(e) : 3;
        return v == 0 ? CU_TENSOR_MAP_L2_PROMOTION_NONE : v == 1 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
               : v == 2 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B : CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
    }();
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, promo,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Index of a step's TMA kernel in the table, or -1 when the step keeps the register-IO kernels.
int tma_index(const PkStep& s) {
    const pkpass::TmaTable* t = tma_kernels();
    if (!t || s.plan <= 0 || s.plan >= kNumPlans || !pkpass::tma_plan(s.plan)) return -1;
    int idx = -1;
    if (s.kind == PK_STEP_X && s.mode == XZ_FWD) idx = pkpass::TMA_X_FWD;
    else if (s.kind == PK_STEP_X && s.mode == XZ_INV) idx = pkpass::TMA_X_INV;
    else if (s.kind == PK_STEP_Z && s.mode == XZ_CONV) idx = pkpass::TMA_Z_CONV;
    if (idx < 0 || !t->k[s.plan][idx][0]) return -1;
    return idx;
}

// ------------------------------------------------------------------ autotuner of the x / z passes
// An x / z step can run on the register-IO kernel (k_xz, variant -1) or on a TMA variant (k_xzt:
// 0 = the plan's 4096-point tile with two buffers; 1, 2 = the alternatives built for the plan).
// The first time a single-volume step of a (pass, plan, size class) is seen, every candidate runs
// once to warm up and twice timed on scratch buffers of that step's geometry (zeroed spectrum and
// OTF; no live data is touched); the fastest is kept for the context and appended to an on-disk
// cache (PK_TUNE_FILE, else ~/.cache/pkdecon/tune-v5.txt), keyed by the device name, so later
// processes skip the timing.  PK_TUNE=0 turns the timing off (the fallback choice everywhere).

std::mutex g_tf_mu;
std::map<std::string, int> g_tf;   // "<device>|<key>" -> variant
bool g_tf_loaded = false;

std::string tune_path() {
    const char* e = getenv("PK_TUNE_FILE");
    if (e && *e) return e;
    const char* h = getenv("HOME");
    if (!h || !*h) return "";
    return std::string(h) + "/.cache/pkdecon/tune-v5.txt";
}

std::string device_tag(int dev) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string n = prop.name;
    for (char& c : n)
        if (c == ' ' || c == '|') c = '_';
    return n + "_sm" + std::to_string(prop.multiProcessorCount);
}

void tf_load() {
    if (g_tf_loaded) return;
    g_tf_loaded = true;
    const std::string path = tune_path();
    if (path.empty()) return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string key;
        int v = 0;
        if (ls >> key >> v) g_tf[key] = v;
    }
}

void tf_store(const std::string& key, int v, float ms) {
    const std::string path = tune_path();
    if (path.empty()) return;
    std::error_code ec;
    std::filesystem::create_directories(std::filesystem::path(path).parent_path(), ec);
    std::ofstream f(path, std::ios::app);
    if (f) f << key << " " << v << " " << ms << "\n";
}

// A candidate's name: "register-IO", or the TMA variant's tile width, compute warps and buffers.
std::string variant_name(int plan, int idx, int v) {
    if (v < 0) return "register-IO";
    const pkpass::TmaTable* t = tma_kernels();
    return "tma-" + std::to_string(t->cols[plan][idx][v]) + "col-" + std::to_string((t->threads[plan][idx][v] - 32) / 32) +
           "warps-" + std::to_string(t->nbuf[plan][idx][v]) + "buf";
}

// Times each candidate of step `s` on scratch buffers: one volume per entry of `geo` (the step's
// own volume, or for a multi-volume step of a batch or a serving round the geometries of its first
// volumes), each with its own zeroed buffers, descriptor and tensor maps; returns the fastest, or -2
// when nothing could be timed. ms[i] receives candidate i's time.
int time_candidates(pk_ctx* ctx, const PkStep& s, const std::vector<VolDesc>& geo, int idx, const std::vector<int>& cands,
                    cudaStream_t st, std::vector<float>& ms) {
    const pkpass::TmaTable* t = tma_kernels();
    const pkpass::KernelTable& kt = kernels();
    const int axis = s.kind == PK_STEP_X ? 1 : 2;
    const bool conv = s.mode == XZ_CONV;
    const int nrep = (int)geo.size();
    if (nrep < 1) return -2;
    std::vector<size_t> off(nrep + 1, 0);
    size_t Sb_all = 0;
    for (int r = 0; r < nrep; r++) {
        const size_t Sb = (size_t)8 * geo[r].Pp * geo[r].nx * geo[r].nz;
        Sb_all += Sb;
        off[r + 1] = off[r] + (conv ? 2 : 1) * ((Sb + 255) & ~(size_t)255);
    }
    if (off[nrep] > ((size_t)3 << 29)) return -2;   // above 1.5 GB of scratch: keep the default
    const size_t moff = ((size_t)nrep * sizeof(VolDesc) + 63) & ~(size_t)63;
    const size_t poff = moff + (size_t)nrep * sizeof(XZMaps);
    const size_t blob = poff + sizeof(int) * (nrep + 1);
    const size_t soff = (blob + 255) & ~(size_t)255;
    char* d = nullptr;   // stream-ordered: a device-wide synchronisation here would wait on a serving dispatcher
    if (cudaMallocAsync((void**)&d, soff + off[nrep], st) != cudaSuccess) {
        cudaGetLastError();
        return -2;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best = -2;
    float best_ms = 1e30f;
    bool ok = cudaMemsetAsync(d + soff, 0, off[nrep], st) == cudaSuccess &&
              cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
    std::vector<VolDesc> dv(geo);
    for (int r = 0; r < nrep; r++) {
        const size_t per = off[r + 1] - off[r];
        dv[r].S = (float2*)(d + soff + off[r]);
        dv[r].otf = conv ? (float2*)(d + soff + off[r] + per / 2) : nullptr;
    }
    std::vector<unsigned char> h(blob, 0);
    memcpy(h.data(), dv.data(), sizeof(VolDesc) * nrep);
    ms.assign(cands.size(), -1.f);
    for (size_t ci = 0; ok && ci < cands.size(); ci++) {
        const int v = cands[ci];
        std::vector<int> pf(nrep + 1, 0);
        int grid;
        size_t smem = 0;
        std::vector<XZMaps> m(nrep);
        memset(m.data(), 0, sizeof(XZMaps) * nrep);
        if (v < 0) {
            for (int r = 0; r < nrep; r++) {
                pf[r + 1] = pf[r] + (axis == 1 ? dv[r].blocksX : dv[r].blocksZ);
                smem = std::max(smem, step_smem(s.kind, s.mode, dv[r]));
            }
            grid = pf[nrep];
        } else {
            const int T = t->cols[s.plan][idx][v];
            bool enc = true;
            for (int r = 0; r < nrep && enc; r++)
                enc = dv[r].Py >= T && encode_spec_map(&m[r].s, dv[r].S, dv[r], axis, s.plan, T) &&
                      (!conv || encode_spec_map(&m[r].otf, dv[r].otf, dv[r], axis, s.plan, T));
            if (!enc) continue;
            for (int r = 0; r < nrep; r++)
                pf[r + 1] = pf[r] + (axis == 1 ? dv[r].nz : dv[r].nx) * ((dv[r].Py + T - 1) / T);
            grid = std::min(pf[nrep], t->per_sm[s.plan][idx][v] * sm_count());
            smem = t->smem[s.plan][idx][v];
        }
        memcpy(h.data() + moff, m.data(), sizeof(XZMaps) * nrep);
        memcpy(h.data() + poff, pf.data(), sizeof(int) * (nrep + 1));
        ok = cudaMemcpyAsync(d, h.data(), blob, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             cudaStreamSynchronize(st) == cudaSuccess;
        const VolDesc* dd = (const VolDesc*)d;
        const XZMaps* dm = (const XZMaps*)(d + moff);
        const int* dp = (const int*)(d + poff);
        auto launch = [&]() {
            if (v < 0) kt.xz[s.plan]<<<grid, PK_THREADS, smem, st>>>(dd, dp, nrep, axis, s.mode);
            else t->k[s.plan][idx][v]<<<grid, t->threads[s.plan][idx][v], smem, st>>>(dd, dm, dp, nrep, ctx->d_err);
        };
        for (int r = 0; ok && r < 1; r++) launch();
        ok = ok && cudaEventRecord(e0, st) == cudaSuccess;
        for (int r = 0; ok && r < 2; r++) launch();
        const cudaError_t le = cudaGetLastError();   // a launch that failed did no work: not a candidate
        ok = ok && cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
        float el = 0.f;
        ok = ok && cudaEventElapsedTime(&el, e0, e1) == cudaSuccess;
        if (!ok) break;
        // a time below the pass's bytes at 10 TB/s (above any B200's HBM) means the launch did not do
        // the work either
        const double floor_ms = (double)(conv ? 3 : 2) * (double)Sb_all / 10e12 * 1e3;
        if (le != cudaSuccess || el / 2.f < floor_ms) continue;
        ms[ci] = el / 2.f;
        if (ms[ci] < best_ms) {
            best_ms = ms[ci];
            best = v;
        }
    }
    if (!ok) {
        cudaGetLastError();
        best = -2;
    }
    cudaFreeAsync(d, st);
    cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGetLastError();
    return best;
}

// Size class of an x / z step: how many waves of variant 0's resident CTAs its tiles make (0: under
// one wave, 1: one to three, 2: three to twelve, 3: more -- a batch's or a serving round's steps).
// Variants are chosen per (pass, plan, size class).
int size_class(const PkProgram& prog, const PkStep& s, int idx) {
    const pkpass::TmaTable* t = tma_kernels();
    const int T = t->cols[s.plan][idx][0];
    long long tiles = 0;
    for (int i = 0; i < s.nvol; i++) {
        const VolDesc& d = prog.descs[s.desc_off + i];
        tiles += (long long)(s.kind == PK_STEP_X ? d.nz : d.nx) * ((d.Py + T - 1) / T);
    }
    const long long wave = (long long)std::max(1, t->per_sm[s.plan][idx][0]) * sm_count();
    return tiles < wave ? 0 : tiles < 3 * wave ? 1 : tiles < 12 * wave ? 2 : 3;
}

// The variant an x / z step runs: the context's earlier choice, the on-disk cache's, or a timing.
// A step times its candidates once per (pass, plan, size class, volume count): on its own volume,
// or for a multi-volume step of a batch or a serving round on its own first volumes; without a timing (inside a stream capture, PK_TUNE=0) it takes the fallback:
// register-IO under one wave of tiles, where the persistent kernel's set-up does not pay, else TMA
// variant 0.
int choose_variant(pk_ctx* ctx, const PkProgram& prog, const PkStep& s, int idx, cudaStream_t st) {
    const pkpass::TmaTable* t = tma_kernels();
    std::vector<int> cands;
    if (kernels().xz[s.plan]) cands.push_back(-1);
    for (int v = 0; v < pkpass::kTmaVariants; v++)
        if (t->k[s.plan][idx][v]) cands.push_back(v);
    const VolDesc& d0 = prog.descs[s.desc_off];
    if (const char* fv = getenv("PK_TMA_VARIANT")) {   // diagnostics: this candidate wherever it exists
        const int v = atoi(fv);
        if (fv[0] && std::find(cands.begin(), cands.end(), v) != cands.end()) return v;
    }
    const int cls = size_class(prog, s, idx);
    const int fallback = (cls == 0 && kernels().xz[s.plan]) ? -1 : 0;
    if (!ctx || cands.size() < 2) return cands.empty() ? 0 : (cands.size() == 1 ? cands[0] : fallback);
    // steps over several volumes (batches, serving rounds) time apart from single volumes, and steps
    // over 8 or more apart again: on the 96-chunk batch the 8-column x kernel of 352- and 416-long
    // lines ran 1.4-2x slower with 20 volumes per launch than the 16-column one, with 2-3 volumes not
    const int multi = s.nvol == 1 ? 0 : s.nvol < 8 ? 1 : 2;
    const std::vector<long long> key = {s.kind, s.mode, s.plan, cls, multi};
    auto it = ctx->tune.find(key);
    if (it != ctx->tune.end()) return it->second;
    std::string fkey = device_tag(ctx->device) + "|";
    for (size_t i = 0; i < key.size(); i++) fkey += (i ? "," : "") + std::to_string(key[i]);
    auto record = [&](int v, const char* source, const std::vector<float>* ms, const VolDesc& g) {
        std::string rec = "{\"pass\": \"" + std::string(pk_step_name(s)) + "\", \"n\": " + std::to_string(kPlans[s.plan].n) +
                          ", \"size_class\": " + std::to_string(cls) + ", \"timed_on\": [" + std::to_string(g.ny) + ", " +
                          std::to_string(g.nx) + ", " + std::to_string(g.nz) + "], \"chosen\": \"" +
                          variant_name(s.plan, idx, v) + "\", \"source\": \"" + source + "\"";
        if (ms) {
            rec += ", \"ms\": {";
            for (size_t i = 0; i < cands.size(); i++) {
                char tmp[96];
                snprintf(tmp, sizeof(tmp), "%s\"%s\": %.5f", i ? ", " : "", variant_name(s.plan, idx, cands[i]).c_str(),
                         ms->size() > i ? (*ms)[i] : -1.f);
                rec += tmp;
            }
            rec += "}";
        }
        rec += "}";
        ctx->tune_log.push_back(rec);
    };
    {
        std::lock_guard<std::mutex> lk(g_tf_mu);
        tf_load();
        auto f = g_tf.find(fkey);
        if (f != g_tf.end() && std::find(cands.begin(), cands.end(), f->second) != cands.end()) {
            ctx->tune[key] = f->second;
            record(f->second, "cache", nullptr, d0);
            return f->second;
        }
    }
    const char* off = getenv("PK_TUNE");
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
    if (capturing) cudaGetLastError();
    if ((off && off[0] == '0') || capturing) return fallback;   // no timing here
    // the timed geometry: the step's volume; for a multi-volume step, its volumes in order (each with
    // its own scratch buffers), up to 16 of them within the scratch limit, so that a batch of mixed
    // shapes is timed on its own mix (copies of one volume ranked the x tiles of a 96-chunk batch the
    // other way round from the batch itself)
    std::vector<VolDesc> geo{d0};
    if (multi) {
        const bool conv = s.mode == XZ_CONV;
        size_t used = 0;
        geo.clear();
        for (int i = 0; i < s.nvol && geo.size() < 16; i++) {
            const VolDesc& d = prog.descs[s.desc_off + i];
            const size_t Sb = (size_t)8 * d.Pp * d.nx * d.nz;
            const size_t need = (conv ? 2 : 1) * ((Sb + 255) & ~(size_t)255);
            if (!geo.empty() && used + need > ((size_t)3 << 29)) break;
            geo.push_back(d);
            used += need;
        }
    }
    const VolDesc& dt = d0;
    std::vector<float> ms;
    PkRange range("pk autotune");
    int best = time_candidates(ctx, s, geo, idx, cands, st, ms);
    if (best == -2) return fallback;
    ctx->tune[key] = best;
    record(best, "timed", &ms, dt);
    {
        std::lock_guard<std::mutex> lk(g_tf_mu);
        g_tf[fkey] = best;
        float bms = 0.f;
        for (size_t i = 0; i < cands.size(); i++)
            if (cands[i] == best && i < ms.size()) bms = ms[i];
        tf_store(fkey, best, bms);
    }
    return best;
}

// Replaces each x forward / z convolution / x inverse triple of one volume by one fused step when a
// fused kernel is built for its plans and the volume's column tiles fit it.
static void fuse_conv3(pk_ctx* ctx, PkProgram& prog) {
    const auto& c3 = conv3_kernels();
    if (c3.empty() || !ctx || !tma_kernels()) return;
    std::vector<PkStep> out;
    out.reserve(prog.steps.size());
    for (size_t i = 0; i < prog.steps.size(); i++) {
        const PkStep& a = prog.steps[i];
        if (i + 2 < prog.steps.size()) {
            const PkStep& z = prog.steps[i + 1];
            const PkStep& c = prog.steps[i + 2];
            const bool shape = a.kind == PK_STEP_X && a.mode == XZ_FWD && z.kind == PK_STEP_Z && z.mode == XZ_CONV &&
                               c.kind == PK_STEP_X && c.mode == XZ_INV && a.nvol == 1 && z.nvol == 1 && c.nvol == 1 &&
                               a.grid > 0 && z.grid > 0 && c.grid > 0 && a.plan == c.plan;
            int k = -1;
            if (shape) {
                const VolDesc& da = prog.descs[a.desc_off];
                const VolDesc& dz = prog.descs[z.desc_off];
                const VolDesc& dc = prog.descs[c.desc_off];
                // the three steps cover the same whole volume (not the z-slab views of a streamed call)
                const auto same = [&](const VolDesc& u) {
                    return u.S == dz.S && u.nx == dz.nx && u.nz == dz.nz && u.Py == dz.Py && u.Pp == dz.Pp;
                };
                if (same(da) && same(dc) && dz.otf)
                    for (size_t e = 0; e < c3.size() && k < 0; e++)
                        if (c3[e].k && c3[e].px == a.plan && c3[e].pz == z.plan && dz.Py >= c3[e].cols) k = (int)e;
                XZMaps m;
                if (k >= 0 && !(encode_spec_map(&m.s, dz.S, dz, 2, z.plan, c3[k].cols) &&
                                encode_spec_map(&m.otf, dz.otf, dz, 2, z.plan, c3[k].cols) &&
                                encode_spec_map(&m.s2, dz.S, dz, 1, a.plan, c3[k].cols)))
                    k = -1;   // the tensor maps cannot describe this volume: keep the separate passes
            }
            if (k >= 0) {
                // the column-tile counters live in the program's prefix array: every upload of the
                // program's blob (before each launch or graph replay) brings them in as zeros, and
                // programs that run at the same time (streams, graphs, device-launched requests)
                // each have their own blob
                const VolDesc& dz = prog.descs[z.desc_off];
                const int K = (dz.Py + c3[k].cols - 1) / c3[k].cols;
                PkStep f = z;
                f.kind = PK_STEP_CONV3;
                f.mode = 0;
                f.plan = a.plan;
                f.plan2 = z.plan;
                f.conv3 = k;
                // claim counter, X and Z counters, one 128-byte line each (from the blob's start,
                // which is 256-byte aligned in device memory)
                const size_t dbytes = sizeof(VolDesc) * prog.descs.size();
                while ((dbytes + sizeof(int) * prog.prefix.size()) % (sizeof(int) * pkpass::kC3Line)) prog.prefix.push_back(0);
                f.prefix_off = (int)prog.prefix.size();
                prog.prefix.insert(prog.prefix.end(), (size_t)pkpass::c3_counter_ints(K), 0);
                static const int grid_cap = getenv("PK_CONV3_GRID") ? atoi(getenv("PK_CONV3_GRID")) : 0;   // diagnostics
                f.grid = grid_cap > 0 ? std::min(grid_cap, sm_count()) : sm_count();
                out.push_back(f);
                i += 2;
                continue;
            }
        }
        out.push_back(a);
    }
    prog.steps.swap(out);
}

void assign_tma(pk_ctx* ctx, PkProgram& prog, cudaStream_t st) {
    fuse_conv3(ctx, prog);
    prog.maps.assign(prog.descs.size(), XZMaps());
    const pkpass::YregTable* yt = yreg_kernels();
    for (PkStep& s : prog.steps) {
        s.tma = -1;
        s.yreg = 0;
        if (s.kind == PK_STEP_CONV3) {
            // z-box map of S, z-box map of the OTF, x-box map of S (fuse_conv3 checked that they encode)
            const pkpass::Conv3Entry& e = conv3_kernels()[s.conv3];
            const VolDesc& d = prog.descs[s.desc_off];
            XZMaps& m = prog.maps[s.desc_off];
            encode_spec_map(&m.s, d.S, d, 2, s.plan2, e.cols);
            encode_spec_map(&m.otf, d.otf, d, 2, s.plan2, e.cols);
            encode_spec_map(&m.s2, d.S, d, 1, s.plan, e.cols);
            continue;
        }
        if (s.kind == PK_STEP_Y && yt && s.plan == pkpass::kYregPlan && s.grid > 0 && s.mode >= 0 &&
            s.mode <= Y_C2R && yt->k[s.mode]) {
            bool ok = true;
            for (int i = 0; i < s.nvol && ok; i++) ok = yreg_ok(prog.descs[s.desc_off + i], s.mode);
            if (ok) {
                s.yreg = 1;
                s.yreg_smem = yt->smem[s.mode];
            }
            continue;
        }
        const int idx = tma_index(s);
        if (idx < 0 || s.grid == 0) continue;
        const int axis = s.kind == PK_STEP_X ? 1 : 2;
        const pkpass::TmaTable* t = tma_kernels();
        int* pf = prog.prefix.data() + s.prefix_off;
        const int var = choose_variant(ctx, prog, s, idx, st);
        if (var < 0) {   // the register-IO kernel: its own tile prefix
            for (int i = 0; i < s.nvol; i++) {
                const VolDesc& d = prog.descs[s.desc_off + i];
                pf[i + 1] = pf[i] + (axis == 1 ? d.blocksX : d.blocksZ);
            }
            s.grid = pf[s.nvol];
            continue;
        }
        const int T = t->cols[s.plan][idx][var];
        bool ok = true;
        for (int i = 0; i < s.nvol && ok; i++) {
            const VolDesc& d = prog.descs[s.desc_off + i];
            XZMaps& m = prog.maps[s.desc_off + i];
            ok = d.Py >= T && encode_spec_map(&m.s, d.S, d, axis, s.plan, T);
            if (ok && s.mode == XZ_CONV) ok = encode_spec_map(&m.otf, d.otf, d, axis, s.plan, T);
        }
        if (!ok) continue;
        // the kernel's tiles are T columns wide: the step's tile prefix follows them
        for (int i = 0; i < s.nvol; i++) {
            const VolDesc& d = prog.descs[s.desc_off + i];
            pf[i + 1] = pf[i] + (axis == 1 ? d.nz : d.nx) * ((d.Py + T - 1) / T);
        }
        s.grid = pf[s.nvol];
        s.tma = idx;
        s.tma_var = var;
        s.tma_smem = t->smem[s.plan][idx][var];
        s.tma_grid = std::min(s.grid, t->per_sm[s.plan][idx][var] * sm_count());
    }
}

// Queues the copy of a page-locked host blob (a multiple of 16 bytes) to device memory on `st`.
pk_status blob_upload(pk_ctx* ctx, void* d, const void* h, size_t bytes, cudaStream_t st) {
    const long long n16 = (long long)((bytes + 15) / 16);
    if (n16 == 0) return PK_OK;
    const void* hd = nullptr;
    if (cudaHostGetDevicePointer((void**)&hd, const_cast<void*>(h), 0) != cudaSuccess || !hd) {
        cudaGetLastError();   // not mapped: fall back to a copy-engine copy
        PK_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
        return PK_OK;
    }
    const int grid = (int)std::min<long long>(64, std::max<long long>(1, n16 / 1024));
    k_blob_copy<<<grid, 256, 0, st>>>((uint4*)d, (const uint4*)hd, n16);
    PK_CUDA(cudaGetLastError());
    if (ctx) ctx->launches++;
    return PK_OK;
}

// Layout of an uploaded program: descriptors | block prefixes | (64-byte aligned) tensor maps.
void blob_layout(const PkProgram& prog, size_t* dbytes, size_t* moff, size_t* total) {
    *dbytes = sizeof(VolDesc) * prog.descs.size();
    const size_t pend = *dbytes + sizeof(int) * prog.prefix.size();
    *moff = (pend + 63) & ~(size_t)63;
    *total = *moff + sizeof(XZMaps) * prog.maps.size();
}

void blob_fill(const PkProgram& prog, void* h) {
    size_t dbytes, moff, total;
    blob_layout(prog, &dbytes, &moff, &total);
    memcpy(h, prog.descs.data(), dbytes);
    memcpy((char*)h + dbytes, prog.prefix.data(), sizeof(int) * prog.prefix.size());
    if (!prog.maps.empty()) memcpy((char*)h + moff, prog.maps.data(), sizeof(XZMaps) * prog.maps.size());
}

// lambda = clamp(sum((J2-Y).*J4) / (sum(J4.*J4) + eps), 0, 1)  (decon_lucy_function.m:126-127),
// one CTA per volume, fixed summation order; the result goes to partials[0].
__global__ void k_lambda(const VolDesc* __restrict__ descs, int nvol) {
    const VolDesc& d = descs[blockIdx.x];
    __shared__ double s0[256], s1[256];
    const int tid = threadIdx.x;
    double a = 0.0, b = 0.0;
    for (int i = tid; i < d.blocksY; i += blockDim.x) {
        a += d.partials[2 + 2 * i];
        b += d.partials[3 + 2 * i];
    }
    s0[tid] = a;
    s1[tid] = b;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (tid < s) {
            s0[tid] += s0[tid + s];
            s1[tid] += s1[tid + s];
        }
        __syncthreads();
    }
    if (tid == 0) {
        double lam = s0[0] / (s1[0] + 2.220446049250313e-16);
        lam = fmax(fmin(lam, 1.0), 0.0);
        d.partials[0] = lam;
    }
}

}  // namespace

// One CTA waits on an mbarrier that nothing arrives on: the bounded wait runs out after limit_ns
// and the failure goes to the context's status word (the self-test of the device waits).
__global__ void k_wait_selftest(int* err, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        pktma::mbar_init(&bar, 1);
        pktma::fence_mbar_init();
    }
    __syncthreads();
    const bool ok = pktma::mbar_wait(&bar, 0, limit_ns);
    if (!__syncthreads_and(ok) && threadIdx.x == 0) pktma::report_wait_failure(err, 1);
}

// ------------------------------------------------------------------ host: plans and tables
bool pk_make_axis_plan(int n, AxisPlan* p) {
    p->n = n;
    p->nst = 0;
    if (n < 1) return false;
    int r = n;
    auto push = [&](int R) {
        if (p->nst >= PK_MAXST) return false;
        p->rad[p->nst++] = R;
        r /= R;
        return true;
    };
    while (r % 16 == 0) if (!push(16)) return false;
    if (r % 8 == 0) { if (!push(8)) return false; }
    else if (r % 4 == 0) { if (!push(4)) return false; }
    else if (r % 2 == 0) { if (!push(2)) return false; }
    while (r % 5 == 0) if (!push(5)) return false;
    while (r % 3 == 0) if (!push(3)) return false;
    for (int f = 7; r > 1; f += 2) {
        while (r % f == 0) if (!push(f)) return false;
        if ((long long)f * f > r && r > 1) { if (!push(r)) return false; }
    }
    return true;
}

// root exp(-2 pi i k / n), exact at the multiples of pi/2 so symmetric bins stay symmetric
static float2 root_of(int k, int n) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    double c = std::cos(a), s = std::sin(a);
    if ((4LL * k) % n == 0) {
        const int q = (int)((4LL * k) / n) & 3;
        c = q == 0 ? 1 : q == 2 ? -1 : 0;
        s = q == 1 ? -1 : q == 3 ? 1 : 0;
    }
    return make_float2((float)c, (float)s);
}

void pk_root_table(int n, float2* h) {
    for (int k = 0; k < n; k++) h[k] = root_of(k, n);
}

pk_status pk_get_twiddles(pk_ctx* ctx, int twN, const float2** out) {
    auto it = ctx->tw.find(twN);
    if (it != ctx->tw.end()) { *out = it->second.d; return PK_OK; }
    std::vector<float2> h(twN);
    pk_root_table(twN, h.data());
    TwTable t;
    t.n = twN;
    PK_CUDA(cudaMalloc(&t.d, sizeof(float2) * twN));
    PK_CUDA(cudaMemcpy(t.d, h.data(), sizeof(float2) * twN, cudaMemcpyHostToDevice));
    ctx->tw[twN] = t;
    *out = t.d;
    return PK_OK;
}

// Axis table of length-n transforms: the stage-ordered table of n's compile-time plan (entries
// taken from the root table), else the root table itself.
int pk_axis_table(int n, float2* out) {
    const int p = pk_find_plan(n);
    if (p == 0) {
        pk_root_table(n, out);
        return n;
    }
    int o = 0;
    int ns = 1;
    for (int s = 0; s < kPlans[p].nst; s++) {
        const int R = kPlans[p].rad[s];
        const int tstep = n / (ns * R);
        if (ns > 1)
            for (int r = 1; r < R; r++)
                for (int k = 0; k < ns; k++) out[o++] = root_of(r * k * tstep, n);
        if (direct_radix(R))
            for (int e = 0; e < R; e++) out[o++] = root_of(e * (n / R), n);
        ns *= R;
    }
    return o;
}

pk_status pk_get_axis_table(pk_ctx* ctx, int n, const float2** out) {
    const int key = -n;   // root tables use the positive keys
    auto it = ctx->tw.find(key);
    if (it != ctx->tw.end()) { *out = it->second.d; return PK_OK; }
    std::vector<float2> h(n + PK_TW_EXTRA);
    const int cnt = pk_axis_table(n, h.data());
    TwTable t;
    t.n = cnt;
    PK_CUDA(cudaMalloc(&t.d, sizeof(float2) * cnt));
    PK_CUDA(cudaMemcpy(t.d, h.data(), sizeof(float2) * cnt, cudaMemcpyHostToDevice));
    ctx->tw[key] = t;
    *out = t.d;
    return PK_OK;
}

pk_status pk_fill_axis(pk_ctx* ctx, int n, int twN, AxisDev* a) {
    AxisPlan p;
    if (!pk_make_axis_plan(n, &p)) return pk_fail(PK_ERR_UNSUPPORTED, "transform length " + std::to_string(n) + " needs too many radix stages");
    memset(a, 0, sizeof(*a));
    a->n = n;
    a->nst = p.nst;
    for (int i = 0; i < p.nst; i++) a->rad[i] = p.rad[i];
    a->twN = twN;
    a->twStride = twN / n;
    a->plan = pk_find_plan(n);
    return pk_get_axis_table(ctx, n, &a->tw);
}

static const int kThreads = PK_THREADS;

pk_status pk_init_desc(pk_ctx* ctx, int ny, int nx, int nz, VolDesc* d) {
    memset(d, 0, sizeof(*d));
    if (ny < 1 || nx < 1 || nz < 1) return pk_fail(PK_ERR_INVALID, "volume dimensions must be positive");
    d->ny = ny; d->nx = nx; d->nz = nz;
    d->odd = ny & 1;
    d->M = d->odd ? ny : ny / 2;
    d->Py = ny / 2 + 1;
    d->Pp = d->Py + (d->Py & 1);
    d->nrows = (long long)nx * nz;
    const int P = PK_TILE_POINTS;  // complex points one CTA holds
    if (d->M > P || nx > P || nz > P)
        return pk_fail(PK_ERR_UNSUPPORTED, "a transform axis is longer than " + std::to_string(P) +
                                               " (" + std::to_string(2 * P) + " along y)");
    pk_status st;
    if ((st = pk_fill_axis(ctx, d->M, d->M, &d->ay)) != PK_OK) return st;
    if ((st = pk_fill_axis(ctx, nx, nx, &d->ax)) != PK_OK) return st;
    if ((st = pk_fill_axis(ctx, nz, nz, &d->az)) != PK_OK) return st;
    if (!d->odd && (st = pk_get_twiddles(ctx, ny, &d->tw_rc)) != PK_OK) return st;
    d->Ly = d->ay.plan ? plan_lines_y(d->M) : std::max(1, P / d->M);
    if ((long long)d->Ly > d->nrows && d->ay.plan == 0) d->Ly = (int)d->nrows;
    d->Tx = d->ax.plan ? plan_cols_xz(nx) : std::max(1, std::min(P / nx, d->Py));
    d->Tz = d->az.plan ? plan_cols_xz(nz) : std::max(1, std::min(P / nz, d->Py));
    auto set_blocks = [&]() {
        const int ct_x = (d->Py + d->Tx - 1) / d->Tx, ct_z = (d->Py + d->Tz - 1) / d->Tz;
        d->blocksY = (int)((d->nrows + d->Ly - 1) / d->Ly);
        d->blocksX = nz * ct_x;
        d->blocksZ = nx * ct_z;
    };
    set_blocks();
    // a volume whose y pass would not give every SM two waves of 3 CTAs runs on 1024-point tiles
    if (small_tile_plan(d->ay.plan) && small_tile_plan(d->ax.plan) && small_tile_plan(d->az.plan) &&
        d->blocksY < 2 * 3 * sm_count()) {
        d->Ly = plan_lines_y(d->M, PK_TILE_SMALL);
        d->Tx = plan_cols_xz(nx, PK_TILE_SMALL);
        d->Tz = plan_cols_xz(nz, PK_TILE_SMALL);
        d->tiles_small = 1;
        set_blocks();
    }
    d->bb0[0] = d->bb0[1] = d->bb0[2] = 0;
    d->bb1[0] = ny - 1; d->bb1[1] = nx - 1; d->bb1[2] = nz - 1;
    d->scale = 1.f;
    d->xz_scale = 1.f;
    return PK_OK;
}

size_t pk_spec_elems(const VolDesc& d) { return (size_t)d.Pp * (size_t)d.nrows; }

// ------------------------------------------------------------------ programs
// A program is the full launch sequence of a call (or of a batch / serving round): every step's
// descriptors and block prefix live in one device buffer uploaded once, so the launches run
// back to back without host synchronisation and can be captured into a CUDA graph.
// Kernel-table index of a pass: the axis plan, offset by kNumPlans for the small-tile kernels.
static int step_plan(int kind, const VolDesc& v) {
    const int p = kind == PK_STEP_Y ? v.ay.plan : kind == PK_STEP_X ? v.ax.plan : kind == PK_STEP_Z ? v.az.plan : 0;
    return (v.tiles_small && kind != PK_STEP_LAMBDA) ? kNumPlans + p : p;
}

// One step per distinct transform plan among `vols` (a launch is instantiated for one plan).
void pk_program_add(PkProgram& prog, int kind, int mode, const std::vector<VolDesc>& vols) {
    std::vector<int> plans;
    for (const VolDesc& v : vols) {
        const int p = step_plan(kind, v);
        if (std::find(plans.begin(), plans.end(), p) == plans.end()) plans.push_back(p);
    }
    for (int plan : plans) {
        PkStep s;
        s.kind = kind;
        s.mode = mode;
        s.plan = plan;
        s.desc_off = (int)prog.descs.size();
        s.prefix_off = (int)prog.prefix.size();
        prog.prefix.push_back(0);
        size_t smem = 0;
        int nv = 0;
        for (const VolDesc& v : vols) {
            if (step_plan(kind, v) != plan) continue;
            int blocks = kind == PK_STEP_Y ? v.blocksY : kind == PK_STEP_X ? v.blocksX : kind == PK_STEP_Z ? v.blocksZ : 1;
            smem = std::max(smem, step_smem(kind, mode, v));
            prog.prefix.push_back(prog.prefix.back() + blocks);
            prog.descs.push_back(v);
            nv++;
        }
        s.nvol = nv;
        s.grid = prog.prefix.back();
        s.smem = smem;
        prog.steps.push_back(s);
    }
}

pk_status pk_program_upload(pk_ctx* ctx, PkProgram& prog, cudaStream_t st) {
    for (VolDesc& d : prog.descs) d.chk = ctx && ctx->d_err ? ctx->d_err + 1 : nullptr;
    assign_tma(ctx, prog, st);
    size_t dbytes, moff, need;
    blob_layout(prog, &dbytes, &moff, &need);
    const int si = ctx->next_slot;
    ctx->next_slot = (ctx->next_slot + 1) % 4;
    pk_ctx::ProgSlot& sl = ctx->slots[si];
    if (sl.used) PK_CUDA(cudaEventSynchronize(sl.ev));   // launches that read this slot are done
    sl.used = false;
    if (!sl.ev) PK_CUDA(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
    if (sl.cap < need) {
        if (sl.d) cudaFree(sl.d);
        if (sl.h) cudaFreeHost(sl.h);
        sl.d = sl.h = nullptr;
        sl.cap = 0;
        const size_t cap = std::max(need, (size_t)64 * 1024);
        PK_CUDA(cudaMalloc(&sl.d, cap));
        PK_CUDA(cudaMallocHost(&sl.h, cap));
        sl.cap = cap;
    }
    blob_fill(prog, sl.h);
    {
        const pk_status bs = blob_upload(ctx, sl.d, sl.h, need, st);
        if (bs != PK_OK) return bs;
    }
    prog.d_desc = (VolDesc*)sl.d;
    prog.d_prefix = (int*)((char*)sl.d + dbytes);
    prog.d_maps = (XZMaps*)((char*)sl.d + moff);
    prog.slot = si;
    return PK_OK;
}

const char* pk_step_name(const PkStep& s) {
    static const char* yn[] = {"y_r2c", "y_pre", "y_ratio", "y_update", "y_final", "y_rlpre", "y_rlupd", "y_rlfinal", "y_c2r"};
    static const char* xn[] = {"x_fwd", "x_inv", "x_conv", "x_fwd_scale"};
    static const char* zn[] = {"z_fwd", "z_inv", "z_conv", "z_fwd_scale"};
    if (s.kind == PK_STEP_Y) return yn[s.mode];
    if (s.kind == PK_STEP_X) return xn[s.mode];
    if (s.kind == PK_STEP_Z) return zn[s.mode];
    if (s.kind == PK_STEP_CONV3) return "xzx_conv";
    return "lambda";
}

// Algorithmic HBM bytes of one launch: the minimum each pass must read and write.
double pk_step_bytes(const PkStep& s, const VolDesc* descs) {
    double b = 0;
    for (int i = 0; i < s.nvol; i++) {
        const VolDesc& d = descs[i];
        const double N = (double)d.nrows * d.ny, Sb = 8.0 * d.Py * (double)d.nrows;
        const double ob = (double)(d.bb1[0] - d.bb0[0] + 1) * (d.bb1[1] - d.bb0[1] + 1) * (d.bb1[2] - d.bb0[2] + 1) * (d.save16 ? 2 : 4);
        if (s.kind == PK_STEP_Y) {
            switch (s.mode) {
                case Y_R2C: b += 4 * N + Sb; break;
                case Y_PRE: b += (d.raw_type == PK_U16 ? 2 : d.raw_type == PK_F32 ? 4 : 8) * N + 4 * N + Sb + (d.write_mask ? N : 0); break;
                case Y_RATIO: b += 2 * Sb + 4 * N; break;
                case Y_UPDATE: b += 2 * Sb + 8 * N; break;
                case Y_FINAL: b += Sb + 4 * N + (d.damp > 1.f ? 4 * N : 0) + ob; break;
                case Y_RLPRE: b += 12 * N + Sb; break;
                case Y_RLUPD: b += Sb + (d.rl_first ? 12 : 16) * N; break;
                case Y_RLFINAL: b += Sb + 4 * N + ob; break;
                case Y_C2R: b += Sb + 4 * N; break;
            }
        } else if (s.kind == PK_STEP_X || s.kind == PK_STEP_Z) {
            b += (s.mode == XZ_CONV ? 3 : 2) * Sb;
        } else if (s.kind == PK_STEP_CONV3) {
            b += 3 * Sb;   // S in, the OTF in, S out: the convolution's ruler
        } else {
            b += 16.0 * d.blocksY;
        }
    }
    return b;
}

// A device-launched request graph's last node: every pass before it is done.
__global__ void k_req_done(int* done) {
    if (threadIdx.x == 0) {
        __threadfence_system();
        *(volatile int*)done = 1;
    }
}

static pk_status launch_steps(pk_ctx* ctx, const PkProgram& prog, cudaStream_t st, size_t b = 0,
                              size_t e = (size_t)-1) {
    const pkpass::KernelTable& kt = kernels();
    e = std::min(e, prog.steps.size());
    for (size_t si = b; si < e; si++) {
        const PkStep& s = prog.steps[si];
        const VolDesc* dd = prog.d_desc + s.desc_off;
        const int* dp = prog.d_prefix + s.prefix_off;
        if (s.grid == 0) continue;
        PkRange range(pk_step_name(s));
        pk_ctx::ProfRec rec;
        if (ctx && ctx->prof_on) {
            auto take = [&]() {
                cudaEvent_t e;
                if (!ctx->ev_pool.empty()) { e = ctx->ev_pool.back(); ctx->ev_pool.pop_back(); }
                else cudaEventCreate(&e);
                return e;
            };
            rec.kind = pk_step_name(s);
            static const bool detail = getenv("PK_PROF_DETAIL") && getenv("PK_PROF_DETAIL")[0] == '1';
            if (detail) {   // diagnostics: the transform length and the kernel family in the kind
                const int pl = s.plan % kNumPlans;
                rec.kind += "@" + std::to_string(kPlans[pl].n) +
                            (s.tma >= 0 ? ":tma" : s.yreg ? ":yreg" : s.kind == PK_STEP_Y ? ":rolled" : ":rio") +
                            (s.plan >= kNumPlans ? "-1k" : "");
            }
            rec.bytes = pk_step_bytes(s, prog.descs.data() + s.desc_off);
            rec.a = take();
            rec.b = take();
            cudaEventRecord(rec.a, st);
        }
        if (s.kind == PK_STEP_CONV3) {
            const pkpass::Conv3Entry& c3 = conv3_kernels()[s.conv3];
            c3.k<<<s.grid, c3.threads, c3.smem, st>>>(dd, prog.d_maps + s.desc_off, const_cast<int*>(dp),
                                                     ctx ? ctx->d_err : nullptr);
        } else if (s.tma >= 0) {
            tma_kernels()->k[s.plan][s.tma][s.tma_var]<<<s.tma_grid, tma_kernels()->threads[s.plan][s.tma][s.tma_var],
                                                         s.tma_smem, st>>>(
                dd, prog.d_maps + s.desc_off, dp, s.nvol, ctx ? ctx->d_err : nullptr);
        } else if (s.yreg) {
            yreg_kernels()->k[s.mode]<<<s.grid, kThreads, s.yreg_smem, st>>>(dd, dp, s.nvol, ctx ? ctx->d_err : nullptr);
        } else if (s.kind == PK_STEP_Y) {
            kt.y[s.plan][s.mode]<<<s.grid, kThreads, s.smem, st>>>(dd, dp, s.nvol, s.mode);
        } else if (s.kind == PK_STEP_X || s.kind == PK_STEP_Z) {
            kt.xz[s.plan]<<<s.grid, kThreads, s.smem, st>>>(dd, dp, s.nvol, s.kind == PK_STEP_X ? 1 : 2, s.mode);
        } else if (s.kind == PK_STEP_LAMBDA) {
            k_lambda<<<s.nvol, 256, 0, st>>>(dd, s.nvol);
        }
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess)
            return pk_fail(PK_ERR_CUDA, std::string("launch of ") + pk_step_name(s) + " (plan " + std::to_string(s.plan) +
                                            ", grid " + std::to_string(s.grid) + ", smem " + std::to_string(s.smem) +
                                            "): " + cudaGetErrorString(le));
        if (ctx && ctx->prof_on) {
            cudaEventRecord(rec.b, st);
            ctx->prof.push_back(rec);
        }
    }
    return PK_OK;
}

// The program's launches as a graph of kernel nodes in launch order, built node by node (no stream
// capture, so other threads' CUDA calls cannot disturb it).

static bool build_graph(const PkProgram& prog, const VolDesc* d_desc, const int* d_prefix, const XZMaps* d_maps,
                        int* d_err, cudaGraphExec_t* out, unsigned long long flags = 0, int* d_done = nullptr) {
    const pkpass::KernelTable& kt = kernels();
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) { cudaGetLastError(); return false; }
    cudaGraphNode_t prev = nullptr;
    bool ok = true;
    for (const PkStep& s : prog.steps) {
        if (s.grid == 0) continue;
        const VolDesc* dd = d_desc + s.desc_off;
        const int* dp = d_prefix + s.prefix_off;
        const XZMaps* dm = d_maps + s.desc_off;
        int* de = d_err;
        int nvol = s.nvol, mode = s.mode, axis = s.kind == PK_STEP_X ? 1 : 2;
        void* args5[] = {(void*)&dd, (void*)&dp, (void*)&nvol, (void*)&axis, (void*)&mode};
        void* args4[] = {(void*)&dd, (void*)&dp, (void*)&nvol, (void*)&mode};
        void* args2[] = {(void*)&dd, (void*)&nvol};
        void* argst[] = {(void*)&dd, (void*)&dm, (void*)&dp, (void*)&nvol, (void*)&de};
        void* argsy[] = {(void*)&dd, (void*)&dp, (void*)&nvol, (void*)&de};
        cudaKernelNodeParams p = {};
        p.blockDim = dim3(kThreads);
        p.gridDim = dim3(s.grid);
        p.sharedMemBytes = (unsigned)s.smem;
        int* cnt = const_cast<int*>(dp);
        void* argsc[] = {(void*)&dd, (void*)&dm, (void*)&cnt, (void*)&de};
        if (s.kind == PK_STEP_CONV3) {
            const pkpass::Conv3Entry& c3 = conv3_kernels()[s.conv3];
            p.func = (void*)c3.k;
            p.blockDim = dim3(c3.threads);
            p.sharedMemBytes = (unsigned)c3.smem;
            p.kernelParams = argsc;
        } else if (s.tma >= 0) {
            p.func = (void*)tma_kernels()->k[s.plan][s.tma][s.tma_var];
            p.gridDim = dim3(s.tma_grid);
            p.blockDim = dim3(tma_kernels()->threads[s.plan][s.tma][s.tma_var]);
            p.sharedMemBytes = (unsigned)s.tma_smem;
            p.kernelParams = argst;
        } else if (s.yreg) {
            p.func = (void*)yreg_kernels()->k[s.mode];
            p.sharedMemBytes = (unsigned)s.yreg_smem;
            p.kernelParams = argsy;
        } else if (s.kind == PK_STEP_Y) {
            p.func = (void*)kt.y[s.plan][s.mode];
            p.kernelParams = args4;
        } else if (s.kind == PK_STEP_X || s.kind == PK_STEP_Z) {
            p.func = (void*)kt.xz[s.plan];
            p.kernelParams = args5;
        } else {
            p.func = (void*)k_lambda;
            p.gridDim = dim3(s.nvol);
            p.blockDim = dim3(256);
            p.sharedMemBytes = 0;
            p.kernelParams = args2;
        }
        cudaGraphNode_t node = nullptr;
        const cudaError_t ea = cudaGraphAddKernelNode(&node, g, prev ? &prev : nullptr, prev ? 1 : 0, &p);
        if (ea != cudaSuccess) {
            if (getenv("PK_DEBUG_GRAPHS")) fprintf(stderr, "graph node %s: %s\n", pk_step_name(s), cudaGetErrorString(ea));
            ok = false;
            break;
        }
        prev = node;
    }
    if (ok && d_done) {
        cudaKernelNodeParams p = {};
        void* args[] = {(void*)&d_done};
        p.func = (void*)k_req_done;
        p.gridDim = dim3(1);
        p.blockDim = dim3(32);
        p.kernelParams = args;
        cudaGraphNode_t node = nullptr;
        ok = cudaGraphAddKernelNode(&node, g, prev ? &prev : nullptr, prev ? 1 : 0, &p) == cudaSuccess;
    }
    if (ok) {
        const cudaError_t ei = cudaGraphInstantiate(out, g, flags);
        if (ei != cudaSuccess) {
            if (getenv("PK_DEBUG_GRAPHS")) fprintf(stderr, "graph instantiate: %s\n", cudaGetErrorString(ei));
            ok = false;
        }
    }
    if (getenv("PK_DEBUG_GRAPHS")) fprintf(stderr, "graph of %zu steps built: %d\n", prog.steps.size(), (int)ok);
    cudaGraphDestroy(g);
    if (!ok) cudaGetLastError();
    return ok;
}

static bool graphs_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("PK_NO_GRAPHS");
        v = (e && e[0] == '1') ? 0 : 1;
    }
    return v == 1;
}

// Launches a program's kernels.  A program seen before with the same launch shapes and descriptor
// layout replays a CUDA graph of its launches, whose descriptor buffer is refreshed on the stream
// before each replay; per-kernel profiling and a stream the caller is capturing take the direct path.
pk_status pk_check_device_waits(pk_ctx* ctx) {
    if (ctx && ctx->h_err && *(volatile int*)ctx->h_err != 0) {
        *(volatile int*)ctx->h_err = 0;
        return pk_fail(PK_ERR_TIMEOUT, "a bounded wait on the device ran out in an earlier call of this context "
                                       "(its results are not valid)");
    }
    if (ctx && ctx->h_err && *(volatile int*)(ctx->h_err + 1) != 0) {
        const int code = *(volatile int*)(ctx->h_err + 1);
        *(volatile int*)(ctx->h_err + 1) = 0;
        return pk_fail(PK_ERR_INTERNAL, "index check " + std::to_string(code) +
                                            " of the bounds-checked build failed (the access was skipped)");
    }
    return PK_OK;
}

extern "C" int32_t pk_checked_build(void) {
#ifdef PK_CHECK
    return 1;
#else
    return 0;
#endif
}

pk_status pk_program_launch(pk_ctx* ctx, PkProgram& prog, cudaStream_t st) {
    PkRange range("pk program launch");
    {
        const pk_status w = pk_check_device_waits(ctx);
        if (w != PK_OK) return w;
    }
    const int nk = pk_program_kernel_count(prog);
    bool direct = !ctx || ctx->prof_on || prog.slot < 0 || prog.no_graph || !graphs_enabled() || nk < 2;
    if (!direct) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
            cudaGetLastError();
            direct = true;
        } else if (cs != cudaStreamCaptureStatusNone) {
            direct = true;
        }
    }
    pk_status rs = PK_OK;
    if (direct) {
        rs = launch_steps(ctx, prog, st);
    } else {
        std::vector<long long> key;
        key.reserve(2 + 8 * prog.steps.size());
        key.push_back((long long)prog.descs.size());
        key.push_back((long long)prog.prefix.size());
        for (const PkStep& s : prog.steps) {
            const long long v[] = {s.kind, s.mode, s.plan, s.nvol, s.grid, (long long)s.smem, s.desc_off, s.prefix_off,
                                   s.tma, s.tma_var, s.tma_grid, s.yreg, s.conv3};
            key.insert(key.end(), v, v + 13);
        }
        auto it = ctx->graphs.find(key);
        if (it == ctx->graphs.end() && ctx->graph_seen.size() >= 4096) ctx->graph_seen.clear();  // bounded
        int* seen = it == ctx->graphs.end() ? &ctx->graph_seen[key] : nullptr;
        if (seen && (*seen < 0 || (*seen)++ == 0)) {
            rs = launch_steps(ctx, prog, st);   // first sighting (or no graph possible): launch directly
        } else {
            if (it == ctx->graphs.end()) {
                if (ctx->graphs.size() >= 64) pk_release_graphs(ctx);   // bounded cache: start over
                size_t dbytes, moff, total;
                blob_layout(prog, &dbytes, &moff, &total);
                pk_ctx::GraphEntry e;
                e.bytes = total;
                bool ok = cudaMalloc(&e.d, e.bytes) == cudaSuccess && cudaMallocHost(&e.h, e.bytes) == cudaSuccess &&
                          cudaEventCreateWithFlags(&e.ev, cudaEventDisableTiming) == cudaSuccess;
                ok = ok && build_graph(prog, (const VolDesc*)e.d, (const int*)((char*)e.d + dbytes),
                                       (const XZMaps*)((char*)e.d + moff), ctx->d_err, &e.exec);
                if (!ok) {
                    cudaGetLastError();
                    if (e.d) cudaFree(e.d);
                    if (e.h) cudaFreeHost(e.h);
                    if (e.ev) cudaEventDestroy(e.ev);
                    *seen = -1;   // never try this program again
                    rs = launch_steps(ctx, prog, st);
                } else {
                    it = ctx->graphs.emplace(key, e).first;
                }
            }
            if (it != ctx->graphs.end()) {
                pk_ctx::GraphEntry& e = it->second;
                if (e.used) PK_CUDA(cudaEventSynchronize(e.ev));   // the previous refresh has been read
                blob_fill(prog, e.h);
                {
                    const pk_status bs = blob_upload(ctx, e.d, e.h, e.bytes, st);
                    if (bs != PK_OK) return bs;
                }
                PK_CUDA(cudaGraphLaunch(e.exec, st));
                PK_CUDA(cudaEventRecord(e.ev, st));
                e.used = true;
            }
        }
    }
    if (rs != PK_OK) return rs;
    if (ctx) ctx->launches += nk;
    if (ctx && prog.slot >= 0) {
        pk_ctx::ProgSlot& sl = ctx->slots[prog.slot];
        PK_CUDA(cudaEventRecord(sl.ev, st));
        sl.used = true;
    }
    return PK_OK;
}

pk_status pk_program_device_graph(pk_ctx* ctx, PkProgram& prog, cudaStream_t st, int* d_done,
                                  const std::function<void*(size_t)>& host_blob, void** d_blob, cudaGraphExec_t* out) {
    *d_blob = nullptr;
    for (VolDesc& d : prog.descs) d.chk = ctx && ctx->d_err ? ctx->d_err + 1 : nullptr;
    assign_tma(ctx, prog, st);
    size_t dbytes, moff, need;
    blob_layout(prog, &dbytes, &moff, &need);
    void* h = host_blob(need);
    void* d = nullptr;
    if (!h || cudaMallocAsync(&d, need, st) != cudaSuccess) {
        cudaGetLastError();
        return pk_fail(PK_ERR_NOMEM, "request graph descriptors: allocation failed");
    }
    blob_fill(prog, h);
    cudaError_t e = cudaMemcpyAsync(d, h, need, cudaMemcpyHostToDevice, st);
    bool ok = e == cudaSuccess && build_graph(prog, (const VolDesc*)d, (const int*)((char*)d + dbytes),
                                              (const XZMaps*)((char*)d + moff), ctx->d_err, out,
                                              cudaGraphInstantiateFlagDeviceLaunch, d_done);
    if (ok) {
        e = cudaGraphUpload(*out, st);
        if (e != cudaSuccess) {
            cudaGraphExecDestroy(*out);
            ok = false;
        }
    }
    if (!ok) {
        cudaGetLastError();
        cudaFreeAsync(d, st);
        return pk_fail(PK_ERR_CUDA, "request graph: device-launch instantiation failed");
    }
    *d_blob = d;
    return PK_OK;
}

// Launches steps [b, e) of an uploaded program directly (the caller orders them against other
// streams between ranges); the last range of a program passes last = true, which marks its
// descriptor slot busy until the work queued so far has run.
pk_status pk_program_launch_range(pk_ctx* ctx, PkProgram& prog, cudaStream_t st, size_t b, size_t e, bool last) {
    pk_status rs = pk_check_device_waits(ctx);
    if (rs != PK_OK) return rs;
    rs = launch_steps(ctx, prog, st, b, e);
    if (rs != PK_OK) return rs;
    for (size_t i = b; i < std::min(e, prog.steps.size()); i++) ctx->launches += prog.steps[i].grid > 0 ? 1 : 0;
    if (last && prog.slot >= 0) {
        pk_ctx::ProgSlot& sl = ctx->slots[prog.slot];
        PK_CUDA(cudaEventRecord(sl.ev, st));
        sl.used = true;
    }
    return PK_OK;
}

void pk_release_graphs(pk_ctx* ctx) {
    for (auto& kv : ctx->graphs) {
        pk_ctx::GraphEntry& e = kv.second;
        if (e.ev) cudaEventSynchronize(e.ev);
        if (e.exec) cudaGraphExecDestroy(e.exec);
        if (e.d) cudaFree(e.d);
        if (e.h) cudaFreeHost(e.h);
        if (e.ev) cudaEventDestroy(e.ev);
    }
    ctx->graphs.clear();
    ctx->graph_seen.clear();
}

int pk_program_kernel_count(const PkProgram& prog) {
    int n = 0;
    for (const PkStep& s : prog.steps) n += s.grid > 0 ? 1 : 0;
    return n;
}


extern "C" pk_status pk_selftest_device_wait(pk_ctx* ctx, int64_t limit_ns) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "NULL context");
    if (limit_ns < 1000 || limit_ns > 1000000000) return pk_fail(PK_ERR_INVALID, "limit_ns must be in [1e3, 1e9]");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    int prev = 0;
    cudaGetDevice(&prev);
    PK_CUDA(cudaSetDevice(ctx->device));
    k_wait_selftest<<<1, 32, 0, ctx->stream>>>(ctx->d_err, (unsigned long long)limit_ns);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return pk_fail(PK_ERR_CUDA, std::string("wait self-test: ") + cudaGetErrorString(e));
    return pk_check_device_waits(ctx);
}

extern "C" int32_t pk_ctx_tune_read(pk_ctx* ctx, char* buf, int32_t cap) {
    if (!ctx) return -1;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    std::string js = "[";
    for (size_t i = 0; i < ctx->tune_log.size(); i++) js += (i ? ", " : "") + ctx->tune_log[i];
    js += "]";
    if (buf && cap > 0) {
        const int n = std::min((int)js.size(), cap - 1);
        memcpy(buf, js.data(), n);
        buf[n] = 0;
    }
    return (int32_t)js.size();
}
