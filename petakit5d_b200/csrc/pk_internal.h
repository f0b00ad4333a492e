// Internal types of libpkdecon: per-volume descriptors read by the pass kernels, transform plans,
// and the context.  Layout conventions:
//   real volume  : float  v[z][x][y]            (column-major [ny nx nz], y fastest)
//   half spectrum: float2 S[z][x][k], k < Py     (Py = floor(ny/2)+1; real transform along y),
//                  row pitch Pp = Py rounded up to even
// A 3D transform is three kinds of pass: a y pass over contiguous rows (real<->half-spectrum,
// with the per-voxel arithmetic of the iteration folded into its load/store), and two strided
// complex passes over x and z on tiles of T adjacent k-columns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pkdecon.h"

#include <nvtx3/nvToolsExt.h>

// NVTX range over a scope (header-only NVTX 3: inert unless a profiler attaches): API calls,
// program launches and each pass launch are named, so a timeline shows where the host time goes.
struct PkRange {
    explicit PkRange(const char* name) { nvtxRangePushA(name); }
    ~PkRange() { nvtxRangePop(); }
    PkRange(const PkRange&) = delete;
    PkRange& operator=(const PkRange&) = delete;
};

#define PK_MAXST 16   // max radix stages per axis
#ifndef PK_PPT
#define PK_PPT 16     // max complex points per thread per stage
#endif

// ------------------------------------------------------------------ device-visible structs
struct AxisDev {
    int n;            // complex transform length along the axis
    int nst;          // number of radix stages (runtime engine)
    int rad[PK_MAXST];
    const float2* tw; // axis table (device, cached per n): stage-ordered for plan > 0, roots for plan 0
    int twN;          // table length (= n)
    int twStride;     // 1
    int plan;         // compile-time plan id (0 = runtime engine)
};

// Pass modes of the y kernel.
enum YMode : int {
    Y_R2C = 0,        // src float rows -> S                           (plain forward / OTF prep)
    Y_PRE = 1,        // raw rows -> I (written), mask8 -> S           (first pass of a call)
    Y_RATIO = 2,      // S -> c; r = I / max(c, eps) -> S              (OMW / RL middle)
    Y_UPDATE = 3,     // S -> c; Jn = max(c * Jo, 0) (written) -> S    (OMW iteration boundary)
    Y_FINAL = 4,      // S -> c; J = max(c * Jo, 0); post -> out       (OMW last)
    Y_RLPRE = 5,      // Y = max(J2 + lam (J2 - J3), 0) (written) -> S (RL iteration start)
    Y_RLUPD = 6,      // S -> c; J2n = max(Y * c, 0), J4 = J2n - Y, lam partials
    Y_RLFINAL = 7,    // S -> c; J = max(Y * c, 0); post -> out
    Y_C2R = 8         // S -> float rows (plain inverse, unnormalised)
};

enum XZMode : int { XZ_FWD = 0, XZ_INV = 1, XZ_CONV = 2, XZ_FWD_SCALE = 3 };

struct VolDesc {
    // geometry
    int ny, nx, nz;
    int M;            // y-pass complex length: ny/2 (even ny) or ny (odd ny)
    int Py;           // spectrum bins per row, floor(ny/2)+1
    int Pp;           // spectrum row pitch (Py rounded up to even: rows start 16-byte aligned)
    int odd;
    long long nrows;  // nx * nz
    int Ly, Tx, Tz;   // lines per CTA (y pass), k-columns per CTA (x / z passes)
    const float2* tw_rc;  // exp(-2 pi i k / ny), k < ny: the real/half-spectrum split (even ny)
    int blocksY, blocksX, blocksZ;
    AxisDev ay, ax, az;
    // buffers
    const void* raw; int raw_type;   // Y_PRE source (pk_dtype)
    int rdims[3]; int padded;        // raw extent; padded = transform extent larger (zeros beyond)
    const float* src; float* dst;    // Y_R2C source / Y_C2R destination
    float* I;                        // background-subtracted input
    const float* Jo; float* Jn;      // OMW estimate (old / new; may alias)
    float* Yb; float* J4; const float* J3;  // RL: Y, J4 buffers, previous estimate
    const float* J2;                 // RL: current estimate (read in Y_RLPRE)
    float* J2n;                      // RL: next estimate (Y_RLUPD / Y_RLFINAL write)
    float2* S;                       // half spectrum (work)
    const float2* otf; int conj;     // XZ_CONV
    int xz_dir;                      // XZ_FWD / XZ_INV selection for an X launch
    float xz_scale;                  // XZ_FWD_SCALE factor
    double* partials;                // RL: 2 doubles per y-pass CTA
    int lam_on;                      // RL: lambda from partials (iteration >= 3) else 0
    int rl_first;                    // RL: Y_RLUPD without an old J4 (iteration 1)
    // pre / post
    float bg_f; int bg16;
    uint8_t* mask8; int write_mask;  // Y_PRE: write raw ~= 0
    unsigned int* zero_count;        // Y_PRE: number of raw zeros (erosion branch choice)
    int mask_mode;                   // post: 0 none, 1 mask8 as is, 2 full-mask border erosion, 3 mask8 eroded
    float damp; float scale; float offset; int erosion; int scale_mode; // scale_mode: 0 none, 1 scale, 2 (J*s+o)*mask
    int save16; void* out;
    int bb0[3], bb1[3];              // 0-based inclusive crop box (y, x, z)
    int crop;                        // crop box smaller than the volume
    int need_xz;                     // post needs x/z of a voxel (crop or border erosion)
    int tiles_small;                 // passes use the 1024-point-tile kernels (small volumes)
    int* chk;                        // bounds-checked build (-DPK_CHECK): where a failed index check is recorded
};

// Bounds-checked build.  With -DPK_CHECK the pass kernels test the indices of their global-memory
// accesses (and their shared-memory layout against the launch's dynamic shared memory); a failed
// test records its check code in the context's status word (VolDesc::chk) and skips the access,
// and the call returns PK_ERR_INTERNAL.  Without it the tests compile to nothing.
#ifdef PK_CHECK
#define PK_IN(d, cond, code) pk_check_in((d).chk, (cond), (code))
__device__ __forceinline__ bool pk_check_in(int* chk, bool ok, int code) {
    if (!ok && chk) *(volatile int*)chk = code;
    return ok;
}
__device__ __forceinline__ unsigned pk_dyn_smem() {
    unsigned v;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
    return v;
}
#define PK_SMEM_OK(d, need, code) pk_check_in((d).chk, pk_dyn_smem() >= (unsigned)(need), (code))
#else
#define PK_IN(d, cond, code) true
#define PK_SMEM_OK(d, need, code) true
#endif

// TMA tensor maps of one descriptor of an x or z step run by the persistent TMA kernel: the
// spectrum S as a 3-D tensor {2 Py floats, nx, nz} (row pitch Pp) with the step's column-tile box,
// and the OTF (same layout) for XZ_CONV.  Encoded on the host when the program is uploaded.
struct alignas(64) XZMaps {
    CUtensorMap s;
    CUtensorMap otf;
    CUtensorMap s2;   // the fused convolution pass: S with the x pass's box (s has the z pass's)
};

// ------------------------------------------------------------------ host side
struct AxisPlan {
    int n = 0, nst = 0;
    int rad[PK_MAXST] = {0};
};

bool pk_make_axis_plan(int n, AxisPlan* p);   // radix factorisation (any n >= 1)

struct TwTable { float2* d = nullptr; int n = 0; };

struct OtfEntry {
    float2* d = nullptr;      // pre-scaled (1/N) half spectrum
    size_t bytes = 0;
    // the PSF it was made from (a cache hit compares the whole PSF); entries of one PSF at several
    // data sizes share this storage, so a PSF confirmed once needs no second comparison
    std::shared_ptr<const std::vector<float>> psf;
    int64_t pd[3] = {0, 0, 0};
};

struct pk_ctx_impl;

struct pk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    std::map<int, TwTable> tw;                                   // twN -> table
    // OTF cache: key = (psf content hash, ny, nx, nz)
    std::map<std::tuple<uint64_t, int, int, int>, OtfEntry> otf;
    std::vector<std::pair<void*, size_t>> scratch;               // reusable device buffers by slot
    // uploaded program descriptors: a ring of pinned-host + device slots, each reused only after
    // the event recorded behind the launches that read it has completed
    struct ProgSlot { void* d = nullptr; void* h = nullptr; size_t cap = 0; cudaEvent_t ev = nullptr; bool used = false; };
    ProgSlot slots[4];
    int next_slot = 0;
    unsigned int* d_counter = nullptr;
    std::vector<void*> host_pinned;
    long long launches = 0;                                      // kernels launched
    // per-kind profiling (pk_ctx_profile)
    bool prof_on = false;
    struct ProfRec { std::string kind; cudaEvent_t a, b; double bytes; };
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
    // CUDA graphs of repeated programs: key = launch shapes and descriptor layout.  A program is
    // built into a graph the second time its key is seen and replayed from then on; each graph reads
    // its descriptors from a device buffer of its own, refreshed (stream-ordered) before each replay.
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        void* d = nullptr;
        void* h = nullptr;
        size_t bytes = 0;
        cudaEvent_t ev = nullptr;
        bool used = false;
    };
    std::map<std::vector<long long>, GraphEntry> graphs;
    std::map<std::vector<long long>, int> graph_seen;
    // copy streams and per-slab events of streamed host calls
    cudaStream_t h2d = nullptr, d2h = nullptr;
    std::vector<cudaEvent_t> io_ev;
    // asynchronous host-buffer calls (pk_decon_submit / pk_decon_wait): two staging slots used in
    // turn, so the upload of call k+1 and the download of call k-1 overlap the compute of call k
    struct AsyncSlot {
        void* d_in = nullptr; size_t in_cap = 0;
        void* d_out = nullptr; size_t out_cap = 0;
        cudaEvent_t up = nullptr, comp = nullptr, down = nullptr;   // upload done, compute done, download done
        bool used = false;
    };
    AsyncSlot aslot[2];
    // small read-only device tables built once per parameter set (e.g. the deskew's skewed-slice table)
    std::map<std::string, void*> dev_tables;
    long long next_ticket = 1;
    std::map<long long, cudaEvent_t> tickets;                  // ticket -> its download's event
    // device-wait status: page-locked word the kernels write when a bounded wait on the device ran
    // out (0 = none); h_err is the host view, d_err the device pointer passed to the kernels
    int* h_err = nullptr;
    int* d_err = nullptr;
    // autotuner of the x / z passes: chosen variant per (pass, plan, geometry) key (-1 = register-IO
    // kernel, 0.. = TMA variant), and a JSON record of each decision (pk_ctx_tune_read)
    std::map<std::vector<long long>, int> tune;
    std::vector<std::string> tune_log;
};

// error helpers (capi.cpp)
void pk_set_error(const std::string& msg);
pk_status pk_fail(pk_status st, const std::string& msg);
#define PK_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess)                                                          \
            return pk_fail(PK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// plans / descriptors (fft_kernels.cu)
void pk_root_table(int n, float2* out);
int pk_axis_table(int n, float2* out);   // writes at most n + PK_TW_EXTRA entries, returns the count
pk_status pk_get_twiddles(pk_ctx* ctx, int twN, const float2** out);
pk_status pk_fill_axis(pk_ctx* ctx, int n, int twN, AxisDev* a);
pk_status pk_init_desc(pk_ctx* ctx, int ny, int nx, int nz, VolDesc* d);
size_t pk_spec_elems(const VolDesc& d);   // complex elements of the half spectrum

// launch programs (passes.cu)
// PK_STEP_CONV3: x forward, z convolution and x inverse of one volume in one launch (pass_conv3.cuh)
enum { PK_STEP_Y = 0, PK_STEP_X = 1, PK_STEP_Z = 2, PK_STEP_LAMBDA = 3, PK_STEP_CONV3 = 4 };
struct PkStep {
    int kind = 0, mode = 0, plan = 0, nvol = 0, desc_off = 0, prefix_off = 0, grid = 0;
    size_t smem = 0;
    // set at upload: index of the persistent TMA kernel that runs this x / z step (-1: none), its
    // grid (resident CTAs, each walking tiles) and dynamic shared memory
    int tma = -1, tma_var = 0, tma_grid = 0;
    // PK_STEP_CONV3: the fused kernel's table index and its z plan (its column-tile counters are the
    // 2K ints of the prefix array at prefix_off)
    int conv3 = -1, plan2 = 0;
    size_t tma_smem = 0;
    // set at upload: this y step runs the register-packing kernel (512-voxel rows), with its smem
    int yreg = 0;
    size_t yreg_smem = 0;
};
struct PkProgram {
    std::vector<VolDesc> descs;
    std::vector<int> prefix;
    std::vector<PkStep> steps;
    std::vector<XZMaps> maps;   // parallel to descs: tensor maps of the steps run by the TMA kernels
    VolDesc* d_desc = nullptr; int* d_prefix = nullptr;   // inside one of the context's program slots
    XZMaps* d_maps = nullptr;
    int slot = -1;
    bool no_graph = false;   // launch directly (e.g. per-slab programs of a streamed call)
};
void pk_program_add(PkProgram& prog, int kind, int mode, const std::vector<VolDesc>& vols);
pk_status pk_program_upload(pk_ctx* ctx, PkProgram& prog, cudaStream_t st);
pk_status pk_program_launch(pk_ctx* ctx, PkProgram& prog, cudaStream_t st);
void pk_release_graphs(pk_ctx* ctx);
// PK_ERR_TIMEOUT (and the status cleared) when a kernel of this context reported that one of its
// bounded device waits ran out since the last check; PK_OK otherwise
pk_status pk_check_device_waits(pk_ctx* ctx);
pk_status pk_program_launch_range(pk_ctx* ctx, PkProgram& prog, cudaStream_t st, size_t b, size_t e, bool last);
double pk_step_bytes(const PkStep& s, const VolDesc* descs);
const char* pk_step_name(const PkStep& s);
int pk_program_kernel_count(const PkProgram& prog);
// The program as a graph that a kernel can launch (the server's device loop): its descriptors in a
// device blob of its own (*d_blob, stream-ordered allocation on st, copied there from a page-locked
// buffer of host_blob(bytes); both must outlive the graph's run), then a node that sets
// *d_done = 1 (page-locked host memory) when every pass is done; instantiated for device launch and
// uploaded on st.
pk_status pk_program_device_graph(pk_ctx* ctx, PkProgram& prog, cudaStream_t st, int* d_done,
                                  const std::function<void*(size_t)>& host_blob, void** d_blob, cudaGraphExec_t* out);

// Device-resident request loop (serve.cu host side, dloop_rdc.cu dispatcher).  The ring lives in
// page-locked host memory: the host appends ready requests' graphs at `tail`; a dispatcher kernel
// takes them at `head` and launches each fire-and-forget from the device.
constexpr int kDlRingCap = 1024;
constexpr int kDlLaunchBudget = 112;   // graphs one dispatcher launches (the device runtime allows 120)
enum DlExit : int { DL_NONE = 0, DL_STOPPED = 1, DL_BUDGET = 2, DL_HEARTBEAT = 3, DL_IDLE = 4 };
struct DlRing {
    volatile long long tail;             // host: entries appended
    volatile long long head;             // dispatcher: entries launched
    volatile long long heartbeat;        // host: bumped by the scheduler thread while it runs
    volatile long long heartbeat_ns;     // host: a dispatcher returns when the heartbeat stalls this long
    volatile long long idle_ns;          // host: a dispatcher returns after this long without an entry
    volatile long long epoch_launched;   // host: dispatcher instances started
    volatile long long epoch_ended;      // dispatcher: instances that have returned
    volatile int stop;                   // host: dispatchers return
    volatile int exit_code;              // dispatcher: why the last instance returned (DlExit)
    cudaGraphExec_t graph[kDlRingCap];
    volatile int status[kDlRingCap];     // dispatcher: 1 + cudaError of the entry's launch
    volatile int epoch[kDlRingCap];      // dispatcher: the instance that launched the entry
};
// One dispatcher instance as a (host-launched) graph of one kernel on ring d_ring.
pk_status pk_dloop_instance(DlRing* d_ring, cudaStream_t st, cudaGraphExec_t* out);

// scratch buffers
pk_status pk_scratch(pk_ctx* ctx, int slot, size_t bytes, void** ptr);

// PSF-size volume helpers (psfvol.cu, decon.cu)
std::vector<int4> pk_ball_offsets(int r);           // strel('sphere', r): (dy, dx, dz, 0), dy^2+dx^2+dz^2 <= r^2
std::vector<int2> pk_disk_offsets(int R);           // strel('disk', R): (dy, dx)
// binary morphology on the GPU: ops is a string of 'd' (dilate) / 'e' (erode) applied in order;
// d_a holds the mask in and out, d_tmp is a mask-sized work buffer
pk_status pk_morph_ops(uint8_t* d_a, uint8_t* d_tmp, int ny, int nx, int nz, const int4* d_offs, int noff,
                       const char* ops, cudaStream_t st);
pk_status pk_morph_host(std::vector<uint8_t>& mask, int ny, int nx, int nz, const std::vector<int4>& offs,
                        const char* ops, cudaStream_t st);
int pk_label26(const uint8_t* m, int ny, int nx, int nz, std::vector<int>& lab, std::vector<long long>& sizes);
std::vector<double2> pk_twiddles64(int n, int sign);   // exp(sign 2 pi i m / n), m < n

// decon drivers (decon.cu)
// OTF of a host PSF at a data size, from the context's cache or made on `st`.  `confirmed` (may be
// null) carries, across the lookups of one call, the cached copy the host PSF has already been
// compared equal to: entries sharing that copy are hits without another comparison.
pk_status pk_get_otf(pk_ctx* ctx, const float* h_psf, const int64_t psf_dims[3], int ny, int nx, int nz,
                     const float2** d_otf, cudaStream_t st,
                     std::shared_ptr<const std::vector<float>>* confirmed = nullptr);
// one volume of a multi-volume run: inputs, transform extent, OTFs, outputs and work buffers
struct DeconJob {
    const void* d_raw = nullptr;
    int rdims[3] = {0, 0, 0};   // raw extent
    int dims[3] = {0, 0, 0};    // transform extent (>= raw; the excess reads as zeros)
    const float2* otf_f = nullptr;
    const float2* otf_b = nullptr;
    void* d_out = nullptr;
    int has_bbox = 0;
    int64_t bbox[6] = {0, 0, 0, 0, 0, 0};
    float *I = nullptr, *J = nullptr, *JB = nullptr, *Yb = nullptr, *J4 = nullptr;
    float2* S = nullptr;
    uint8_t* mask = nullptr;
    double* part = nullptr;
};
size_t pk_job_bytes(int method, const int dims[3], bool need_mask, int blocksY);
void pk_job_carve(DeconJob& j, int method, bool need_mask, int blocksY, char* arena);
// Host buffers of a single-volume call whose copies are streamed by z-slab: slab s of the input is
// uploaded on h2d while the first passes of slab s-1 run, and slab s of the result is downloaded on
// d2h as soon as the last passes of slab s are done.  The caller synchronises d2h.
struct HostStreamIO {
    const void* h_in = nullptr;
    void* h_out = nullptr;
    size_t in_esize = 0, out_esize = 0;
    bool active = false;   // set by pk_decon_multi when the call could be streamed
};
// Debug run of one volume (decon_lucy_omw_function.m:114-144, decon_lucy_function.m:144-175): the
// last iteration also writes J, and after the launches of iteration k, after_iter(k, J) queues the
// caller's per-iteration work (error measure, snapshot) on the stream.
struct DebugHook {
    std::function<pk_status(int k, const float* J, const float* I)> after_iter;
};
// debug-run helpers (decon.cu): mean((J - I).^2) in float64 (fixed order) into *out, uint16(J) into o
pk_status pk_debug_error(const float* J, const float* I, long long n, double* part, int nb, double* out, cudaStream_t st);
pk_status pk_debug_u16(const float* J, long long n, uint16_t* o, cudaStream_t st);
pk_status pk_decon_multi(pk_ctx* ctx, int method, std::vector<DeconJob>& jobs, pk_dtype in_type, int numit,
                         const pk_decon_params* p, cudaStream_t st, HostStreamIO* io = nullptr,
                         const DebugHook* dbg = nullptr);
pk_status pk_check_params(const int64_t dims[3], const pk_decon_params* p);

pk_status pk_decon_run(pk_ctx* ctx, int method, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                       const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                       const int64_t psf_b_dims[3], int numit, const pk_decon_params* p, void* d_out,
                       cudaStream_t st, HostStreamIO* io = nullptr, const DebugHook* dbg = nullptr);
