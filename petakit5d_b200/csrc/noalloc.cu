// pk_decon_lucy_omw_noalloc: the OMW deconvolution for callers that cannot allocate GPU memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another runtime's memory manager
// (a host application that owns the whole device pool, a plugin loaded into a process whose
// allocator must not be bypassed), or code on a path where an allocation could fail or stall
// (an instrument's acquisition loop, an allocation-free real-time section).  This entry point
// runs the same pass kernels as pk_decon_lucy_omw_device but takes every work buffer -- the
// background-subtracted input, the estimate, the spectrum, both OTFs, the twiddle tables and the
// launch descriptors -- from one file-scope device array, g_noalloc_scratch, so it allocates no
// device memory and calls no allocating CUDA or library routine.  The caller passes the input and
// output volumes as device pointers (and the two PSFs as host arrays, copied into the array).
//
// Limits and sharing:
//   * at most PK_NOALLOC_MAX_VOXELS voxels per volume (1,048,576, e.g. 128 x 128 x 64); larger
//     volumes are rejected with PK_ERR_UNSUPPORTED.  The array (about 32.4 MB) is held on every
//     GPU that loads the library until the process exits;
//   * deconOffset and EdgeErosion (which need a mask volume) and NUMIT = 0 are rejected with
//     PK_ERR_UNSUPPORTED; dampFactor, scaleFactor, save16bit and bbox are supported;
//   * every call uses the same array and the array keeps the last call's contents: the call
//     clears what must start at zero (the OTF scatter volume) itself.  Calls whose work overlaps
//     on the GPU (two host threads, or two streams) race on the array and corrupt each other's
//     results -- issue them one after another on one stream;
//   * the call runs on the calling thread's current device.  The first call on a device looks up
//     the array's device address (cudaGetSymbolAddress, once per device, with that device
//     current) and sets the kernels' shared-memory limits.  Both are kept for the life of the
//     process: a program that resets a device (cudaDeviceReset) must not call this entry point on
//     that device afterwards.
#include <cmath>
#include <cstring>
#include <mutex>

#include "pass_kernels.cuh"
#include "pk_internal.h"
#include "plans.h"

void pk_fill_all_kernels(pkpass::KernelTable& t);
void set_post(VolDesc& d, const pk_decon_params* p, int mask_mode, void* d_out);

#define PK_NOALLOC_MAX_VOXELS (1u << 20)
#define PK_NOALLOC_MAX_DEVICES 64

namespace {

constexpr size_t kWorkBytes = 32ull * PK_NOALLOC_MAX_VOXELS + 4096;   // I, J, S, OTF_f, OTF_b
constexpr int kTwEntries = 4096 + 8192 + 4096 + 4096;                 // y FFT, y split, x, z tables
constexpr int kDescs = 12;
constexpr size_t kTwBytes = sizeof(float2) * kTwEntries;
constexpr size_t kMetaBytes = sizeof(VolDesc) * kDescs + 64 + 256;
constexpr size_t kScratchBytes = kWorkBytes + kTwBytes + kMetaBytes;

// The scratch of every call.  Host code never takes its address directly: it passes the device
// address looked up per device by cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_addr[PK_NOALLOC_MAX_DEVICES] = {nullptr};

// host staging for the tables and descriptors (static storage: no heap allocation per call)
struct Staging {
    float2 tw[kTwEntries];
    VolDesc desc[kDescs];
    int prefix[8];
};
Staging g_stage;

__global__ void k_na_psf_sum(const float* __restrict__ psf, long long n, double* out) {
    __shared__ double s[256];
    double a = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) a += (double)psf[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// pad (post) to the volume, circshift by -floor(psz/2), normalise by the float64 sum
__global__ void k_na_psf_scatter(const float* __restrict__ psf, int py, int px, int pz, const double* __restrict__ sum,
                                 float* __restrict__ vol, int ny, int nx, int nz) {
    const long long n = (long long)py * px * pz;
    const double s = *sum;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % py);
        const int x = (int)((i / py) % px);
        const int z = (int)(i / ((long long)py * px));
        int ty = y - py / 2; if (ty < 0) ty += ny;
        int tx = x - px / 2; if (tx < 0) tx += nx;
        int tz = z - pz / 2; if (tz < 0) tz += nz;
        vol[(long long)ty + (long long)ny * (tx + (long long)nx * tz)] = (float)((double)psf[i] / s);
    }
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

bool axis(int n, const float2* dtw, AxisDev* a) {
    AxisPlan p;
    if (!pk_make_axis_plan(n, &p)) return false;
    memset(a, 0, sizeof(*a));
    a->n = n;
    a->nst = p.nst;
    for (int i = 0; i < p.nst; i++) a->rad[i] = p.rad[i];
    a->tw = dtw;
    a->twN = n;
    a->twStride = 1;
    a->plan = pk_find_plan(n);
    return true;
}

size_t smem_for(int kind, int mode, const VolDesc& v) {
    if (kind == PK_STEP_Y)
        return sizeof(float2) * (tw_slots(v.M) + (v.odd ? 0 : v.M + 1) + pkfft::padded_size(v.Ly * v.M) + v.Ly +
                                 (size_t)pkpass::y_aux_arrays(mode) * v.Ly * v.M);
    const AxisDev& A = kind == PK_STEP_X ? v.ax : v.az;
    const int T = kind == PK_STEP_X ? v.Tx : v.Tz;
    return sizeof(float2) * (tw_slots(A.n) + pkfft::padded_size2(T * A.n) + (mode == XZ_CONV ? T * A.n : 0));
}

pkpass::KernelTable g_kt;
bool g_kt_dev[PK_NOALLOC_MAX_DEVICES] = {false};

}  // namespace

extern "C" pk_status pk_decon_lucy_omw_noalloc(const void* d_in, pk_dtype in_type, const int64_t dims[3],
                                               const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                                               const int64_t psf_b_dims[3], int32_t numit,
                                               const pk_decon_params* params, void* d_out, void* stream) {
    if (!d_in || !d_out || !dims || !psf_f || !psf_f_dims || !psf_b || !psf_b_dims)
        return pk_fail(PK_ERR_INVALID, "NULL argument");
    if (in_type != PK_U16 && in_type != PK_F32 && in_type != PK_F64) return pk_fail(PK_ERR_INVALID, "bad input dtype");
    if (numit < 0) return pk_fail(PK_ERR_INVALID, "NUMIT must be non-negative");
    if (numit == 0)
        return pk_fail(PK_ERR_UNSUPPORTED, "the no-allocation call needs NUMIT >= 1 (use pk_decon_lucy_omw_device for 0)");
    pk_decon_params def;
    if (!params) {
        pk_params_default(&def);
        params = &def;
    }
    pk_status s = pk_check_params(dims, params);
    if (s != PK_OK) return s;
    if (params->decon_offset != 0.0 || params->edge_erosion > 0)
        return pk_fail(PK_ERR_UNSUPPORTED, "the no-allocation call does not support deconOffset or EdgeErosion");
    // every axis of a volume that fits the array is below 2^20; checked before the int conversion,
    // so a huge extent cannot wrap to a small one
    for (int i = 0; i < 3; i++)
        if (dims[i] > (int64_t)PK_NOALLOC_MAX_VOXELS)
            return pk_fail(PK_ERR_UNSUPPORTED, "volume has more voxels than the no-allocation scratch holds (1048576)");
    const int ny = (int)dims[0], nx = (int)dims[1], nz = (int)dims[2];
    const long long N = (long long)ny * nx * nz;
    if (N > (long long)PK_NOALLOC_MAX_VOXELS)
        return pk_fail(PK_ERR_UNSUPPORTED, "volume has more voxels than the no-allocation scratch holds (1048576)");
    const int M = (ny & 1) ? ny : ny / 2;
    if (M > PK_TILE_POINTS || nx > PK_TILE_POINTS || nz > PK_TILE_POINTS)
        return pk_fail(PK_ERR_UNSUPPORTED, "a transform axis is longer than the tile");
    for (int i = 0; i < 3; i++)
        if (psf_f_dims[i] < 1 || psf_b_dims[i] < 1 || psf_f_dims[i] > dims[i] || psf_b_dims[i] > dims[i])
            return pk_fail(PK_ERR_INVALID, "outSizeIsSmallerThanPsfSize");

    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= PK_NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return pk_fail(PK_ERR_CUDA, "no current CUDA device");
    }
    if (!g_addr[dev]) {
        // once per device, with that device current: the array's device address
        void* a = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
        if (e != cudaSuccess || !a) {
            cudaGetLastError();
            return pk_fail(PK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        }
        g_addr[dev] = a;
    }
    if (!g_kt_dev[dev]) {
        pk_fill_all_kernels(g_kt);
        g_kt_dev[dev] = true;
    }
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)g_addr[dev];

    // ---- layout of the array: work buffers | twiddle tables | descriptors | prefixes | sum
    const int Pyv = ny / 2 + 1;
    const size_t spec_b = sizeof(float2) * (size_t)(Pyv + (Pyv & 1)) * nx * nz;
    if (2 * al256(4 * N) + 3 * al256(spec_b) > kWorkBytes)
        return pk_fail(PK_ERR_UNSUPPORTED, "volume's spectrum does not fit the no-allocation scratch (1048576 voxels)");
    float* I = (float*)base;
    float* J = (float*)(base + al256(4 * N));
    float2* S = (float2*)(base + 2 * al256(4 * N));
    float2* OF = (float2*)((char*)S + al256(spec_b));
    float2* OB = (float2*)((char*)OF + al256(spec_b));
    char* twb = base + kWorkBytes;
    VolDesc* ddesc = (VolDesc*)(twb + kTwBytes);
    int* dprefix = (int*)((char*)ddesc + sizeof(VolDesc) * kDescs);
    double* dsum = (double*)((char*)dprefix + 64);
    const float2* tw_y = (const float2*)twb;
    const float2* tw_rc = tw_y + 4096;
    const float2* tw_x = tw_rc + 8192;
    const float2* tw_z = tw_x + 4096;

    // ---- descriptors (the same geometry rules as the context path)
    pk_axis_table(M, g_stage.tw);
    if (!(ny & 1)) pk_root_table(ny, g_stage.tw + 4096);
    pk_axis_table(nx, g_stage.tw + 4096 + 8192);
    pk_axis_table(nz, g_stage.tw + 4096 + 8192 + 4096);
    VolDesc v;
    memset(&v, 0, sizeof(v));
    v.ny = ny; v.nx = nx; v.nz = nz;
    v.odd = ny & 1;
    v.M = M;
    v.Py = ny / 2 + 1;
    v.Pp = v.Py + (v.Py & 1);
    v.nrows = (long long)nx * nz;
    if (!axis(M, tw_y, &v.ay) || !axis(nx, tw_x, &v.ax) || !axis(nz, tw_z, &v.az))
        return pk_fail(PK_ERR_UNSUPPORTED, "transform length needs too many radix stages");
    v.tw_rc = v.odd ? nullptr : tw_rc;
    const int P = PK_TILE_POINTS;
    v.Ly = v.ay.plan ? plan_lines_y(M) : (P / M > 1 ? P / M : 1);
    if ((long long)v.Ly > v.nrows && v.ay.plan == 0) v.Ly = (int)v.nrows;
    v.Tx = v.ax.plan ? plan_cols_xz(nx) : std::max(1, std::min(P / nx, v.Py));
    v.Tz = v.az.plan ? plan_cols_xz(nz) : std::max(1, std::min(P / nz, v.Py));
    v.blocksY = (int)((v.nrows + v.Ly - 1) / v.Ly);
    v.blocksX = nz * ((v.Py + v.Tx - 1) / v.Tx);
    v.blocksZ = nx * ((v.Py + v.Tz - 1) / v.Tz);
    v.bb1[0] = ny - 1; v.bb1[1] = nx - 1; v.bb1[2] = nz - 1;
    v.scale = 1.f;
    v.S = S;
    v.I = I;
    for (int k = 0; k < 3; k++) v.rdims[k] = (int)dims[k];
    enum { D_OTFF, D_OTFB, D_PRE, D_BASE, D_ZF, D_ZB, D_UPD1, D_UPDN, D_FIN1, D_FINN };
    VolDesc* h = g_stage.desc;
    for (int i = 0; i < kDescs; i++) h[i] = v;
    h[D_OTFF].src = I; h[D_OTFF].S = OF; h[D_OTFF].xz_scale = (float)(1.0 / (double)N);
    h[D_OTFB].src = I; h[D_OTFB].S = OB; h[D_OTFB].xz_scale = (float)(1.0 / (double)N);
    h[D_PRE].raw = d_in;
    h[D_PRE].raw_type = in_type;
    h[D_PRE].bg_f = (float)params->background;
    {
        double b = std::floor(std::fabs(params->background) + 0.5);
        if (params->background < 0 || !(b == b)) b = 0;
        h[D_PRE].bg16 = (int)std::min(b, 65535.0);
    }
    h[D_ZF].otf = OF;
    h[D_ZB].otf = OB;
    h[D_UPD1].Jo = I; h[D_UPD1].Jn = J;
    h[D_UPDN].Jo = J; h[D_UPDN].Jn = J;
    h[D_FIN1].Jo = I; h[D_FIN1].Jn = J;
    h[D_FINN].Jo = J; h[D_FINN].Jn = J;
    set_post(h[D_FIN1], params, 0, d_out);
    set_post(h[D_FINN], params, 0, d_out);
    int* pf = g_stage.prefix;   // [0, blocksY], [0, blocksX], [0, blocksZ]
    pf[0] = 0; pf[1] = v.blocksY;
    pf[2] = 0; pf[3] = v.blocksX;
    pf[4] = 0; pf[5] = v.blocksZ;

    // ---- uploads (pageable sources are staged before the calls return, so the static staging
    //      area can be rewritten by the next call)
#define NA_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess) return pk_fail(PK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)
    NA_CUDA(cudaMemcpyAsync(twb, g_stage.tw, kTwBytes, cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemcpyAsync(ddesc, g_stage.desc, sizeof(VolDesc) * kDescs, cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemcpyAsync(dprefix, g_stage.prefix, sizeof(int) * 6, cudaMemcpyHostToDevice, st));

    auto launch = [&](int kind, int mode, int di) -> pk_status {
        const VolDesc& hv = h[di];
        const size_t smem = smem_for(kind, mode, hv);
        if (kind == PK_STEP_Y)
            g_kt.y[hv.ay.plan][mode]<<<hv.blocksY, PK_THREADS, smem, st>>>(ddesc + di, dprefix, 1, mode);
        else if (kind == PK_STEP_X)
            g_kt.xz[hv.ax.plan]<<<hv.blocksX, PK_THREADS, smem, st>>>(ddesc + di, dprefix + 2, 1, 1, mode);
        else
            g_kt.xz[hv.az.plan]<<<hv.blocksZ, PK_THREADS, smem, st>>>(ddesc + di, dprefix + 4, 1, 2, mode);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return pk_fail(PK_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
        return PK_OK;
    };

    // ---- both OTFs: the PSF goes to J, the zeroed scatter volume is I (both rewritten later)
    for (int which = 0; which < 2; which++) {
        const float* hp = which ? psf_b : psf_f;
        const int64_t* pd = which ? psf_b_dims : psf_f_dims;
        const long long pn = pd[0] * pd[1] * pd[2];
        NA_CUDA(cudaMemcpyAsync(J, hp, sizeof(float) * pn, cudaMemcpyHostToDevice, st));
        NA_CUDA(cudaMemsetAsync(I, 0, sizeof(float) * N, st));
        k_na_psf_sum<<<1, 256, 0, st>>>(J, pn, dsum);
        const long long g = std::min<long long>((pn + 255) / 256, 148LL * 16);
        k_na_psf_scatter<<<(int)std::max(1LL, g), 256, 0, st>>>(J, (int)pd[0], (int)pd[1], (int)pd[2], dsum, I, ny, nx, nz);
        NA_CUDA(cudaGetLastError());
        const int di = which ? D_OTFB : D_OTFF;
        if ((s = launch(PK_STEP_Y, Y_R2C, di)) != PK_OK) return s;
        if ((s = launch(PK_STEP_X, XZ_FWD, di)) != PK_OK) return s;
        if ((s = launch(PK_STEP_Z, XZ_FWD_SCALE, di)) != PK_OK) return s;
    }

    // ---- the OMW iterations (decon_lucy_omw_function.m:105-113), as in the context path
    if ((s = launch(PK_STEP_Y, Y_PRE, D_PRE)) != PK_OK) return s;
    for (int it = 1; it <= numit; it++) {
        if ((s = launch(PK_STEP_X, XZ_FWD, D_BASE)) != PK_OK) return s;
        if ((s = launch(PK_STEP_Z, XZ_CONV, D_ZF)) != PK_OK) return s;
        if ((s = launch(PK_STEP_X, XZ_INV, D_BASE)) != PK_OK) return s;
        if ((s = launch(PK_STEP_Y, Y_RATIO, D_BASE)) != PK_OK) return s;
        if ((s = launch(PK_STEP_X, XZ_FWD, D_BASE)) != PK_OK) return s;
        if ((s = launch(PK_STEP_Z, XZ_CONV, D_ZB)) != PK_OK) return s;
        if ((s = launch(PK_STEP_X, XZ_INV, D_BASE)) != PK_OK) return s;
        if (it < numit) s = launch(PK_STEP_Y, Y_UPDATE, it == 1 ? D_UPD1 : D_UPDN);
        else s = launch(PK_STEP_Y, Y_FINAL, it == 1 ? D_FIN1 : D_FINN);
        if (s != PK_OK) return s;
    }
#undef NA_CUDA
    return PK_OK;
}
