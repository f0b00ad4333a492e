// Drivers of the two iterations: OTF preparation and the launch programs of
// decon_lucy_omw_function (OMW / WB backprojector RL) and decon_lucy_function (Biggs RL).
//
// Per OMW iteration (decon_lucy_omw_function.m:105-113) the program is
//   [y: c = C2R(S); Jn = max(c*Jo,0); S = R2C(Jn)] x-fwd  z(OTF_f)  x-inv
//   [y: c = C2R(S); r = I / max(c,eps); S = R2C(r)] x-fwd  z(OTF_b)  x-inv
// where the first y pass of a call is [raw -> I; S = R2C(I)] and the last one writes the
// post-processed, cropped output directly (decon_lucy_omw_function.m:146-177).
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

// Float64 sum of the PSF in a fixed order (deterministic): block b sums its contiguous slice
// (thread-strided, then a tree), and k_psf_sum_final adds the block partials in block order.
constexpr int kPsfSumBlocks = 64;
__global__ void k_psf_sum(const float* __restrict__ psf, long long n, double* part) {
    __shared__ double s[256];
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    const long long b0 = per * blockIdx.x, b1 = min(n, b0 + per);
    double a = 0.0;
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) a += (double)psf[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void k_psf_sum_final(const double* __restrict__ part, int nb, double* out) {
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int b = 0; b < nb; b++) a += part[b];
        *out = a;
    }
}

// Pad (post) to the volume, circshift by -floor(psz/2), normalise by the float64 sum
// (decon_psf2otf.m:25-27 with PSF./sum(PSF(:)) in float64).
__global__ void k_psf_scatter(const float* __restrict__ psf, int py, int px, int pz, const double* __restrict__ sum,
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

// Post-processing of a materialised estimate `src` into the output (numit == 0: src = I; debug
// runs: the last iteration's J).
__global__ void k_post_from(VolDesc d, const float* __restrict__ src) {
    const long long n = d.nrows * d.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / d.ny;
        const int y = (int)(i - row * d.ny);
        const int x = (int)(row % d.nx), z = (int)(row / d.nx);
        if (y < d.bb0[0] || y > d.bb1[0] || x < d.bb0[1] || x > d.bb1[1] || z < d.bb0[2] || z > d.bb1[2]) continue;
        float J = src[i];
        if (d.damp > 1.f) {
            const float dI = __fmul_rn(d.damp, d.I[i]);
            J = __fadd_rn((J <= dI) ? J : 0.f, fminf(J, (J >= dI) ? dI : 0.f));
        }
        if (d.scale_mode == 1) J = __fmul_rn(J, d.scale);
        else if (d.scale_mode == 2) {
            int m = 1;
            if (d.mask_mode == 1 || d.mask_mode == 3) m = d.mask8[i] != 0;
            else if (d.mask_mode == 2) {
                const int E = d.erosion;
                m = d.mask8[i] != 0 && y >= E && y < d.ny - E && x >= E && x < d.nx - E &&
                    (d.nz == 1 || (z >= E && z < d.nz - E));      // one plane: MATLAB's 2-D case
            }
            J = __fmul_rn(__fadd_rn(__fmul_rn(J, d.scale), d.offset), (float)m);
        }
        const long long oy = d.bb1[0] - d.bb0[0] + 1, ox = d.bb1[1] - d.bb0[1] + 1;
        const long long oi = (long long)(y - d.bb0[0]) + oy * ((long long)(x - d.bb0[1]) + ox * (long long)(z - d.bb0[2]));
        if (d.save16) {
            float r = roundf(J);
            if (!(r >= 0.f)) r = 0.f;
            if (r > 65535.f) r = 65535.f;
            ((uint16_t*)d.out)[oi] = (uint16_t)r;
        } else {
            ((float*)d.out)[oi] = J;
        }
    }
}

// ---- debug runs: per-iteration float64 MSE of J against I and uint16 snapshots of J
constexpr int kSqBlocks = 64;
__global__ void k_sqdiff_part(const float* __restrict__ J, const float* __restrict__ I, long long n, double* part) {
    __shared__ double s[256];
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    const long long b0 = per * blockIdx.x, b1 = min(n, b0 + per);
    double a = 0.0;
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double d = (double)J[i] - (double)I[i];
        a += d * d;
    }
    s[threadIdx.x] = a;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void k_sqdiff_final(const double* __restrict__ part, int nb, long long n, double* out) {
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int b = 0; b < nb; b++) a += part[b];
        *out = a / (double)n;
    }
}

__global__ void k_to_u16(const float* __restrict__ J, long long n, uint16_t* __restrict__ o) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float r = roundf(J[i]);             // MATLAB uint16(): half away from zero, saturate, NaN -> 0
        if (!(r >= 0.f)) r = 0.f;
        if (r > 65535.f) r = 65535.f;
        o[i] = (uint16_t)r;
    }
}

// ---- irregular-mask edge erosion (decon_mask_edge_erosion.m:18-29)
__global__ void k_mask_faces(uint8_t* m, int ny, int nx, int nz) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny);
        const int x = (int)((i / ny) % nx);
        const int z = (int)(i / ((long long)ny * nx));
        // one plane is MATLAB's 2-D case (ndims 2): no z faces
        if (y == 0 || y == ny - 1 || x == 0 || x == nx - 1 || (nz > 1 && (z == 0 || z == nz - 1))) m[i] = 0;
    }
}

// erosion with a 2D (per z-slice) neighbourhood given as (dy, dx) offsets; outside counts as true
__global__ void k_erode_xy(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int ny, int nx, int nz,
                           const int2* __restrict__ offs, int noff) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny);
        const int x = (int)((i / ny) % nx);
        const long long zo = (i / ((long long)ny * nx)) * (long long)ny * nx;
        uint8_t v = in[i];
        for (int k = 0; v && k < noff; k++) {
            const int yy = y + offs[k].x, xx = x + offs[k].y;
            if (yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
            v = in[zo + yy + (long long)ny * xx];
        }
        out[i] = v;
    }
}

__global__ void k_erode_z(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int ny, int nx, int nz, int h) {
    const long long n = (long long)ny * nx * nz;
    const long long plane = (long long)ny * nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i / plane);
        uint8_t v = in[i];
        for (int o = -h; v && o <= h; o++) {
            const int zz = z + o;
            if (zz < 0 || zz >= nz) continue;
            v = in[i + (long long)o * plane];
        }
        out[i] = v;
    }
}

// Cache key of a PSF: a 64-bit hash of its dims, its size and 256 evenly spaced values.  It only
// picks the candidate entry; a hit is confirmed by comparing the whole PSF (memcmp runs near memory
// speed, a full-content hash would cost a serial pass over the PSF on every call).
uint64_t psf_key(const float* psf, const int64_t pd[3]) {
    const size_t n = (size_t)pd[0] * pd[1] * pd[2];
    uint64_t h = 0x243F6A8885A308D3ULL;
    auto mix = [&](uint64_t w) {
        h ^= w;
        h *= 0x9E3779B97F4A7C15ULL;
        h ^= h >> 29;
    };
    for (int i = 0; i < 3; i++) mix((uint64_t)pd[i]);
    const size_t samples = n < 256 ? n : 256;
    for (size_t k = 0; k < samples; k++) {
        uint32_t w;
        memcpy(&w, psf + (n - 1) * k / (samples > 1 ? samples - 1 : 1), 4);
        mix(w);
    }
    return h;
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    if (g > 148LL * 32) g = 148LL * 32;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

pk_status pk_debug_error(const float* J, const float* I, long long n, double* part, int nb, double* out, cudaStream_t st) {
    k_sqdiff_part<<<nb, 256, 0, st>>>(J, I, n, part);
    k_sqdiff_final<<<1, 32, 0, st>>>(part, nb, n, out);
    PK_CUDA(cudaGetLastError());
    return PK_OK;
}

pk_status pk_debug_u16(const float* J, long long n, uint16_t* o, cudaStream_t st) {
    k_to_u16<<<grid_for(n), 256, 0, st>>>(J, n, o);
    PK_CUDA(cudaGetLastError());
    return PK_OK;
}

// strel('disk', R) neighbourhood (default N = 4 approximation), as (dy, dx) offsets.
std::vector<int2> pk_disk_offsets(int R) {
    std::vector<std::pair<int, int>> pts;
    if (R < 3) {
        for (int a = -R; a <= R; a++)
            for (int b = -R; b <= R; b++)
                if (a * a + b * b <= R * R) pts.push_back({a, b});
    } else {
        // radial decomposition into four periodic lines (Adams 1993; Jones & Soille 1996)
        const double theta = M_PI / 8.0;
        const double k = 2.0 * R / (1.0 / std::tan(theta) + 1.0 / std::sin(theta));
        const int vy[4] = {1, 1, 0, -1}, vx[4] = {0, 1, 1, 1};
        std::vector<std::pair<int, int>> cur{{0, 0}};
        auto minkowski = [&](int dy, int dx, int rp) {
            std::vector<std::pair<int, int>> nxt;
            for (auto& p : cur)
                for (int m = -rp; m <= rp; m++) nxt.push_back({p.first + m * dy, p.second + m * dx});
            std::sort(nxt.begin(), nxt.end());
            nxt.erase(std::unique(nxt.begin(), nxt.end()), nxt.end());
            cur.swap(nxt);
        };
        for (int q = 0; q < 4; q++) {
            const int rp = (int)std::floor(k / std::sqrt((double)(vy[q] * vy[q] + vx[q] * vx[q])));
            minkowski(vy[q], vx[q], rp);
        }
        int rmax = 0;
        for (auto& p : cur) rmax = std::max(rmax, p.first);
        const int len = 2 * (R - rmax - 1) + 1;
        if (len >= 3) {
            minkowski(0, 1, len / 2);
            minkowski(1, 0, len / 2);
        }
        pts = cur;
    }
    std::vector<int2> out;
    for (auto& p : pts) out.push_back(make_int2(p.first, p.second));
    return out;
}

pk_status pk_scratch(pk_ctx* ctx, int slot, size_t bytes, void** ptr) {
    if ((int)ctx->scratch.size() <= slot) ctx->scratch.resize(slot + 1, {nullptr, 0});
    auto& s = ctx->scratch[slot];
    if (s.second < bytes) {
        if (s.first) cudaFree(s.first);
        s.first = nullptr;
        s.second = 0;
        cudaError_t e = cudaMalloc(&s.first, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return pk_fail(PK_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        }
        s.second = bytes;
    }
    *ptr = s.first;
    return PK_OK;
}

enum { SL_ARENA = 0, SL_JB = 2, SL_S = 5, SL_MASK2 = 7, SL_IN = 9, SL_OUT = 10, SL_PSF = 11, SL_SUM = 12,
       SL_OFFS = 13, SL_ZC = 14 };

// Half-spectrum OTF of a PSF at the volume size, scaled by `scale` (1/N for the iterations).
pk_status pk_make_otf(pk_ctx* ctx, const float* h_psf, const int64_t pd[3], int ny, int nx, int nz, double scale,
                      float2* d_otf, cudaStream_t st) {
    const long long pn = (long long)pd[0] * pd[1] * pd[2];
    if (pd[0] > ny || pd[1] > nx || pd[2] > nz) return pk_fail(PK_ERR_INVALID, "outSizeIsSmallerThanPsfSize");
    void *d_psf, *d_sum, *d_vol;
    pk_status s;
    if ((s = pk_scratch(ctx, SL_PSF, sizeof(float) * pn, &d_psf)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, SL_SUM, sizeof(double) * (kPsfSumBlocks + 1), &d_sum)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, SL_JB, sizeof(float) * (size_t)ny * nx * nz, &d_vol)) != PK_OK) return s;
    PK_CUDA(cudaMemcpyAsync(d_psf, h_psf, sizeof(float) * pn, cudaMemcpyHostToDevice, st));
    PK_CUDA(cudaMemsetAsync(d_vol, 0, sizeof(float) * (size_t)ny * nx * nz, st));
    k_psf_sum<<<kPsfSumBlocks, 256, 0, st>>>((const float*)d_psf, pn, (double*)d_sum + 1);
    k_psf_sum_final<<<1, 32, 0, st>>>((const double*)d_sum + 1, kPsfSumBlocks, (double*)d_sum);
    k_psf_scatter<<<grid_for(pn), 256, 0, st>>>((const float*)d_psf, (int)pd[0], (int)pd[1], (int)pd[2],
                                                 (const double*)d_sum, (float*)d_vol, ny, nx, nz);
    PK_CUDA(cudaGetLastError());
    VolDesc d;
    if ((s = pk_init_desc(ctx, ny, nx, nz, &d)) != PK_OK) return s;
    d.src = (const float*)d_vol;
    d.S = d_otf;
    d.xz_scale = (float)scale;
    PkProgram prog;
    pk_program_add(prog, PK_STEP_Y, Y_R2C, {d});
    pk_program_add(prog, PK_STEP_X, XZ_FWD, {d});
    pk_program_add(prog, PK_STEP_Z, XZ_FWD_SCALE, {d});
    if ((s = pk_program_upload(ctx, prog, st)) == PK_OK) s = pk_program_launch(ctx, prog, st);
    return s;
}

pk_status pk_get_otf(pk_ctx* ctx, const float* h_psf, const int64_t pd[3], int ny, int nx, int nz,
                     const float2** d_otf, cudaStream_t st, std::shared_ptr<const std::vector<float>>* confirmed) {
    const long long pn = (long long)pd[0] * pd[1] * pd[2];
    // open addressing on the key: an entry with the same key but another PSF moves this one on
    uint64_t hk = psf_key(h_psf, pd);
    for (;; hk++) {
        auto it = ctx->otf.find(std::make_tuple(hk, ny, nx, nz));
        if (it == ctx->otf.end()) break;
        const OtfEntry& c = it->second;
        if (c.pd[0] != pd[0] || c.pd[1] != pd[1] || c.pd[2] != pd[2] || (long long)c.psf->size() != pn) continue;
        const bool same = (confirmed && *confirmed && c.psf == *confirmed) ||
                          memcmp(c.psf->data(), h_psf, sizeof(float) * pn) == 0;
        if (same) {
            if (confirmed && !*confirmed) *confirmed = c.psf;
            *d_otf = c.d;
            return PK_OK;
        }
    }
    const auto key = std::make_tuple(hk, ny, nx, nz);
    OtfEntry e;
    if (confirmed && *confirmed && (long long)(*confirmed)->size() == pn) {
        e.psf = *confirmed;
    } else {
        // share the copy of an entry of the same PSF at another data size (compared once, here), so a
        // later call that confirms one of them hits the others by pointer
        const uint64_t k0 = psf_key(h_psf, pd);
        for (const auto& kv : ctx->otf) {
            const OtfEntry& o = kv.second;
            if (std::get<0>(kv.first) != k0 || o.pd[0] != pd[0] || o.pd[1] != pd[1] || o.pd[2] != pd[2] ||
                (long long)o.psf->size() != pn)
                continue;
            if (memcmp(o.psf->data(), h_psf, sizeof(float) * pn) == 0) {
                e.psf = o.psf;
                break;
            }
        }
        if (!e.psf) e.psf = std::make_shared<const std::vector<float>>(h_psf, h_psf + pn);
    }
    if (confirmed) *confirmed = e.psf;
    for (int i = 0; i < 3; i++) e.pd[i] = pd[i];
    const int Py = ny / 2 + 1;
    e.bytes = sizeof(float2) * (size_t)(Py + (Py & 1)) * nx * nz;
    cudaError_t ce = cudaMalloc(&e.d, e.bytes);
    if (ce != cudaSuccess) { cudaGetLastError(); return pk_fail(PK_ERR_NOMEM, "OTF allocation failed"); }
    const double N = (double)ny * nx * nz;
    pk_status s = pk_make_otf(ctx, h_psf, pd, ny, nx, nz, 1.0 / N, e.d, st);
    if (s != PK_OK) { cudaFree(e.d); return s; }
    ctx->otf[key] = e;
    *d_otf = e.d;
    return PK_OK;
}

void set_post(VolDesc& d, const pk_decon_params* p, int mask_mode, void* d_out) {
    const bool off = p->decon_offset != 0.0, ero = p->edge_erosion > 0;
    d.damp = (float)p->damp_factor;
    d.scale = (float)p->scale_factor;
    d.offset = (float)p->decon_offset;
    d.erosion = p->edge_erosion;
    if (p->scale_factor != 1.0 || off || ero) d.scale_mode = (off || ero) ? 2 : 1;
    else d.scale_mode = 0;
    d.mask_mode = d.scale_mode == 2 ? mask_mode : 0;
    d.save16 = p->save16bit ? 1 : 0;
    d.out = d_out;
    if (p->has_bbox) {
        for (int i = 0; i < 3; i++) {
            d.bb0[i] = (int)p->bbox[i] - 1;
            d.bb1[i] = (int)p->bbox[i + 3] - 1;
        }
    }
    const int dims[3] = {d.ny, d.nx, d.nz};
    d.crop = 0;
    for (int i = 0; i < 3; i++)
        if (d.bb0[i] != 0 || d.bb1[i] != dims[i] - 1) d.crop = 1;
    d.need_xz = d.crop || d.mask_mode == 2;
}

pk_status pk_check_params(const int64_t dims[3], const pk_decon_params* p) {
    if (!p) return pk_fail(PK_ERR_INVALID, "params must not be NULL");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return pk_fail(PK_ERR_INVALID, "empty input volume");
    if (p->has_bbox) {
        for (int i = 0; i < 3; i++) {
            if (p->bbox[i] < 1 || p->bbox[i + 3] > dims[i] || p->bbox[i] > p->bbox[i + 3])
                return pk_fail(PK_ERR_INVALID, "bbox is outside the volume (Index exceeds array bounds)");
        }
    }
    return PK_OK;
}

// ------------------------------------------------------------------ multi-volume runner
// Bytes of the work buffers one job needs (256-byte aligned pieces).
static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

static size_t spec_bytes(const int dims[3]) {
    const int Py = dims[0] / 2 + 1;
    return sizeof(float2) * (size_t)(Py + (Py & 1)) * dims[1] * dims[2];
}

size_t pk_job_bytes(int method, const int dims[3], bool need_mask, int blocksY) {
    const size_t N = (size_t)dims[0] * dims[1] * dims[2];
    const size_t spec = spec_bytes(dims);
    size_t b = al256(4 * N) * 2 + al256(spec);                       // I, J, S
    if (method == 0) b += al256(4 * N) * 3 + al256(sizeof(double) * (2 + 2 * (size_t)blocksY));  // JB, Y, J4, partials
    if (need_mask) b += al256(N);
    return b;
}

void pk_job_carve(DeconJob& j, int method, bool need_mask, int blocksY, char* arena) {
    const size_t N = (size_t)j.dims[0] * j.dims[1] * j.dims[2];
    const size_t spec = spec_bytes(j.dims);
    size_t o = 0;
    auto take = [&](size_t b) { char* p = arena + o; o += al256(b); return p; };
    j.I = (float*)take(4 * N);
    j.J = (float*)take(4 * N);
    j.S = (float2*)take(spec);
    if (method == 0) {
        j.JB = (float*)take(4 * N);
        j.Yb = (float*)take(4 * N);
        j.J4 = (float*)take(4 * N);
        j.part = (double*)take(sizeof(double) * (2 + 2 * (size_t)blocksY));
    }
    if (need_mask) j.mask = (uint8_t*)take(N);
}

static void set_post_job(VolDesc& d, const pk_decon_params* p, int mask_mode, const DeconJob& j) {
    pk_decon_params q = *p;
    q.has_bbox = j.has_bbox;
    for (int i = 0; i < 6; i++) q.bbox[i] = j.bbox[i];
    if (!j.has_bbox && (j.rdims[0] != j.dims[0] || j.rdims[1] != j.dims[1] || j.rdims[2] != j.dims[2])) {
        // padded transform: the output is the raw extent
        q.has_bbox = 1;
        for (int i = 0; i < 3; i++) {
            q.bbox[i] = 1;
            q.bbox[i + 3] = j.rdims[i];
        }
    }
    set_post(d, &q, mask_mode, j.d_out);
}

// The z-slab [z0, z0 + nzs) of a volume descriptor as a volume of its own: y and x passes work
// plane by plane, so a slab view runs them on those planes only.
static VolDesc slab_view(const VolDesc& d, int z0, int nzs, size_t raw_esize, size_t out_esize) {
    VolDesc v = d;
    const size_t plane = (size_t)d.ny * d.nx;
    const size_t off = (size_t)z0 * plane;
    const int ctx_tiles = d.blocksX / d.nz;
    v.nz = nzs;
    v.nrows = (long long)d.nx * nzs;
    v.blocksY = (int)((v.nrows + v.Ly - 1) / v.Ly);
    v.blocksX = nzs * ctx_tiles;
    v.blocksZ = 0;
    v.rdims[2] = nzs;
    v.bb1[2] = nzs - 1;
    if (d.raw) v.raw = (const char*)d.raw + off * raw_esize;
    if (d.src) v.src = d.src + off;
    if (d.dst) v.dst = d.dst + off;
    if (d.I) v.I = d.I + off;
    if (d.Jo) v.Jo = d.Jo + off;
    if (d.Jn) v.Jn = d.Jn + off;
    if (d.Yb) v.Yb = d.Yb + off;
    if (d.J4) v.J4 = d.J4 + off;
    if (d.J3) v.J3 = d.J3 + off;
    if (d.J2) v.J2 = d.J2 + off;
    if (d.J2n) v.J2n = d.J2n + off;
    if (d.mask8) v.mask8 = d.mask8 + off;
    if (d.out) v.out = (char*)d.out + off * out_esize;
    if (d.S) v.S = d.S + (size_t)z0 * d.nx * d.Pp;
    return v;
}

static pk_status get_io_event(pk_ctx* ctx, size_t i, cudaEvent_t* e) {
    while (ctx->io_ev.size() <= i) {
        cudaEvent_t ev;
        PK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        ctx->io_ev.push_back(ev);
    }
    *e = ctx->io_ev[i];
    return PK_OK;
}

pk_status pk_decon_multi(pk_ctx* ctx, int method, std::vector<DeconJob>& jobs, pk_dtype in_type, int numit,
                         const pk_decon_params* p, cudaStream_t st, HostStreamIO* io, const DebugHook* dbg) {
    pk_status s;
    if (numit < 0) return pk_fail(PK_ERR_INVALID, "NUMIT must be non-negative");
    const size_t nj = jobs.size();
    if (nj == 0) return PK_OK;
    if (dbg && (nj != 1 || io)) return pk_fail(PK_ERR_INVALID, "debug runs take one volume on device buffers");
    const bool need_mask = p->decon_offset != 0.0 || p->edge_erosion > 0;
    // a single-volume call with host buffers streams its copies by z-slab when its first and last
    // passes work plane by plane on the raw layout (no padding, crop, erosion or scalar raw path)
    bool stream_io = false;
    static const bool io_off = getenv("PK_NO_STREAM_IO") && getenv("PK_NO_STREAM_IO")[0] == '1';
    if (io && io_off) {
        const DeconJob& j = jobs[0];
        const size_t N = (size_t)j.rdims[0] * j.rdims[1] * j.rdims[2];
        PK_CUDA(cudaMemcpyAsync((void*)j.d_raw, io->h_in, N * io->in_esize, cudaMemcpyHostToDevice, st));
    } else if (io) {
        const DeconJob& j = jobs[0];
        bool full_box = true;
        if (j.has_bbox)
            for (int i = 0; i < 3; i++)
                if (j.bbox[i] != 1 || j.bbox[i + 3] != j.dims[i]) full_box = false;
        stream_io = nj == 1 && numit >= 1 && full_box && p->edge_erosion == 0 && in_type != PK_F64 &&
                    !(in_type == PK_U16 && (j.dims[0] & 1)) && j.dims[2] >= 16 && j.rdims[0] == j.dims[0] &&
                    j.rdims[1] == j.dims[1] && j.rdims[2] == j.dims[2];
        if (!stream_io) {
            const size_t N = (size_t)j.rdims[0] * j.rdims[1] * j.rdims[2];
            PK_CUDA(cudaMemcpyAsync((void*)j.d_raw, io->h_in, N * io->in_esize, cudaMemcpyHostToDevice, st));
        }
    }
    std::vector<VolDesc> base(nj);
    unsigned int* zc = nullptr;
    if (p->edge_erosion > 0) {
        void* z;
        if ((s = pk_scratch(ctx, SL_ZC, sizeof(unsigned int) * nj, &z)) != PK_OK) return s;
        zc = (unsigned int*)z;
        PK_CUDA(cudaMemsetAsync(zc, 0, sizeof(unsigned int) * nj, st));
    }
    double b16 = std::floor(std::fabs(p->background) + 0.5);
    if (p->background < 0 || !(b16 == b16)) b16 = 0;
    for (size_t i = 0; i < nj; i++) {
        DeconJob& j = jobs[i];
        VolDesc& d = base[i];
        if ((s = pk_init_desc(ctx, j.dims[0], j.dims[1], j.dims[2], &d)) != PK_OK) return s;
        d.raw = j.d_raw;
        d.raw_type = in_type;
        for (int k = 0; k < 3; k++) d.rdims[k] = j.rdims[k];
        d.padded = j.rdims[0] != j.dims[0] || j.rdims[1] != j.dims[1] || j.rdims[2] != j.dims[2];
        d.bg_f = (float)p->background;
        d.bg16 = (int)std::min(b16, 65535.0);
        d.I = j.I;
        d.mask8 = j.mask;
        d.write_mask = need_mask ? 1 : 0;
        d.zero_count = zc ? zc + i : nullptr;
        d.S = j.S;
        d.partials = j.part;
    }
    PkProgram prog;
    pk_program_add(prog, PK_STEP_Y, Y_PRE, base);
    std::vector<int> mask_mode(nj, need_mask ? 1 : 0);
    if (p->edge_erosion > 0) {
        // the erosion branch depends on whether the raw mask is full (decon_mask_edge_erosion.m:8)
        if ((s = pk_program_upload(ctx, prog, st)) != PK_OK) return s;
        if ((s = pk_program_launch(ctx, prog, st)) != PK_OK) return s;
        prog = PkProgram();
        std::vector<unsigned int> zeros(nj, 0);
        PK_CUDA(cudaMemcpyAsync(zeros.data(), zc, sizeof(unsigned int) * nj, cudaMemcpyDeviceToHost, st));
        PK_CUDA(cudaStreamSynchronize(st));
        std::vector<int2> disk = pk_disk_offsets(p->edge_erosion - 1);
        for (size_t i = 0; i < nj; i++) {
            if (zeros[i] == 0) { mask_mode[i] = 2; continue; }
            mask_mode[i] = 3;
            DeconJob& j = jobs[i];
            const int ny = j.dims[0], nx = j.dims[1], nz = j.dims[2];
            const size_t N = (size_t)ny * nx * nz;
            void *m2, *offs;
            if ((s = pk_scratch(ctx, SL_MASK2, N, &m2)) != PK_OK) return s;
            if ((s = pk_scratch(ctx, SL_OFFS, sizeof(int2) * disk.size(), &offs)) != PK_OK) return s;
            PK_CUDA(cudaMemcpyAsync(offs, disk.data(), sizeof(int2) * disk.size(), cudaMemcpyHostToDevice, st));
            k_mask_faces<<<grid_for((long long)N), 256, 0, st>>>(j.mask, ny, nx, nz);
            k_erode_xy<<<grid_for((long long)N), 256, 0, st>>>(j.mask, (uint8_t*)m2, ny, nx, nz, (const int2*)offs,
                                                                (int)disk.size());
            k_erode_z<<<grid_for((long long)N), 256, 0, st>>>((const uint8_t*)m2, j.mask, ny, nx, nz, p->edge_erosion - 1);
            PK_CUDA(cudaGetLastError());
            PK_CUDA(cudaStreamSynchronize(st));  // the offsets are a host temporary, m2 is reused
        }
    }
    for (VolDesc& d : base) {
        d.raw = nullptr;
        d.zero_count = nullptr;
        d.write_mask = 0;
    }
    if (numit == 0) {
        if (!prog.steps.empty()) {
            if ((s = pk_program_upload(ctx, prog, st)) != PK_OK) return s;
            if ((s = pk_program_launch(ctx, prog, st)) != PK_OK) return s;
        }
        for (size_t i = 0; i < nj; i++) {
            VolDesc f = base[i];
            set_post_job(f, p, mask_mode[i], jobs[i]);
            k_post_from<<<grid_for((long long)f.nrows * f.ny), 256, 0, st>>>(f, f.I);
            PK_CUDA(cudaGetLastError());
        }
        return PK_OK;
    }
    auto with = [&](auto fn) {
        std::vector<VolDesc> v(nj);
        for (size_t i = 0; i < nj; i++) {
            v[i] = base[i];
            fn(v[i], jobs[i], (int)i);
        }
        return v;
    };
    auto conv = [&](int which) {
        pk_program_add(prog, PK_STEP_X, XZ_FWD, base);
        pk_program_add(prog, PK_STEP_Z, XZ_CONV, with([&](VolDesc& d, DeconJob& j, int) {
            if (method == 1) { d.otf = which ? j.otf_b : j.otf_f; d.conj = 0; }
            else { d.otf = j.otf_f; d.conj = which; }
        }));
        pk_program_add(prog, PK_STEP_X, XZ_INV, base);
    };
    // debug runs launch each iteration's program on its own, then the caller's per-iteration work
    auto flush = [&]() -> pk_status {
        if (prog.steps.empty()) return PK_OK;
        pk_status r = pk_program_upload(ctx, prog, st);
        if (r == PK_OK) r = pk_program_launch(ctx, prog, st);
        prog = PkProgram();
        return r;
    };
    if (method == 1) {
        for (int it = 1; it <= numit; it++) {
            conv(0);
            pk_program_add(prog, PK_STEP_Y, Y_RATIO, base);
            conv(1);
            const bool last = it == numit && !dbg;
            pk_program_add(prog, PK_STEP_Y, last ? Y_FINAL : Y_UPDATE, with([&](VolDesc& d, DeconJob& j, int i) {
                d.Jo = it == 1 ? j.I : j.J;
                d.Jn = j.J;
                if (last) set_post_job(d, p, mask_mode[i], j);
            }));
            if (dbg) {
                if ((s = flush()) != PK_OK) return s;
                if ((s = dbg->after_iter(it, jobs[0].J, jobs[0].I)) != PK_OK) return s;
            }
        }
    } else {
        for (int k = 1; k <= numit; k++) {
            if (k >= 2) {
                pk_program_add(prog, PK_STEP_Y, Y_RLPRE, with([&](VolDesc& d, DeconJob& j, int) {
                    float* Jb[2] = {j.J, j.JB};
                    d.J2 = Jb[k % 2];
                    d.J3 = k == 2 ? j.I : Jb[(k - 1) % 2];
                    d.Yb = j.Yb;
                    d.lam_on = k >= 3 ? 1 : 0;
                }));
            }
            conv(0);
            pk_program_add(prog, PK_STEP_Y, Y_RATIO, base);
            conv(1);
            if (k < numit || dbg) {
                auto u = with([&](VolDesc& d, DeconJob& j, int) {
                    float* Jb[2] = {j.J, j.JB};
                    d.Yb = k == 1 ? j.I : j.Yb;
                    d.J4 = j.J4;
                    d.rl_first = k == 1 ? 1 : 0;
                    d.J2n = Jb[(k + 1) % 2];
                });
                pk_program_add(prog, PK_STEP_Y, Y_RLUPD, u);
                pk_program_add(prog, PK_STEP_LAMBDA, 0, u);
                if (dbg) {
                    if ((s = flush()) != PK_OK) return s;
                    if ((s = dbg->after_iter(k, (k + 1) % 2 ? jobs[0].JB : jobs[0].J, jobs[0].I)) != PK_OK) return s;
                }
            } else {
                pk_program_add(prog, PK_STEP_Y, Y_RLFINAL, with([&](VolDesc& d, DeconJob& j, int i) {
                    d.Yb = k == 1 ? j.I : j.Yb;
                    set_post_job(d, p, mask_mode[i], j);
                }));
            }
        }
    }
    if (dbg) {   // the last estimate is materialised: post-process it into the output
        if ((s = flush()) != PK_OK) return s;
        VolDesc f = base[0];
        set_post_job(f, p, mask_mode[0], jobs[0]);
        const float* Jlast = method == 1 ? jobs[0].J : ((numit + 1) % 2 ? jobs[0].JB : jobs[0].J);
        k_post_from<<<grid_for((long long)f.nrows * f.ny), 256, 0, st>>>(f, Jlast);
        PK_CUDA(cudaGetLastError());
        return PK_OK;
    }
    // streamed host call: the first two passes (y pre-pass, x forward) and the last two (x inverse,
    // final y pass) run slab by slab behind the slab copies
    const size_t ns = prog.steps.size();
    const DeconJob& j0 = jobs[0];
    const bool io_uploaded = io && !stream_io;
    if (stream_io)   // the program has the expected shape (checked, not assumed)
        stream_io = ns >= 5 && prog.steps[0].kind == PK_STEP_Y && prog.steps[0].mode == Y_PRE &&
                    prog.steps[1].kind == PK_STEP_X && prog.steps[1].mode == XZ_FWD &&
                    prog.steps[ns - 2].kind == PK_STEP_X && prog.steps[ns - 2].mode == XZ_INV &&
                    prog.steps[ns - 1].kind == PK_STEP_Y &&
                    (prog.steps[ns - 1].mode == Y_FINAL || prog.steps[ns - 1].mode == Y_RLFINAL) &&
                    !prog.descs[prog.steps[ns - 1].desc_off].need_xz;
    if (!stream_io) {
        if (io && !io_uploaded) {   // decided late: whole-volume upload before the program
            const size_t N = (size_t)j0.rdims[0] * j0.rdims[1] * j0.rdims[2];
            PK_CUDA(cudaMemcpyAsync((void*)j0.d_raw, io->h_in, N * io->in_esize, cudaMemcpyHostToDevice, st));
        }
        if ((s = pk_program_upload(ctx, prog, st)) != PK_OK) return s;
        return pk_program_launch(ctx, prog, st);
    }
    if (!ctx->h2d) PK_CUDA(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
    if (!ctx->d2h) PK_CUDA(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
    io->active = true;
    const int nz = j0.dims[2];
    const int nslab = std::min(8, nz / 8);
    const size_t plane = (size_t)j0.dims[0] * j0.dims[1];
    const PkStep head[2] = {prog.steps[0], prog.steps[1]};
    const PkStep tail[2] = {prog.steps[ns - 2], prog.steps[ns - 1]};
    // one program for the whole call (per-slab heads, the middle, per-slab tails), so its descriptors
    // go up in one small copy queued ahead of the slab uploads
    PkProgram all;
    all.no_graph = true;
    std::vector<int> zb(nslab + 1);
    for (int sl = 0; sl <= nslab; sl++) zb[sl] = (int)((long long)nz * sl / nslab);
    for (int sl = 0; sl < nslab; sl++)
        for (const PkStep& h : head)
            pk_program_add(all, h.kind, h.mode, {slab_view(prog.descs[h.desc_off], zb[sl], zb[sl + 1] - zb[sl],
                                                           io->in_esize, io->out_esize)});
    const size_t mid0 = all.steps.size();
    for (size_t k = 2; k + 2 < ns; k++) pk_program_add(all, prog.steps[k].kind, prog.steps[k].mode, {prog.descs[prog.steps[k].desc_off]});
    const size_t tail0 = all.steps.size();
    for (int sl = 0; sl < nslab; sl++)
        for (const PkStep& t : tail)
            pk_program_add(all, t.kind, t.mode, {slab_view(prog.descs[t.desc_off], zb[sl], zb[sl + 1] - zb[sl],
                                                           io->in_esize, io->out_esize)});
    if (all.steps.size() != tail0 + 2 * (size_t)nslab || mid0 != 2 * (size_t)nslab)
        return pk_fail(PK_ERR_UNSUPPORTED, "streamed program layout");
    if ((s = pk_program_upload(ctx, all, st)) != PK_OK) return s;
    // the upload may fuse convolution triples of the middle part (not the per-slab head or tail):
    // the tail starts 2 nslab steps from the end
    const size_t tail0u = all.steps.size() - 2 * (size_t)nslab;
    cudaEvent_t ev;
    for (int sl = 0; sl < nslab; sl++) {   // every slab upload is queued before any wait on the host
        if ((s = get_io_event(ctx, sl, &ev)) != PK_OK) return s;
        PK_CUDA(cudaMemcpyAsync((char*)j0.d_raw + zb[sl] * plane * io->in_esize,
                                (const char*)io->h_in + zb[sl] * plane * io->in_esize,
                                (size_t)(zb[sl + 1] - zb[sl]) * plane * io->in_esize, cudaMemcpyHostToDevice, ctx->h2d));
        PK_CUDA(cudaEventRecord(ev, ctx->h2d));
    }
    for (int sl = 0; sl < nslab; sl++) {
        PK_CUDA(cudaStreamWaitEvent(st, ctx->io_ev[sl], 0));
        if ((s = pk_program_launch_range(ctx, all, st, 2 * sl, 2 * sl + 2, false)) != PK_OK) return s;
    }
    if ((s = pk_program_launch_range(ctx, all, st, mid0, tail0u, false)) != PK_OK) return s;
    for (int sl = 0; sl < nslab; sl++) {
        if ((s = pk_program_launch_range(ctx, all, st, tail0u + 2 * sl, tail0u + 2 * sl + 2, sl == nslab - 1)) != PK_OK)
            return s;
        if ((s = get_io_event(ctx, nslab + sl, &ev)) != PK_OK) return s;
        PK_CUDA(cudaEventRecord(ev, st));
        PK_CUDA(cudaStreamWaitEvent(ctx->d2h, ev, 0));
        PK_CUDA(cudaMemcpyAsync((char*)io->h_out + zb[sl] * plane * io->out_esize,
                                (const char*)j0.d_out + zb[sl] * plane * io->out_esize,
                                (size_t)(zb[sl + 1] - zb[sl]) * plane * io->out_esize, cudaMemcpyDeviceToHost, ctx->d2h));
    }
    return PK_OK;
}

pk_status pk_decon_run(pk_ctx* ctx, int method, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                       const float* psf_f, const int64_t psf_f_dims[3], const float* psf_b,
                       const int64_t psf_b_dims[3], int numit, const pk_decon_params* p, void* d_out,
                       cudaStream_t st, HostStreamIO* io, const DebugHook* dbg) {
    PkRange range(method == 1 ? "pk_decon omw" : "pk_decon rl");
    pk_status s;
    if ((s = pk_check_params(dims, p)) != PK_OK) return s;
    if (numit < 0) return pk_fail(PK_ERR_INVALID, "NUMIT must be non-negative");
    DeconJob j;
    for (int i = 0; i < 3; i++) j.dims[i] = j.rdims[i] = (int)dims[i];
    VolDesc d;
    if ((s = pk_init_desc(ctx, j.dims[0], j.dims[1], j.dims[2], &d)) != PK_OK) return s;
    if ((s = pk_get_otf(ctx, psf_f, psf_f_dims, j.dims[0], j.dims[1], j.dims[2], &j.otf_f, st)) != PK_OK) return s;
    if (method == 1 && (s = pk_get_otf(ctx, psf_b, psf_b_dims, j.dims[0], j.dims[1], j.dims[2], &j.otf_b, st)) != PK_OK)
        return s;
    const bool need_mask = p->decon_offset != 0.0 || p->edge_erosion > 0;
    void* arena;
    if ((s = pk_scratch(ctx, SL_ARENA, pk_job_bytes(method, j.dims, need_mask, d.blocksY), &arena)) != PK_OK) return s;
    pk_job_carve(j, method, need_mask, d.blocksY, (char*)arena);
    j.d_raw = d_in;
    j.d_out = d_out;
    j.has_bbox = p->has_bbox;
    for (int i = 0; i < 6; i++) j.bbox[i] = p->bbox[i];
    std::vector<DeconJob> jobs{j};
    return pk_decon_multi(ctx, method, jobs, in_type, numit, p, st, io, dbg);
}

// ---- decon_mask_edge_erosion(im > 0, E) on its own (decon/decon_mask_edge_erosion.m:1-30), for the
// eroded-mask files that XR_RLdeconFrame3D saves; the irregular branch runs the kernels above
namespace {

template <typename T>
__global__ void k_positive(const T* __restrict__ im, long long n, uint8_t* __restrict__ m,
                           unsigned long long* __restrict__ zeros) {
    unsigned long long z = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const bool p = im[i] > (T)0;
        m[i] = p;
        z += !p;
    }
    if (z) atomicAdd(zeros, z);
}

// full mask: E voxels cleared at each face (:8-15), z only for more than one plane
__global__ void k_full_faces(uint8_t* m, int ny, int nx, int nz, int E) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny);
        const int x = (int)((i / ny) % nx);
        const int z = (int)(i / ((long long)ny * nx));
        if (y < E || y >= ny - E || x < E || x >= nx - E || (nz > 1 && (z < E || z >= nz - E))) m[i] = 0;
    }
}

}  // namespace

extern "C" pk_status pk_mask_edge_erosion(pk_ctx* ctx, const void* im, pk_dtype type, const int64_t dims[3],
                                          int32_t erosion, uint8_t* mask) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!im || !dims || !mask) return pk_fail(PK_ERR_INVALID, "NULL volume/dims/mask");
    if (type != PK_U16 && type != PK_F32) return pk_fail(PK_ERR_INVALID, "volume must be uint16 or single");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || dims[0] > INT32_MAX || dims[1] > INT32_MAX || dims[2] > INT32_MAX)
        return pk_fail(PK_ERR_INVALID, "bad volume size");
    if (erosion < 1 || erosion > 180) return pk_fail(PK_ERR_INVALID, "EdgeErosion must be in [1, 180]");
    const int ny = (int)dims[0], nx = (int)dims[1], nz = (int)dims[2];
    const long long n = (long long)ny * nx * nz;
    const size_t es = type == PK_U16 ? 2 : 4;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    pk_status s;
    void *din, *dm, *dm2, *dz, *doffs;
    const std::vector<int2> disk = pk_disk_offsets(erosion - 1);
    if ((s = pk_scratch(ctx, 37, es * n, &din)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 38, n, &dm)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 39, n, &dm2)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 40, sizeof(unsigned long long), &dz)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 41, sizeof(int2) * disk.size(), &doffs)) != PK_OK) return s;
    PK_CUDA(cudaMemcpyAsync(din, im, es * n, cudaMemcpyHostToDevice, st));
    PK_CUDA(cudaMemsetAsync(dz, 0, sizeof(unsigned long long), st));
    if (type == PK_U16) k_positive<<<grid_for(n), 256, 0, st>>>((const uint16_t*)din, n, (uint8_t*)dm, (unsigned long long*)dz);
    else k_positive<<<grid_for(n), 256, 0, st>>>((const float*)din, n, (uint8_t*)dm, (unsigned long long*)dz);
    unsigned long long zeros = 0;
    PK_CUDA(cudaMemcpyAsync(&zeros, dz, sizeof(zeros), cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    if (zeros == 0) {
        k_full_faces<<<grid_for(n), 256, 0, st>>>((uint8_t*)dm, ny, nx, nz, erosion);
        ctx->launches += 2;
    } else {                                                     // :18-29; k_erode_z is a copy for one plane
        PK_CUDA(cudaMemcpyAsync(doffs, disk.data(), sizeof(int2) * disk.size(), cudaMemcpyHostToDevice, st));
        k_mask_faces<<<grid_for(n), 256, 0, st>>>((uint8_t*)dm, ny, nx, nz);
        k_erode_xy<<<grid_for(n), 256, 0, st>>>((const uint8_t*)dm, (uint8_t*)dm2, ny, nx, nz, (const int2*)doffs,
                                                (int)disk.size());
        k_erode_z<<<grid_for(n), 256, 0, st>>>((const uint8_t*)dm2, (uint8_t*)dm, ny, nx, nz, erosion - 1);
        ctx->launches += 4;
    }
    PK_CUDA(cudaGetLastError());
    PK_CUDA(cudaMemcpyAsync(mask, dm, n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    return PK_OK;
}
