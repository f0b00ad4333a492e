// Edge taper of the raw volume (decon/RLdecon.m:351-357): every z slice goes through MATLAB's
// edgetaper(I, PSF) with PSF = fspecial('gaussian', nTapering + 30, nTapering):
//   B = real(ifft2(fft2(I) .* psf2otf(PSF, [ny nx])))            circular blur, PSF centred at floor(h/2)
//     = sum_ij PSF(i, j) I((y + hy/2 - i) mod ny, (x + hx/2 - j) mod nx)
//   alpha(y, x) = (1 - beta_y(y)) (1 - beta_x(x))
//   J = alpha .* I + (1 - alpha) .* B                           (uint16 by round-half-away, saturated)
// beta_d is the circular autocorrelation (period n_d - 1) of the PSF's projection on axis d, normalised
// to 1 at lag 0, with the lag-0 value repeated at index n_d - 1; it is 1 at both borders and 0 once
// the lag is beyond the PSF's width.  The weights are tiny host work in float64.
//
// The blur is a direct circular sum instead of a 2-D FFT.  A rank-1 PSF (the Gaussian is one) runs as
// two 1-D passes, y then x, each a grid-stride loop whose neighbouring threads read neighbouring y
// (coalesced; the h taps of a thread hit L1/L2), the second fused with the weighting and the
// conversion: 2 + 4 + 4 + 2 + 2 = 14 B of HBM per uint16 voxel.  Any other PSF runs as one direct
// 2-D sum.  Indexes wrap by one compare, which is exact because h_d <= n_d - 1 is checked.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

int grid_of(long long n) { return (int)std::max(1LL, std::min((n + 255) / 256, 148LL * 32)); }

template <typename T>
__device__ __forceinline__ float ld(const T* a, long long i) { return (float)a[i]; }

// uint16 by MATLAB's conversion (round half away from zero, saturate, NaN -> 0); single unchanged
__device__ __forceinline__ void st(uint16_t* o, long long i, float v) {
    float r = roundf(v);
    if (!(r >= 0.f)) r = 0.f;
    if (r > 65535.f) r = 65535.f;
    o[i] = (uint16_t)r;
}
__device__ __forceinline__ void st(float* o, long long i, float v) { o[i] = v; }

// y pass of a rank-1 PSF: T(y, x, z) = sum_i u(i) I((y + hy/2 - i) mod ny, x, z)
template <typename TI>
__global__ void k_taper_y(const TI* __restrict__ im, const float* __restrict__ u, int hy, float* __restrict__ t,
                          int ny, long long n) {
    const int cy = hy / 2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(q % ny);
        const long long col = q - y;
        int s = y + cy;
        if (s >= ny) s -= ny;
        float acc = 0.f;
        for (int i = 0; i < hy; i++) {
            acc = fmaf(u[i], ld(im, col + s), acc);
            s = s == 0 ? ny - 1 : s - 1;
        }
        t[q] = acc;
    }
}

// x pass of a rank-1 PSF fused with the weighting: B(y, x, z) = sum_j v(j) T(y, (x + hx/2 - j) mod nx, z)
template <typename TI, typename TO>
__global__ void k_taper_x(const TI* __restrict__ im, const float* __restrict__ t, const float* __restrict__ v, int hx,
                          const float* __restrict__ ay, const float* __restrict__ ax, TO* __restrict__ out, int ny,
                          int nx, long long n) {
    const int cx = hx / 2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(q % ny);
        const int x = (int)((q / ny) % nx);
        const long long row = q - (long long)x * ny;        // voxel (y, 0, z)
        int s = x + cx;
        if (s >= nx) s -= nx;
        float acc = 0.f;
        for (int j = 0; j < hx; j++) {
            acc = fmaf(v[j], t[row + (long long)s * ny], acc);
            s = s == 0 ? nx - 1 : s - 1;
        }
        const float a = ay[y] * ax[x];
        st(out, q, a * ld(im, q) + (1.f - a) * acc);
    }
}

// any other PSF: the direct 2-D circular sum, PSF column-major [hy hx]
template <typename TI, typename TO>
__global__ void k_taper_2d(const TI* __restrict__ im, const float* __restrict__ h, int hy, int hx,
                           const float* __restrict__ ay, const float* __restrict__ ax, TO* __restrict__ out, int ny,
                           int nx, long long n) {
    const int cy = hy / 2, cx = hx / 2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(q % ny);
        const int x = (int)((q / ny) % nx);
        const long long slice = q - y - (long long)x * ny;  // voxel (0, 0, z)
        int sy0 = y + cy, sx = x + cx;
        if (sy0 >= ny) sy0 -= ny;
        if (sx >= nx) sx -= nx;
        float acc = 0.f;
        for (int j = 0; j < hx; j++) {
            const long long colb = slice + (long long)sx * ny;
            int sy = sy0;
            for (int i = 0; i < hy; i++) {
                acc = fmaf(h[i + (long long)j * hy], ld(im, colb + sy), acc);
                sy = sy == 0 ? ny - 1 : sy - 1;
            }
            sx = sx == 0 ? nx - 1 : sx - 1;
        }
        const float a = ay[y] * ax[x];
        st(out, q, a * ld(im, q) + (1.f - a) * acc);
    }
}

// 1 - beta_d for an axis of n samples from the PSF's projection p (length h <= n - 1)
std::vector<float> one_minus_beta(const std::vector<double>& p, int n) {
    const int h = (int)p.size(), L = n - 1;
    std::vector<double> c(h, 0.0);                  // linear autocorrelation at lag d < h
    for (int d = 0; d < h; d++)
        for (int m = 0; m + d < h; m++) c[d] += p[m] * p[m + d];
    std::vector<double> r(L, 0.0);                  // circular, period L: r(l) = c(l) + c(L - l)
    for (int l = 0; l < L; l++) {
        if (l < h) r[l] += c[l];
        if (l > 0 && L - l < h) r[l] += c[L - l];
    }
    double mx = 0.0;
    for (double v : r) mx = std::max(mx, v);
    std::vector<float> w(n);
    for (int l = 0; l < n; l++) w[l] = (float)(1.0 - (mx > 0.0 ? r[l < L ? l : 0] / mx : 0.0));
    return w;
}

size_t es(pk_dtype t) { return t == PK_U16 ? 2 : 4; }

template <typename TI, typename TO>
void launch(bool sep, const void* din, float* dt, const float* dsmall, int hy, int hx, int ny, int nx, long long n,
            void* dout, cudaStream_t st) {
    const int g = grid_of(n);
    const float* ay = dsmall + hy + hx;
    const float* ax = ay + ny;
    if (sep) {
        k_taper_y<<<g, 256, 0, st>>>((const TI*)din, dsmall, hy, dt, ny, n);
        k_taper_x<<<g, 256, 0, st>>>((const TI*)din, dt, dsmall + hy, hx, ay, ax, (TO*)dout, ny, nx, n);
    } else {
        k_taper_2d<<<g, 256, 0, st>>>((const TI*)din, ax + nx, hy, hx, ay, ax, (TO*)dout, ny, nx, n);
    }
}

}  // namespace

extern "C" pk_status pk_edgetaper(pk_ctx* ctx, const void* in, pk_dtype type, const int64_t dims[3], const double* psf,
                                  const int64_t psf_dims[2], void* out) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!in || !out || !dims || !psf || !psf_dims) return pk_fail(PK_ERR_INVALID, "NULL volume/PSF/output");
    if (type != PK_U16 && type != PK_F32) return pk_fail(PK_ERR_INVALID, "edgetaper: volume must be uint16 or single");
    if (dims[0] < 2 || dims[1] < 2 || dims[2] < 1 || dims[0] > INT32_MAX || dims[1] > INT32_MAX)
        return pk_fail(PK_ERR_INVALID, "edgetaper: bad volume size");
    if (psf_dims[0] < 1 || psf_dims[1] < 1) return pk_fail(PK_ERR_INVALID, "edgetaper: empty PSF");
    if (psf_dims[0] > dims[0] - 1 || psf_dims[1] > dims[1] - 1)
        return pk_fail(PK_ERR_INVALID, "edgetaper: the PSF must be smaller than the image in y and x");
    const int ny = (int)dims[0], nx = (int)dims[1], hy = (int)psf_dims[0], hx = (int)psf_dims[1];
    const long long n = (long long)ny * nx * dims[2];
    double mx = 0.0;
    int i0 = 0, j0 = 0;
    for (int j = 0; j < hx; j++)
        for (int i = 0; i < hy; i++) {
            const double v = psf[i + (long long)j * hy];
            if (!std::isfinite(v)) return pk_fail(PK_ERR_INVALID, "edgetaper: PSF is not finite");
            if (std::fabs(v) > mx) mx = std::fabs(v), i0 = i, j0 = j;
        }
    // rank-1 test: PSF(i, j) = u(i) v(j) with u = PSF(:, j0), v = PSF(i0, :) / PSF(i0, j0)
    bool sep = mx > 0.0;
    for (int j = 0; sep && j < hx; j++)
        for (int i = 0; i < hy; i++) {
            const double uv = psf[i + (long long)j0 * hy] * psf[i0 + (long long)j * hy] / psf[i0 + (long long)j0 * hy];
            if (std::fabs(psf[i + (long long)j * hy] - uv) > 1e-6 * mx) { sep = false; break; }
        }
    if (!sep && (double)hy * hx * (double)n > 1.1e12)
        return pk_fail(PK_ERR_INVALID, "edgetaper: a PSF that is not rank-1 is limited to hy*hx*numel <= 1.1e12");
    std::vector<double> py(hy, 0.0), px(hx, 0.0);
    for (int j = 0; j < hx; j++)
        for (int i = 0; i < hy; i++) py[i] += psf[i + (long long)j * hy], px[j] += psf[i + (long long)j * hy];
    const std::vector<float> ay = one_minus_beta(py, ny), ax = one_minus_beta(px, nx);
    // small device table: u (hy) | v (hx) | 1 - beta_y (ny) | 1 - beta_x (nx) | PSF (hy*hx, non-separable)
    std::vector<float> small((size_t)hy + hx + ny + nx + (sep ? 0 : (size_t)hy * hx), 0.f);
    if (sep)
        for (int i = 0; i < hy; i++) small[i] = (float)psf[i + (long long)j0 * hy];
    if (sep)
        for (int j = 0; j < hx; j++) small[hy + j] = (float)(psf[i0 + (long long)j * hy] / psf[i0 + (long long)j0 * hy]);
    std::copy(ay.begin(), ay.end(), small.begin() + hy + hx);
    std::copy(ax.begin(), ax.end(), small.begin() + hy + hx + ny);
    if (!sep)
        for (long long k = 0; k < (long long)hy * hx; k++) small[hy + hx + ny + nx + k] = (float)psf[k];

    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    pk_status s;
    void *din, *dout, *dsmall, *dt = nullptr;
    if ((s = pk_scratch(ctx, 33, es(type) * n, &din)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 34, es(type) * n, &dout)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 35, sizeof(float) * small.size(), &dsmall)) != PK_OK) return s;
    if (sep && (s = pk_scratch(ctx, 36, sizeof(float) * n, &dt)) != PK_OK) return s;
    PK_CUDA(cudaMemcpyAsync(dsmall, small.data(), sizeof(float) * small.size(), cudaMemcpyHostToDevice, st));
    PK_CUDA(cudaMemcpyAsync(din, in, es(type) * n, cudaMemcpyHostToDevice, st));
    if (type == PK_U16) launch<uint16_t, uint16_t>(sep, din, (float*)dt, (const float*)dsmall, hy, hx, ny, nx, n, dout, st);
    else launch<float, float>(sep, din, (float*)dt, (const float*)dsmall, hy, hx, ny, nx, n, dout, st);
    PK_CUDA(cudaGetLastError());
    ctx->launches += sep ? 2 : 1;
    PK_CUDA(cudaMemcpyAsync(out, dout, es(type) * n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    return PK_OK;
}
