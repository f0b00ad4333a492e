// PSF preparation: psf_gen_new.m:1-140, called for every measured PSF before deconvolution
// (RLdecon.m:241-248 with psfGen = true, its default; RLdecon_large_in_memory.m:107;
// RLdecon_large_in_place.m:127; XR_decon_data_wrapper.m:279).
//
// Device work: the 3x3x3 (3x3 in 2D) median filter, the border-row threshold of the 'masked'
// method, the closing of the peak component with strel('sphere', 3) (strel('disk', 3) in 2D), the
// masked background subtraction, the z padding + circular shift that centres the peak, and the
// axial resampling (z-only float64 DFT pair: the x/y transforms of the reference's fftn / ifftn
// cancel because the truncation acts on z alone).  Host work: the 26-connected labelling
// (bwareaopen, bwlabeln), the median of the border slices of the 'median' method, the peak and
// the z extent.
//
// Fixed orders of operations (the reference leaves them to MATLAB): the means of the border rows
// are float64 sums in row order (then z) rounded to float32; the median of an even count is the
// float64 mean of the middle pair rounded to float32; a*3 + b is two rounded float operations.
// The resampled PSF is returned in float32 (MATLAB returns double there).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

constexpr int kMasked = 0, kMedian = 1;

int grid_of(long long n) {
    long long g = (n + 255) / 256;
    return (int)std::max(1LL, std::min(g, 148LL * 16));
}

// median of K values by rank (exact for every ordering of equal values; NaN is never selected)
template <int K>
__device__ __forceinline__ float median_rank(const float (&v)[K]) {
    constexpr int mid = K / 2;
    float r = v[mid];
#pragma unroll
    for (int i = 0; i < K; i++) {
        int lt = 0, le = 0;
#pragma unroll
        for (int j = 0; j < K; j++) {
            lt += v[j] < v[i];
            le += v[j] <= v[i];
        }
        if (lt <= mid && mid < le) r = v[i];
    }
    return r;
}

// medfilt3(a, [3 3 3]) ('symmetric' padding = edge voxel repeated for a 3-wide window)
__global__ void k_medfilt3(const float* __restrict__ a, float* __restrict__ out, int ny, int nx, int nz) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny), x = (int)((i / ny) % nx), z = (int)(i / ((long long)ny * nx));
        float v[27];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const int yy = min(max(y + q - 1, 0), ny - 1);
                    const int xx = min(max(x + b - 1, 0), nx - 1);
                    const int zz = min(max(z + c - 1, 0), nz - 1);
                    v[q + 3 * b + 9 * c] = a[yy + (long long)ny * (xx + (long long)nx * zz)];
                }
        out[i] = median_rank<27>(v);
    }
}

// medfilt2(a, [3 3]) (zero padding), nz == 1
__global__ void k_medfilt2(const float* __restrict__ a, float* __restrict__ out, int ny, int nx) {
    const long long n = (long long)ny * nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny), x = (int)(i / ny);
        float v[9];
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const int yy = y + q - 1, xx = x + b - 1;
                v[q + 3 * b] = (yy < 0 || yy >= ny || xx < 0 || xx >= nx) ? 0.f : a[yy + (long long)ny * xx];
            }
        out[i] = median_rank<9>(v);
    }
}

__device__ __forceinline__ int border_row(int r, int ny) { return r < 10 ? r : ny - 20 + r; }   // [1:10, end-9:end]

// 'masked' threshold (psf_gen_new.m:49-51, 2D :79-81): per (x, z) column
//   a = max_r sqrt(|med(r) - 100|) * 3 + mean_r med(r)   (2D: sqrt(med(r)), no offset)
// over the 20 border rows; BW = med > a
__global__ void k_border_thresh(const float* __restrict__ med, uint8_t* __restrict__ bw, int ny, int nx, int nz, int twod) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long col = i / ny;
        const float* c = med + col * ny;
        float mx = 0.f;
        double s = 0.0;
        for (int r = 0; r < 20; r++) {
            const float v = c[border_row(r, ny)];
            const float q = twod ? __fsqrt_rn(v) : __fsqrt_rn(fabsf(__fsub_rn(v, 100.f)));
            mx = r == 0 ? q : fmaxf(mx, q);
            s += (double)v;
        }
        const float a = __fadd_rn(__fmul_rn(mx, 3.f), (float)(s / 20.0));
        bw[i] = med[i] > a;
    }
}

// mean over the border rows and z, per x (psf_gen_new.m:57): float64, rows outer, z inner
__global__ void k_border_colmean(const float* __restrict__ raw, float* __restrict__ colmean, int ny, int nx, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    double s = 0.0;
    for (int r = 0; r < 20; r++) {
        const int y = border_row(r, ny);
        for (int z = 0; z < nz; z++) s += (double)raw[y + (long long)ny * (x + (long long)nx * z)];
    }
    colmean[x] = (float)(s / (20.0 * nz));
}

// raw = max(psf - s, 0)  (psf_gen_new.m:33-35)
__global__ void k_sub_clamp(const float* __restrict__ a, float s, float* __restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = fmaxf(__fsub_rn(a[i], s), 0.f);
}

// masked: out = raw .* BW - colmean(x), negatives to 0 (:57-58);  median: out = raw .* BW (:41)
__global__ void k_apply_mask(const float* __restrict__ raw, const uint8_t* __restrict__ bw,
                             const float* __restrict__ colmean, float* __restrict__ out, int ny, int nx, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float v = __fmul_rn(raw[i], bw[i] ? 1.f : 0.f);
        if (colmean) {
            v = __fsub_rn(v, colmean[(i / ny) % nx]);
            if (v < 0.f) v = 0.f;
        }
        out[i] = v;
    }
}

// z padding (pre slices of zeros, total nz2) + circshift by (sy, sx, sz)  (:109-121); clamp at 0
// when the result is final (no resampling, :139)
__global__ void k_place(const float* __restrict__ raw, float* __restrict__ out, int ny, int nx, int nz, int nz2,
                        int pre, int sy, int sx, int sz, int clamp0) {
    const long long n = (long long)ny * nx * nz2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny), x = (int)((i / ny) % nx), z = (int)(i / ((long long)ny * nx));
        const int ys = ((y - sy) % ny + ny) % ny, xs = ((x - sx) % nx + nx) % nx;
        const int zs = ((z - sz) % nz2 + nz2) % nz2 - pre;
        float v = (zs >= 0 && zs < nz) ? raw[ys + (long long)ny * (xs + (long long)nx * zs)] : 0.f;
        if (clamp0) v = fmaxf(v, 0.f);
        out[i] = v;
    }
}

// kept axial frequencies (:128-131): plane m of the truncated spectrum comes from plane src(m) of
// the full one; the second band wins where the two overlap (odd new_nz)
__device__ __forceinline__ int kept_src(int m, int nz, int new_nz, int h) {
    if (m >= new_nz - h) return nz - new_nz + m;
    return m < h ? m : -1;
}

// G[y,x,m] = sum_j c[y,x,j] exp(-2 pi i j src(m) / nz)   (float64)
__global__ void k_dft_z_kept(const float* __restrict__ c, double2* __restrict__ G, int ny, int nx, int nz, int new_nz,
                             int h, const double2* __restrict__ tw) {
    const long long plane = (long long)ny * nx, n = plane * new_nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long p = i % plane;
        const int m = (int)(i / plane);
        const int k = kept_src(m, nz, new_nz, h);
        double re = 0.0, im = 0.0;
        if (k >= 0) {
            long long jk = 0;
            for (int j = 0; j < nz; j++) {
                const double v = (double)c[p + plane * j];
                const double2 w = tw[jk];
                re += v * w.x;
                im += v * w.y;
                jk += k;
                if (jk >= nz) jk -= nz;
            }
        }
        G[i] = make_double2(re, im);
    }
}

// out[y,x,j] = max(real(sum_m G[y,x,m] exp(+2 pi i m j / new_nz)) / new_nz, 0)
__global__ void k_idft_z_real(const double2* __restrict__ G, float* __restrict__ out, int ny, int nx, int new_nz,
                              const double2* __restrict__ tw) {
    const long long plane = (long long)ny * nx, n = plane * new_nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long p = i % plane;
        const int j = (int)(i / plane);
        double re = 0.0;
        long long mj = 0;
        for (int m = 0; m < new_nz; m++) {
            const double2 g = G[p + plane * m];
            const double2 w = tw[mj];
            re += g.x * w.x - g.y * w.y;
            mj += j;
            if (mj >= new_nz) mj -= new_nz;
        }
        const double v = re / (double)new_nz;
        out[i] = (float)(v > 0.0 ? v : 0.0);
    }
}

long long round_half_away(double v) { return v >= 0 ? (long long)std::floor(v + 0.5) : (long long)std::ceil(v - 0.5); }

struct Buf {
    void* p = nullptr;
    ~Buf() { if (p) cudaFree(p); }
    template <typename T> T* as() { return (T*)p; }
};

pk_status balloc(Buf& b, size_t bytes) {
    if (cudaMalloc(&b.p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
        cudaGetLastError();
        return pk_fail(PK_ERR_NOMEM, "psf_gen: device allocation failed");
    }
    return PK_OK;
}

// bwareaopen(BW, P) then L = bwlabeln(BW), BW = L == L(peak)  (:36-39, :52-55, :70-72, :83-86)
std::vector<uint8_t> peak_component(const std::vector<uint8_t>& bw, int ny, int nx, int nz, long long P, long long peak) {
    std::vector<int> lab;
    std::vector<long long> sz;
    pk_label26(bw.data(), ny, nx, nz, lab, sz);
    std::vector<uint8_t> kept(bw.size());
    for (size_t i = 0; i < bw.size(); i++) kept[i] = lab[i] && sz[lab[i]] >= P;
    pk_label26(kept.data(), ny, nx, nz, lab, sz);
    const int lp = lab[(size_t)peak];
    std::vector<uint8_t> out(bw.size());
    for (size_t i = 0; i < bw.size(); i++) out[i] = lab[i] == lp;   // lp == 0: every voxel outside the components
    return out;
}

long long first_max(const std::vector<float>& v) {
    long long k = 0;
    for (size_t i = 1; i < v.size(); i++)
        if (v[i] > v[(size_t)k]) k = (long long)i;
    return k;
}

}  // namespace

extern "C" pk_status pk_psf_gen(pk_ctx* ctx, const float* psf, const int64_t dims[3], double dz_psf, double dz_data,
                                double med_factor, int32_t method, float* out, int64_t out_capacity, int64_t out_dims[3]) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!psf || !dims || !out_dims) return pk_fail(PK_ERR_INVALID, "NULL psf/dims/out_dims");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || dims[0] * dims[1] * dims[2] > (1LL << 31))
        return pk_fail(PK_ERR_INVALID, "psf_gen: bad PSF size");
    if (method != kMasked && method != kMedian) return pk_fail(PK_ERR_INVALID, "PSFGenMethod must be 0 ('masked') or 1 ('median')");
    const int ny = (int)dims[0], nx = (int)dims[1], nz = (int)dims[2];
    const long long n = (long long)ny * nx * nz;
    const long long plane = (long long)ny * nx;
    const bool twod = nz == 1;
    if (twod && method == kMedian)
        return pk_fail(PK_ERR_UNSUPPORTED, "psf_gen_new.m:68 calls medfilt, which neither MATLAB nor the reference defines");
    if (!twod && nz < 5) return pk_fail(PK_ERR_INVALID, "psf_gen_new.m:26 indexes slices [1:5, end-4:end]: the PSF needs 5 or more slices");

    // does the cleanup run?  (:25-29: any positive value in the first / last five slices; 2D: always)
    bool clean = twod;
    std::vector<float> fl;
    if (!twod) {
        const int zl[10] = {0, 1, 2, 3, 4, nz - 5, nz - 4, nz - 3, nz - 2, nz - 1};
        for (int k = 0; k < 10; k++)
            for (long long q = 0; q < plane; q++) {
                const float v = psf[plane * zl[k] + q];
                if (v > 0.f) {
                    clean = true;
                    if (method == kMedian) fl.push_back(v);
                }
            }
    }
    if (clean && method == kMasked && ny < 10)
        return pk_fail(PK_ERR_INVALID, "psf_gen_new.m:49 indexes rows [1:10, end-9:end]: the PSF needs 10 or more rows");

    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    pk_status s;
    Buf dpsf, draw, dmed, dbw, dcol, doffs;
    if ((s = balloc(dpsf, 4 * n)) || (s = balloc(draw, 4 * n)))
        return s;
    PK_CUDA(cudaMemcpyAsync(dpsf.p, psf, 4 * n, cudaMemcpyHostToDevice, st));
    const float* dres = dpsf.as<float>();      // the cleaned PSF (psf_raw after :95)
    if (clean) {
        if ((s = balloc(dmed, 4 * n)) || (s = balloc(dbw, 2 * n)) || (s = balloc(dcol, 4 * nx)))
            return s;
        std::vector<float> med(n);
        std::vector<uint8_t> bw(n);
        const float* dsrc = dpsf.as<float>();
        if (method == kMedian) {                                   // :31-35
            const size_t k = fl.size();
            std::sort(fl.begin(), fl.end());
            const float m = k % 2 ? fl[k / 2] : (float)(((double)fl[k / 2 - 1] + (double)fl[k / 2]) / 2.0);
            const float sub = (float)med_factor * m;
            k_sub_clamp<<<grid_of(n), 256, 0, st>>>(dpsf.as<float>(), sub, draw.as<float>(), n);
            dsrc = draw.as<float>();
        }
        if (twod) k_medfilt2<<<grid_of(n), 256, 0, st>>>(dsrc, dmed.as<float>(), ny, nx);
        else k_medfilt3<<<grid_of(n), 256, 0, st>>>(dsrc, dmed.as<float>(), ny, nx, nz);
        if (method == kMasked) k_border_thresh<<<grid_of(n), 256, 0, st>>>(dmed.as<float>(), dbw.as<uint8_t>(), ny, nx, nz, twod);
        PK_CUDA(cudaGetLastError());
        PK_CUDA(cudaMemcpyAsync(med.data(), dmed.p, 4 * n, cudaMemcpyDeviceToHost, st));
        if (method == kMasked) PK_CUDA(cudaMemcpyAsync(bw.data(), dbw.p, n, cudaMemcpyDeviceToHost, st));
        PK_CUDA(cudaStreamSynchronize(st));
        if (method == kMedian)
            for (long long i = 0; i < n; i++) bw[i] = med[i] > 0.f;
        if (twod)
            for (int r = 0; r < 20; r++)
                for (int x = 0; x < nx; x++)
                    if (med[(r < 10 ? r : ny - 20 + r) + (long long)ny * x] < 0.f)
                        return pk_fail(PK_ERR_UNSUPPORTED, "psf_gen_new.m:79 takes sqrt of negative border values (complex in MATLAB)");
        bw = peak_component(bw, ny, nx, nz, twod ? 50 : 300, first_max(med));
        // imclose(BW, strel('sphere', 3)) / strel('disk', 3) on the GPU
        std::vector<int4> offs;
        if (twod) {
            for (const int2& d : pk_disk_offsets(3)) offs.push_back(make_int4(d.x, d.y, 0, 0));
        } else {
            offs = pk_ball_offsets(3);
        }
        if ((s = balloc(doffs, sizeof(int4) * offs.size())) != PK_OK) return s;
        PK_CUDA(cudaMemcpyAsync(doffs.p, offs.data(), sizeof(int4) * offs.size(), cudaMemcpyHostToDevice, st));
        PK_CUDA(cudaMemcpyAsync(dbw.p, bw.data(), n, cudaMemcpyHostToDevice, st));
        if ((s = pk_morph_ops(dbw.as<uint8_t>(), dbw.as<uint8_t>() + n, ny, nx, nz, doffs.as<int4>(), (int)offs.size(), "de", st)) != PK_OK)
            return s;
        const float* colmean = nullptr;
        if (method == kMasked) {
            k_border_colmean<<<(nx + 127) / 128, 128, 0, st>>>(dpsf.as<float>(), dcol.as<float>(), ny, nx, nz);
            colmean = dcol.as<float>();
        }
        // the input of the mask product: psf (masked) or max(psf - s, 0) (median); result into dmed
        k_apply_mask<<<grid_of(n), 256, 0, st>>>(method == kMedian ? draw.as<float>() : dpsf.as<float>(), dbw.as<uint8_t>(),
                                                 colmean, dmed.as<float>(), ny, nx, n);
        PK_CUDA(cudaGetLastError());
        dres = dmed.as<float>();
    }

    // peak, z extent and the centring shift (:97-121)
    std::vector<float> raw(n);
    PK_CUDA(cudaMemcpyAsync(raw.data(), dres, 4 * n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    const long long pk = first_max(raw);
    const int py = (int)(pk % ny) + 1, px = (int)((pk / ny) % nx) + 1;
    int pz = (int)(pk / plane) + 1;
    int zs = 0, zt = 0;
    for (int z = 0; z < nz; z++) {
        double zsum = 0.0;
        for (long long q = 0; q < plane; q++) zsum += (double)raw[plane * z + q];
        if (zsum != 0.0) {
            if (!zs) zs = z + 1;
            zt = z + 1;
        }
    }
    if (!zs) return pk_fail(PK_ERR_INVALID, "psf_gen_new.m:105: the cleaned PSF is all zero");
    int nz2 = nz, pre = 0;
    if (pz - zs > nz2 / 2.0) nz2 += (int)(pz - zs - round_half_away((nz2 - 1) / 2.0) + 3);            // :109-112
    if (zt - pz > nz2 / 2.0) {                                                                        // :113-117
        pre = (int)(zt - pz - round_half_away((nz2 - 1) / 2.0) + 3);
        pz += pre;
        nz2 += pre;
    }
    const int sy = (int)round_half_away((ny + 1) / 2.0 - py);
    const int sx = (int)round_half_away((nx + 1) / 2.0 - px);
    const int sz = (int)round_half_away((nz2 + 1) / 2.0 - pz);

    const double ratio = dz_data / dz_psf;
    const bool resample = ratio > 1;
    long long new_nz = nz2;
    if (resample) new_nz = std::min<long long>(std::max<long long>(round_half_away(nz2 / ratio), 0), 65535);   // uint16(round(.))
    out_dims[0] = ny;
    out_dims[1] = nx;
    out_dims[2] = new_nz;
    if (!out) return PK_OK;
    const long long nout = plane * new_nz;
    if (out_capacity < nout) return pk_fail(PK_ERR_INVALID, "psf_gen: output buffer too small (see out_dims)");
    if (nout == 0) return PK_OK;

    Buf dc, dG, dtwf, dtwi, dout;
    if ((s = balloc(dc, 4 * plane * nz2)) != PK_OK) return s;
    k_place<<<grid_of(plane * nz2), 256, 0, st>>>(dres, dc.as<float>(), ny, nx, nz, nz2, pre, sy, sx, sz, resample ? 0 : 1);
    PK_CUDA(cudaGetLastError());
    const float* dfinal = dc.as<float>();
    if (resample) {                                                                                   // :126-135
        const int h = (int)((new_nz + 1) / 2);                                                        // uint16 new_nz/2
        const std::vector<double2> twf = pk_twiddles64(nz2, -1), twi = pk_twiddles64((int)new_nz, +1);
        if ((s = balloc(dG, 16 * nout)) || (s = balloc(dtwf, 16 * twf.size())) || (s = balloc(dtwi, 16 * twi.size())) ||
            (s = balloc(dout, 4 * nout)))
            return s;
        PK_CUDA(cudaMemcpyAsync(dtwf.p, twf.data(), 16 * twf.size(), cudaMemcpyHostToDevice, st));
        PK_CUDA(cudaMemcpyAsync(dtwi.p, twi.data(), 16 * twi.size(), cudaMemcpyHostToDevice, st));
        k_dft_z_kept<<<grid_of(nout), 256, 0, st>>>(dc.as<float>(), dG.as<double2>(), ny, nx, nz2, (int)new_nz, h,
                                                    dtwf.as<double2>());
        k_idft_z_real<<<grid_of(nout), 256, 0, st>>>(dG.as<double2>(), dout.as<float>(), ny, nx, (int)new_nz, dtwi.as<double2>());
        PK_CUDA(cudaGetLastError());
        dfinal = dout.as<float>();
    }
    PK_CUDA(cudaMemcpyAsync(out, dfinal, 4 * nout, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    return PK_OK;
}
