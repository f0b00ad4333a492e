// Edge erosion of the large-file runner (RLdecon_large_in_memory.m:146-168, 267-270):
//   im_bw_erode = im > 0 with the six faces cleared;  im_bw_erode = bwdist(~im_bw_erode) > E - 1;
//   result = result .* im_bw_erode.
// bwdist is the Euclidean distance to the nearest cleared voxel.  Only the test d^2 > R^2 (R = E - 1)
// is needed, and the squared Euclidean distance is a sum over the three axes, so it is computed
// exactly as three windowed min-plus passes (Saito-Toriwaki decomposition) restricted to |d| <= R:
//   A(v) = min_{|dy|<=R, v+dy cleared} dy^2
//   B(v) = min_{|dx|<=R} A(v + dx) + dx^2
//   C(v) = min_{|dz|<=R} B(v + dz) + dz^2,      keep v  <=>  C(v) > R^2
// Values are capped at R^2 + 1 (anything larger cannot change the test), so each pass is 2R + 1
// reads of 16-bit values per voxel, all HBM-bound and coalesced along y.
#include <algorithm>
#include <string>

#include "pk_internal.h"

namespace {

int grid_of(long long n) { return (int)std::max(1LL, std::min((n + 255) / 256, 148LL * 32)); }

template <typename T>
__device__ __forceinline__ bool positive(const T* a, long long i) { return a[i] > (T)0; }

// pass along y from the raw volume: the cleared set is {im <= 0} plus the faces
template <typename T>
__global__ void k_edt_y(const T* __restrict__ im, uint16_t* __restrict__ A, int ny, int nx, int nz, int R, int cap) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny);
        const long long col = i / ny;
        const int x = (int)(col % nx), z = (int)(col / nx);
        const bool xz_face = x == 0 || x == nx - 1 || z == 0 || z == nz - 1;
        int best = cap;
        for (int d = -R; d <= R; d++) {
            const int yy = y + d;
            if (yy < 0 || yy >= ny) continue;
            const bool cleared = xz_face || yy == 0 || yy == ny - 1 || !positive(im, i + d);
            if (cleared) best = min(best, d * d);
        }
        A[i] = (uint16_t)best;
    }
}

// min-plus pass along an axis with element stride `stride` and extent `len`
__global__ void k_edt_pass(const uint16_t* __restrict__ in, uint16_t* __restrict__ out, long long n, long long stride,
                           int len, long long inner, int R, int cap) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)((i / inner) % len);
        int best = cap;
        for (int d = -R; d <= R; d++) {
            const int cc = c + d;
            if (cc < 0 || cc >= len) continue;
            best = min(best, (int)in[i + (long long)d * stride] + d * d);
        }
        out[i] = (uint16_t)min(best, cap);
    }
}

// last pass along z fused with the multiply of the result
template <typename TO>
__global__ void k_edt_z_apply(const uint16_t* __restrict__ B, TO* __restrict__ out, uint8_t* __restrict__ mask,
                              int ny, int nx, int nz, int R, int cap) {
    const long long plane = (long long)ny * nx, n = plane * nz;
    const int r2 = R * R;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i / plane);
        int best = cap;
        for (int d = -R; d <= R; d++) {
            const int zz = z + d;
            if (zz < 0 || zz >= nz) continue;
            best = min(best, (int)B[i + (long long)d * plane] + d * d);
        }
        const bool keep = best > r2;
        if (mask) mask[i] = keep;
        if (out && !keep) out[i] = (TO)0;
    }
}

size_t es(pk_dtype t) { return t == PK_U16 ? 2 : t == PK_F32 ? 4 : 8; }

}  // namespace

extern "C" pk_status pk_edge_erosion_edt(pk_ctx* ctx, const void* im, pk_dtype im_type, const int64_t dims[3],
                                         int32_t erosion, void* out, pk_dtype out_type, uint8_t* mask) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!im || !dims) return pk_fail(PK_ERR_INVALID, "NULL volume/dims");
    if (im_type != PK_U16 && im_type != PK_F32) return pk_fail(PK_ERR_INVALID, "volume must be uint16 or single");
    if (out && out_type != PK_U16 && out_type != PK_F32) return pk_fail(PK_ERR_INVALID, "result must be uint16 or single");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return pk_fail(PK_ERR_INVALID, "bad volume size");
    if (erosion < 1 || erosion > 180) return pk_fail(PK_ERR_INVALID, "EdgeErosion must be in [1, 180]");
    const int ny = (int)dims[0], nx = (int)dims[1], nz = (int)dims[2];
    const long long n = (long long)ny * nx * nz;
    const int R = erosion - 1, cap = R * R + 1;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    pk_status s;
    void *dim, *dA, *dB, *dout = nullptr, *dmask = nullptr;
    if ((s = pk_scratch(ctx, 28, es(im_type) * n, &dim)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 29, 2 * n, &dA)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 30, 2 * n, &dB)) != PK_OK) return s;
    if (out && (s = pk_scratch(ctx, 31, es(out_type) * n, &dout)) != PK_OK) return s;
    if (mask && (s = pk_scratch(ctx, 32, n, &dmask)) != PK_OK) return s;
    PK_CUDA(cudaMemcpyAsync(dim, im, es(im_type) * n, cudaMemcpyHostToDevice, st));
    if (out) PK_CUDA(cudaMemcpyAsync(dout, out, es(out_type) * n, cudaMemcpyHostToDevice, st));
    const int g = grid_of(n);
    if (im_type == PK_U16) k_edt_y<<<g, 256, 0, st>>>((const uint16_t*)dim, (uint16_t*)dA, ny, nx, nz, R, cap);
    else k_edt_y<<<g, 256, 0, st>>>((const float*)dim, (uint16_t*)dA, ny, nx, nz, R, cap);
    k_edt_pass<<<g, 256, 0, st>>>((const uint16_t*)dA, (uint16_t*)dB, n, ny, nx, ny, R, cap);
    if (out_type == PK_U16 || !out)
        k_edt_z_apply<<<g, 256, 0, st>>>((const uint16_t*)dB, (uint16_t*)dout, (uint8_t*)dmask, ny, nx, nz, R, cap);
    else
        k_edt_z_apply<<<g, 256, 0, st>>>((const uint16_t*)dB, (float*)dout, (uint8_t*)dmask, ny, nx, nz, R, cap);
    PK_CUDA(cudaGetLastError());
    ctx->launches += 3;
    if (out) PK_CUDA(cudaMemcpyAsync(out, dout, es(out_type) * n, cudaMemcpyDeviceToHost, st));
    if (mask) PK_CUDA(cudaMemcpyAsync(mask, dmask, n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    return PK_OK;
}
