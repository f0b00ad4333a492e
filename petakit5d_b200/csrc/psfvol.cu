// Helpers for the PSF-size volumes of the backprojector generation and the PSF preparation
// (a few hundred thousand voxels, once per PSF):
//   * binary dilation / erosion with an arbitrary neighbourhood on the GPU -- imdilate / imerode of
//     MATLAB's Image Processing Toolbox as called at omw_backprojector_generation.m:44-48,122 and
//     psf_gen_new.m:39,55 (dilation: voxels outside the volume count as false; erosion: as true);
//   * 26-connected component labelling on the host (bwlabeln / bwconncomp / bwareaopen, conn 26),
//     components numbered by their first voxel in column-major order;
//   * float64 DFT twiddle tables with the quarter-turn points exact.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pk_internal.h"

namespace {

__global__ void k_morph(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int ny, int nx, int nz,
                        const int4* __restrict__ offs, int noff, int erode) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % ny), x = (int)((i / ny) % nx), z = (int)(i / ((long long)ny * nx));
        bool v = erode != 0;
        for (int k = 0; k < noff; k++) {
            const int4 o = __ldg(offs + k);
            const int yy = y + o.x, xx = x + o.y, zz = z + o.z;
            bool s;
            if (yy < 0 || yy >= ny || xx < 0 || xx >= nx || zz < 0 || zz >= nz) s = erode != 0;
            else s = in[yy + (long long)ny * (xx + (long long)nx * zz)] != 0;
            if (erode) {
                if (!s) { v = false; break; }
            } else if (s) {
                v = true;
                break;
            }
        }
        out[i] = v;
    }
}

int grid_of(long long n) {
    long long g = (n + 255) / 256;
    return (int)std::max(1LL, std::min(g, 148LL * 16));
}

}  // namespace

std::vector<int4> pk_ball_offsets(int r) {
    std::vector<int4> o;
    for (int c = -r; c <= r; c++)
        for (int b = -r; b <= r; b++)
            for (int a = -r; a <= r; a++)
                if (a * a + b * b + c * c <= r * r) o.push_back(make_int4(a, b, c, 0));
    return o;
}

pk_status pk_morph_ops(uint8_t* d_a, uint8_t* d_tmp, int ny, int nx, int nz, const int4* d_offs, int noff,
                       const char* ops, cudaStream_t st) {
    const long long n = (long long)ny * nx * nz;
    for (const char* p = ops; *p; p++) {
        k_morph<<<grid_of(n), 256, 0, st>>>(d_a, d_tmp, ny, nx, nz, d_offs, noff, *p == 'e' ? 1 : 0);
        PK_CUDA(cudaGetLastError());
        PK_CUDA(cudaMemcpyAsync(d_a, d_tmp, (size_t)n, cudaMemcpyDeviceToDevice, st));
    }
    return PK_OK;
}

pk_status pk_morph_host(std::vector<uint8_t>& mask, int ny, int nx, int nz, const std::vector<int4>& offs,
                        const char* ops, cudaStream_t st) {
    const size_t n = (size_t)ny * nx * nz;
    if (mask.size() != n) return pk_fail(PK_ERR_INVALID, "morphology: mask size mismatch");
    uint8_t *d = nullptr;
    int4* dof = nullptr;
    auto done = [&](pk_status s) {
        cudaStreamSynchronize(st);
        if (d) cudaFree(d);
        if (dof) cudaFree(dof);
        return s;
    };
    if (cudaMalloc(&d, 2 * n + 16) != cudaSuccess || cudaMalloc(&dof, sizeof(int4) * std::max<size_t>(1, offs.size())) != cudaSuccess) {
        cudaGetLastError();
        return done(pk_fail(PK_ERR_NOMEM, "morphology: device allocation failed"));
    }
    if (cudaMemcpyAsync(d, mask.data(), n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dof, offs.data(), sizeof(int4) * offs.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return done(pk_fail(PK_ERR_CUDA, "morphology: upload failed"));
    pk_status s = pk_morph_ops(d, d + n, ny, nx, nz, dof, (int)offs.size(), ops, st);
    if (s != PK_OK) return done(s);
    if (cudaMemcpyAsync(mask.data(), d, n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return done(pk_fail(PK_ERR_CUDA, "morphology: download failed"));
    if (cudaStreamSynchronize(st) != cudaSuccess) return done(pk_fail(PK_ERR_CUDA, "morphology: kernel failed"));
    return done(PK_OK);
}

int pk_label26(const uint8_t* m, int ny, int nx, int nz, std::vector<int>& lab, std::vector<long long>& sizes) {
    const long long N = (long long)ny * nx * nz;
    lab.assign((size_t)N, 0);
    sizes.assign(1, 0);
    int n = 0;
    std::vector<long long> stack;
    for (long long i = 0; i < N; i++) {
        if (!m[i] || lab[i]) continue;
        n++;
        long long cnt = 0;
        lab[i] = n;
        stack.push_back(i);
        while (!stack.empty()) {
            const long long v = stack.back();
            stack.pop_back();
            cnt++;
            const int y = (int)(v % ny), x = (int)((v / ny) % nx), z = (int)(v / ((long long)ny * nx));
            for (int c = -1; c <= 1; c++)
                for (int b = -1; b <= 1; b++)
                    for (int a = -1; a <= 1; a++) {
                        const int yy = y + a, xx = x + b, zz = z + c;
                        if (yy < 0 || yy >= ny || xx < 0 || xx >= nx || zz < 0 || zz >= nz) continue;
                        const long long w = yy + (long long)ny * (xx + (long long)nx * zz);
                        if (m[w] && !lab[w]) {
                            lab[w] = n;
                            stack.push_back(w);
                        }
                    }
        }
        sizes.push_back(cnt);
    }
    return n;
}

std::vector<double2> pk_twiddles64(int n, int sign) {
    std::vector<double2> t(n);
    for (int m = 0; m < n; m++) {
        double c, s;
        if ((4LL * m) % n == 0) {
            const int q = (int)((4LL * m) / n) & 3;
            c = q == 0 ? 1 : q == 2 ? -1 : 0;
            s = q == 1 ? 1 : q == 3 ? -1 : 0;
        } else {
            const double a = 2.0 * M_PI * (double)m / (double)n;
            c = std::cos(a);
            s = std::sin(a);
        }
        t[m] = make_double2(c, sign * s);
    }
    return t;
}
