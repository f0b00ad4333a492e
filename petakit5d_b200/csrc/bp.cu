// Backprojector generation at PSF size:
//   pk_omw_backprojector  -- omw_backprojector_generation.m:1-166 (OTF-masked Wiener)
//   pk_backprojector      -- third_parties/WBDeconvolution/BackProjector.m:67-233 (every bp_type;
//                            pk_wb_backprojector is its 'wiener-butterworth' form)
//
// Device work: float64 PSF normalisation sum, float64 direct DFTs along each axis (any length),
// |OTF|, the descending sort + sequential float64 cumulative sum of the OTF threshold search,
// the K=2 nearest-edge search of the star distance, the Wiener / window products, and the binary
// openings / closings / erosion of the OTF mask (psfvol.cu).  Host work (a few hundred thousand
// voxels, once per PSF): connected components, the per-slice convex hulls and the mask edge list.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

// ------------------------------------------------------------------ device kernels
__global__ void k_sum_f32_to_f64(const float* __restrict__ a, long long n, double* out) {
    __shared__ double s[256];
    double v = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) v += (double)a[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// p = float(psf / sum) (float64 divide), then circshift(-floor(psz/2)) into a complex128 array
__global__ void k_norm_shift(const float* __restrict__ psf, const double* __restrict__ sum, int ny, int nx, int nz,
                             float* __restrict__ pnorm, double2* __restrict__ shifted) {
    const long long n = (long long)ny * nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = (float)((double)psf[i] / *sum);
        pnorm[i] = v;
        const int y = (int)(i % ny), x = (int)((i / ny) % nx), z = (int)(i / ((long long)ny * nx));
        int ty = y - ny / 2; if (ty < 0) ty += ny;
        int tx = x - nx / 2; if (tx < 0) tx += nx;
        int tz = z - nz / 2; if (tz < 0) tz += nz;
        shifted[ty + (long long)ny * (tx + (long long)nx * tz)] = make_double2((double)v, 0.0);
    }
}

// direct DFT along one axis: out[..k..] = sum_j in[..j..] * tw[(j*k) mod n]; tw = exp(sign 2 pi i m / n)
__global__ void k_dft_axis(const double2* __restrict__ in, double2* __restrict__ out, int ny, int nx, int nz, int axis,
                           const double2* __restrict__ tw) {
    const long long N = (long long)ny * nx * nz;
    const int n = axis == 0 ? ny : axis == 1 ? nx : nz;
    const long long stride = axis == 0 ? 1 : axis == 1 ? ny : (long long)ny * nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((i / stride) % n);
        const long long base = i - (long long)k * stride;
        double re = 0.0, im = 0.0;
        int e = 0;
        for (int j = 0; j < n; j++) {
            const double2 a = in[base + (long long)j * stride];
            const double2 w = tw[e];
            re += a.x * w.x - a.y * w.y;
            im += a.x * w.y + a.y * w.x;
            e += k;
            if (e >= n) e -= n;
        }
        out[i] = make_double2(re, im);
    }
}

// OTF rounded to complex64 and |OTF| = float(sqrt(re^2 + im^2)) from the rounded parts (float64 math)
__global__ void k_round_abs(const double2* __restrict__ O, long long n, float2* __restrict__ O32, float* __restrict__ absO) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float re = (float)O[i].x, im = (float)O[i].y;
        O32[i] = make_float2(re, im);
        const double r = (double)re, q = (double)im;
        absO[i] = (float)sqrt(__dadd_rn(__dmul_rn(r, r), __dmul_rn(q, q)));
    }
}

// sequential float64 cumulative sum over the descending sort (omw_backprojector_generation.m:35-41)
__global__ void k_cum_threshold(const float* __restrict__ sorted_desc, long long n, double thresh, const float* __restrict__ abs0,
                                double min_int, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double total = 0.0;
    for (long long i = 0; i < n; i++) total += (double)sorted_desc[i];
    const double target = total * thresh;
    double cs = 0.0;
    long long tind = n - 1;
    for (long long i = 0; i < n; i++) {
        cs += (double)sorted_desc[i];
        if (cs > target) { tind = i; break; }
    }
    double dc = (double)sorted_desc[tind] / (double)(*abs0);
    if (dc < min_int) dc = min_int;
    out[0] = dc;
    out[1] = (double)tind;
    out[2] = total;
}

// K = 2 nearest edge directions for every voxel direction; ties go to the lower edge index
__global__ void k_knn2(const double3* __restrict__ Q, long long nq, const double3* __restrict__ E, int ne,
                       int2* __restrict__ inds, double2* __restrict__ dmat) {
    extern __shared__ double3 tile[];
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double3 p = make_double3(0, 0, 0);
    if (q < nq) p = Q[q];
    double b1 = INFINITY, b2 = INFINITY;
    int i1 = 0, i2 = 0;
    for (int t0 = 0; t0 < ne; t0 += blockDim.x) {
        const int cnt = min((int)blockDim.x, ne - t0);
        __syncthreads();
        if ((int)threadIdx.x < cnt) tile[threadIdx.x] = E[t0 + threadIdx.x];
        __syncthreads();
        for (int j = 0; j < cnt; j++) {
            const double3 e = tile[j];
            const double dy = __dsub_rn(p.x, e.x), dx = __dsub_rn(p.y, e.y), dz = __dsub_rn(p.z, e.z);
            const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dy, dy), __dmul_rn(dx, dx)), __dmul_rn(dz, dz));
            if (d2 < b1) { b2 = b1; i2 = i1; b1 = d2; i1 = t0 + j; }
            else if (d2 < b2) { b2 = d2; i2 = t0 + j; }
        }
    }
    if (q < nq) {
        inds[q] = make_int2(i1, i2);
        dmat[q] = make_double2(sqrt(b1), sqrt(b2));
    }
}

// rn, bw_dist and the cos^2 window (omw_backprojector_generation.m:136-148), column-major voxel order
__global__ void k_star_window(const int2* __restrict__ inds, const double2* __restrict__ dmat, const double* __restrict__ Rn,
                              const double* __restrict__ rs, long long nq, double l, double u, double* __restrict__ win) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq; q += (long long)gridDim.x * blockDim.x) {
        const int2 id = inds[q];
        const double d1 = dmat[id.x].x;   // d_mat(inds(:,1), 1): rows indexed by edge indices, as the reference does
        const double d2 = dmat[id.y].y;
        const double rn = __ddiv_rn(__dadd_rn(__dmul_rn(Rn[id.x], d2), __dmul_rn(Rn[id.y], d1)), __dadd_rn(d1, d2));
        const double x = __ddiv_rn(rs[q], rn);
        const double c = cos(__ddiv_rn(__ddiv_rn(__dmul_rn(M_PI, __dsub_rn(x, l)), 2.0), __dsub_rn(u, l)));
        const double lt = (x < l) ? 1.0 : 0.0;
        const double band = (x >= l && x < u) ? 1.0 : 0.0;
        win[q] = __dadd_rn(lt, __dmul_rn(__dmul_rn(c, c), band));
    }
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    if (g > 148LL * 16) g = 148LL * 16;
    return (int)std::max(1LL, g);
}

// ------------------------------------------------------------------ host helpers
struct Dims {
    int ny, nx, nz;
    long long n() const { return (long long)ny * nx * nz; }
    long long at(int y, int x, int z) const { return y + (long long)ny * (x + (long long)nx * z); }
};

// 3D DFT in place (through a ping-pong buffer) on the device; sign -1 forward, +1 inverse (unnormalised)
pk_status dft3(const Dims& D, double2* a, double2* tmp, int sign, cudaStream_t st) {
    const int ns[3] = {D.ny, D.nx, D.nz};
    double2* src = a;
    double2* dst = tmp;
    for (int ax = 0; ax < 3; ax++) {
        std::vector<double2> tw = pk_twiddles64(ns[ax], sign);
        double2* dtw;
        PK_CUDA(cudaMallocAsync(&dtw, sizeof(double2) * tw.size(), st));
        PK_CUDA(cudaMemcpyAsync(dtw, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice, st));
        k_dft_axis<<<grid_for(D.n()), 256, 0, st>>>(src, dst, D.ny, D.nx, D.nz, ax, dtw);
        PK_CUDA(cudaGetLastError());
        PK_CUDA(cudaStreamSynchronize(st));   // tw is a host temporary
        PK_CUDA(cudaFreeAsync(dtw, st));
        std::swap(src, dst);
    }
    if (src != a) PK_CUDA(cudaMemcpyAsync(a, src, sizeof(double2) * D.n(), cudaMemcpyDeviceToDevice, st));
    return PK_OK;
}

// fftshift / ifftshift index maps (column-major): shift each axis by floor(n/2) / -floor(n/2)
template <typename T>
std::vector<T> shift3(const std::vector<T>& a, const Dims& D, bool inverse) {
    std::vector<T> o(a.size());
    for (int z = 0; z < D.nz; z++)
        for (int x = 0; x < D.nx; x++)
            for (int y = 0; y < D.ny; y++) {
                int ty, tx, tz;
                if (!inverse) {
                    ty = (y + D.ny / 2) % D.ny; tx = (x + D.nx / 2) % D.nx; tz = (z + D.nz / 2) % D.nz;
                } else {
                    ty = (y - D.ny / 2 + D.ny) % D.ny; tx = (x - D.nx / 2 + D.nx) % D.nx; tz = (z - D.nz / 2 + D.nz) % D.nz;
                }
                o[D.at(ty, tx, tz)] = a[D.at(y, x, z)];
            }
    return o;
}

// 26-connected components numbered by their first voxel in column-major order (1..n)
int label26(const std::vector<uint8_t>& m, const Dims& D, std::vector<int>& lab, std::vector<long long>& sizes) {
    return pk_label26(m.data(), D.ny, D.nx, D.nz, lab, sizes);
}

std::vector<uint8_t> bwareaopen(const std::vector<uint8_t>& m, const Dims& D, double P) {
    std::vector<int> lab;
    std::vector<long long> sz;
    label26(m, D, lab, sz);
    std::vector<uint8_t> o(m.size(), 0);
    for (long long i = 0; i < D.n(); i++) o[i] = lab[i] && (double)sz[lab[i]] >= P;
    return o;
}

// 2D 8-connected component count
int count8(const std::vector<uint8_t>& img, int h, int w) {
    std::vector<int> lab(img.size(), 0);
    int n = 0;
    std::vector<int> st;
    for (int i = 0; i < h * w; i++) {
        if (!img[i] || lab[i]) continue;
        lab[i] = ++n;
        st.push_back(i);
        while (!st.empty()) {
            const int v = st.back();
            st.pop_back();
            const int r = v % h, c = v / h;
            for (int dc = -1; dc <= 1; dc++)
                for (int dr = -1; dr <= 1; dr++) {
                    const int rr = r + dr, cc = c + dc;
                    if (rr < 0 || rr >= h || cc < 0 || cc >= w) continue;
                    const int u = rr + h * cc;
                    if (img[u] && !lab[u]) { lab[u] = n; st.push_back(u); }
                }
        }
    }
    return n;
}

// bwconvhull(img, 'union'): hull of the pixel corners, pixels with centre inside or on the hull set.
// img is h x w (column-major); coordinates are doubled so corners and centres are integers.
void convhull_fill(std::vector<uint8_t>& img, int h, int w) {
    std::vector<std::pair<long long, long long>> pts;
    int r0 = h, r1 = -1, c0 = w, c1 = -1;
    for (int c = 0; c < w; c++)
        for (int r = 0; r < h; r++)
            if (img[r + (long long)h * c]) {
                for (int da = -1; da <= 1; da += 2)
                    for (int db = -1; db <= 1; db += 2) pts.push_back({2LL * r + da, 2LL * c + db});
                r0 = std::min(r0, r); r1 = std::max(r1, r); c0 = std::min(c0, c); c1 = std::max(c1, c);
            }
    if (pts.empty()) return;
    std::sort(pts.begin(), pts.end());
    pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
    auto cross = [](const std::pair<long long, long long>& o, const std::pair<long long, long long>& a,
                    const std::pair<long long, long long>& b) {
        return (a.first - o.first) * (b.second - o.second) - (a.second - o.second) * (b.first - o.first);
    };
    std::vector<std::pair<long long, long long>> lower, upper;
    for (auto& p : pts) {
        while (lower.size() >= 2 && cross(lower[lower.size() - 2], lower.back(), p) <= 0) lower.pop_back();
        lower.push_back(p);
    }
    for (auto it = pts.rbegin(); it != pts.rend(); ++it) {
        while (upper.size() >= 2 && cross(upper[upper.size() - 2], upper.back(), *it) <= 0) upper.pop_back();
        upper.push_back(*it);
    }
    std::vector<std::pair<long long, long long>> hull(lower.begin(), lower.end() - 1);
    hull.insert(hull.end(), upper.begin(), upper.end() - 1);
    const size_t m = hull.size();
    for (int c = c0; c <= c1; c++)
        for (int r = r0; r <= r1; r++) {
            const long long X = 2LL * r, Y = 2LL * c;
            bool in = true;
            for (size_t k = 0; k < m && in; k++) {
                const auto& o = hull[k];
                const auto& a = hull[(k + 1) % m];
                if ((a.first - o.first) * (Y - o.second) - (a.second - o.second) * (X - o.first) < 0) in = false;
            }
            if (in) img[r + (long long)h * c] = 1;
        }
}

// Threshold .. convex hulls of omw_backprojector_generation.m:43-109 on the host.
pk_status omw_mask_host(const std::vector<float>& abs_c, const Dims& D0, float abs0, double dc, int skewed_in,
                        double area, std::vector<uint8_t>& mask, Dims& D, int& skewed, cudaStream_t st) {
    D = D0;
    const float thr = abs0 * (float)dc;
    mask.assign(D.n(), 0);
    for (long long i = 0; i < D.n(); i++) mask[i] = abs_c[i] > thr;
    const std::vector<int4> ball2 = pk_ball_offsets(2);
    pk_status s;
    if ((s = pk_morph_host(mask, D.ny, D.nx, D.nz, ball2, "ed", st)) != PK_OK) return s;     // imopen (GPU)
    mask = bwareaopen(mask, D, area);
    if ((s = pk_morph_host(mask, D.ny, D.nx, D.nz, ball2, "deed", st)) != PK_OK) return s;   // imclose, imopen
    mask = bwareaopen(mask, D, area);
    if (std::find(mask.begin(), mask.end(), 1) == mask.end())
        return pk_fail(PK_ERR_EMPTY_OTF_MASK, "The OTF mask is empty, check the PSF and OTF-related parameters!");
    skewed = skewed_in;
    if (skewed < 0) {                                      // :57-71 auto-detection
        skewed = 0;
        std::vector<uint8_t> xz((size_t)D.nx * D.nz, 0);
        for (int z = 0; z < D.nz; z++)
            for (int x = 0; x < D.nx; x++)
                for (int y = 0; y < D.ny; y++)
                    if (mask[D.at(y, x, z)]) xz[x + (size_t)D.nx * z] = 1;
        if (count8(xz, D.nx, D.nz) > 1) {
            std::vector<int> line(D.nz, 0);
            for (int z = 0; z < D.nz; z++)
                for (int x = 0; x < D.nx; x++) line[z] += xz[x + (size_t)D.nx * z];
            const int pind = (int)(std::max_element(line.begin(), line.end()) - line.begin()) + 1;
            bool all = true;
            for (int v : line) all = all && v > 0;
            if (all && std::fabs(pind - (D.nz + 1) / 2.0) > 1) skewed = 1;
        }
    }
    std::vector<int> lab;
    std::vector<long long> sz;
    int n = label26(mask, D, lab, sz);
    if (skewed) {                                          // :73-88
        if (n + 1 > 4) {
            std::vector<int> order(n);
            std::iota(order.begin(), order.end(), 1);
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sz[a] > sz[b]; });
            std::vector<uint8_t> keep(n + 1, 0);
            for (int i = 0; i < 3; i++) keep[order[i]] = 1;
            for (long long i = 0; i < D.n(); i++) mask[i] = lab[i] && keep[lab[i]];
            n = label26(mask, D, lab, sz);
        } else if (n + 1 == 2) {
            for (long long i = 0; i < D.n(); i++) lab[i] = (lab[i] + 1) * (mask[i] ? 1 : 0);
        }
        Dims D3{D.ny, D.nx, 3 * D.nz};
        std::vector<uint8_t> m3(D3.n(), 0);
        const int part_label[3] = {3, 2, 1};               // cat(3, OTF_mask_r, OTF_mask_c, OTF_mask_l)
        for (int p = 0; p < 3; p++)
            for (int z = 0; z < D.nz; z++)
                for (int x = 0; x < D.nx; x++)
                    for (int y = 0; y < D.ny; y++)
                        m3[D3.at(y, x, z + p * D.nz)] = lab[D.at(y, x, z)] == part_label[p];
        mask.swap(m3);
        D = D3;
    } else {                                               // :89-94
        int best = 1;
        for (int i = 2; i <= n; i++)
            if (sz[i] > sz[best]) best = i;
        for (long long i = 0; i < D.n(); i++) mask[i] = lab[i] == best;
    }
    // per-slice convex hulls in z, y, x (slice lists taken before any hull, :98-100)
    std::vector<uint8_t> hz(D.nz, 0), hy(D.ny, 0), hx(D.nx, 0);
    for (int z = 0; z < D.nz; z++)
        for (int x = 0; x < D.nx; x++)
            for (int y = 0; y < D.ny; y++)
                if (mask[D.at(y, x, z)]) { hz[z] = 1; hy[y] = 1; hx[x] = 1; }
    std::vector<uint8_t> sl;
    for (int z = 0; z < D.nz; z++) {
        if (!hz[z]) continue;
        sl.assign((size_t)D.ny * D.nx, 0);
        for (int x = 0; x < D.nx; x++)
            for (int y = 0; y < D.ny; y++) sl[y + (size_t)D.ny * x] = mask[D.at(y, x, z)];
        convhull_fill(sl, D.ny, D.nx);
        for (int x = 0; x < D.nx; x++)
            for (int y = 0; y < D.ny; y++) mask[D.at(y, x, z)] = sl[y + (size_t)D.ny * x];
    }
    for (int y = 0; y < D.ny; y++) {
        if (!hy[y]) continue;
        sl.assign((size_t)D.nx * D.nz, 0);
        for (int z = 0; z < D.nz; z++)
            for (int x = 0; x < D.nx; x++) sl[x + (size_t)D.nx * z] = mask[D.at(y, x, z)];
        convhull_fill(sl, D.nx, D.nz);
        for (int z = 0; z < D.nz; z++)
            for (int x = 0; x < D.nx; x++) mask[D.at(y, x, z)] = sl[x + (size_t)D.nx * z];
    }
    for (int x = 0; x < D.nx; x++) {
        if (!hx[x]) continue;
        sl.assign((size_t)D.ny * D.nz, 0);
        for (int z = 0; z < D.nz; z++)
            for (int y = 0; y < D.ny; y++) sl[y + (size_t)D.ny * z] = mask[D.at(y, x, z)];
        convhull_fill(sl, D.ny, D.nz);
        for (int z = 0; z < D.nz; z++)
            for (int y = 0; y < D.ny; y++) mask[D.at(y, x, z)] = sl[y + (size_t)D.ny * z];
    }
    return PK_OK;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    template <typename T> T* as() { return (T*)p; }
};

pk_status dalloc(DevBuf& b, size_t bytes) {
    cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) { cudaGetLastError(); return pk_fail(PK_ERR_NOMEM, "backprojector: device allocation failed"); }
    return PK_OK;
}

}  // namespace

extern "C" {

pk_status pk_omw_backprojector(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], double alpha, int32_t skewed,
                               double otf_cum_thresh, double otf_area_thresh, double hann_lo, double hann_hi,
                               double min_int_thresh, float* b_omw, float* otf_bp_omw, float* abs_otf_c,
                               uint8_t* otf_mask) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!psf || !psf_dims || !b_omw) return pk_fail(PK_ERR_INVALID, "NULL psf/output");
    if (psf_dims[0] < 1 || psf_dims[1] < 1 || psf_dims[2] < 1)
        return pk_fail(PK_ERR_INVALID, "A valid nonzero PSF needs to be provided!");
    const Dims D0{(int)psf_dims[0], (int)psf_dims[1], (int)psf_dims[2]};
    const long long n = D0.n();
    bool any = false;
    for (long long i = 0; i < n && !any; i++) any = psf[i] != 0.f;
    if (!any) return pk_fail(PK_ERR_INVALID, "A valid nonzero PSF needs to be provided!");   // :25-27
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    pk_status s;
    DevBuf dpsf, dsum, dp, dO, dT, dO32, dabs, dsorted, dtmp, dthr;
    if ((s = dalloc(dpsf, 4 * n)) || (s = dalloc(dsum, 8)) || (s = dalloc(dp, 4 * n)) || (s = dalloc(dO, 16 * n)) ||
        (s = dalloc(dT, 16 * n)) || (s = dalloc(dO32, 8 * n)) || (s = dalloc(dabs, 4 * n)) || (s = dalloc(dsorted, 4 * n)) ||
        (s = dalloc(dthr, 32)))
        return s;
    PK_CUDA(cudaMemcpyAsync(dpsf.p, psf, 4 * n, cudaMemcpyHostToDevice, st));
    k_sum_f32_to_f64<<<1, 256, 0, st>>>(dpsf.as<float>(), n, dsum.as<double>());          // :29-30 (float64 sum)
    k_norm_shift<<<grid_for(n), 256, 0, st>>>(dpsf.as<float>(), dsum.as<double>(), D0.ny, D0.nx, D0.nz,
                                              dp.as<float>(), dO.as<double2>());
    PK_CUDA(cudaGetLastError());
    if ((s = dft3(D0, dO.as<double2>(), dT.as<double2>(), -1, st)) != PK_OK) return s;       // :32 OTF = fftn
    k_round_abs<<<grid_for(n), 256, 0, st>>>(dO.as<double2>(), n, dO32.as<float2>(), dabs.as<float>());
    // descending sort of |OTF| (non-negative floats sort as their bit patterns) + cumulative threshold
    size_t tmpb = 0;
    cub::DeviceRadixSort::SortKeysDescending(nullptr, tmpb, dabs.as<float>(), dsorted.as<float>(), (int)n, 0, 32, st);
    if ((s = dalloc(dtmp, tmpb)) != PK_OK) return s;
    cub::DeviceRadixSort::SortKeysDescending(dtmp.p, tmpb, dabs.as<float>(), dsorted.as<float>(), (int)n, 0, 32, st);
    k_cum_threshold<<<1, 1, 0, st>>>(dsorted.as<float>(), n, otf_cum_thresh, dabs.as<float>(), min_int_thresh,
                                     dthr.as<double>());
    PK_CUDA(cudaGetLastError());
    std::vector<float> absO(n);
    std::vector<float2> O32(n);
    double thr[3];
    PK_CUDA(cudaMemcpyAsync(absO.data(), dabs.p, 4 * n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaMemcpyAsync(O32.data(), dO32.p, 8 * n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaMemcpyAsync(thr, dthr.p, sizeof(thr), cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    const std::vector<float> abs_c = shift3(absO, D0, false);                               // :34 fftshift
    if (abs_otf_c) memcpy(abs_otf_c, abs_c.data(), 4 * n);
    std::vector<uint8_t> mask;
    Dims D;
    int sk = 0;
    if ((s = omw_mask_host(abs_c, D0, absO[0], thr[0], skewed, otf_area_thresh, mask, D, sk, st)) != PK_OK) return s;
    // edge = mask & ~imerode(mask, sphere(1)) (:122) and the star geometry (:123-133)
    std::vector<uint8_t> er = mask;
    if ((s = pk_morph_host(er, D.ny, D.nx, D.nz, pk_ball_offsets(1), "e", st)) != PK_OK) return s;
    const long long nq = D.n();
    std::vector<double3> Q(nq), E;
    std::vector<double> rs(nq), Rn;
    const double cy = (D.ny + 1) / 2.0, cx = (D.nx + 1) / 2.0, cz = (D.nz + 1) / 2.0;
    for (int z = 0; z < D.nz; z++)
        for (int x = 0; x < D.nx; x++)
            for (int y = 0; y < D.ny; y++) {
                const long long i = D.at(y, x, z);
                const double Y = (y + 1) - cy, X = (x + 1) - cx, Z = (z + 1) - cz;
                const double r = std::sqrt((X * X + Y * Y) + Z * Z);
                rs[i] = r;
                Q[i] = r > 0 ? make_double3(Y / r, X / r, Z / r) : make_double3(0.0, 1.0, 0.0);
                if (mask[i] && !er[i]) {
                    E.push_back(Q[i]);
                    Rn.push_back(r);
                }
            }
    if (E.size() < 2) return pk_fail(PK_ERR_EMPTY_OTF_MASK, "The OTF mask edge has fewer than two voxels");
    DevBuf dQ, dE, dI, dD, dRn, drs, dwin;
    if ((s = dalloc(dQ, sizeof(double3) * nq)) || (s = dalloc(dE, sizeof(double3) * E.size())) ||
        (s = dalloc(dI, sizeof(int2) * nq)) || (s = dalloc(dD, sizeof(double2) * nq)) ||
        (s = dalloc(dRn, 8 * Rn.size())) || (s = dalloc(drs, 8 * nq)) || (s = dalloc(dwin, 8 * nq)))
        return s;
    PK_CUDA(cudaMemcpyAsync(dQ.p, Q.data(), sizeof(double3) * nq, cudaMemcpyHostToDevice, st));
    PK_CUDA(cudaMemcpyAsync(dE.p, E.data(), sizeof(double3) * E.size(), cudaMemcpyHostToDevice, st));
    PK_CUDA(cudaMemcpyAsync(dRn.p, Rn.data(), 8 * Rn.size(), cudaMemcpyHostToDevice, st));
    PK_CUDA(cudaMemcpyAsync(drs.p, rs.data(), 8 * nq, cudaMemcpyHostToDevice, st));
    k_knn2<<<(int)((nq + 127) / 128), 128, 128 * sizeof(double3), st>>>(dQ.as<double3>(), nq, dE.as<double3>(),
                                                                          (int)E.size(), dI.as<int2>(), dD.as<double2>());
    k_star_window<<<grid_for(nq), 256, 0, st>>>(dI.as<int2>(), dD.as<double2>(), dRn.as<double>(), drs.as<double>(), nq,
                                                hann_lo, hann_hi, dwin.as<double>());
    PK_CUDA(cudaGetLastError());
    std::vector<double> win(nq);
    PK_CUDA(cudaMemcpyAsync(win.data(), dwin.p, 8 * nq, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    if (sk) {                                              // :150-153 fold the three parts back
        std::vector<double> w0(n, 0.0);
        std::vector<uint8_t> m0(n, 0);
        for (int p = 0; p < 3; p++)
            for (int z = 0; z < D0.nz; z++)
                for (int x = 0; x < D0.nx; x++)
                    for (int y = 0; y < D0.ny; y++) {
                        const long long i0 = D0.at(y, x, z), i3 = D.at(y, x, z + p * D0.nz);
                        w0[i0] += win[i3];
                        m0[i0] = (uint8_t)(m0[i0] + mask[i3]);
                    }
        win.swap(w0);
        mask.swap(m0);
    }
    if (otf_mask) memcpy(otf_mask, mask.data(), n);
    // OTF_bp_omw = single(ifftshift(mask)) .* conj(OTF) ./ (|OTF|.^2 + alpha)  (:155-161)
    const std::vector<double> om = shift3(win, D0, true);
    std::vector<double2> omw(n);
    std::vector<float2> omw32(n);
    const float af = (float)alpha;
    for (long long i = 0; i < n; i++) {
        const float a = absO[i];
        const float den = a * a + af;
        const float wr = O32[i].x / den, wi = -O32[i].y / den;
        const float m = (float)om[i];
        omw32[i] = make_float2(m * wr, m * wi);
        omw[i] = make_double2((double)omw32[i].x, (double)omw32[i].y);
    }
    if (otf_bp_omw) memcpy(otf_bp_omw, omw32.data(), 8 * n);
    // b_omw = fftshift(real(ifftn(OTF_bp_omw)))  (:163)
    PK_CUDA(cudaMemcpyAsync(dO.p, omw.data(), 16 * n, cudaMemcpyHostToDevice, st));
    if ((s = dft3(D0, dO.as<double2>(), dT.as<double2>(), +1, st)) != PK_OK) return s;
    std::vector<double2> res(n);
    PK_CUDA(cudaMemcpyAsync(res.data(), dO.p, 16 * n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    std::vector<float> b(n);
    for (long long i = 0; i < n; i++) b[i] = (float)(res[i].x / (double)n);
    const std::vector<float> bs = shift3(b, D0, false);
    memcpy(b_omw, bs.data(), 4 * n);
    return PK_OK;
}

}  // extern "C"

namespace {

int sgnf(float v) { return v > 0.f ? 1 : (v < 0.f ? -1 : 0); }

long long mround(double v) { return v >= 0 ? (long long)std::floor(v + 0.5) : (long long)std::ceil(v - 0.5); }

// fwhm (BackProjector.m:443-483) in single precision, x = 1..N; NaN when there is no trailing edge
bool fwhm_line(std::vector<float> y, float* out) {
    const int N = (int)y.size();
    if (N < 2) { *out = NAN; return true; }
    float mx = y[0];
    for (float v : y) mx = std::max(mx, v);
    for (float& v : y) v = v / mx;
    const float lev = 0.5f;
    int center;
    if (y[0] < lev) center = (int)(std::max_element(y.begin(), y.end()) - y.begin());
    else center = (int)(std::min_element(y.begin(), y.end()) - y.begin());
    int i = 1;
    while (i < N && sgnf(y[i] - lev) == sgnf(y[i - 1] - lev)) i++;
    if (i >= N) return false;                     // no leading crossing (MATLAB indexes past the end)
    float interp = (lev - y[i - 1]) / (y[i] - y[i - 1]);
    const float tlead = (float)i + interp * 1.0f;
    i = center + 1;
    if (i >= N) { *out = NAN; return true; }
    while (sgnf(y[i] - lev) == sgnf(y[i - 1] - lev) && i <= N - 2) i++;
    if (i != N - 1) {
        interp = (lev - y[i - 1]) / (y[i] - y[i - 1]);
        const float ttrail = (float)i + interp * 1.0f;
        *out = ttrail - tlead;
    } else {
        *out = NAN;
    }
    return true;
}

}  // namespace

extern "C" {

pk_status pk_backprojector(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], int32_t bp_type, double alpha,
                           double beta, int32_t nord, int32_t res_flag, const double ires[3], double* psf_bp,
                           double* otf_bp) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!psf || !psf_dims || !psf_bp) return pk_fail(PK_ERR_INVALID, "NULL psf/output");
    if (bp_type < PK_BP_TRADITIONAL || bp_type > PK_BP_WIENER_BUTTERWORTH)
        return pk_fail(PK_ERR_INVALID, "bp_type does not match any back-projector type");
    if (psf_dims[0] < 2 || psf_dims[1] < 2 || psf_dims[2] < 2) return pk_fail(PK_ERR_INVALID, "PSF must be 3D");
    if (res_flag < 0 || res_flag > 2) return pk_fail(PK_ERR_INVALID, "Processing terminated, please set resFlag as 0, 1, or 2");
    const Dims D{(int)psf_dims[0], (int)psf_dims[1], (int)psf_dims[2]};
    const long long n = D.n();
    const int Sx = D.ny, Sy = D.nx, Sz = D.nz;   // the reference names MATLAB dims 1..3 x, y, z
    const double Scx = (Sx + 1) / 2.0, Scy = (Sy + 1) / 2.0, Scz = (Sz + 1) / 2.0;
    const int Soz = (int)mround((Sz + 1) / 2.0);
    // FWHM through the maximum (fwhm_PSF, cFlag = 0, fitFlag = 0)
    long long imax = 0;
    for (long long i = 1; i < n; i++)
        if (psf[i] > psf[imax]) imax = i;
    const int ix = (int)(imax % Sx), iy = (int)((imax / Sx) % Sy), iz = (int)(imax / ((long long)Sx * Sy));
    std::vector<float> lx(Sx), ly(Sy), lz(Sz);
    for (int i = 0; i < Sx; i++) lx[i] = psf[D.at(i, iy, iz)];
    for (int j = 0; j < Sy; j++) ly[j] = psf[D.at(ix, j, iz)];
    for (int k = 0; k < Sz; k++) lz[k] = psf[D.at(ix, iy, k)];
    float Fx, Fy, Fz;
    if (!fwhm_line(lx, &Fx) || !fwhm_line(ly, &Fy) || !fwhm_line(lz, &Fz))
        return pk_fail(PK_ERR_INVALID, "PSF profile has no half-maximum crossing (fwhm)");
    float rx, ry, rz;
    if (res_flag == 0) {
        const float s2 = (float)std::sqrt(2.0);
        rx = Fx / s2; ry = Fy / s2; rz = Fz / s2;
    } else if (res_flag == 1) {
        rx = Fx; ry = Fy; rz = Fz;
    } else {
        if (!ires) return pk_fail(PK_ERR_INVALID, "iRes required for resFlag 2");
        rx = (float)ires[0]; ry = (float)ires[1]; rz = (float)ires[2];
    }
    const float tx = (1.0f / rx) / (float)(1.0 / Sx), ty = (1.0f / ry) / (float)(1.0 / Sy), tz = (1.0f / rz) / (float)(1.0 / Sz);
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    pk_status s;
    // OTF_flip = fftn(ifftshift(flipPSF(PSF)))  (float64)
    std::vector<double> flipped(n);
    for (int k = 0; k < Sz; k++)
        for (int j = 0; j < Sy; j++)
            for (int i = 0; i < Sx; i++) flipped[D.at(i, j, k)] = (double)psf[D.at(Sx - 1 - i, Sy - 1 - j, Sz - 1 - k)];
    const std::vector<double> fs = shift3(flipped, D, true);
    std::vector<double2> a(n);
    for (long long i = 0; i < n; i++) a[i] = make_double2(fs[i], 0.0);
    DevBuf dA, dT;
    if ((s = dalloc(dA, 16 * n)) || (s = dalloc(dT, 16 * n))) return s;
    PK_CUDA(cudaMemcpyAsync(dA.p, a.data(), 16 * n, cudaMemcpyHostToDevice, st));
    if ((s = dft3(D, dA.as<double2>(), dT.as<double2>(), -1, st)) != PK_OK) return s;
    std::vector<double2> F(n);
    PK_CUDA(cudaMemcpyAsync(F.data(), dA.p, 16 * n, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    std::vector<double> absF(n);
    for (long long i = 0; i < n; i++) absF[i] = std::hypot(F[i].x, F[i].y);
    const std::vector<double> Fabs = shift3(absF, D, false);
    double Mx = Fabs[0];
    for (double v : Fabs) Mx = std::max(Mx, v);
    if (alpha == 1 || beta == 1) {                          // BackProjector.m:114-156
        std::vector<double> t1(Sx, -INFINITY), t2(Sy, -INFINITY), t3(Sz, -INFINITY);
        for (int k = 0; k < Sz; k++)
            for (int j = 0; j < Sy; j++)
                for (int i = 0; i < Sx; i++) {
                    const double v = Fabs[D.at(i, j, k)] / Mx;
                    t1[i] = std::max(t1[i], v);
                    t2[j] = std::max(t2[j], v);
                    t3[k] = std::max(t3[k], v);
                }
        auto cut = [](const std::vector<double>& t, double c, float tt, int S) {
            const long long o1 = std::max(mround((double)((float)c - tt)), 1LL);
            const long long o2 = std::min(mround((double)((float)c + tt)), (long long)S);
            return (t[o1 - 1] + t[o2 - 1]) / 2;
        };
        const double bfp = (cut(t1, Scx, tx, Sx) + cut(t2, Scy, ty, Sy) + cut(t3, Scz, tz, Sz)) / 3;
        if (alpha == 1) alpha = bfp;
        if (beta == 1) beta = bfp;
    }
    // PSF_bp = fftshift(real(ifftn(OTF_bp))) of the OTF in `a` (:174, 187, 191, 230)
    auto psf_of_otf = [&]() -> pk_status {
        PK_CUDA(cudaMemcpyAsync(dA.p, a.data(), 16 * n, cudaMemcpyHostToDevice, st));
        pk_status r = dft3(D, dA.as<double2>(), dT.as<double2>(), +1, st);
        if (r != PK_OK) return r;
        PK_CUDA(cudaMemcpyAsync(F.data(), dA.p, 16 * n, cudaMemcpyDeviceToHost, st));
        PK_CUDA(cudaStreamSynchronize(st));
        std::vector<double> re(n);
        for (long long i = 0; i < n; i++) re[i] = F[i].x / (double)n;
        const std::vector<double> out = shift3(re, D, false);
        memcpy(psf_bp, out.data(), 8 * n);
        return PK_OK;
    };
    // Butterworth mask 1/sqrt(1 + ee w^n), w = ((i-Scx)/kcx)^2 + ... in single precision (ee meets the
    // single-precision w, so the product is single) (:178-186, :214-227), as ifftshift(mask)
    auto butterworth = [&](double ee) {
        std::vector<double> mask(n);
        const float eef = (float)ee;
        for (int k = 0; k < Sz; k++)
            for (int j = 0; j < Sy; j++)
                for (int i = 0; i < Sx; i++) {
                    const float aa = ((float)(i + 1) - (float)Scx) / tx;
                    const float bb = ((float)(j + 1) - (float)Scy) / ty;
                    const float cc = ((float)(k + 1) - (float)Scz) / tz;
                    const float w = (aa * aa + bb * bb) + cc * cc;
                    const float wn = (float)std::pow((double)w, (double)nord);
                    mask[D.at(i, j, k)] = (double)(1.0f / std::sqrt(1.0f + eef * wn));
                }
        return shift3(mask, D, true);
    };
    if (bp_type == PK_BP_TRADITIONAL) {   // PSF_bp = flipPSF(PSF_fp), OTF_bp = fftn(ifftshift(PSF_bp)) (:164-166)
        if (otf_bp) memcpy(otf_bp, F.data(), 16 * n);
        memcpy(psf_bp, flipped.data(), 8 * n);
        return PK_OK;
    }
    if (bp_type == PK_BP_GAUSSIAN) {
        // gen_gaussianPSF_3D(Sx, Sy, Sz, FWHMx, FWHMy, FWHMz) (:168-171, :485-514): the FWHMs are single,
        // so sigma, the exponent and the normalisation are single-precision arithmetic and the PSF
        // is single; its OTF is a single-precision transform (here float64, rounded to single)
        const float sgx = Fx / 2.3548f, sgy = Fy / 2.3548f, sgz = Fz / 2.3548f;
        const float qx = sgx * sgx * 2.0f, qy = sgy * sgy * 2.0f, qz = sgz * sgz * 2.0f;
        const float c2pi = (float)std::pow(6.283185307179586, 1.5);   // (2 pi)^(3/2) meets single sigmas
        const float coef = 1.0f / (((c2pi * sgx) * sgy) * sgz);
        std::vector<double> g(n);
        for (int k = 0; k < Sz; k++)
            for (int j = 0; j < Sy; j++)
                for (int i = 0; i < Sx; i++) {
                    const double di = (i + 1) - Scx, dj = (j + 1) - Scy, dk = (k + 1) - Scz;
                    const float d = ((float)(di * di) / qx + (float)(dj * dj) / qy) + (float)(dk * dk) / qz;
                    g[D.at(i, j, k)] = (double)(coef * std::exp(-d));
                }
        const std::vector<double> gs = shift3(g, D, true);
        for (long long i = 0; i < n; i++) a[i] = make_double2(gs[i], 0.0);
        PK_CUDA(cudaMemcpyAsync(dA.p, a.data(), 16 * n, cudaMemcpyHostToDevice, st));
        if ((s = dft3(D, dA.as<double2>(), dT.as<double2>(), -1, st)) != PK_OK) return s;
        PK_CUDA(cudaMemcpyAsync(F.data(), dA.p, 16 * n, cudaMemcpyDeviceToHost, st));
        PK_CUDA(cudaStreamSynchronize(st));
        if (otf_bp) {
            for (long long i = 0; i < n; i++) F[i] = make_double2((double)(float)F[i].x, (double)(float)F[i].y);
            memcpy(otf_bp, F.data(), 16 * n);
        }
        memcpy(psf_bp, g.data(), 8 * n);
        return PK_OK;
    }
    if (bp_type == PK_BP_BUTTERWORTH) {   // ee = 1/beta^2 - 1; OTF_bp = ifftshift(mask) (:173-187)
        const std::vector<double> mk = butterworth(1 / (beta * beta) - 1);
        for (long long i = 0; i < n; i++) a[i] = make_double2(mk[i], 0.0);
        if (otf_bp) memcpy(otf_bp, a.data(), 16 * n);
        return psf_of_otf();
    }
    // Wiener filter of the normalised flipped OTF (:190, :202-203)
    std::vector<double2> W(n);
    std::vector<double> absW(n);
    for (long long i = 0; i < n; i++) {
        const double re = F[i].x / Mx, im = F[i].y / Mx;
        const double ab = std::hypot(re, im);
        const double den = ab * ab + alpha;
        W[i] = make_double2(re / den, im / den);
        absW[i] = std::hypot(W[i].x, W[i].y);
    }
    if (bp_type == PK_BP_WIENER) {
        a = W;
        if (otf_bp) memcpy(otf_bp, a.data(), 16 * n);
        return psf_of_otf();
    }
    // its cutoff gain on the central z slice (:205-209), then the Wiener-Butterworth product (:228)
    const std::vector<double> Wabs = shift3(absW, D, false);
    std::vector<double> tline(Sx, -INFINITY);
    for (int j = 0; j < Sy; j++)
        for (int i = 0; i < Sx; i++) tline[i] = std::max(tline[i], std::fabs(Wabs[D.at(i, j, Soz - 1)]));
    const long long to1 = std::max(mround((double)((float)Scx - tx)), 1LL);
    const long long to2 = std::min(mround((double)((float)Scx + tx)), (long long)Sx);
    const double beta_wx = (tline[to1 - 1] + tline[to2 - 1]) / 2;
    const std::vector<double> mk = butterworth(beta_wx / (beta * beta) - 1);
    for (long long i = 0; i < n; i++) a[i] = make_double2(mk[i] * W[i].x, mk[i] * W[i].y);
    if (otf_bp) memcpy(otf_bp, a.data(), 16 * n);
    return psf_of_otf();
}

pk_status pk_wb_backprojector(pk_ctx* ctx, const float* psf, const int64_t psf_dims[3], double alpha, double beta,
                              int32_t nord, int32_t res_flag, const double ires[3], double* psf_bp, double* otf_bp) {
    return pk_backprojector(ctx, psf, psf_dims, PK_BP_WIENER_BUTTERWORTH, alpha, beta, nord, res_flag, ires, psf_bp,
                            otf_bp);
}

}  // extern "C"
