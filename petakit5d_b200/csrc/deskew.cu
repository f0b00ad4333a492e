// Combined deskew / rotate of a light-sheet volume: deskewRotateFrame3D.m:1-260 on its default
// path (linear interpolation, no resampling), whose work the reference does in two MEX files:
//   volume_deskew_rotate_warp_mex.cpp                 -- |dx| <= xStepThresh
//   skewed_space_interp_volume_deskew_rotate_warp_mex.cpp -- |dx| > xStepThresh: intermediate slices
//     interpolated in the skewed space first, then the same warp.
// Both are HBM-bound gathers.  The warp keeps the first axis (MATLAB y, contiguous) and
// interpolates bilinearly over (x, z): an output row is a weighted sum of four input rows, so one
// warp computes a whole row with 16-byte loads of the four source rows and 16-byte stores.
//
// The float arithmetic follows the x86-64 build of those MEX files (the reference's platform):
//   float input:  ((a*wa + b*wb) + c*wc) + d*wd at every position;
//   uint16 input: (a*wa + b*wb) + (c*wc + d*wd) at the positions of whole 16-element blocks of a row,
//                 ((a*wa + b*wb) + c*wc) + d*wd for the last len % 16;
//   uint16 output: blocks round res + 0.5 to nearest even, the last len % 16 truncate res + 0.5;
//   the float64 coordinates and float32 weights as the MEX files form them; no fused multiply-adds.
// Rows whose source falls outside the volume are zero.
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

constexpr int kRowThreads = 256;   // 8 warps, one output row each
int grid_rows(long long rows) { return (int)std::max(1LL, std::min((rows + 7) / 8, 148LL * 16)); }

long long mround(double v) { return v >= 0 ? (long long)std::floor(v + 0.5) : (long long)std::ceil(v - 0.5); }

// uint16 <-> float without the conversion unit: with 2^23 added, a float's low mantissa bits hold an
// integer exactly, and a round-to-nearest-even add of 2^23 rounds a value in [0, 2^23) to an integer
// the way rintf does.  (The conversion instructions run on a quarter-rate pipe and bounded these
// kernels; these forms use only the integer and FMA pipes and give identical results.)
constexpr float kMagic = 8388608.f;
__device__ __forceinline__ float u16f(unsigned v) { return __fsub_rn(__uint_as_float(0x4B000000u | v), kMagic); }

__device__ __forceinline__ float ld(const float* p, long long i) { return __ldg(p + i); }
__device__ __forceinline__ float ld(const uint16_t* p, long long i) { return u16f(__ldg(p + i)); }

// 2- or 4-term weighted sum of one row position with the association of the MEX helper for the
// operand types (pairs: uint16 helpers' whole blocks; otherwise left to right)
template <int NT>
__device__ __forceinline__ float wsum(float a, float b, float c, float d, float wa, float wb, float wc, float wd,
                                      bool pairs) {
    const float pa = __fmul_rn(a, wa), pb = __fmul_rn(b, wb);
    if (NT == 2) return __fadd_rn(pa, pb);
    const float pc = __fmul_rn(c, wc), pd = __fmul_rn(d, wd);
    return pairs ? __fadd_rn(__fadd_rn(pa, pb), __fadd_rn(pc, pd)) : __fadd_rn(__fadd_rn(__fadd_rn(pa, pb), pc), pd);
}

// res + 0.5 rounded to nearest even (whole blocks) or truncated (tail), saturated to [0, 65535]
__device__ __forceinline__ uint16_t to_u16(float v, bool body) {
    const float h = fminf(fmaxf(__fadd_rn(v, 0.5f), 0.f), 65536.f);
    unsigned r = __float_as_uint(__fadd_rn(h, kMagic)) & 0x7FFFFFu;                  // rintf(h)
    if (!body && __fsub_rn(__uint_as_float(0x4B000000u | r), kMagic) > h) r -= 1;     // truncf(h), h >= 0
    return (uint16_t)min(r, 65535u);
}
__device__ __forceinline__ void store(float* o, long long i, float v, bool) { o[i] = v; }
__device__ __forceinline__ void store(uint16_t* o, long long i, float v, bool body) { o[i] = to_u16(v, body); }

// 8 consecutive row elements (16-byte aligned) to / from registers
__device__ __forceinline__ void ld8(const float* p, float (&v)[8]) {
    const float4 x = __ldg((const float4*)p), y = __ldg((const float4*)p + 1);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w; v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
}
__device__ __forceinline__ void ld8(const uint16_t* p, float (&v)[8]) {
    const uint4 x = __ldg((const uint4*)p);
    const unsigned int w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[2 * k] = u16f(w[k] & 0xffffu);
        v[2 * k + 1] = u16f(w[k] >> 16);
    }
}
__device__ __forceinline__ void st8(float* o, const float (&v)[8], bool) {
    ((float4*)o)[0] = make_float4(v[0], v[1], v[2], v[3]);
    ((float4*)o)[1] = make_float4(v[4], v[5], v[6], v[7]);
}
__device__ __forceinline__ void st8(uint16_t* o, const float (&v)[8], bool body) {
    unsigned int w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) w[k] = (unsigned int)to_u16(v[2 * k], body) | ((unsigned int)to_u16(v[2 * k + 1], body) << 16);
    *(uint4*)o = make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ bool al16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// One weighted row, computed by one warp: out[i] = sum_k w_k * src_k[i], i < len.  u16 selects the
// uint16-helper rules.  When every row start is 16-byte aligned and len is a multiple of 8, each
// lane moves 8 elements per source with 16-byte accesses (whole 16-element blocks and the tail
// never share an 8-element group then); otherwise element by element.
template <int NT, typename TA, typename TB, typename TO>
__device__ __forceinline__ void row_blend(const TA* a, const TB* b, const TA* c, const TB* d, float wa, float wb,
                                          float wc, float wd, TO* o, int len, bool u16, int lane) {
    const int body = len - len % 16;
    const bool vec = (len & 7) == 0 && al16(a) && al16(b) && al16(o) && (NT == 2 || (al16(c) && al16(d)));
    if (vec) {
#pragma unroll 2
        for (int i = lane * 8; i < len; i += 256) {
            float va[8], vb[8], vc[8], vd[8], r[8];
            ld8(a + i, va);
            ld8(b + i, vb);
            if (NT == 4) {
                ld8(c + i, vc);
                ld8(d + i, vd);
            }
            const bool in_body = i < body;
#pragma unroll
            for (int k = 0; k < 8; k++)
                r[k] = wsum<NT>(va[k], vb[k], NT == 4 ? vc[k] : 0.f, NT == 4 ? vd[k] : 0.f, wa, wb, wc, wd, u16 && in_body);
            st8(o + i, r, in_body);
        }
        return;
    }
    for (int i = lane; i < len; i += 32) {
        const bool in_body = i < body;
        const float v = wsum<NT>(ld(a, i), ld(b, i), NT == 4 ? ld(c, i) : 0.f, NT == 4 ? ld(d, i) : 0.f, wa, wb, wc, wd,
                                 u16 && in_body);
        store(o, i, v, in_body);
    }
}

template <typename TO>
__device__ __forceinline__ void row_zero(TO* o, int len, int lane) {
    for (int i = lane; i < len; i += 32) o[i] = (TO)0;
}

// per interpolated slice (skewed_space_interp_defined_stepsize, :430-584): source slice, row offsets
// s and t, and the four weights
struct SkewSlice {
    int zo, s, t, pad;
    float c00, c01, c10, c11;
};

// Interpolated slices in the skewed space.  Row y of slice k blends rows of slices zo and zo + 1
// shifted along x by s - xa / t (reverse) or s / t - xa; rows that would leave the volume read zero.
template <typename TI, typename TO>
__global__ void k_skew_interp(const TI* __restrict__ im, TO* __restrict__ out, int ny, int nx, int nz,
                              const SkewSlice* __restrict__ sl, int nint, int xa, int reverse) {
    const long long rows = (long long)nint * nx;
    const long long plane = (long long)ny * nx;
    const bool u16 = sizeof(TI) == 2;
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
        const int y = (int)(r % nx), k = (int)(r / nx);
        const SkewSlice q = sl[k];
        TO* o = out + (long long)k * plane + (long long)y * ny;
        auto row = [&](int yy, int zz) -> const TI* {
            return (yy >= 0 && yy < nx && zz >= 0 && zz < nz) ? im + (long long)zz * plane + (long long)yy * ny : nullptr;
        };
        const TI *a, *b, *c = nullptr, *d = nullptr;
        float wa, wb, wc = 0.f, wd = 0.f;
        int nt;
        if (reverse) {
            if (y < xa - q.s) {
                a = row(y + q.t, q.zo + 1); b = row(y + q.t + 1, q.zo + 1); wa = q.c10; wb = q.c11; nt = 2;
            } else if (y < nx - q.t - 1) {
                a = row(y + q.s - xa, q.zo); b = row(y + q.s - xa + 1, q.zo); c = row(y + q.t, q.zo + 1);
                d = row(y + q.t + 1, q.zo + 1); wa = q.c00; wb = q.c01; wc = q.c10; wd = q.c11; nt = 4;
            } else {
                a = row(y + q.s - xa, q.zo); b = row(y + q.s - xa + 1, q.zo); wa = q.c00; wb = q.c01; nt = 2;
            }
        } else {
            if (y < xa - q.s) {
                a = row(y + q.s, q.zo); b = row(y + q.s + 1, q.zo); wa = q.c00; wb = q.c01; nt = 2;
            } else if (y < nx - q.t - 1) {
                a = row(y + q.s, q.zo); b = row(y + q.s + 1, q.zo); c = row(y + q.t - xa, q.zo + 1);
                d = row(y + q.t - xa + 1, q.zo + 1); wa = q.c00; wb = q.c01; wc = q.c10; wd = q.c11; nt = 4;
            } else {
                a = row(y + q.t - xa, q.zo + 1); b = row(y + q.t - xa + 1, q.zo + 1); wa = q.c10; wb = q.c11; nt = 2;
            }
        }
        if (!a || !b || (nt == 4 && (!c || !d))) {
            // a source row outside the volume reads as zero (only for volumes narrower than ~2 shifts)
            const int body = ny - ny % 16;
            for (int i = lane; i < ny; i += 32) {
                const float va = a ? ld(a, i) : 0.f, vb = b ? ld(b, i) : 0.f;
                const float vc = c ? ld(c, i) : 0.f, vd = d ? ld(d, i) : 0.f;
                const float v = nt == 4 ? wsum<4>(va, vb, vc, vd, wa, wb, wc, wd, u16 && i < body)
                                        : wsum<2>(va, vb, 0.f, 0.f, wa, wb, 0.f, 0.f, false);
                store(o, i, v, i < body);
            }
        } else if (nt == 4) {
            row_blend<4>(a, b, c, d, wa, wb, wc, wd, o, ny, u16, lane);
        } else {
            row_blend<2>(a, b, a, b, wa, wb, 0.f, 0.f, o, ny, u16, lane);
        }
    }
}

// the MEX files' rule for a coordinate exactly one below the last index: move it just inside
__device__ __forceinline__ double nudge(double t, long long n) {
    double c = 1.0;
    for (int it = 0; it < 64 && (long long)floor(t) + 1 == n; it++) {
        t = __dsub_rn(t, __dmul_rn(1e-9, c));
        c *= 2.0;
    }
    return t;
}

struct WarpArgs {
    int ny, nx, nzt;          // source rows / row count per slice / slices (after interpolation)
    int x0, ox, oy, oz;       // first source element of a row; output size
    float sy, sz;             // output box start (0-based) in x and z
    double t12, t13, t21, t22, t23;
};

// transformVolume* (volume_deskew_rotate_warp_mex.cpp:215-380; skewed variant :885-1150)
template <typename TI, typename TN, typename TO>
__global__ void k_dsr_warp(const TI* __restrict__ im, const TN* __restrict__ imi, const int* __restrict__ zindex,
                           const uint8_t* __restrict__ zorig, TO* __restrict__ out, WarpArgs w) {
    const long long rows = (long long)w.oy * w.oz;
    const long long plane = (long long)w.ny * w.nx;
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
        const int y = (int)(r % w.oy), z = (int)(r / w.oy);
        TO* o = out + r * w.ox;
        const float fz = __fadd_rn((float)z, w.sz), fy = __fadd_rn((float)y, w.sy);
        double ty = __dadd_rn(__dmul_rn(w.t12, (double)fz), w.t13);
        if (ty < 0 || ty + 1 >= w.nx) {
            if (ty + 1 == w.nx) ty = nudge(ty, w.nx);
            else { row_zero(o, w.ox, lane); continue; }
        }
        double tz = __dadd_rn(__dadd_rn(__dmul_rn(w.t21, (double)fy), __dmul_rn(w.t22, (double)fz)), w.t23);
        if (tz < 0 || tz + 1 >= w.nzt) {
            if (tz + 1 == w.nzt) tz = nudge(tz, w.nzt);
            else { row_zero(o, w.ox, lane); continue; }
        }
        const long long y0 = (long long)floor(ty), z0 = (long long)floor(tz);
        const float wy = (float)(ty - (double)y0), wz = (float)(tz - (double)z0);
        const float w00 = __fmul_rn(1.f - wy, 1.f - wz), w01 = __fmul_rn(1.f - wy, wz);
        const float w10 = __fmul_rn(wy, 1.f - wz), w11 = __fmul_rn(wy, wz);
        const long long ind = w.x0 + y0 * w.ny;
        const bool o0 = !imi || zorig[z0], o1 = !imi || zorig[z0 + 1];
        const long long p0 = (imi ? zindex[z0] : z0) * plane + ind, p1 = (imi ? zindex[z0 + 1] : z0 + 1) * plane + ind;
        const bool uin = sizeof(TI) == 2, uint_ = sizeof(TN) == 2;
        if (o0 && o1) {
            row_blend<4>(im + p0, im + p1, im + p0 + w.ny, im + p1 + w.ny, w00, w01, w10, w11, o, w.ox, uin, lane);
        } else if (!o0 && !o1) {
            row_blend<4>(imi + p0, imi + p1, imi + p0 + w.ny, imi + p1 + w.ny, w00, w01, w10, w11, o, w.ox, uint_, lane);
        } else if (o0) {          // source slice z0 original, z0 + 1 interpolated
            row_blend<4>(im + p0, imi + p1, im + p0 + w.ny, imi + p1 + w.ny, w00, w01, w10, w11, o, w.ox, uin || uint_, lane);
        } else if (uin == uint_) {  // same types: the helper keeps the slice order
            row_blend<4>(imi + p0, im + p1, imi + p0 + w.ny, im + p1 + w.ny, w00, w01, w10, w11, o, w.ox, uin, lane);
        } else {                  // uint16 original at z0 + 1, float interpolated at z0: operands swapped
            row_blend<4>(im + p1, imi + p0, im + p1 + w.ny, imi + p0 + w.ny, w01, w00, w11, w10, o, w.ox, true, lane);
        }
    }
}

// ------------------------------------------------------------------ host plan
struct DsrPlan {
    int64_t out[3];
    bool do_interp = false;
    double stepsize = 1, xstep = 0;
    long long ntotal = 0;
    double tmat[4][4];
    int64_t bbox[6];
};

typedef double M4[4][4];

void mul4(const M4 a, const M4 b, M4 c) {
    M4 t;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double s = 0;
            for (int k = 0; k < 4; k++) s += a[i][k] * b[k][j];
            t[i][j] = s;
        }
    memcpy(c, t, sizeof(M4));
}

bool inv4(const M4 a, M4 out) {      // Gauss-Jordan with partial pivoting
    double m[4][8];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 8; j++) m[i][j] = j < 4 ? a[i][j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (m[p][c] == 0.0) return false;
        if (p != c)
            for (int j = 0; j < 8; j++) std::swap(m[p][j], m[c][j]);
        const double d = m[c][c];
        for (int j = 0; j < 8; j++) m[c][j] /= d;
        for (int r = 0; r < 4; r++) {
            if (r == c || m[r][c] == 0.0) continue;
            const double f = m[r][c];
            for (int j = 0; j < 8; j++) m[r][j] -= f * m[c][j];
        }
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[i][j] = m[i][j + 4];
    return true;
}

long long n_total(long long nz, double step) {
    return (long long)std::floor((double)mround((double)(nz - 1) / step * 100000) / 100000) + 1;
}

// deskewRotateFrame3D.m:53-208 on the fast path
pk_status dsr_plan(const int64_t dims[3], double angle, double dz, double px, int reverse, int objective_scan,
                   double xstep_thresh, const int64_t* bbox, DsrPlan* P) {
    const long long ny = dims[0], nx = dims[1];
    long long nz = dims[2];
    double theta = angle * M_PI / 180;
    double dx = std::cos(theta) * dz / px;
    double zaniso = objective_scan ? dz / px : std::sin(std::fabs(theta)) * dz / px;
    double os[3];
    if (!objective_scan) {
        os[0] = (double)ny;
        os[1] = (nx - 1) * std::cos(theta) + (nz - 1) * zaniso / std::sin(std::fabs(theta));
        os[2] = (nx - 1) * std::sin(std::fabs(theta)) - 4;
    } else {
        os[0] = (double)ny;
        os[1] = nx * std::cos(theta) + nz * zaniso * std::sin(std::fabs(theta));
        os[2] = nz * zaniso * std::cos(theta) + nx * std::sin(std::fabs(theta));
    }
    for (int k = 0; k < 3; k++) P->out[k] = mround(os[k]);
    P->do_interp = !objective_scan && std::fabs(dx) > xstep_thresh;
    P->xstep = std::fabs(dx);
    if (P->do_interp) {                                           // :71-118
        double dzout;
        if (std::fabs(dx) / xstep_thresh < 1.5) {
            const double thr = px * xstep_thresh / std::cos(theta);
            dzout = dz / (std::ceil((dz / thr) / (1.0 / 1)) * (1.0 / 1));
            int counter = 1;
            while (dzout / thr < 0.4 && counter < 1000000) {
                dzout = dz / (std::ceil((dz / thr) / (1.0 / (counter + 1))) * (1.0 / (counter + 1)));
                counter++;
            }
        } else {
            dzout = dz / std::ceil(std::fabs(dx) / xstep_thresh);
        }
        P->stepsize = dzout / dz;
        nz = n_total(nz, P->stepsize);
        dz = dzout;
        dx = std::cos(theta) * dz / px;
        zaniso = std::sin(std::fabs(theta)) * dz / px;
    }
    P->ntotal = nz;
    double xshift, xstep;                                         // :121-139
    if (!reverse) { xshift = -dx; xstep = dx; }
    else { xshift = dx + std::ceil((nz - 1) * dx); xstep = -dx; }
    double nx_ds = std::ceil((nz - 1) * dx) + nx;
    M4 dsS = {{1, 0, 0, 0}, {0, 1, 0, 0}, {xstep, 0, 1, 0}, {xshift, 0, 0, 1}};
    if (objective_scan) {
        nx_ds = (double)nx;
        const M4 I = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
        memcpy(dsS, I, sizeof(M4));
    }
    if (reverse) theta = -theta;                                  // :143-145
    const double cy = (ny + 1) / 2.0, cx = (nx_ds + 1) / 2.0, cz = (nz + 1) / 2.0;
    const M4 T1o = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {-cx + 1, -cy + 1, -cz + 1, 1}};   // T1 + offset
    const M4 S = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, zaniso, 0}, {0, 0, 0, 1}};
    const double c = std::cos(theta), s = std::sin(theta);
    const M4 R = {{c, 0, -s, 0}, {0, 1, 0, 0}, {s, 0, c, 0}, {0, 0, 0, 1}};
    const M4 T2o = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0},                                  // T2 - offset
                    {(P->out[1] + 1) / 2.0 - 1, (P->out[0] + 1) / 2.0 - 1, (P->out[2] + 1) / 2.0 - 1, 1}};
    if (!objective_scan && reverse) dsS[3][0] -= dx;              // :186-188
    M4 m;
    mul4(T1o, S, m);
    mul4(m, R, m);
    mul4(m, T2o, m);
    mul4(dsS, m, m);
    M4 mt, inv;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) mt[i][j] = m[j][i];
    if (!inv4(mt, inv)) return pk_fail(PK_ERR_INVALID, "deskewRotateFrame3D: singular transform");
    const int perm[4] = {1, 0, 2, 3};                             // tmat([2 1 3 4], [2 1 3 4])
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) P->tmat[i][j] = inv[perm[i]][perm[j]];
    if (bbox) for (int k = 0; k < 6; k++) P->bbox[k] = bbox[k];
    else {
        P->bbox[0] = P->bbox[1] = P->bbox[2] = 1;
        for (int k = 0; k < 3; k++) P->bbox[3 + k] = P->out[k];
    }
    return PK_OK;
}

// skewed_space_interp_defined_stepsize (:430-476) and determine_interpolation_indexing (:1152-1170)
void skew_tables(long long nz, const DsrPlan& P, int reverse, std::vector<int>& zindex, std::vector<uint8_t>& zorig,
                 std::vector<SkewSlice>& sl) {
    const long long nt = P.ntotal;
    zindex.assign(nt, 0);
    zorig.assign(nt, 0);
    sl.clear();
    const double xs = P.xstep;
    for (long long i = 0; i < nt; i++) {
        const double cs = (double)i * P.stepsize;
        const double cr = (double)mround(cs);
        if (std::fabs(cs - cr) < 1e-3) {
            zorig[i] = 1;
            zindex[i] = (int)cr;
            continue;
        }
        zindex[i] = (int)sl.size();
        const double zout = P.stepsize * (double)i;
        const double zw = zout - std::floor(zout);
        double s, t;
        if (reverse) { s = std::ceil(xs) - xs * zw; t = xs * (1 - zw); }
        else { s = xs * (1 - zw); t = std::ceil(xs) - xs * zw; }
        const double sw = s - std::floor(s), tw = t - std::floor(t);
        const float swf = (float)sw, twf = (float)tw, zwf = (float)zw;
        SkewSlice q;
        q.zo = (int)std::floor(zout);
        q.s = (int)std::floor(s);
        q.t = (int)std::floor(t);
        q.pad = 0;
        q.c00 = (float)((1.0 - swf) * (1.0 - zwf));
        q.c01 = (float)(swf * (1.0 - zwf));
        q.c10 = (float)((1.0 - twf) * zwf);
        q.c11 = twf * zwf;                  // a float product in the reference
        sl.push_back(q);
    }
    (void)nz;
}

size_t esize(pk_dtype t) { return t == PK_U16 ? 2 : 4; }

// per-kernel events for pk_ctx_profile (kind = kernel name, bytes = algorithmic bytes: each input,
// interpolated slice and output voxel moved once)
struct KernelProf {
    pk_ctx* ctx;
    pk_ctx::ProfRec rec;
    KernelProf(pk_ctx* c, const char* kind, double bytes, cudaStream_t st) : ctx(c) {
        ctx->launches++;
        if (!ctx->prof_on) return;
        auto take = [&]() {
            cudaEvent_t e;
            if (!ctx->ev_pool.empty()) { e = ctx->ev_pool.back(); ctx->ev_pool.pop_back(); }
            else cudaEventCreate(&e);
            return e;
        };
        rec.kind = kind;
        rec.bytes = bytes;
        rec.a = take();
        rec.b = take();
        cudaEventRecord(rec.a, st);
    }
    void done(cudaStream_t st) {
        if (!ctx->prof_on) return;
        cudaEventRecord(rec.b, st);
        ctx->prof.push_back(rec);
    }
};

pk_status dsr_run(pk_ctx* ctx, const void* d_in, pk_dtype t, const int64_t dims[3], const DsrPlan& P, int reverse,
                  bool u16_out, void* d_out, cudaStream_t st) {
    const int ny = (int)dims[0], nx = (int)dims[1], nz = (int)dims[2];
    const float sx = (float)P.bbox[0] - 1.f, sy = (float)P.bbox[1] - 1.f, sz = (float)P.bbox[2] - 1.f;
    const float ex = (float)P.bbox[3], ey = (float)P.bbox[4], ez = (float)P.bbox[5];
    WarpArgs w;
    w.ny = ny; w.nx = nx; w.nzt = (int)P.ntotal;
    w.x0 = (int)std::floor(sx);
    w.ox = (int)(ex - sx); w.oy = (int)(ey - sy); w.oz = (int)(ez - sz);
    w.sy = sy; w.sz = sz;
    w.t12 = P.tmat[1][2]; w.t13 = P.tmat[1][3]; w.t21 = P.tmat[2][1]; w.t22 = P.tmat[2][2]; w.t23 = P.tmat[2][3];
    const long long rows = (long long)w.oy * w.oz;
    pk_status s;
    const void* imi = nullptr;
    const int* dzi = nullptr;
    const uint8_t* dzo = nullptr;
    if (P.do_interp) {
        std::vector<int> zindex;
        std::vector<uint8_t> zorig;
        std::vector<SkewSlice> sl;
        skew_tables(nz, P, reverse, zindex, zorig, sl);
        const int nint = (int)sl.size();
        const size_t ie = (t == PK_U16 && u16_out) ? 2 : 4;
        void* dint;
        const size_t nsl = std::max<size_t>(1, sl.size());
        if ((s = pk_scratch(ctx, 25, ie * (size_t)ny * nx * std::max(1, nint), &dint)) != PK_OK) return s;
        // the slice tables depend only on the geometry: built and uploaded once per context
        char key[160];
        snprintf(key, sizeof(key), "dsr:%d:%a:%a:%d", nz, P.stepsize, P.xstep, reverse);
        void*& dtab = ctx->dev_tables[key];
        if (!dtab) {
            const size_t tb = sizeof(SkewSlice) * nsl + 4 * zindex.size() + zorig.size();
            std::vector<char> host(tb, 0);
            memcpy(host.data(), sl.data(), sizeof(SkewSlice) * sl.size());
            memcpy(host.data() + sizeof(SkewSlice) * nsl, zindex.data(), 4 * zindex.size());
            memcpy(host.data() + sizeof(SkewSlice) * nsl + 4 * zindex.size(), zorig.data(), zorig.size());
            if (cudaMalloc(&dtab, tb) != cudaSuccess) {
                cudaGetLastError();
                ctx->dev_tables.erase(key);
                return pk_fail(PK_ERR_NOMEM, "deskew: table allocation failed");
            }
            PK_CUDA(cudaMemcpy(dtab, host.data(), tb, cudaMemcpyHostToDevice));
        }
        char* tp = (char*)dtab;
        SkewSlice* dsl = (SkewSlice*)tp;
        int* dzindex = (int*)(tp + sizeof(SkewSlice) * nsl);
        uint8_t* dzorig = (uint8_t*)(dzindex + zindex.size());
        const int xa = (int)std::ceil(P.xstep);
        const int g = grid_rows((long long)nint * nx);
        if (nint > 0) {
            const double ib = (double)esize(t) * ny * nx * nz + (double)ie * ny * nx * nint;
            KernelProf kp(ctx, "k_skew_interp", ib, st);
            if (t == PK_F32)
                k_skew_interp<float, float><<<g, kRowThreads, 0, st>>>((const float*)d_in, (float*)dint, ny, nx, nz, dsl, nint, xa, reverse);
            else if (u16_out)
                k_skew_interp<uint16_t, uint16_t><<<g, kRowThreads, 0, st>>>((const uint16_t*)d_in, (uint16_t*)dint, ny, nx, nz, dsl, nint, xa, reverse);
            else
                k_skew_interp<uint16_t, float><<<g, kRowThreads, 0, st>>>((const uint16_t*)d_in, (float*)dint, ny, nx, nz, dsl, nint, xa, reverse);
            PK_CUDA(cudaGetLastError());
            kp.done(st);
        }
        imi = dint;
        dzi = dzindex;
        dzo = dzorig;
    }
    const int g = grid_rows(rows);
    if (rows == 0 || w.ox == 0) return PK_OK;
    const size_t oe = (t == PK_U16 && u16_out) ? 2 : 4;
    double wb = (double)esize(t) * ny * nx * nz + (double)oe * w.ox * rows;
    if (P.do_interp) wb += (double)oe * ny * nx * (P.ntotal - nz);
    KernelProf kp(ctx, "k_dsr_warp", wb, st);
    if (t == PK_F32)
        k_dsr_warp<float, float, float><<<g, kRowThreads, 0, st>>>((const float*)d_in, (const float*)imi, dzi, dzo, (float*)d_out, w);
    else if (u16_out)
        k_dsr_warp<uint16_t, uint16_t, uint16_t><<<g, kRowThreads, 0, st>>>((const uint16_t*)d_in, (const uint16_t*)imi, dzi, dzo,
                                                                   (uint16_t*)d_out, w);
    else
        k_dsr_warp<uint16_t, float, float><<<g, kRowThreads, 0, st>>>((const uint16_t*)d_in, (const float*)imi, dzi, dzo,
                                                             (float*)d_out, w);
    PK_CUDA(cudaGetLastError());
    kp.done(st);
    return PK_OK;
}

pk_status dsr_check(pk_ctx* ctx, pk_dtype t, const int64_t dims[3], double angle, double dz, double px,
                    double xstep_thresh, const int64_t* bbox, int64_t out_dims[3]) {
    if (!ctx) return pk_fail(PK_ERR_INVALID, "null pk_ctx");
    if (!dims || !out_dims) return pk_fail(PK_ERR_INVALID, "NULL dims/out_dims");
    if (t != PK_U16 && t != PK_F32) return pk_fail(PK_ERR_INVALID, "deskewRotateFrame3D: input must be uint16 or single");
    if (dims[0] < 1 || dims[1] < 2 || dims[2] < 2 || dims[0] * dims[1] * dims[2] > (1LL << 40))
        return pk_fail(PK_ERR_INVALID, "deskewRotateFrame3D: bad volume size");
    if (!(dz > 0) || !(px > 0) || !(xstep_thresh > 0) || !std::isfinite(angle))
        return pk_fail(PK_ERR_INVALID, "deskewRotateFrame3D: dz, xyPixelSize and xStepThresh must be positive");
    if (std::fabs(std::sin(angle * M_PI / 180)) < 1e-6)
        return pk_fail(PK_ERR_INVALID, "deskewRotateFrame3D: the skew angle must not be a multiple of 180 degrees");
    if (bbox) {
        for (int k = 0; k < 3; k++)
            if (bbox[k] < 1 || bbox[k + 3] < bbox[k] - 1)
                return pk_fail(PK_ERR_INVALID, "Input bbox is invalid, the numbers must be nonnegative and the end ranges must be nonless than the start ranges.");
        if (bbox[3] > dims[0]) return pk_fail(PK_ERR_INVALID, "deskewRotateFrame3D: bbox(4) exceeds the first dimension of the volume");
    }
    return PK_OK;
}

}  // namespace

extern "C" pk_status pk_deskew_rotate_device(pk_ctx* ctx, const void* d_in, pk_dtype in_type, const int64_t dims[3],
                                             double angle, double dz, double xy_pixel_size, int32_t reverse,
                                             int32_t objective_scan, double xstep_thresh, const int64_t* bbox,
                                             int32_t save16bit, void* d_out, int64_t out_dims[3], void* stream) {
    pk_status s;
    if ((s = dsr_check(ctx, in_type, dims, angle, dz, xy_pixel_size, xstep_thresh, bbox, out_dims)) != PK_OK) return s;
    DsrPlan P;
    if ((s = dsr_plan(dims, angle, dz, xy_pixel_size, reverse, objective_scan, xstep_thresh, bbox, &P)) != PK_OK) return s;
    for (int k = 0; k < 3; k++) out_dims[k] = P.bbox[3 + k] - P.bbox[k] + 1;
    if (!d_out) return PK_OK;
    if (!d_in) return pk_fail(PK_ERR_INVALID, "NULL input");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    return dsr_run(ctx, d_in, in_type, dims, P, reverse, save16bit && in_type == PK_U16, d_out, st);
}

extern "C" pk_status pk_deskew_rotate(pk_ctx* ctx, const void* in, pk_dtype in_type, const int64_t dims[3], double angle,
                                      double dz, double xy_pixel_size, int32_t reverse, int32_t objective_scan,
                                      double xstep_thresh, const int64_t* bbox, int32_t save16bit, void* out,
                                      int64_t out_dims[3]) {
    pk_status s;
    if ((s = dsr_check(ctx, in_type, dims, angle, dz, xy_pixel_size, xstep_thresh, bbox, out_dims)) != PK_OK) return s;
    DsrPlan P;
    if ((s = dsr_plan(dims, angle, dz, xy_pixel_size, reverse, objective_scan, xstep_thresh, bbox, &P)) != PK_OK) return s;
    for (int k = 0; k < 3; k++) out_dims[k] = P.bbox[3 + k] - P.bbox[k] + 1;
    if (!out) return PK_OK;
    if (!in) return pk_fail(PK_ERR_INVALID, "NULL input");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const bool u16_out = save16bit && in_type == PK_U16;
    const size_t inb = esize(in_type) * (size_t)dims[0] * dims[1] * dims[2];
    const size_t outb = (u16_out ? 2 : 4) * (size_t)out_dims[0] * out_dims[1] * out_dims[2];
    void *din, *dout;
    if ((s = pk_scratch(ctx, 24, inb, &din)) != PK_OK) return s;
    if ((s = pk_scratch(ctx, 27, std::max<size_t>(outb, 16), &dout)) != PK_OK) return s;
    PK_CUDA(cudaMemcpyAsync(din, in, inb, cudaMemcpyHostToDevice, st));
    if ((s = dsr_run(ctx, din, in_type, dims, P, reverse, u16_out, dout, st)) != PK_OK) return s;
    if (outb) PK_CUDA(cudaMemcpyAsync(out, dout, outb, cudaMemcpyDeviceToHost, st));
    PK_CUDA(cudaStreamSynchronize(st));
    return PK_OK;
}
