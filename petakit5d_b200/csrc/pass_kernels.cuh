// Pass kernels, templated on the transform plan of the axis they transform (plan 0 = runtime
// engine), on the tile size (4096 points, or 1024 for small volumes) and, for the y pass, on the
// per-voxel mode (one kernel per mode).  The x/z passes load their tiles from HBM straight into the
// first radix stage's registers and store from the last stage's registers; the y pass stages rows
// and per-voxel inputs with cp.async and, where the plan allows, runs the per-voxel arithmetic on
// registers between the inverse and the forward transform.
#pragma once
#include "fft_ct.cuh"
#include "pk_internal.h"

#define PK_EPS_F 2.220446049250313e-16f  // single(eps) = 2^-52

namespace pkpass {
using namespace pkfft;

__device__ __forceinline__ int find_vol(const int* __restrict__ prefix, int nvol, int b) {
    int lo = 0, hi = nvol - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ float u16_of(float J) {
    float r = roundf(J);             // half away from zero, like MATLAB uint16()
    if (!(r >= 0.f)) r = 0.f;        // negatives and NaN -> 0
    if (r > 65535.f) r = 65535.f;
    return r;
}

// Ampere-style asynchronous global->shared copies (LDGSTS): issued without registers, completed
// by commit/wait groups, so a CTA keeps its whole tile (and the epilogue's inputs) in flight.
__device__ __forceinline__ void cp8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The descriptor fields the per-voxel helpers below read, copied into registers once per CTA.  Read
// through the descriptor itself, every store to one of the volume's arrays would make the compiler
// load them again from memory (the store might alias the descriptor) before the next voxel.
struct VoxFields {
    int ny, nx, nz;
    long long nrows;
    int rdims[3];
    const void* raw;
    int raw_type, bg16;
    float bg_f;
    float *I, *Jn, *Yb, *J4, *J2n, *dst;
    uint8_t* mask8;
    int write_mask, rl_first, mask_mode, erosion, scale_mode, save16, crop, need_xz;
    float damp, scale, offset;
    void* out;
    int bb0[3], bb1[3];
    int* chk;
    __device__ __forceinline__ explicit VoxFields(const VolDesc& d)
        : ny(d.ny), nx(d.nx), nz(d.nz), nrows(d.nrows), raw(d.raw), raw_type(d.raw_type), bg16(d.bg16),
          bg_f(d.bg_f), I(d.I), Jn(d.Jn), Yb(d.Yb), J4(d.J4), J2n(d.J2n), dst(d.dst), mask8(d.mask8),
          write_mask(d.write_mask), rl_first(d.rl_first), mask_mode(d.mask_mode), erosion(d.erosion),
          scale_mode(d.scale_mode), save16(d.save16), crop(d.crop), need_xz(d.need_xz), damp(d.damp),
          scale(d.scale), offset(d.offset), out(d.out), chk(d.chk) {
        for (int i = 0; i < 3; i++) {
            rdims[i] = d.rdims[i];
            bb0[i] = d.bb0[i];
            bb1[i] = d.bb1[i];
        }
    }
};

// Value of one voxel after the post-processing of decon_lucy_omw_function.m:146-177 (damping, then
// scaling with offset and mask); x/z only matter to the border-erosion mask.
template <class D>
__device__ __forceinline__ float post_value(const D& d, float J, long long vi, int x, int y, int z) {
    if (d.damp > 1.f) {
        const float dI = __fmul_rn(d.damp, d.I[vi]);
        const float a = (J <= dI) ? J : 0.f;
        const float b = (J >= dI) ? dI : 0.f;
        J = __fadd_rn(a, fminf(J, b));
    }
    if (d.scale_mode == 1) {
        J = __fmul_rn(J, d.scale);
    } else if (d.scale_mode == 2) {
        int m = 1;
        if (d.mask_mode == 1 || d.mask_mode == 3) m = d.mask8[vi] != 0;
        else if (d.mask_mode == 2) {
            const int E = d.erosion;
            m = d.mask8[vi] != 0 && y >= E && y < d.ny - E && x >= E && x < d.nx - E &&
                (d.nz == 1 || (z >= E && z < d.nz - E));          // one plane: MATLAB's 2-D case
        }
        J = __fmul_rn(__fadd_rn(__fmul_rn(J, d.scale), d.offset), (float)m);
    }
    return J;
}

template <class D>
__device__ __forceinline__ void row_xz(const D& d, long long row, int& x, int& z) {
    const unsigned r = (unsigned)row;
    z = (int)(r / (unsigned)d.nx);
    x = (int)(r - (unsigned)z * (unsigned)d.nx);
}

template <class D>
__device__ __forceinline__ bool in_box(const D& d, int x, int y, int z) {
    return !(y < d.bb0[0] || y > d.bb1[0] || x < d.bb0[1] || x > d.bb1[1] || z < d.bb0[2] || z > d.bb1[2]);
}

// Store of one post-processed voxel into the (cropped) output.
template <class D>
__device__ __forceinline__ void out_store(const D& d, float J, long long vi, int x, int y, int z) {
    long long oi = vi;
    if (d.crop) {
        const long long oy = d.bb1[0] - d.bb0[0] + 1, ox = d.bb1[1] - d.bb0[1] + 1;
        oi = (long long)(y - d.bb0[0]) + oy * ((long long)(x - d.bb0[1]) + ox * (long long)(z - d.bb0[2]));
    }
    if (!PK_IN(d, oi >= 0 && oi < (long long)(d.bb1[0] - d.bb0[0] + 1) * (d.bb1[1] - d.bb0[1] + 1) * (d.bb1[2] - d.bb0[2] + 1), 20))
        return;
    if (d.save16) ((uint16_t*)d.out)[oi] = (uint16_t)u16_of(J);
    else ((float*)d.out)[oi] = J;
}

// Whether rows row0 .. row0 + n - 1 (row = x + nx z) hold a voxel of the crop box: the rows of a
// y-pass tile are consecutive, so they cover one x range of one z plane or reach over whole planes.
__device__ __forceinline__ bool rows_meet_box(const VolDesc& d, long long row0, int n) {
    const unsigned nx = (unsigned)d.nx;
    const int z0 = (int)((unsigned)row0 / nx), z1 = (int)((unsigned)(row0 + n - 1) / nx);
    if (z1 < d.bb0[2] || z0 > d.bb1[2]) return false;
    if (z0 != z1) return true;
    const int x0 = (int)((unsigned)row0 - (unsigned)z0 * nx), x1 = x0 + n - 1;
    return !(x1 < d.bb0[1] || x0 > d.bb1[1]);
}

// post-processing of one voxel and the cropped store.  x/z of the row are only derived when a crop
// box or the border-erosion mask needs them.
template <class D>
__device__ __forceinline__ void post_store(const D& d, float J, long long row, int y) {
    const long long vi = row * d.ny + y;
    int x = 0, z = 0;
    if (d.need_xz) {
        row_xz(d, row, x, z);
        if (!in_box(d, x, y, z)) return;
    }
    out_store(d, post_value(d, J, vi, x, y, z), vi, x, y, z);
}

__device__ __forceinline__ bool mode_from_spec(int m) {
    return m == Y_RATIO || m == Y_UPDATE || m == Y_FINAL || m == Y_RLUPD || m == Y_RLFINAL || m == Y_C2R;
}
__device__ __forceinline__ bool mode_to_spec(int m) {
    return m == Y_R2C || m == Y_PRE || m == Y_RATIO || m == Y_UPDATE || m == Y_RLPRE;
}

// Load two consecutive reals (even ny) or one (odd ny) of a float volume.
__device__ __forceinline__ float2 ld2(const float* p, long long vi, bool odd) {
    if (!odd) return *reinterpret_cast<const float2*>(p + vi);
    return make_float2(p[vi], 0.f);
}
__device__ __forceinline__ void st2(float* p, long long vi, float2 v, bool odd) {
    if (!odd) *reinterpret_cast<float2*>(p + vi) = v;
    else p[vi] = v.x;
}

template <int P, bool INV, int TP>
__device__ __forceinline__ void fft_y(float2* buf, const AxisDev& A, const float2* tw, int L, int tid) {
    if constexpr (P == 0) {
        TileGeom g{L, A.n, A.n, 1, false};
        fft_lines<INV>(buf, A, tw, g, tid, PK_THREADS);
    } else {
        run_plan<P, 0, 1, plan_lines_y(kPlans[P].n, TP), false, INV>(buf, tw, tid);
    }
}

template <int P, bool INV, int TP>
__device__ __forceinline__ void fft_xz(float2* buf, const AxisDev& A, const float2* tw, int T, int tid) {
    if constexpr (P == 0) {
        TileGeom g{T, A.n, 1, T, true};
        fft_lines<INV>(buf, A, tw, g, tid, PK_THREADS);
    } else {
        run_plan<P, 0, 1, plan_cols_xz(kPlans[P].n, TP), true, INV>(buf, tw, tid);
    }
}

// Per-voxel operation of a y-pass mode on a pair of reals (x = element y, y = element y+1; for odd
// ny only .x is live).  a0/a1 are the mode's gathered inputs for the same voxels.
template <class D>
__device__ __forceinline__ float2 voxel_pair(const D& d, int mode, float2 c, float2 a0, float2 a1, long long row,
                                             int y, bool two, float lam, double& acc0, double& acc1) {
    float2 r = make_float2(0.f, 0.f);
    const long long vi = row * d.ny + y;
    switch (mode) {
        case Y_R2C: r = a0; break;
        case Y_RATIO:
            // __fdividef: at most 2 ulp from the rounded quotient for divisors in [2^-126, 2^126]
            // (here max(c, eps) >= 2^-52), and no out-of-line slow path in the unrolled loop
            r.x = __fdividef(a0.x, fmaxf(c.x, PK_EPS_F));
            r.y = two ? __fdividef(a0.y, fmaxf(c.y, PK_EPS_F)) : 0.f;
            break;
        case Y_UPDATE:
            r.x = fmaxf(__fmul_rn(c.x, a0.x), 0.f);
            r.y = two ? fmaxf(__fmul_rn(c.y, a0.y), 0.f) : 0.f;
            st2(d.Jn, vi, r, !two);
            break;
        case Y_FINAL:
            post_store(d, fmaxf(__fmul_rn(c.x, a0.x), 0.f), row, y);
            if (two) post_store(d, fmaxf(__fmul_rn(c.y, a0.y), 0.f), row, y + 1);
            break;
        case Y_RLPRE: {
            r.x = fmaxf(__fadd_rn(a0.x, __fmul_rn(lam, __fsub_rn(a0.x, a1.x))), 0.f);
            r.y = two ? fmaxf(__fadd_rn(a0.y, __fmul_rn(lam, __fsub_rn(a0.y, a1.y))), 0.f) : 0.f;
            st2(d.Yb, vi, r, !two);
            break;
        }
        case Y_RLUPD: {
            float2 j2n, diff;
            j2n.x = fmaxf(__fmul_rn(a0.x, c.x), 0.f);
            j2n.y = two ? fmaxf(__fmul_rn(a0.y, c.y), 0.f) : 0.f;
            diff.x = __fsub_rn(j2n.x, a0.x);
            diff.y = __fsub_rn(j2n.y, a0.y);
            if (!d.rl_first) {
                acc0 += (double)__fmul_rn(diff.x, a1.x);
                acc1 += (double)__fmul_rn(a1.x, a1.x);
                if (two) {
                    acc0 += (double)__fmul_rn(diff.y, a1.y);
                    acc1 += (double)__fmul_rn(a1.y, a1.y);
                }
            }
            st2(d.J4, vi, diff, !two);
            st2(d.J2n, vi, j2n, !two);
            break;
        }
        case Y_RLFINAL:
            post_store(d, fmaxf(__fmul_rn(a0.x, c.x), 0.f), row, y);
            if (two) post_store(d, fmaxf(__fmul_rn(a0.y, c.y), 0.f), row, y + 1);
            break;
        case Y_C2R: st2(d.dst, vi, c, !two); break;
        default: break;
    }
    return r;
}

// Y_PRE on a pair of voxels: raw -> I = sat(raw - bg) (uint16) or max(raw - bg, 0) (written), mask =
// raw ~= 0 (decon_lucy_omw_function.m:79-98).  a0 is the staged raw pair.
template <class D>
__device__ __forceinline__ float2 pre_pair(const D& d, bool raw_sync, bool odd, float2 a0, long long row, int y,
                                           unsigned& zeros) {
    // raw -> I = sat(raw - bg) (uint16) or max(raw - bg, 0); mask = raw ~= 0
    const long long vi = row * (long long)d.ny + y;
    float2 I;
    bool nz0, nz1 = true;
    if (raw_sync) {
        // scalar loads through the raw extent (padded transforms read zeros outside it)
        const unsigned ur = (unsigned)row;
        const int z = (int)(ur / (unsigned)d.nx), x = (int)(ur - (unsigned)z * (unsigned)d.nx);
        float v[2] = {0.f, 0.f};
        bool nzv[2] = {true, true};
        for (int e = 0; e < (odd ? 1 : 2); e++) {
            const int yy = y + e;
            if (yy >= d.rdims[0] || x >= d.rdims[1] || z >= d.rdims[2]) { v[e] = 0.f; continue; }
            const long long ri = yy + (long long)d.rdims[0] * (x + (long long)d.rdims[1] * z);
            if (d.raw_type == PK_U16) {
                const unsigned r = ((const uint16_t*)d.raw)[ri];
                nzv[e] = r != 0;
                v[e] = r > (unsigned)d.bg16 ? (float)(r - (unsigned)d.bg16) : 0.f;
            } else if (d.raw_type == PK_F32) {
                const float r = ((const float*)d.raw)[ri];
                nzv[e] = r != 0.f;
                v[e] = fmaxf(__fsub_rn(r, d.bg_f), 0.f);
            } else {
                const double r = ((const double*)d.raw)[ri];
                nzv[e] = r != 0.0;
                v[e] = fmaxf(__fsub_rn((float)r, d.bg_f), 0.f);
            }
        }
        I = make_float2(v[0], v[1]);
        nz0 = nzv[0];
        nz1 = nzv[1];
    } else if (d.raw_type == PK_U16) {
        const ushort2 q = *reinterpret_cast<const ushort2*>(&a0);
        const unsigned r0 = q.x, r1 = q.y;
        nz0 = r0 != 0;
        nz1 = r1 != 0;
        I.x = r0 > (unsigned)d.bg16 ? (float)(r0 - (unsigned)d.bg16) : 0.f;
        I.y = r1 > (unsigned)d.bg16 ? (float)(r1 - (unsigned)d.bg16) : 0.f;
    } else {
        const float2 r = a0;
        nz0 = r.x != 0.f;
        if (!odd) nz1 = r.y != 0.f;
        I.x = fmaxf(__fsub_rn(r.x, d.bg_f), 0.f);
        I.y = fmaxf(__fsub_rn(r.y, d.bg_f), 0.f);
    }
    if (odd) {
        I.y = 0.f;
        nz1 = true;
    }
    st2(d.I, vi, I, odd);
    if (d.write_mask) {
        d.mask8[vi] = nz0 ? 1 : 0;
        if (!odd) d.mask8[vi + 1] = nz1 ? 1 : 0;
    }
    zeros += (nz0 ? 0u : 1u) + (nz1 ? 0u : 1u);
    return I;
}

// Y_PRE value of a staged raw pair (even ny, raw in the volume's own layout): I and the raw-zero count.
__device__ __forceinline__ float2 pre_value(bool u16, unsigned bg16, float bgf, float2 a0, unsigned& zeros) {
    float2 I;
    bool nz0, nz1;
    if (u16) {
        const ushort2 q = *reinterpret_cast<const ushort2*>(&a0);
        const unsigned r0 = q.x, r1 = q.y;
        nz0 = r0 != 0;
        nz1 = r1 != 0;
        I.x = r0 > bg16 ? (float)(r0 - bg16) : 0.f;
        I.y = r1 > bg16 ? (float)(r1 - bg16) : 0.f;
    } else {
        nz0 = a0.x != 0.f;
        nz1 = a0.y != 0.f;
        I.x = fmaxf(__fsub_rn(a0.x, bgf), 0.f);
        I.y = fmaxf(__fsub_rn(a0.y, bgf), 0.f);
    }
    zeros += (nz0 ? 0u : 1u) + (nz1 ? 0u : 1u);
    return I;
}

// The plan's first and last radix agree: after a transform's last stage each thread holds the elements
// the next transform's first stage needs.
constexpr bool same_end_radix(int p) {
    return p > 0 && kPlans[p].nst >= 2 && kPlans[p].rad[0] == kPlans[p].rad[kPlans[p].nst - 1];
}

// Number of per-voxel input arrays a y-pass mode stages in shared memory.
__host__ __device__ inline int y_aux_arrays(int mode) {
    switch (mode) {
        case Y_RLPRE: case Y_RLUPD: return 2;
        case Y_C2R: return 0;
        default: return 1;
    }
}

template <int P, int MODE, int TP = PK_TILE_POINTS>
__global__ void __launch_bounds__(PK_THREADS, 3) k_y(const VolDesc* __restrict__ descs, const int* __restrict__ prefix,
                                                     int nvol, int) {
    constexpr int mode = MODE;   // one kernel per mode: only that mode's code is in the kernel
    extern __shared__ float2 smem[];
    constexpr int NT = PK_THREADS;
    const int vol = find_vol(prefix, nvol, blockIdx.x);
    const VolDesc& d = descs[vol];
    const int lb = blockIdx.x - prefix[vol];
    const int tid = threadIdx.x;
    const AxisDev& A = d.ay;
    const int M = P == 0 ? d.M : kPlans[P].n;
    const int L = P == 0 ? d.Ly : plan_lines_y(kPlans[P].n, TP);
    const bool odd = d.odd;
    const int Py = d.Py, ny = d.ny;
    // shared memory: tw[tw_slots(M)] | twrc[M+1] (even ny) | buf[padded L*M] | nyq[L] | aux0[L*M] | aux1[L*M]
    float2* tw = smem;
    float2* twrc = smem + tw_slots(M);
    float2* buf = twrc + (odd ? 0 : M + 1);
    float2* nyq = buf + padded_size(L * M);
    float2* aux0 = nyq + L;
    float2* aux1 = aux0 + L * M;
    const long long row0 = (long long)lb * L;
    const int Lc = (int)min((long long)L, d.nrows - row0);
    const bool spec_in = mode_from_spec(mode), spec_out = mode_to_spec(mode);
    if (!PK_SMEM_OK(d, sizeof(float2) * (tw_slots(M) + (odd ? 0 : M + 1) + padded_size(L * M) + L +
                                         (size_t)y_aux_arrays(mode) * L * M), 1) ||
        !PK_IN(d, row0 < d.nrows && Lc >= 1, 2))
        return;   // uniform over the CTA, before any barrier
    if constexpr (mode == Y_FINAL || mode == Y_RLFINAL) {
        if (d.crop && !rows_meet_box(d, row0, Lc)) return;   // none of these rows has a stored voxel
    }

    // ---- issue the asynchronous loads: group A = spectrum rows, group B = per-voxel inputs
    if (spec_in) {
        const int Pp = d.Pp;
        const float2* S0 = d.S + row0 * (long long)Pp;
        if (P > 0 && !odd) {
            // Py = M + 1: bins 0..M-1 of each row into the tile, bin M (Nyquist) aside
            for (int idx = tid; idx < Lc * M; idx += NT) {
                const int l = idx / M, k = idx - l * M;
                if (PK_IN(d, k < Pp, 11)) cp8(&buf[pad(idx)], S0 + l * Pp + k);
            }
            for (int l = tid; l < Lc; l += NT)
                if (PK_IN(d, M < Pp, 11)) cp8(&nyq[l], S0 + l * Pp + M);
        } else {
            const int nin = Lc * Py;
            for (int idx = tid; idx < nin; idx += NT) {
                const int l = idx / Py, k = idx - l * Py;
                if (!odd && k == M) cp8(&nyq[l], S0 + l * Pp + k);
                else cp8(&buf[pad(l * M + k)], S0 + l * Pp + k);
            }
        }
    }
    cp_commit();
    const float* pa0 = nullptr;
    const float* pa1 = nullptr;
    switch (mode) {
        case Y_R2C: pa0 = d.src; break;
        case Y_RATIO: pa0 = d.I; break;
        case Y_UPDATE: case Y_FINAL: pa0 = d.Jo; break;
        case Y_RLPRE: pa0 = d.J2; pa1 = d.J3; break;
        case Y_RLUPD: pa0 = d.Yb; pa1 = d.rl_first ? nullptr : d.J4; break;
        case Y_RLFINAL: pa0 = d.Yb; break;
        default: break;
    }
    const int nvox = Lc * M;
    const long long v0 = row0 * (long long)ny;
    const bool raw_sync = mode == Y_PRE && (d.padded || d.raw_type == PK_F64 || (d.raw_type == PK_U16 && odd));
    // 16-byte copies of two voxel pairs where rows, pairs and both buffers allow it (even ny divisible
    // by 4, even M, 16-byte aligned bases), else one pair per copy
    const bool wide_ok = !odd && M % 2 == 0 && ny % 4 == 0 && (reinterpret_cast<uintptr_t>(aux0) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(aux1) & 15) == 0;
    if (mode == Y_PRE && !raw_sync) {
        if (d.raw_type == PK_F32 && wide_ok && (reinterpret_cast<uintptr_t>(d.raw) & 15) == 0) {
            for (int idx = 2 * tid; idx < nvox; idx += 2 * NT) {
                const int l = idx / M, k = idx - l * M;
                cp16(&aux0[idx], (const float*)d.raw + v0 + (long long)l * ny + 2 * k);
            }
        } else {
            for (int idx = tid; idx < nvox; idx += NT) {
                const int l = idx / M, k = idx - l * M;
                const long long vi = v0 + (long long)l * ny + (odd ? k : 2 * k);
                if (d.raw_type == PK_U16) cp4(&aux0[idx], (const uint16_t*)d.raw + vi);
                else if (!odd) cp8(&aux0[idx], (const float*)d.raw + vi);
                else cp4(&aux0[idx], (const float*)d.raw + vi);
            }
        }
    } else if (pa0 && wide_ok && ((reinterpret_cast<uintptr_t>(pa0) | reinterpret_cast<uintptr_t>(pa1)) & 15) == 0) {
        for (int idx = 2 * tid; idx < nvox; idx += 2 * NT) {
            const int l = idx / M, k = idx - l * M;
            const long long vi = v0 + (long long)l * ny + 2 * k;
            if (!PK_IN(d, vi + 3 < d.nrows * (long long)ny, 12)) continue;
            cp16(&aux0[idx], pa0 + vi);
            if (pa1) cp16(&aux1[idx], pa1 + vi);
        }
    } else if (pa0) {
        for (int idx = tid; idx < nvox; idx += NT) {
            const int l = idx / M, k = idx - l * M;
            const long long vi = v0 + (long long)l * ny + (odd ? k : 2 * k);
            if (!odd) {
                cp8(&aux0[idx], pa0 + vi);
                if (pa1) cp8(&aux1[idx], pa1 + vi);
            } else {
                cp4(&aux0[idx], pa0 + vi);
                if (pa1) cp4(&aux1[idx], pa1 + vi);
            }
        }
    }
    cp_commit();
    // tables (plain loads; they stay in L2)
    for (int i = tid; i < (P == 0 ? M : plan_tw_size(P)); i += NT) tw[i] = A.tw[i];
    if (!odd)
        for (int i = tid; i <= M; i += NT) twrc[i] = d.tw_rc[i];
    double acc0 = 0.0, acc1 = 0.0;
    unsigned zeros = 0;
    const float lam = (mode == Y_RLPRE && d.lam_on) ? (float)d.partials[0] : 0.f;  // partials[0] = lambda

    if (spec_in) {
        cp_wait<1>();
        __syncthreads();
        // packed inverse sequence, in place: Z[k] = (X[k] + X*[M-k]) + i (X[k] - X*[M-k]) W_ny^{-k}
        if (!odd) {
            const int half = M / 2 + 1;
            const int np = Lc * half;
            for (int p = tid; p < np; p += NT) {
                const int l = p / half, k = p - l * half;
                const float2 xk = buf[pad(l * M + k)];
                const float2 xm = k == 0 ? nyq[l] : buf[pad(l * M + (M - k))];
                {
                    const float2 a = xk, b = conjf2(xm);
                    float2 w = twrc[k];
                    w.y = -w.y;
                    const float2 s2 = cadd(a, b), t2 = cmul(csub(a, b), w);
                    buf[pad(l * M + k)] = make_float2(s2.x - t2.y, s2.y + t2.x);
                }
                if (k != 0 && 2 * k != M) {
                    const float2 a = xm, b = conjf2(xk);
                    float2 w = twrc[M - k];
                    w.y = -w.y;
                    const float2 s2 = cadd(a, b), t2 = cmul(csub(a, b), w);
                    buf[pad(l * M + (M - k))] = make_float2(s2.x - t2.y, s2.y + t2.x);
                }
            }
        } else {
            const int nf = Lc * (ny - Py);
            for (int p = tid; p < nf; p += NT) {
                const int l = p / (ny - Py), k = Py + (p - l * (ny - Py));
                buf[pad(l * M + k)] = conjf2(buf[pad(l * M + (ny - k))]);
            }
        }
        __syncthreads();
    }

    bool fused = false;
    if constexpr (same_end_radix(P)) {
        // the common cases only: damping, scaling, masks, crops and the scalar raw path keep the rolled
        // per-voxel loop below, so their code is not unrolled into this one
        constexpr bool kPostMode = mode == Y_FINAL || mode == Y_RLFINAL;
        const bool fuse_ok = !odd && !(mode == Y_PRE && raw_sync) &&
                             !(kPostMode && (d.damp > 1.f || d.scale_mode != 0 || d.need_xz));
        if (fuse_ok) {
            // The inverse transform's last stage and the forward transform's first stage have the
            // same radix, so each thread holds the same elements after the one and before the
            // other: the per-voxel phase runs on registers between them.
            constexpr int N = kPlans[P].n, NST = kPlans[P].nst, R = kPlans[P].rad[0];
            constexpr int LL = plan_lines_y(N, TP), MS = N / R, MAXB = (LL * MS + NT - 1) / NT;
            float2 v[MAXB][R];
            if (spec_in) run_mid<P, 0, NST - 1, 1, LL, false, true>(buf, tw, tid);
            cp_wait<0>();
            __syncthreads();
            if (spec_in)
                stage_s2r<R, plan_ns_before(P, NST - 1), N, LL, false, true, stage_tw_off(P, NST - 1)>(buf, tw, tid, v);
            // phase 1: every value of the thread's elements, no global stores (so the descriptor
            // fields stay in registers); phase 2: the stores of the mode's per-voxel outputs
            constexpr bool kPost = kPostMode;
            // block-uniform settings read once
            const bool raw_u16 = d.raw_type == PK_U16;
            const unsigned bg16 = (unsigned)d.bg16;
            const float bgf = d.bg_f;
#pragma unroll
            for (int i = 0; i < MAXB; i++) {
                const int b = tid + i * NT;
                if (MAXB * NT == LL * MS || b < LL * MS) {
                    const int l = b / MS, j = b - l * MS;
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        const int e = j + r * MS;
                        float2 out = make_float2(0.f, 0.f);
                        if (l < Lc) {
                            const int idx = l * M + e;
                            const float2 c = spec_in ? v[i][r] : make_float2(0.f, 0.f);
                            const float2 a0 = pa0 || mode == Y_PRE ? aux0[idx] : make_float2(0.f, 0.f);
                            const float2 a1 = pa1 ? aux1[idx] : make_float2(0.f, 0.f);
                            if constexpr (mode == Y_PRE) {
                                out = pre_value(raw_u16, bg16, bgf, a0, zeros);
                            } else if constexpr (mode == Y_R2C) {
                                out = a0;
                            } else if constexpr (mode == Y_RATIO) {
                                out.x = __fdividef(a0.x, fmaxf(c.x, PK_EPS_F));
                                out.y = __fdividef(a0.y, fmaxf(c.y, PK_EPS_F));
                            } else if constexpr (mode == Y_UPDATE) {
                                out.x = fmaxf(__fmul_rn(c.x, a0.x), 0.f);
                                out.y = fmaxf(__fmul_rn(c.y, a0.y), 0.f);
                            } else if constexpr (kPost) {   // no damping, scaling or mask here
                                out.x = fmaxf(__fmul_rn(c.x, a0.x), 0.f);
                                out.y = fmaxf(__fmul_rn(c.y, a0.y), 0.f);
                            } else if constexpr (mode == Y_RLPRE) {
                                out.x = fmaxf(__fadd_rn(a0.x, __fmul_rn(lam, __fsub_rn(a0.x, a1.x))), 0.f);
                                out.y = fmaxf(__fadd_rn(a0.y, __fmul_rn(lam, __fsub_rn(a0.y, a1.y))), 0.f);
                            } else if constexpr (mode == Y_RLUPD) {
                                out.x = fmaxf(__fmul_rn(a0.x, c.x), 0.f);
                                out.y = fmaxf(__fmul_rn(a0.y, c.y), 0.f);
                                if (pa1) {   // not rl_first
                                    acc0 += (double)__fmul_rn(__fsub_rn(out.x, a0.x), a1.x);
                                    acc1 += (double)__fmul_rn(a1.x, a1.x);
                                    acc0 += (double)__fmul_rn(__fsub_rn(out.y, a0.y), a1.y);
                                    acc1 += (double)__fmul_rn(a1.y, a1.y);
                                }
                            } else if constexpr (mode == Y_C2R) {
                                out = c;
                            }
                        }
                        v[i][r] = out;
                    }
                }
            }
            if constexpr (mode != Y_RATIO && mode != Y_R2C) {
                float* p1 = nullptr;
                float* p2 = nullptr;
                uint8_t* mk = nullptr;
                if constexpr (mode == Y_PRE) { p1 = d.I; mk = d.write_mask ? d.mask8 : nullptr; }
                if constexpr (mode == Y_UPDATE) p1 = d.Jn;
                if constexpr (mode == Y_RLPRE) p1 = d.Yb;
                if constexpr (mode == Y_RLUPD) { p1 = d.J2n; p2 = d.J4; }
                if constexpr (mode == Y_C2R) p1 = d.dst;
                void* const o = kPost ? d.out : nullptr;   // no crop here: the output has the volume's layout
                const bool vec_out = kPost && ((reinterpret_cast<uintptr_t>(o) & (d.save16 ? 3 : 7)) == 0);
                const bool s16 = kPost && d.save16;
#pragma unroll
                for (int i = 0; i < MAXB; i++) {
                    const int b = tid + i * NT;
                    if (MAXB * NT == LL * MS || b < LL * MS) {
                        const int l = b / MS, j = b - l * MS;
                        if (l < Lc) {
                            const long long row = row0 + l;
#pragma unroll
                            for (int r = 0; r < R; r++) {
                                const int e = j + r * MS;
                                const long long vi = row * (long long)ny + 2 * e;
                                const float2 val = v[i][r];
                                if (!PK_IN(d, vi + 1 < d.nrows * (long long)ny, 13)) continue;
                                if constexpr (kPost) {
                                    if (vec_out) {
                                        if (s16) {
                                            const unsigned lo = (unsigned)u16_of(val.x), hi = (unsigned)u16_of(val.y);
                                            *reinterpret_cast<unsigned*>((uint16_t*)o + vi) = lo | (hi << 16);
                                        } else {
                                            *reinterpret_cast<float2*>((float*)o + vi) = val;
                                        }
                                    } else if (s16) {
                                        ((uint16_t*)o)[vi] = (uint16_t)u16_of(val.x);
                                        ((uint16_t*)o)[vi + 1] = (uint16_t)u16_of(val.y);
                                    } else {
                                        ((float*)o)[vi] = val.x;
                                        ((float*)o)[vi + 1] = val.y;
                                    }
                                } else {
                                    if (p1) *reinterpret_cast<float2*>(p1 + vi) = val;
                                    if constexpr (mode == Y_RLUPD) {
                                        const float2 a0 = aux0[l * M + e];
                                        *reinterpret_cast<float2*>(p2 + vi) =
                                            make_float2(__fsub_rn(val.x, a0.x), __fsub_rn(val.y, a0.y));
                                    }
                                    if constexpr (mode == Y_PRE) {
                                        if (mk) {
                                            const float2 a0 = aux0[l * M + e];
                                            unsigned m2;
                                            if (d.raw_type == PK_U16) {
                                                const ushort2 q = *reinterpret_cast<const ushort2*>(&a0);
                                                m2 = (q.x != 0 ? 1u : 0u) | (q.y != 0 ? 0x100u : 0u);
                                            } else {
                                                m2 = (a0.x != 0.f ? 1u : 0u) | (a0.y != 0.f ? 0x100u : 0u);
                                            }
                                            *reinterpret_cast<uint16_t*>(mk + vi) = (uint16_t)m2;
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
            }
            if (spec_out) {
                int tid2 = tid;  // opaque copy: the inverse's index arithmetic is not kept live for reuse
                asm volatile("mov.b32 %0, %0;" : "+r"(tid2));
                stage_r2s<R, N, LL, false, false>(buf, tid2, v);
                run_mid<P, 1, NST, R, LL, false, false>(buf, tw, tid2);
            }
            fused = true;
        }
    }
    if (!fused) {
    if (spec_in) fft_y<P, true, TP>(buf, A, tw, L, tid);
    cp_wait<0>();
    __syncthreads();

    // ---- per-voxel phase (descriptor fields in registers: the loop stores to the volume's arrays)
    const VoxFields f(d);
    for (int idx = tid; idx < nvox; idx += NT) {
        const int l = idx / M, k = idx - l * M;
        const long long row = row0 + l;
        const int y = odd ? k : 2 * k;
        float2 out;
        if (mode == Y_PRE) {
            out = pre_pair(f, raw_sync, odd, aux0[idx], row, y, zeros);
        } else {
            const float2 cval = spec_in ? buf[pad(idx)] : make_float2(0.f, 0.f);
            out = voxel_pair(f, mode, cval, pa0 ? aux0[idx] : make_float2(0.f, 0.f), pa1 ? aux1[idx] : make_float2(0.f, 0.f),
                             row, y, !odd, lam, acc0, acc1);
        }
        if (spec_out) buf[pad(idx)] = odd ? make_float2(out.x, 0.f) : out;
    }
    if (spec_out) {
        __syncthreads();
        fft_y<P, false, TP>(buf, A, tw, L, tid);
    }
    }

    if (spec_out) {
        const int nout = Lc * Py;
        const int Pp = d.Pp;
        float2* S0 = d.S + row0 * (long long)Pp;
        if (P > 0 && !odd) {
            // X[k] = (Z[k] + Z*[M-k]) / 2 + W^k (Z[k] - Z*[M-k]) / 2i for k < M; X[M] from Z[0]
            auto split = [&](int l, int k) {
                const float2 zk = buf[pad(l * M + k)];
                const float2 zc = conjf2(buf[pad(l * M + (k == 0 ? 0 : M - k))]);
                const float2 fe = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
                const float2 df = csub(zk, zc);
                const float2 fo = make_float2(0.5f * df.y, -0.5f * df.x);
                return cadd(fe, cmul(twrc[k], fo));
            };
            if (M % 2 == 0 && (reinterpret_cast<uintptr_t>(S0) & 15) == 0) {
                // two bins per thread, one 16-byte store (even M and row pitch keep the pairs aligned)
                for (int idx = 2 * tid; idx < Lc * M; idx += 2 * NT) {
                    const int l = idx / M, k = idx - l * M;
                    const float2 x0 = split(l, k), x1 = split(l, k + 1);
                    if (PK_IN(d, k + 1 < Pp, 14))
                        *reinterpret_cast<float4*>(S0 + l * Pp + k) = make_float4(x0.x, x0.y, x1.x, x1.y);
                }
            } else {
                for (int idx = tid; idx < Lc * M; idx += NT) {
                    const int l = idx / M, k = idx - l * M;
                    S0[l * Pp + k] = split(l, k);
                }
            }
            for (int l = tid; l < Lc; l += NT) {
                const float2 zk = buf[pad(l * M)];
                const float2 zc = conjf2(zk);
                const float2 fe = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
                const float2 df = csub(zk, zc);
                const float2 fo = make_float2(0.5f * df.y, -0.5f * df.x);
                S0[l * Pp + M] = cadd(fe, cmul(twrc[M], fo));
            }
        } else {
            for (int idx = tid; idx < nout; idx += NT) {
                const int l = idx / Py, k = idx - l * Py;
                float2 X;
                if (!odd) {
                    const float2 zk = buf[pad(l * M + (k == M ? 0 : k))];
                    const float2 zc = conjf2(buf[pad(l * M + (k == 0 ? 0 : M - k))]);
                    const float2 fe = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
                    const float2 df = csub(zk, zc);
                    const float2 fo = make_float2(0.5f * df.y, -0.5f * df.x);  // (zk - zc) / (2i)
                    X = cadd(fe, cmul(twrc[k], fo));
                } else {
                    X = buf[pad(l * M + k)];
                }
                S0[l * Pp + k] = X;
            }
        }
    }

    if (mode == Y_RLUPD) {
        // deterministic block reduction of the two lambda sums
        __shared__ double r0[NT], r1[NT];
        r0[tid] = acc0;
        r1[tid] = acc1;
        __syncthreads();
        for (int s = NT / 2; s > 0; s >>= 1) {
            if (tid < s) {
                r0[tid] += r0[tid + s];
                r1[tid] += r1[tid + s];
            }
            __syncthreads();
        }
        if (tid == 0) {
            d.partials[2 + 2 * lb] = r0[0];
            d.partials[3 + 2 * lb] = r1[0];
        }
    }
    if (mode == Y_PRE && d.zero_count) {
        __shared__ unsigned zc;
        if (tid == 0) zc = 0;
        __syncthreads();
        if (zeros) atomicAdd(&zc, zeros);
        __syncthreads();
        if (tid == 0 && zc) atomicAdd(d.zero_count, zc);
    }
}

// Tile of an x/z pass as seen by the register-IO stages: element e of column t is p[e*es + t];
// columns at or beyond ncol read as zero and are not stored.  The tables (twiddles, OTF tile)
// are staged into shared memory right after the first loads are issued.
struct XZTile {
    float2* p;             // S + tile origin
    long long es;          // element stride along the transformed axis
    int ncol;              // valid columns of the tile
#ifdef PK_CHECK
    long long lim;         // elements of S from p on (the checked build tests every access against it)
    int* chk;
#endif
    float sc;              // output scale (XZ_FWD_SCALE), else 1
    const float2* gtw;     // twiddle table (global)
    const float2* gh;      // OTF at the tile origin (XZ_CONV), else null
    float2* tw;            // shared twiddles
    float2* h;             // shared OTF tile
    int T, n, ntw, conj;
    __device__ __forceinline__ float2 ld(int l, int e) const {
#ifdef PK_CHECK
        if (l < ncol && !pk_check_in(chk, e * es + l < lim, 30)) return make_float2(0.f, 0.f);
#endif
        return l < ncol ? p[e * es + l] : make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void st(int l, int e, float2 v) const {
#ifdef PK_CHECK
        if (l < ncol && !pk_check_in(chk, e * es + l < lim, 31)) return;
#endif
        if (l < ncol) p[e * es + l] = make_float2(v.x * sc, v.y * sc);
    }
    __device__ __forceinline__ float2 otf(int l, int e) const {
        float2 v = h[e * T + l];
        if (conj) v.y = -v.y;
        return v;
    }
    __device__ __forceinline__ void after_loads() const {
        const int tid = threadIdx.x;
        if (gh) {
            if (T % 2 == 0 && n % 2 == 0) {   // column pairs, one 16-byte copy each: with even T, n, Pp and
                                              // column offsets, source and shared tile are 16-byte aligned
#pragma unroll 1
                for (int idx = 2 * tid; idx < T * n; idx += 2 * PK_THREADS) {
                    const int e = idx / T, t = idx - e * T;
                    if (t + 1 < ncol) cp16(&h[idx], gh + e * es + t);
                    else if (t < ncol) cp8(&h[idx], gh + e * es + t);
                }
            } else {
#pragma unroll 1
                for (int idx = tid; idx < T * n; idx += PK_THREADS) {
                    const int e = idx / T, t = idx - e * T;
                    if (t < ncol) cp8(&h[idx], gh + e * es + t);
                }
            }
            cp_commit();
        }
#pragma unroll 1
        for (int i = tid; i < ntw; i += PK_THREADS) tw[i] = gtw[i];
    }
    __device__ __forceinline__ void before_last() const {
        cp_wait<0>();
        __syncthreads();
    }
    // Copy whose address fields the compiler cannot see through, so address arithmetic of a later
    // transform is not hoisted into (and kept live across) an earlier one.
    __device__ __forceinline__ XZTile fenced() const {
        XZTile r = *this;
        asm volatile("mov.b64 %0, %0;" : "+l"(r.p));
        asm volatile("mov.b64 %0, %0;" : "+l"(r.es));
        asm volatile("mov.b32 %0, %0;" : "+r"(r.ncol));
        return r;
    }
};

// CTAs per SM the x/z kernel of plan P is compiled for: 4 (64 registers) for length 512, where that
// measured faster, else 3 (80 registers; 1024 and 2048 measured slower at 4).
constexpr int xz_min_blocks(int p) {
    return p > 0 && kPlans[p].n == 512 ? 4 : 3;
}

template <int P, int TP = PK_TILE_POINTS>
__global__ void __launch_bounds__(PK_THREADS, xz_min_blocks(P)) k_xz(const VolDesc* __restrict__ descs, const int* __restrict__ prefix,
                                                      int nvol, int axis, int mode) {
    extern __shared__ float2 smem[];
    constexpr int NT = PK_THREADS;
    const int vol = find_vol(prefix, nvol, blockIdx.x);
    const VolDesc& d = descs[vol];
    const int lb = blockIdx.x - prefix[vol];
    const int tid = threadIdx.x;
    const AxisDev& A = axis == 1 ? d.ax : d.az;
    const int n = P == 0 ? A.n : kPlans[P].n;
    const int T = P == 0 ? (axis == 1 ? d.Tx : d.Tz) : plan_cols_xz(kPlans[P].n, TP);
    const int Py = d.Py;
    const int ctiles = (Py + T - 1) / T;
    const int outer = lb / ctiles;
    const int k0 = (lb - outer * ctiles) * T;
    long long base, es;
    if (axis == 1) { base = (long long)outer * d.nx * d.Pp; es = d.Pp; }
    else { base = (long long)outer * d.Pp; es = (long long)d.nx * d.Pp; }
    // shared memory: tw[tw_slots(n)] | buf[padded T*n, rounded up to even] | otf[T*n] (XZ_CONV)
    float2* tw = smem;
    float2* buf = smem + tw_slots(n);
    float2* hbuf = buf + padded_size2(T * n);   // 16-byte aligned: the OTF tile takes 16-byte copies
    const int P_ = T * n;
    const bool conv = mode == XZ_CONV;
    if constexpr (P > 0 && kPlans[P].nst >= 2) {
        // first stage loads from HBM into registers, last stage stores from registers to HBM; the
        // OTF multiply runs inside the last forward stage
        constexpr int TT = plan_cols_xz(kPlans[P].n, TP);
#ifdef PK_CHECK
        if (!PK_SMEM_OK(d, sizeof(float2) * (tw_slots(n) + padded_size2(TT * n) + (conv ? TT * n : 0)), 3)) return;
        const XZTile g{d.S + base + k0, es, Py - k0, d.Pp * d.nrows - (base + k0), d.chk,
                       mode == XZ_FWD_SCALE ? d.xz_scale : 1.f, A.tw, conv ? d.otf + base + k0 : nullptr, tw, hbuf, TT,
                       kPlans[P].n, plan_tw_size(P), d.conj};
#else
        const XZTile g{d.S + base + k0, es, Py - k0, mode == XZ_FWD_SCALE ? d.xz_scale : 1.f, A.tw,
                       conv ? d.otf + base + k0 : nullptr, tw, hbuf, TT, kPlans[P].n, plan_tw_size(P), d.conj};
#endif
        if (mode == XZ_INV) fft_g<P, TT, true, true, false, true>(buf, tw, g, tid);
        else if (!conv) fft_g<P, TT, true, false, false, true>(buf, tw, g, tid);
        else if constexpr (same_end_radix(P)) {
            // first and last radix agree: the forward transform's last stage leaves each thread the
            // elements the inverse transform's first stage needs, so the OTF multiply runs on registers
            // between them
            constexpr int N = kPlans[P].n, NST = kPlans[P].nst, R = kPlans[P].rad[0];
            constexpr int MS = N / R, MAXB = (TT * MS + NT - 1) / NT;
            float2 v[MAXB][R];
            stage_g2s<R, N, TT, true, false>(buf, g, tid);
            run_mid<P, 1, NST - 1, R, TT, true, false>(buf, tw, tid);
            g.before_last();
            stage_s2r<R, plan_ns_before(P, NST - 1), N, TT, true, false, stage_tw_off(P, NST - 1)>(buf, tw, tid, v);
#pragma unroll
            for (int i = 0; i < MAXB; i++) {
                const int b = tid + i * NT;
                if (MAXB * NT == TT * MS || b < TT * MS) {
                    const int l = b % TT, j = b / TT;
#pragma unroll
                    for (int r = 0; r < R; r++) v[i][r] = cmul(v[i][r], g.otf(l, j + r * MS));
                }
            }
            int tid2 = tid;  // opaque copy: keeps the forward's index arithmetic from being reused here
            asm volatile("mov.b32 %0, %0;" : "+r"(tid2));
            stage_r2s<R, N, TT, true, true>(buf, tid2, v);
            run_mid<P, 1, NST - 1, R, TT, true, true>(buf, tw, tid2);
            stage_s2x<kPlans[P].rad[NST - 1], plan_ns_before(P, NST - 1), N, TT, true, true, stage_tw_off(P, NST - 1),
                      false, true>(buf, tw, g.fenced(), tid2);
        } else {
            fft_g<P, TT, true, false, true, false>(buf, tw, g, tid);
            int tid2 = tid;  // opaque copy: keeps the forward's index arithmetic from being reused here
            asm volatile("mov.b32 %0, %0;" : "+r"(tid2));
            fft_s2g<P, TT, true, true>(buf, tw, g.fenced(), tid2);
        }
    } else {
        for (int idx = tid; idx < P_; idx += NT) {
            const int e = idx / T, t = idx - e * T;
            if (k0 + t < Py) cp8(&buf[pad(idx)], d.S + base + e * es + k0 + t);
            else buf[pad(idx)] = make_float2(0.f, 0.f);
        }
        cp_commit();
        if (conv) {
            for (int idx = tid; idx < P_; idx += NT) {
                const int e = idx / T, t = idx - e * T;
                if (k0 + t < Py) cp8(&hbuf[idx], d.otf + base + e * es + k0 + t);
            }
        }
        cp_commit();
        for (int i = tid; i < (P == 0 ? n : plan_tw_size(P)); i += NT) tw[i] = A.tw[i];
        cp_wait<1>();
        __syncthreads();
        if (mode == XZ_INV) fft_xz<P, true, TP>(buf, A, tw, T, tid);
        else fft_xz<P, false, TP>(buf, A, tw, T, tid);
        if (conv) {
            cp_wait<0>();
            __syncthreads();
            const bool cj = d.conj;
            for (int idx = tid; idx < P_; idx += NT) {
                const int t = idx % T;
                if (k0 + t < Py) {
                    float2 hv = hbuf[idx];
                    if (cj) hv.y = -hv.y;
                    buf[pad(idx)] = cmul(buf[pad(idx)], hv);
                }
            }
            __syncthreads();
            fft_xz<P, true, TP>(buf, A, tw, T, tid);
        }
        const float sc = mode == XZ_FWD_SCALE ? d.xz_scale : 1.f;
        for (int idx = tid; idx < P_; idx += NT) {
            const int e = idx / T, t = idx - e * T;
            if (k0 + t < Py) {
                float2 v = buf[pad(idx)];
                if (mode == XZ_FWD_SCALE) v = make_float2(v.x * sc, v.y * sc);
                d.S[base + e * es + k0 + t] = v;
            }
        }
    }
}

constexpr int kYModes = Y_C2R + 1;

// Entries [0, kNumPlans) hold the 4096-point-tile kernels, [kNumPlans + p] the small-tile kernels
// of plan p (small_tile_plan(p)); a program step's plan id carries that offset.
struct KernelTable {
    void (*y[2 * kNumPlans][kYModes])(const VolDesc*, const int*, int, int);
    void (*xz[2 * kNumPlans])(const VolDesc*, const int*, int, int, int);
};

template <int P, int MD>
struct RegisterY {
    static void fill(KernelTable& t) {
        t.y[P][MD] = k_y<P, MD>;
        cudaFuncSetAttribute(k_y<P, MD>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if constexpr (small_tile_plan(P)) {
            t.y[kNumPlans + P][MD] = k_y<P, MD, PK_TILE_SMALL>;
            cudaFuncSetAttribute(k_y<P, MD, PK_TILE_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        }
        RegisterY<P, MD + 1>::fill(t);
    }
};
template <int P>
struct RegisterY<P, kYModes> {
    static void fill(KernelTable&) {}
};

template <int P, int HI>
struct Register {
    static void fill(KernelTable& t) {
        RegisterY<P, 0>::fill(t);
        t.xz[P] = k_xz<P>;
        cudaFuncSetAttribute(k_xz<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if constexpr (small_tile_plan(P)) {
            t.xz[kNumPlans + P] = k_xz<P, PK_TILE_SMALL>;
            cudaFuncSetAttribute(k_xz<P, PK_TILE_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        }
        Register<P + 1, HI>::fill(t);
    }
};
template <int HI>
struct Register<HI, HI> {
    static void fill(KernelTable&) {}
};

}  // namespace pkpass
