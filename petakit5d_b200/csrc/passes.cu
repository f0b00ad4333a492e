// Pass kernels of the 3D real transform with the RL / OMW per-voxel arithmetic folded in.
//
// y pass   (k_ypass<MODE>): one CTA = Ly consecutive rows (contiguous in HBM).  Forward: real row
//          -> length-ny/2 complex FFT -> split into the ny/2+1 half-spectrum bins.  Inverse: the
//          reverse, then the mode's per-voxel epilogue; modes that continue into the next
//          convolution transform the epilogue's output straight back, so a row makes one HBM
//          round trip between the two convolutions of an iteration.
// x/z pass (k_xzpass<MODE>): one CTA = T adjacent spectrum columns k along a full x (or z) line;
//          XZ_CONV runs forward FFT, OTF multiply and inverse FFT on the tile in shared memory.
// Every launch covers a list of volumes (descriptors + block prefix), so the batched and served
// paths reuse the same kernels as the single-volume call.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fft_engine.cuh"
#include "pk_internal.h"

using namespace pkfft;

#define PK_EPS_F 2.220446049250313e-16f  // single(eps) = 2^-52

namespace {

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

// post-processing of one voxel (decon_lucy_omw_function.m:146-177)
__device__ __forceinline__ void post_store(const VolDesc& d, float J, long long row, int y) {
    const int x = (int)(row % d.nx);
    const int z = (int)(row / d.nx);
    if (y < d.bb0[0] || y > d.bb1[0] || x < d.bb0[1] || x > d.bb1[1] || z < d.bb0[2] || z > d.bb1[2]) return;
    const long long vi = row * d.ny + y;
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
            m = d.mask8[vi] != 0 && y >= E && y < d.ny - E && x >= E && x < d.nx - E && z >= E && z < d.nz - E;
        }
        J = __fmul_rn(__fadd_rn(__fmul_rn(J, d.scale), d.offset), (float)m);
    }
    const long long oy = d.bb1[0] - d.bb0[0] + 1, ox = d.bb1[1] - d.bb0[1] + 1;
    const long long oi = (long long)(y - d.bb0[0]) + oy * ((long long)(x - d.bb0[1]) + ox * (long long)(z - d.bb0[2]));
    if (d.save16) ((uint16_t*)d.out)[oi] = (uint16_t)u16_of(J);
    else ((float*)d.out)[oi] = J;
}

template <int MODE>
struct YTraits {
    static constexpr bool from_spec = MODE == Y_RATIO || MODE == Y_UPDATE || MODE == Y_FINAL || MODE == Y_RLUPD ||
                                      MODE == Y_RLFINAL || MODE == Y_C2R;
    static constexpr bool to_spec = MODE == Y_R2C || MODE == Y_PRE || MODE == Y_RATIO || MODE == Y_UPDATE || MODE == Y_RLPRE;
};

// Per-voxel operation of the mode.  v: value at (row, y) after the inverse transform (scaled to the
// convolution) or the raw-source value; returns the value the forward transform consumes.
template <int MODE>
__device__ __forceinline__ float voxel_op(const VolDesc& d, float v, long long row, int y, float lam, double& acc0,
                                          double& acc1, unsigned& zeros) {
    const long long vi = row * d.ny + y;
    if constexpr (MODE == Y_R2C) {
        return d.src[vi];
    } else if constexpr (MODE == Y_PRE) {
        float I;
        bool nz;
        if (d.raw_type == PK_U16) {
            const unsigned r = ((const uint16_t*)d.raw)[vi];
            nz = r != 0;
            I = r > (unsigned)d.bg16 ? (float)(r - (unsigned)d.bg16) : 0.f;
        } else if (d.raw_type == PK_F32) {
            const float r = ((const float*)d.raw)[vi];
            nz = r != 0.f;
            I = fmaxf(__fsub_rn(r, d.bg_f), 0.f);
        } else {
            const float r = (float)((const double*)d.raw)[vi];
            nz = ((const double*)d.raw)[vi] != 0.0;
            I = fmaxf(__fsub_rn(r, d.bg_f), 0.f);
        }
        d.I[vi] = I;
        if (d.write_mask) d.mask8[vi] = nz ? 1 : 0;
        zeros += nz ? 0u : 1u;
        return I;
    } else if constexpr (MODE == Y_RATIO) {
        return __fdiv_rn(d.I[vi], fmaxf(v, PK_EPS_F));
    } else if constexpr (MODE == Y_UPDATE) {
        const float j = fmaxf(__fmul_rn(v, d.Jo[vi]), 0.f);
        d.Jn[vi] = j;
        return j;
    } else if constexpr (MODE == Y_FINAL) {
        post_store(d, fmaxf(__fmul_rn(v, d.Jo[vi]), 0.f), row, y);
        return 0.f;
    } else if constexpr (MODE == Y_RLPRE) {
        const float j2 = d.J2[vi], j3 = d.J3[vi];
        const float yv = fmaxf(__fadd_rn(j2, __fmul_rn(lam, __fsub_rn(j2, j3))), 0.f);
        d.Yb[vi] = yv;
        return yv;
    } else if constexpr (MODE == Y_RLUPD) {
        const float yv = d.Yb[vi];
        const float j2n = fmaxf(__fmul_rn(yv, v), 0.f);
        const float diff = __fsub_rn(j2n, yv);
        if (!d.rl_first) {
            const float j4 = d.J4[vi];
            acc0 += (double)__fmul_rn(diff, j4);
            acc1 += (double)__fmul_rn(j4, j4);
        }
        d.J4[vi] = diff;
        d.J2n[vi] = j2n;
        return 0.f;
    } else if constexpr (MODE == Y_RLFINAL) {
        post_store(d, fmaxf(__fmul_rn(d.Yb[vi], v), 0.f), row, y);
        return 0.f;
    } else {  // Y_C2R
        d.dst[vi] = v;
        return 0.f;
    }
}

template <int MODE>
__global__ void __launch_bounds__(512) k_ypass(const VolDesc* __restrict__ descs, const int* __restrict__ prefix,
                                               int nvol) {
    extern __shared__ float2 smem[];
    const int vol = find_vol(prefix, nvol, blockIdx.x);
    const VolDesc& d = descs[vol];
    const int lb = blockIdx.x - prefix[vol];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const AxisDev& A = d.ay;
    float2* tw = smem;
    for (int i = tid; i < A.twN; i += nthr) tw[i] = A.tw[i];
    float2* buf = smem + A.twN;
    const long long row0 = (long long)lb * d.Ly;
    const int Lc = (int)min((long long)d.Ly, d.nrows - row0);
    const int M = d.M, Py = d.Py, ny = d.ny;
    const int npts = Lc * M;
    TileGeom g{Lc, M, M, 1, false};
    float lam = 0.f;
    if constexpr (MODE == Y_RLPRE) lam = d.lam_on ? (float)(*d.partials) : 0.f;  // partials[0] holds lambda
    double acc0 = 0.0, acc1 = 0.0;
    unsigned zeros = 0;
    __syncthreads();

    if constexpr (YTraits<MODE>::from_spec) {
        // gather the half spectrum into the length-M complex sequence of the packed inverse
        for (int idx = tid; idx < npts; idx += nthr) {
            const int l = idx / M, k = idx - l * M;
            const float2* Srow = d.S + (row0 + l) * (long long)Py;
            float2 Z;
            if (!d.odd) {
                const float2 a = Srow[k], b = conjf2(Srow[M - k]);
                float2 w = tw[k];
                w.y = -w.y;  // W_N^{-k}
                const float2 s = cadd(a, b);
                const float2 t = cmul(csub(a, b), w);
                Z = make_float2(s.x - t.y, s.y + t.x);  // s + i t
            } else {
                Z = k < Py ? Srow[k] : conjf2(Srow[ny - k]);
            }
            buf[pad(l * M + k)] = Z;
        }
        __syncthreads();
        fft_lines<true>(buf, A, tw, g, tid, nthr);
        for (int idx = tid; idx < npts; idx += nthr) {
            const int l = idx / M, k = idx - l * M;
            const long long row = row0 + l;
            float2 z = buf[pad(l * M + k)];
            if (!d.odd) {
                z.x = voxel_op<MODE>(d, z.x, row, 2 * k, lam, acc0, acc1, zeros);
                z.y = voxel_op<MODE>(d, z.y, row, 2 * k + 1, lam, acc0, acc1, zeros);
            } else {
                z.x = voxel_op<MODE>(d, z.x, row, k, lam, acc0, acc1, zeros);
                z.y = 0.f;
            }
            if constexpr (YTraits<MODE>::to_spec) buf[pad(l * M + k)] = z;
        }
    } else {
        for (int idx = tid; idx < npts; idx += nthr) {
            const int l = idx / M, k = idx - l * M;
            const long long row = row0 + l;
            float2 z;
            if (!d.odd) {
                z.x = voxel_op<MODE>(d, 0.f, row, 2 * k, lam, acc0, acc1, zeros);
                z.y = voxel_op<MODE>(d, 0.f, row, 2 * k + 1, lam, acc0, acc1, zeros);
            } else {
                z.x = voxel_op<MODE>(d, 0.f, row, k, lam, acc0, acc1, zeros);
                z.y = 0.f;
            }
            buf[pad(l * M + k)] = z;
        }
    }

    if constexpr (YTraits<MODE>::to_spec) {
        __syncthreads();
        fft_lines<false>(buf, A, tw, g, tid, nthr);
        const int nout = Lc * Py;
        for (int idx = tid; idx < nout; idx += nthr) {
            const int l = idx / Py, k = idx - l * Py;
            float2 X;
            if (!d.odd) {
                const float2 zk = buf[pad(l * M + (k == M ? 0 : k))];
                const float2 zc = conjf2(buf[pad(l * M + (k == 0 ? 0 : M - k))]);
                const float2 fe = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
                const float2 df = csub(zk, zc);
                const float2 fo = make_float2(0.5f * df.y, -0.5f * df.x);  // (zk - zc) / (2i)
                X = cadd(fe, cmul(tw[k], fo));
            } else {
                X = buf[pad(l * M + k)];
            }
            d.S[(row0 + l) * (long long)Py + k] = X;
        }
    }

    if constexpr (MODE == Y_RLUPD) {
        // deterministic block reduction of the two lambda sums
        __shared__ double r0[512], r1[512];
        r0[tid] = acc0;
        r1[tid] = acc1;
        __syncthreads();
        for (int s = 256; s > 0; s >>= 1) {
            if (tid < s && tid + s < nthr) {
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
    if constexpr (MODE == Y_PRE) {
        if (d.zero_count) {
            __shared__ unsigned zc;
            if (tid == 0) zc = 0;
            __syncthreads();
            if (zeros) atomicAdd(&zc, zeros);
            __syncthreads();
            if (tid == 0 && zc) atomicAdd(d.zero_count, zc);
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(512) k_xzpass(const VolDesc* __restrict__ descs, const int* __restrict__ prefix,
                                                int nvol, int axis) {
    extern __shared__ float2 smem[];
    const int vol = find_vol(prefix, nvol, blockIdx.x);
    const VolDesc& d = descs[vol];
    const int lb = blockIdx.x - prefix[vol];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const AxisDev& A = axis == 1 ? d.ax : d.az;
    const int T = axis == 1 ? d.Tx : d.Tz;
    const int Py = d.Py;
    const int ctiles = (Py + T - 1) / T;
    const int outer = lb / ctiles;
    const int k0 = (lb - outer * ctiles) * T;
    long long base, es;
    if (axis == 1) { base = (long long)outer * d.nx * Py; es = Py; }
    else { base = (long long)outer * Py; es = (long long)d.nx * Py; }
    float2* tw = smem;
    for (int i = tid; i < A.twN; i += nthr) tw[i] = A.tw[i];
    float2* buf = smem + A.twN;
    const int n = A.n;
    const int P = T * n;
    for (int idx = tid; idx < P; idx += nthr) {
        const int e = idx / T, t = idx - e * T;
        const int k = k0 + t;
        buf[pad(idx)] = k < Py ? d.S[base + e * es + k] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    TileGeom g{T, n, 1, T, true};
    if constexpr (MODE == XZ_INV) fft_lines<true>(buf, A, tw, g, tid, nthr);
    else fft_lines<false>(buf, A, tw, g, tid, nthr);
    if constexpr (MODE == XZ_CONV) {
        for (int idx = tid; idx < P; idx += nthr) {
            const int e = idx / T, t = idx - e * T;
            const int k = k0 + t;
            if (k < Py) {
                float2 h = d.otf[base + e * es + k];
                if (d.conj) h.y = -h.y;
                buf[pad(idx)] = cmul(buf[pad(idx)], h);
            }
        }
        __syncthreads();
        fft_lines<true>(buf, A, tw, g, tid, nthr);
    }
    for (int idx = tid; idx < P; idx += nthr) {
        const int e = idx / T, t = idx - e * T;
        const int k = k0 + t;
        if (k < Py) {
            float2 v = buf[pad(idx)];
            if constexpr (MODE == XZ_FWD_SCALE) v = make_float2(v.x * d.xz_scale, v.y * d.xz_scale);
            d.S[base + e * es + k] = v;
        }
    }
}

// lambda = clamp(sum((J2-Y).*J4) / (sum(J4.*J4) + eps), 0, 1)  (decon_lucy_function.m:126-127),
// one CTA per volume, fixed summation order; the result goes to partials[0].
__global__ void k_lambda(const VolDesc* __restrict__ descs, int nvol) {
    const VolDesc& d = descs[blockIdx.x];
    __shared__ double s0[256], s1[256];
    const int tid = threadIdx.x;
    double a = 0.0, b = 0.0;
    for (int i = tid; i < d.blocksY; i += blockDim.x) {
        a += d.partials[2 + 2 * i];
        b += d.partials[3 + 2 * i];
    }
    s0[tid] = a;
    s1[tid] = b;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (tid < s) {
            s0[tid] += s0[tid + s];
            s1[tid] += s1[tid + s];
        }
        __syncthreads();
    }
    if (tid == 0) {
        double lam = s0[0] / (s1[0] + 2.220446049250313e-16);
        lam = fmax(fmin(lam, 1.0), 0.0);
        d.partials[0] = lam;
    }
}

}  // namespace

// ------------------------------------------------------------------ host: plans and tables
bool pk_make_axis_plan(int n, AxisPlan* p) {
    p->n = n;
    p->nst = 0;
    if (n < 1) return false;
    int r = n;
    auto push = [&](int R) {
        if (p->nst >= PK_MAXST) return false;
        p->rad[p->nst++] = R;
        r /= R;
        return true;
    };
    while (r % 16 == 0) if (!push(16)) return false;
    if (r % 8 == 0) { if (!push(8)) return false; }
    else if (r % 4 == 0) { if (!push(4)) return false; }
    else if (r % 2 == 0) { if (!push(2)) return false; }
    while (r % 5 == 0) if (!push(5)) return false;
    while (r % 3 == 0) if (!push(3)) return false;
    for (int f = 7; r > 1; f += 2) {
        while (r % f == 0) if (!push(f)) return false;
        if ((long long)f * f > r && r > 1) { if (!push(r)) return false; }
    }
    return true;
}

pk_status pk_get_twiddles(pk_ctx* ctx, int twN, const float2** out) {
    auto it = ctx->tw.find(twN);
    if (it != ctx->tw.end()) { *out = it->second.d; return PK_OK; }
    std::vector<float2> h(twN);
    for (int k = 0; k < twN; k++) {
        // exact for the multiples of pi/2 so symmetric bins stay symmetric
        const double a = -2.0 * M_PI * (double)k / (double)twN;
        double c = std::cos(a), s = std::sin(a);
        if ((4LL * k) % twN == 0) {
            const int q = (int)((4LL * k) / twN) & 3;
            c = q == 0 ? 1 : q == 2 ? -1 : 0;
            s = q == 1 ? -1 : q == 3 ? 1 : 0;
        }
        h[k] = make_float2((float)c, (float)s);
    }
    TwTable t;
    t.n = twN;
    PK_CUDA(cudaMalloc(&t.d, sizeof(float2) * twN));
    PK_CUDA(cudaMemcpy(t.d, h.data(), sizeof(float2) * twN, cudaMemcpyHostToDevice));
    ctx->tw[twN] = t;
    *out = t.d;
    return PK_OK;
}

pk_status pk_fill_axis(pk_ctx* ctx, int n, int twN, AxisDev* a) {
    AxisPlan p;
    if (!pk_make_axis_plan(n, &p)) return pk_fail(PK_ERR_UNSUPPORTED, "transform length " + std::to_string(n) + " needs too many radix stages");
    memset(a, 0, sizeof(*a));
    a->n = n;
    a->nst = p.nst;
    for (int i = 0; i < p.nst; i++) a->rad[i] = p.rad[i];
    a->twN = twN;
    a->twStride = twN / n;
    return pk_get_twiddles(ctx, twN, &a->tw);
}

static const int kThreads = 256;

pk_status pk_init_desc(pk_ctx* ctx, int ny, int nx, int nz, VolDesc* d) {
    memset(d, 0, sizeof(*d));
    if (ny < 1 || nx < 1 || nz < 1) return pk_fail(PK_ERR_INVALID, "volume dimensions must be positive");
    d->ny = ny; d->nx = nx; d->nz = nz;
    d->odd = ny & 1;
    d->M = d->odd ? ny : ny / 2;
    d->Py = ny / 2 + 1;
    d->nrows = (long long)nx * nz;
    const int P = PK_PPT * kThreads;  // complex points one CTA holds
    if (d->M > P || nx > P || nz > P)
        return pk_fail(PK_ERR_UNSUPPORTED, "a transform axis is longer than " + std::to_string(P) +
                                               " (" + std::to_string(2 * P) + " along y)");
    d->Ly = (int)std::max(1, P / d->M);
    if ((long long)d->Ly > d->nrows) d->Ly = (int)d->nrows;
    d->Tx = std::max(1, std::min(P / nx, d->Py));
    d->Tz = std::max(1, std::min(P / nz, d->Py));
    const int ct_x = (d->Py + d->Tx - 1) / d->Tx, ct_z = (d->Py + d->Tz - 1) / d->Tz;
    d->blocksY = (int)((d->nrows + d->Ly - 1) / d->Ly);
    d->blocksX = nz * ct_x;
    d->blocksZ = nx * ct_z;
    pk_status st;
    if ((st = pk_fill_axis(ctx, d->M, d->odd ? ny : ny, &d->ay)) != PK_OK) return st;
    if ((st = pk_fill_axis(ctx, nx, nx, &d->ax)) != PK_OK) return st;
    if ((st = pk_fill_axis(ctx, nz, nz, &d->az)) != PK_OK) return st;
    d->bb0[0] = d->bb0[1] = d->bb0[2] = 0;
    d->bb1[0] = ny - 1; d->bb1[1] = nx - 1; d->bb1[2] = nz - 1;
    d->scale = 1.f;
    d->xz_scale = 1.f;
    return PK_OK;
}

size_t pk_spec_elems(const VolDesc& d) { return (size_t)d.Py * (size_t)d.nrows; }

// ------------------------------------------------------------------ programs
// A program is the full launch sequence of a call (or of a batch / serving round): every step's
// descriptors and block prefix live in one device buffer uploaded once, so the launches run
// back to back without host synchronisation and can be captured into a CUDA graph.
template <int MODE>
static void launch_y_mode(int grid, size_t smem, const VolDesc* dd, const int* dp, int nvol, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_ypass<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    k_ypass<MODE><<<grid, kThreads, smem, st>>>(dd, dp, nvol);
}

template <int MODE>
static void launch_xz_mode(int grid, size_t smem, const VolDesc* dd, const int* dp, int nvol, int axis, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_xzpass<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    k_xzpass<MODE><<<grid, kThreads, smem, st>>>(dd, dp, nvol, axis);
}

void pk_program_add(PkProgram& prog, int kind, int mode, const std::vector<VolDesc>& vols) {
    PkStep s;
    s.kind = kind;
    s.mode = mode;
    s.nvol = (int)vols.size();
    s.desc_off = (int)prog.descs.size();
    s.prefix_off = (int)prog.prefix.size();
    prog.prefix.push_back(0);
    size_t smem = 0;
    for (const VolDesc& v : vols) {
        int blocks = 0;
        if (kind == PK_STEP_Y) {
            blocks = v.blocksY;
            smem = std::max(smem, sizeof(float2) * (v.ay.twN + padded_size(v.Ly * v.M)));
        } else if (kind == PK_STEP_X) {
            blocks = v.blocksX;
            smem = std::max(smem, sizeof(float2) * (v.ax.twN + padded_size(v.Tx * v.ax.n)));
        } else if (kind == PK_STEP_Z) {
            blocks = v.blocksZ;
            smem = std::max(smem, sizeof(float2) * (v.az.twN + padded_size(v.Tz * v.az.n)));
        } else {
            blocks = 1;
        }
        prog.prefix.push_back(prog.prefix.back() + blocks);
        prog.descs.push_back(v);
    }
    s.grid = prog.prefix.back();
    s.smem = smem;
    prog.steps.push_back(s);
}

pk_status pk_program_upload(pk_ctx* ctx, PkProgram& prog, cudaStream_t st) {
    const size_t dbytes = sizeof(VolDesc) * prog.descs.size();
    const size_t pbytes = sizeof(int) * prog.prefix.size();
    const size_t need = dbytes + pbytes;
    const int si = ctx->next_slot;
    ctx->next_slot = (ctx->next_slot + 1) % 4;
    pk_ctx::ProgSlot& sl = ctx->slots[si];
    if (sl.used) PK_CUDA(cudaEventSynchronize(sl.ev));   // launches that read this slot are done
    sl.used = false;
    if (!sl.ev) PK_CUDA(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
    if (sl.cap < need) {
        if (sl.d) cudaFree(sl.d);
        if (sl.h) cudaFreeHost(sl.h);
        sl.d = sl.h = nullptr;
        sl.cap = 0;
        const size_t cap = std::max(need, (size_t)64 * 1024);
        PK_CUDA(cudaMalloc(&sl.d, cap));
        PK_CUDA(cudaMallocHost(&sl.h, cap));
        sl.cap = cap;
    }
    memcpy(sl.h, prog.descs.data(), dbytes);
    memcpy((char*)sl.h + dbytes, prog.prefix.data(), pbytes);
    PK_CUDA(cudaMemcpyAsync(sl.d, sl.h, need, cudaMemcpyHostToDevice, st));
    prog.d_desc = (VolDesc*)sl.d;
    prog.d_prefix = (int*)((char*)sl.d + dbytes);
    prog.slot = si;
    return PK_OK;
}

const char* pk_step_name(const PkStep& s) {
    static const char* yn[] = {"y_r2c", "y_pre", "y_ratio", "y_update", "y_final", "y_rlpre", "y_rlupd", "y_rlfinal", "y_c2r"};
    static const char* xn[] = {"x_fwd", "x_inv", "x_conv", "x_fwd_scale"};
    static const char* zn[] = {"z_fwd", "z_inv", "z_conv", "z_fwd_scale"};
    if (s.kind == PK_STEP_Y) return yn[s.mode];
    if (s.kind == PK_STEP_X) return xn[s.mode];
    if (s.kind == PK_STEP_Z) return zn[s.mode];
    return "lambda";
}

// Algorithmic HBM bytes of one launch: the minimum each pass must read and write.
double pk_step_bytes(const PkStep& s, const VolDesc* descs) {
    double b = 0;
    for (int i = 0; i < s.nvol; i++) {
        const VolDesc& d = descs[i];
        const double N = (double)d.nrows * d.ny, Sb = 8.0 * d.Py * (double)d.nrows;
        const double ob = (double)(d.bb1[0] - d.bb0[0] + 1) * (d.bb1[1] - d.bb0[1] + 1) * (d.bb1[2] - d.bb0[2] + 1) * (d.save16 ? 2 : 4);
        if (s.kind == PK_STEP_Y) {
            switch (s.mode) {
                case Y_R2C: b += 4 * N + Sb; break;
                case Y_PRE: b += (d.raw_type == PK_U16 ? 2 : d.raw_type == PK_F32 ? 4 : 8) * N + 4 * N + Sb + (d.write_mask ? N : 0); break;
                case Y_RATIO: b += 2 * Sb + 4 * N; break;
                case Y_UPDATE: b += 2 * Sb + 8 * N; break;
                case Y_FINAL: b += Sb + 4 * N + (d.damp > 1.f ? 4 * N : 0) + ob; break;
                case Y_RLPRE: b += 12 * N + Sb; break;
                case Y_RLUPD: b += Sb + (d.rl_first ? 12 : 16) * N; break;
                case Y_RLFINAL: b += Sb + 4 * N + ob; break;
                case Y_C2R: b += Sb + 4 * N; break;
            }
        } else if (s.kind == PK_STEP_X || s.kind == PK_STEP_Z) {
            b += (s.mode == XZ_CONV ? 3 : 2) * Sb;
        } else {
            b += 16.0 * d.blocksY;
        }
    }
    return b;
}

pk_status pk_program_launch(pk_ctx* ctx, PkProgram& prog, cudaStream_t st) {
    for (const PkStep& s : prog.steps) {
        const VolDesc* dd = prog.d_desc + s.desc_off;
        const int* dp = prog.d_prefix + s.prefix_off;
        if (s.grid == 0) continue;
        pk_ctx::ProfRec rec;
        if (ctx && ctx->prof_on) {
            auto take = [&]() {
                cudaEvent_t e;
                if (!ctx->ev_pool.empty()) { e = ctx->ev_pool.back(); ctx->ev_pool.pop_back(); }
                else cudaEventCreate(&e);
                return e;
            };
            rec.kind = pk_step_name(s);
            rec.bytes = pk_step_bytes(s, prog.descs.data() + s.desc_off);
            rec.a = take();
            rec.b = take();
            cudaEventRecord(rec.a, st);
        }
        if (s.kind == PK_STEP_Y) {
            switch (s.mode) {
                case Y_R2C: launch_y_mode<Y_R2C>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_PRE: launch_y_mode<Y_PRE>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_RATIO: launch_y_mode<Y_RATIO>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_UPDATE: launch_y_mode<Y_UPDATE>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_FINAL: launch_y_mode<Y_FINAL>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_RLPRE: launch_y_mode<Y_RLPRE>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_RLUPD: launch_y_mode<Y_RLUPD>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_RLFINAL: launch_y_mode<Y_RLFINAL>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                case Y_C2R: launch_y_mode<Y_C2R>(s.grid, s.smem, dd, dp, s.nvol, st); break;
                default: return pk_fail(PK_ERR_INVALID, "bad y mode");
            }
        } else if (s.kind == PK_STEP_X || s.kind == PK_STEP_Z) {
            const int axis = s.kind == PK_STEP_X ? 1 : 2;
            switch (s.mode) {
                case XZ_FWD: launch_xz_mode<XZ_FWD>(s.grid, s.smem, dd, dp, s.nvol, axis, st); break;
                case XZ_INV: launch_xz_mode<XZ_INV>(s.grid, s.smem, dd, dp, s.nvol, axis, st); break;
                case XZ_CONV: launch_xz_mode<XZ_CONV>(s.grid, s.smem, dd, dp, s.nvol, axis, st); break;
                case XZ_FWD_SCALE: launch_xz_mode<XZ_FWD_SCALE>(s.grid, s.smem, dd, dp, s.nvol, axis, st); break;
                default: return pk_fail(PK_ERR_INVALID, "bad xz mode");
            }
        } else if (s.kind == PK_STEP_LAMBDA) {
            k_lambda<<<s.nvol, 256, 0, st>>>(dd, s.nvol);
        }
        PK_CUDA(cudaGetLastError());
        if (ctx) ctx->launches++;
        if (ctx && ctx->prof_on) {
            cudaEventRecord(rec.b, st);
            ctx->prof.push_back(rec);
        }
    }
    if (ctx && prog.slot >= 0) {
        pk_ctx::ProgSlot& sl = ctx->slots[prog.slot];
        PK_CUDA(cudaEventRecord(sl.ev, st));
        sl.used = true;
    }
    return PK_OK;
}

int pk_program_kernel_count(const PkProgram& prog) {
    int n = 0;
    for (const PkStep& s : prog.steps) n += s.grid > 0 ? 1 : 0;
    return n;
}

