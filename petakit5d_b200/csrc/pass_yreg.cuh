// y pass with the real/half-spectrum packing in registers, for 512-voxel rows (the 256-point complex
// plan 16 x 16 on 4096-point tiles: 16 rows per CTA, 16 threads per row).
//
// The rolled y pass stages a tile's spectrum rows in shared memory with one 8-byte cp.async per
// bin, packs them (Z[k] from X[k] and X[M-k]) in a separate shared-memory sweep, and splits the
// forward result in another; those sweeps and their index arithmetic cost about as many
// instructions as the two transforms.  Here:
//   * each thread loads the 16 bins j + 16 r of its row straight into registers (coalesced: a
//     half-warp reads 128 contiguous bytes); the partner bin M - k of bin k = j + 16 r is bin
//     (16 - j) + 16 (15 - r), which the thread 16 - j of the same row holds in the same register
//     slot 15 - r, so it arrives by one warp shuffle per register (thread 0 pairs with itself and
//     with the Nyquist bin); the pack feeds the inverse transform's first radix-16 stage directly;
//   * after the forward transform's last stage each thread holds Z[j + 16 r] and the split takes
//     its partner the same way, then stores X[k] straight to HBM (coalesced);
//   * the per-voxel inputs of the tile (contiguous rows) arrive by one bulk copy (cp.async.bulk)
//     per array into shared memory, completing on an mbarrier with a bounded wait.
// The arithmetic and its rounding order are those of the rolled kernel (pass_kernels.cuh), so the
// results are the same.
#pragma once
#include "pass_kernels.cuh"
#include "tma.cuh"

namespace pkpass {

constexpr bool yreg_plan(int p) {
    return p > 0 && kPlans[p].n == 256 && kPlans[p].nst == 2 && kPlans[p].rad[0] == 16 && kPlans[p].rad[1] == 16;
}

constexpr int find_yreg_plan() {
    for (int p = 1; p < kNumPlans; p++)
        if (yreg_plan(p)) return p;
    return -1;
}
constexpr int kYregPlan = find_yreg_plan();

constexpr bool y_spec_in(int m) {
    return m == Y_RATIO || m == Y_UPDATE || m == Y_FINAL || m == Y_RLUPD || m == Y_RLFINAL || m == Y_C2R;
}
constexpr bool y_spec_out(int m) {
    return m == Y_R2C || m == Y_PRE || m == Y_RATIO || m == Y_UPDATE || m == Y_RLPRE;
}
constexpr int y_naux(int m) { return (m == Y_RLPRE || m == Y_RLUPD) ? 2 : (m == Y_C2R ? 0 : 1); }

// shared memory of k_yr<P, MODE>: aux arrays | padded tile | twiddles | split table | barrier (+ slack
// to align the base to 128 bytes)
__host__ __device__ constexpr size_t yreg_smem_bytes(int mode) {
    return 128 + sizeof(float2) * ((size_t)y_naux(mode) * 4096 + (size_t)(4096 + 4096 / 16 + 1 + 1) + (256 + 32) + 258) + 16;
}

// Volume descriptor fields the kernel needs for a voxel's post-processing are those of the rolled
// kernel's fused path: no damping, scaling, mask or crop (the host only picks this kernel then).
template <int P, int MODE>
__global__ void __launch_bounds__(PK_THREADS, y_naux(MODE) == 2 ? 2 : 3)
    k_yr(const VolDesc* __restrict__ descs, const int* __restrict__ prefix, int nvol, int* err) {
    constexpr int N = 256, R = 16, MS = 16, LL = 16, NT = PK_THREADS;
    constexpr int M = N;                       // complex points per row (ny = 2M = 512)
    constexpr bool SIN = y_spec_in(MODE), SOUT = y_spec_out(MODE);
    constexpr int NAUX = y_naux(MODE);
    constexpr int OFF1 = stage_tw_off(P, 1);
    extern __shared__ unsigned char yraw[];
    unsigned char* base = yraw + ((128 - (pktma::smem_u32(yraw) & 127)) & 127);
    float2* aux0 = (float2*)base;
    float2* aux1 = aux0 + LL * M;
    float2* buf = aux0 + NAUX * LL * M;
    float2* tw = buf + (4096 + 4096 / 16 + 2);
    float2* twrc = tw + (256 + 32);
    uint64_t* bar = (uint64_t*)(twrc + 258);

    const int vol = find_vol(prefix, nvol, blockIdx.x);
    const VolDesc& d = descs[vol];
    const int lb = blockIdx.x - prefix[vol];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int l = tid / MS, j = tid % MS;
    const long long row0 = (long long)lb * LL;
    const int Lc = (int)min((long long)LL, d.nrows - row0);
    const bool valid = l < Lc;
    const long long row = row0 + l;
    const int ny = d.ny;
    const long long v0 = row0 * (long long)ny;
    if (!PK_SMEM_OK(d, yreg_smem_bytes(MODE), 4) || !PK_IN(d, row0 < d.nrows && Lc >= 1 && d.Pp >= M + 1, 5))
        return;   // uniform over the CTA, before any barrier

    // ---- the tile's per-voxel inputs: one bulk copy per array (contiguous rows row0 .. row0+Lc-1)
    const void* src0 = nullptr;
    const void* src1 = nullptr;
    uint32_t esz = 4;
    if constexpr (MODE == Y_PRE) { src0 = d.raw; esz = d.raw_type == PK_U16 ? 2 : 4; }
    else if constexpr (MODE == Y_R2C) src0 = d.src;
    else if constexpr (MODE == Y_RATIO) src0 = d.I;
    else if constexpr (MODE == Y_UPDATE || MODE == Y_FINAL) src0 = d.Jo;
    else if constexpr (MODE == Y_RLPRE) { src0 = d.J2; src1 = d.J3; }
    else if constexpr (MODE == Y_RLUPD) { src0 = d.Yb; src1 = d.rl_first ? nullptr : d.J4; }
    else if constexpr (MODE == Y_RLFINAL) src0 = d.Yb;
    if (tid == 0 && NAUX > 0) {
        pktma::mbar_init(bar, 1);
        pktma::fence_mbar_init();
        uint32_t bytes = (uint32_t)Lc * (uint32_t)ny * esz;
        if (!PK_IN(d, (row0 + Lc) * (long long)ny <= d.nrows * (long long)ny && bytes <= LL * M * 8u, 15)) bytes = 0;
        pktma::mbar_expect_tx(bar, src1 ? 2 * bytes : bytes);
        if (bytes) {
            pktma::bulk_load(aux0, (const char*)src0 + (size_t)v0 * esz, bytes, bar);
            if (src1) pktma::bulk_load(aux1, (const char*)src1 + (size_t)v0 * esz, bytes, bar);
        }
    }

    float2 v[1][R];
    const int partner = (lane & 16) | ((16 - j) & 15);   // the thread holding bin M - k, same row
    if constexpr (SIN) {
        // spectrum bins j + 16 r of the row (and the Nyquist bin for thread 0), straight to registers
        const float2* Srow = d.S + row * (long long)d.Pp;
        float2 x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = valid ? Srow[j + 16 * r] : make_float2(0.f, 0.f);
        const float2 nyq = (valid && j == 0) ? Srow[M] : make_float2(0.f, 0.f);
        for (int i = tid; i < plan_tw_size(P); i += NT) tw[i] = d.ay.tw[i];
        for (int i = tid; i <= M; i += NT) twrc[i] = d.tw_rc[i];
        __syncthreads();
        float2 t[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            t[q].x = __shfl_sync(0xffffffffu, x[q].x, partner);
            t[q].y = __shfl_sync(0xffffffffu, x[q].y, partner);
        }
        // packed inverse sequence Z[k] = (X[k] + X*[M-k]) + i (X[k] - X*[M-k]) W_ny^{-k}
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = j + 16 * r;
            float2 xm = t[R - 1 - r];
            if (j == 0) xm = r == 0 ? nyq : x[(R - r) & (R - 1)];
            const float2 a = x[r], b = conjf2(xm);
            float2 w = twrc[k];
            w.y = -w.y;
            const float2 s2 = cadd(a, b), t2 = cmul(csub(a, b), w);
            v[0][r] = make_float2(s2.x - t2.y, s2.y + t2.x);
        }
        stage_r2s<R, N, LL, false, true>(buf, tid, v);                  // inverse stage 1 of 2
        stage_s2r<R, 16, N, LL, false, true, OFF1>(buf, tw, tid, v);    // stage 2: v = c at bins j + 16 r
    } else {
        for (int i = tid; i < plan_tw_size(P); i += NT) tw[i] = d.ay.tw[i];
        for (int i = tid; i <= M; i += NT) twrc[i] = d.tw_rc[i];
        __syncthreads();
    }

    // ---- per-voxel phase on element e = j + 16 r (voxels 2e, 2e + 1 of the row)
    if constexpr (NAUX > 0) {
        const bool ok = pktma::mbar_wait(bar, 0);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) pktma::report_wait_failure(err, 1);
            return;
        }
    }
    double acc0 = 0.0, acc1 = 0.0;
    unsigned zeros = 0;
    const float lam = (MODE == Y_RLPRE && d.lam_on) ? (float)d.partials[0] : 0.f;
    const bool raw_u16 = d.raw_type == PK_U16;
    const unsigned bg16 = (unsigned)d.bg16;
    const float bgf = d.bg_f;
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int e = j + 16 * r;
        const int idx = l * M + e;
        float2 out = make_float2(0.f, 0.f);
        if (valid) {
            const float2 c = v[0][r];
            if constexpr (MODE == Y_PRE) {
                if (raw_u16) {   // pre_value's uint16 branch on the dense uint16 rows
                    const ushort2 q = ((const ushort2*)aux0)[idx];
                    const unsigned q0 = q.x, q1 = q.y;
                    zeros += (q0 != 0 ? 0u : 1u) + (q1 != 0 ? 0u : 1u);
                    out.x = q0 > bg16 ? (float)(q0 - bg16) : 0.f;
                    out.y = q1 > bg16 ? (float)(q1 - bg16) : 0.f;
                } else {
                    out = pre_value(false, bg16, bgf, aux0[idx], zeros);
                }
            } else if constexpr (MODE == Y_R2C) {
                out = aux0[idx];
            } else if constexpr (MODE == Y_RATIO) {
                const float2 a0 = aux0[idx];
                out.x = __fdividef(a0.x, fmaxf(c.x, PK_EPS_F));
                out.y = __fdividef(a0.y, fmaxf(c.y, PK_EPS_F));
            } else if constexpr (MODE == Y_UPDATE || MODE == Y_FINAL) {
                const float2 a0 = aux0[idx];
                out.x = fmaxf(__fmul_rn(c.x, a0.x), 0.f);
                out.y = fmaxf(__fmul_rn(c.y, a0.y), 0.f);
            } else if constexpr (MODE == Y_RLPRE) {
                const float2 a0 = aux0[idx], a1 = aux1[idx];
                out.x = fmaxf(__fadd_rn(a0.x, __fmul_rn(lam, __fsub_rn(a0.x, a1.x))), 0.f);
                out.y = fmaxf(__fadd_rn(a0.y, __fmul_rn(lam, __fsub_rn(a0.y, a1.y))), 0.f);
            } else if constexpr (MODE == Y_RLUPD) {
                const float2 a0 = aux0[idx];
                out.x = fmaxf(__fmul_rn(a0.x, c.x), 0.f);
                out.y = fmaxf(__fmul_rn(a0.y, c.y), 0.f);
                if (src1) {   // not the first iteration
                    const float2 a1 = aux1[idx];
                    acc0 += (double)__fmul_rn(__fsub_rn(out.x, a0.x), a1.x);
                    acc1 += (double)__fmul_rn(a1.x, a1.x);
                    acc0 += (double)__fmul_rn(__fsub_rn(out.y, a0.y), a1.y);
                    acc1 += (double)__fmul_rn(a1.y, a1.y);
                }
            } else if constexpr (MODE == Y_RLFINAL) {
                const float2 a0 = aux0[idx];
                out.x = fmaxf(__fmul_rn(a0.x, c.x), 0.f);
                out.y = fmaxf(__fmul_rn(a0.y, c.y), 0.f);
            } else if constexpr (MODE == Y_C2R) {
                out = c;
            }
        }
        v[0][r] = out;
    }
    // stores of the per-voxel outputs (coalesced: a half-warp writes 128 contiguous bytes)
    if (valid && MODE != Y_RATIO && MODE != Y_R2C) {
        constexpr bool kPost = MODE == Y_FINAL || MODE == Y_RLFINAL;
        float* p1 = nullptr;
        float* p2 = nullptr;
        uint8_t* mk = nullptr;
        if constexpr (MODE == Y_PRE) { p1 = d.I; mk = d.write_mask ? d.mask8 : nullptr; }
        if constexpr (MODE == Y_UPDATE) p1 = d.Jn;
        if constexpr (MODE == Y_RLPRE) p1 = d.Yb;
        if constexpr (MODE == Y_RLUPD) { p1 = d.J2n; p2 = d.J4; }
        if constexpr (MODE == Y_C2R) p1 = d.dst;
        void* const o = kPost ? d.out : nullptr;
        const bool vec_out = kPost && ((reinterpret_cast<uintptr_t>(o) & (d.save16 ? 3 : 7)) == 0);
        const bool s16 = kPost && d.save16;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int e = j + 16 * r;
            const long long vi = row * (long long)ny + 2 * e;
            const float2 val = v[0][r];
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
                if constexpr (MODE == Y_RLUPD) {
                    const float2 a0 = aux0[l * M + e];
                    *reinterpret_cast<float2*>(p2 + vi) = make_float2(__fsub_rn(val.x, a0.x), __fsub_rn(val.y, a0.y));
                }
                if constexpr (MODE == Y_PRE) {
                    if (mk) {
                        unsigned m2;
                        if (raw_u16) {
                            const ushort2 q = ((const ushort2*)aux0)[l * M + e];
                            m2 = (q.x != 0 ? 1u : 0u) | (q.y != 0 ? 0x100u : 0u);
                        } else {
                            const float2 a0 = aux0[l * M + e];
                            m2 = (a0.x != 0.f ? 1u : 0u) | (a0.y != 0.f ? 0x100u : 0u);
                        }
                        *reinterpret_cast<uint16_t*>(mk + vi) = (uint16_t)m2;
                    }
                }
            }
        }
    }

    if constexpr (SOUT) {
        int tid2 = tid;   // opaque copy: the inverse's index arithmetic is not kept live for reuse
        asm volatile("mov.b32 %0, %0;" : "+r"(tid2));
        stage_r2s<R, N, LL, false, false>(buf, tid2, v);                  // forward stage 1 of 2
        stage_s2r<R, 16, N, LL, false, false, OFF1>(buf, tw, tid2, v);    // stage 2: v = Z[j + 16 r]
        // split into the half spectrum: X[k] = (Z[k] + Z*[M-k]) / 2 + W^k (Z[k] - Z*[M-k]) / 2i
        float2 t[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            t[q].x = __shfl_sync(0xffffffffu, v[0][q].x, partner);
            t[q].y = __shfl_sync(0xffffffffu, v[0][q].y, partner);
        }
        float2* Srow = d.S + row * (long long)d.Pp;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = j + 16 * r;
            const float2 zk = v[0][r];
            const float2 zp = j == 0 ? v[0][(R - r) & (R - 1)] : t[R - 1 - r];
            const float2 zc = conjf2(zp);
            const float2 fe = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
            const float2 df = csub(zk, zc);
            const float2 fo = make_float2(0.5f * df.y, -0.5f * df.x);
            if (valid) Srow[k] = cadd(fe, cmul(twrc[k], fo));
        }
        if (valid && j == 0) {   // Nyquist bin from Z[0]
            const float2 zk = v[0][0];
            const float2 zc = conjf2(zk);
            const float2 fe = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
            const float2 df = csub(zk, zc);
            const float2 fo = make_float2(0.5f * df.y, -0.5f * df.x);
            Srow[M] = cadd(fe, cmul(twrc[M], fo));
        }
    }

    if constexpr (MODE == Y_RLUPD) {
        // deterministic block reduction of the two lambda sums (the rolled kernel's order)
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

// The register-packing y kernels of plan P by mode, with their shared memory and whether they loaded.
struct YregTable {
    void (*k[Y_C2R + 1])(const VolDesc*, const int*, int, int*);
    size_t smem[Y_C2R + 1];
};

template <int P, int MD>
struct RegisterYreg {
    static void fill(YregTable& t) {
        auto fn = k_yr<P, MD>;
        const size_t smem = yreg_smem_bytes(MD);
        t.k[MD] = fn;
        t.smem[MD] = smem;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            t.k[MD] = nullptr;
        }
        RegisterYreg<P, MD + 1>::fill(t);
    }
};
template <int P>
struct RegisterYreg<P, Y_C2R + 1> {
    static void fill(YregTable&) {}
};

}  // namespace pkpass
