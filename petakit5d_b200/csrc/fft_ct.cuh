// Compile-time FFT stages: radix, Stockham stride Ns, length, tile lines and layout are template
// constants, so each stage is straight-line code with constant index arithmetic.
#pragma once
#include "fft_engine.cuh"
#include "plans.h"

namespace pkfft {

// Direct DFT butterfly for a compile-time odd radix (7, 9, 11, 13, 17), in its symmetric form: with
// a_m = v_m + v_{R-m}, b_m = v_m - v_{R-m} (m = 1..H, H = (R-1)/2) and W_R^e = c_e + i s_e (the
// direction's sign in s), y_q = t1 + i t2 and y_{R-q} = t1 - i t2 for
//   t1 = v_0 + sum_m a_m c_{qm},  t2 = sum_m b_m s_{qm}
// which takes about a quarter of the multiply-adds of sum_m v_m W^{qm}.  W_R^e = tw[e * wstep] (forward
// roots; the inverse negates their imaginary parts).  Only the H roots W_R^1 .. W_R^H are read: the
// table's W_R^{R-e} is the conjugate of its W_R^e, bit for bit (both come from the same angle), so
// c_{R-e} = c_e and s_{R-e} = -s_e select, at compile time, among H loads instead of H^2.
template <int R, bool INV>
__device__ __forceinline__ void bf_direct(float2* v, const float2* __restrict__ tw, int wstep) {
    static_assert(R % 2 == 1, "symmetric direct DFT needs an odd radix");
    constexpr int H = (R - 1) / 2;
    float2 a[H + 1], b[H + 1], w[H + 1];
    w[0] = make_float2(1.f, 0.f);   // W_R^0, as the table holds it (q m = 0 mod R for a composite R)
    float2 y0 = v[0];
#pragma unroll
    for (int m = 1; m <= H; m++) {
        w[m] = tw[m * wstep];   // roots stay in shared memory until here
        a[m] = make_float2(v[m].x + v[R - m].x, v[m].y + v[R - m].y);
        b[m] = make_float2(v[m].x - v[R - m].x, v[m].y - v[R - m].y);
        y0.x += a[m].x;
        y0.y += a[m].y;
    }
    float2 out[R];
    out[0] = y0;
#pragma unroll
    for (int q = 1; q <= H; q++) {
        float2 t1 = v[0], t2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 1; m <= H; m++) {
            const int e = (q * m) % R;
            const float c = e <= H ? w[e].x : w[R - e].x;
            const float sn = e <= H ? w[e].y : -w[R - e].y;
            const float sw = INV ? -sn : sn;
            t1.x += a[m].x * c;
            t1.y += a[m].y * c;
            t2.x += b[m].x * sw;
            t2.y += b[m].y * sw;
        }
        out[q] = make_float2(t1.x - t2.y, t1.y + t2.x);
        out[R - q] = make_float2(t1.x + t2.y, t1.y - t2.x);
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = out[q];
}

// Padded shared-memory index of a + r*STEP given pa = pad(a), with the carries of pad() resolved at
// compile time where possible: STEP a multiple of 16 adds STEP*17/16 per step; RUN16 says that
// (a mod 16) + r*STEP stays below 16 for every r used, so no spare slot is crossed.
template <int STEP, bool RUN16>
__device__ __forceinline__ int pstep(int a, int pa, int r) {
    if constexpr (STEP % 16 == 0) return pa + r * (STEP + STEP / 16);
    else if constexpr (RUN16) return pa + r * STEP;
    else return pad(a + r * STEP);
}

// Stores of a first stage (Ns = 1) start at a multiple of R along a line of a line-major tile; with
// R dividing 16 and lines a multiple of 16 long, the R outputs stay inside one 16-slot run.
template <int R, int N, bool LF>
constexpr bool first_run16() { return !LF && N % 16 == 0 && 16 % R == 0; }

// One Stockham stage, shared -> shared.  tw is the plan's stage-ordered table; OFF is this stage's
// section in it.
template <int R, int NS, int N, int L, bool LF, bool INV, int OFF>
__device__ __forceinline__ void stage_ct(float2* __restrict__ buf, const float2* __restrict__ tw, int tid) {
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = PK_THREADS;
    constexpr int MAXB = (B + NT - 1) / NT;
    constexpr int LS = LF ? 1 : N;
    constexpr int ES = LF ? L : 1;
    float2 v[MAXB][R];
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            const int a0 = l * LS + j * ES;
            const int p0 = pad(a0);
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[pstep<M * ES, false>(a0, p0, r)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            const int k = j % NS;
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 w = tw[OFF + (r - 1) * NS + k];
                    if (INV) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            if constexpr (!direct_radix(R)) bfly<R, INV>(v[i]);
            else bf_direct<R, INV>(v[i], tw + OFF + (NS > 1 ? (R - 1) * NS : 0), 1);
            const int a0 = l * LS + ((j - k) * R + k) * ES;
            const int p0 = pad(a0);
#pragma unroll
            for (int r = 0; r < R; r++)
                buf[pstep<NS * ES, NS == 1 && first_run16<R, N, LF>()>(a0, p0, r)] = v[i][r];
        }
    }
    __syncthreads();
}

template <int P, int S, int NS, int L, bool LF, bool INV>
__device__ __forceinline__ void run_plan(float2* buf, const float2* tw, int tid) {
    if constexpr (S < kPlans[P].nst) {
        constexpr int R = kPlans[P].rad[S];
        stage_ct<R, NS, kPlans[P].n, L, LF, INV, stage_tw_off(P, S)>(buf, tw, tid);
        run_plan<P, S + 1, NS * R, L, LF, INV>(buf, tw, tid);
    }
}

// ---- stages whose inputs come from / outputs go to HBM directly (registers <-> global), so a
// transform makes two fewer passes over shared memory.  G is an accessor of the tile with
//   float2 ld(l, e); void st(l, e, v); float2 otf(l, e); void after_loads(); void before_last()
// for element e of line l (ld reads zero and st skips outside the tile's valid columns).

// first stage (Ns = 1, no twiddles): global -> registers -> butterfly -> shared.  g.after_loads()
// runs once the loads are issued (the caller stages tables and side inputs there).
template <int R, int N, int L, bool LF, bool INV, class G>
__device__ __forceinline__ void stage_g2s(float2* __restrict__ buf, const G& g, int tid) {
    static_assert(R == 2 || R == 3 || R == 4 || R == 5 || R == 8 || R == 16, "first stage needs a register butterfly");
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = PK_THREADS;
    constexpr int MAXB = (B + NT - 1) / NT;
    constexpr int LS = LF ? 1 : N;
    constexpr int ES = LF ? L : 1;
    float2 v[MAXB][R];
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = g.ld(l, j + r * M);
        }
    }
    g.after_loads();
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            bfly<R, INV>(v[i]);
            const int a0 = l * LS + j * R * ES;
            const int p0 = pad(a0);
#pragma unroll
            for (int r = 0; r < R; r++) buf[pstep<ES, first_run16<R, N, LF>()>(a0, p0, r)] = v[i][r];
        }
    }
    __syncthreads();
}

// last stage: shared -> registers -> twiddle, butterfly [x OTF] -> global (TO_GLOBAL) or shared
template <int R, int NS, int N, int L, bool LF, bool INV, int OFF, bool MUL, bool TO_GLOBAL, class G>
__device__ __forceinline__ void stage_s2x(float2* __restrict__ buf, const float2* __restrict__ tw, const G& g, int tid) {
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = PK_THREADS;
    constexpr int MAXB = (B + NT - 1) / NT;
    constexpr int LS = LF ? 1 : N;
    constexpr int ES = LF ? L : 1;
    float2 v[MAXB][R];
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            const int a0 = l * LS + j * ES;
            const int p0 = pad(a0);
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[pstep<M * ES, false>(a0, p0, r)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            const int k = j % NS;
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 w = tw[OFF + (r - 1) * NS + k];
                    if (INV) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            if constexpr (!direct_radix(R)) bfly<R, INV>(v[i]);
            else bf_direct<R, INV>(v[i], tw + OFF + (NS > 1 ? (R - 1) * NS : 0), 1);
            const int aw = l * LS + ((j - k) * R + k) * ES;
            const int pw = pad(aw);
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int e = (j - k) * R + k + r * NS;
                float2 o = v[i][r];
                if constexpr (MUL) o = cmul(o, g.otf(l, e));
                if constexpr (TO_GLOBAL) g.st(l, e, o);
                else buf[pstep<NS * ES, NS == 1 && first_run16<R, N, LF>()>(aw, pw, r)] = o;
            }
        }
    }
    if constexpr (!TO_GLOBAL) __syncthreads();
}

// Last stage kept in registers: shared -> registers, twiddle and butterfly; v[i][r] is then element
// (j - k) R + k + r NS of line l (b = tid + i * PK_THREADS as in stage_ct).
template <int R, int NS, int N, int L, bool LF, bool INV, int OFF>
__device__ __forceinline__ void stage_s2r(const float2* __restrict__ buf, const float2* __restrict__ tw, int tid,
                                          float2 (&v)[(L * (N / R) + PK_THREADS - 1) / PK_THREADS][R]) {
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = PK_THREADS;
    constexpr int MAXB = (B + NT - 1) / NT;
    constexpr int LS = LF ? 1 : N;
    constexpr int ES = LF ? L : 1;
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            const int a0 = l * LS + j * ES;
            const int p0 = pad(a0);
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[pstep<M * ES, false>(a0, p0, r)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int j = LF ? b / L : b % M;
            const int k = j % NS;
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 w = tw[OFF + (r - 1) * NS + k];
                    if (INV) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            if constexpr (!direct_radix(R)) bfly<R, INV>(v[i]);
            else bf_direct<R, INV>(v[i], tw + OFF + (NS > 1 ? (R - 1) * NS : 0), 1);
        }
    }
}

// First stage from registers: v[i][r] is element j + r (N / R) of line l; butterfly, store to shared.
template <int R, int N, int L, bool LF, bool INV>
__device__ __forceinline__ void stage_r2s(float2* __restrict__ buf, int tid,
                                          float2 (&v)[(L * (N / R) + PK_THREADS - 1) / PK_THREADS][R]) {
    static_assert(!direct_radix(R), "first stage needs a register butterfly");
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = PK_THREADS;
    constexpr int MAXB = (B + NT - 1) / NT;
    constexpr int LS = LF ? 1 : N;
    constexpr int ES = LF ? L : 1;
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = LF ? b % L : b / M;
            const int j = LF ? b / L : b % M;
            bfly<R, INV>(v[i]);
            const int a0 = l * LS + j * R * ES;
            const int p0 = pad(a0);
#pragma unroll
            for (int r = 0; r < R; r++) buf[pstep<ES, first_run16<R, N, LF>()>(a0, p0, r)] = v[i][r];
        }
    }
    __syncthreads();
}

// middle stages S in [S0, S1) of plan P (shared -> shared)
template <int P, int S, int S1, int NS, int L, bool LF, bool INV>
__device__ __forceinline__ void run_mid(float2* buf, const float2* tw, int tid) {
    if constexpr (S < S1) {
        constexpr int R = kPlans[P].rad[S];
        stage_ct<R, NS, kPlans[P].n, L, LF, INV, stage_tw_off(P, S)>(buf, tw, tid);
        run_mid<P, S + 1, S1, NS * R, L, LF, INV>(buf, tw, tid);
    }
}

// Whole transform of plan P (>= 2 stages) with HBM input and HBM or shared output.
//   TO_GLOBAL: the last stage stores through g.st; else it leaves the result in shared memory
//   MUL: the last stage multiplies by g.otf before storing (g.before_last() makes that table ready)
template <int P, int L, bool LF, bool INV, bool MUL, bool TO_GLOBAL, class G>
__device__ __forceinline__ void fft_g(float2* buf, const float2* tw, const G& g, int tid) {
    constexpr int nst = kPlans[P].nst;
    constexpr int N = kPlans[P].n;
    static_assert(nst >= 2, "fft_g needs at least two stages");
    stage_g2s<kPlans[P].rad[0], N, L, LF, INV>(buf, g, tid);
    run_mid<P, 1, nst - 1, kPlans[P].rad[0], L, LF, INV>(buf, tw, tid);
    if constexpr (MUL) g.before_last();
    stage_s2x<kPlans[P].rad[nst - 1], plan_ns_before(P, nst - 1), N, L, LF, INV, stage_tw_off(P, nst - 1), MUL,
              TO_GLOBAL>(buf, tw, g, tid);
}

// Transform of plan P starting from shared memory with the last stage going to HBM.
template <int P, int L, bool LF, bool INV, class G>
__device__ __forceinline__ void fft_s2g(float2* buf, const float2* tw, const G& g, int tid) {
    constexpr int nst = kPlans[P].nst;
    constexpr int N = kPlans[P].n;
    run_mid<P, 0, nst - 1, 1, L, LF, INV>(buf, tw, tid);
    stage_s2x<kPlans[P].rad[nst - 1], plan_ns_before(P, nst - 1), N, L, LF, INV, stage_tw_off(P, nst - 1), false,
              true>(buf, tw, g, tid);
}

}  // namespace pkfft
