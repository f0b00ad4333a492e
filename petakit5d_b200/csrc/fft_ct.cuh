// Compile-time FFT stages: radix, Stockham stride Ns, length, tile lines and layout are template
// constants, so each stage is straight-line code with constant index arithmetic.
#pragma once
#include "fft_engine.cuh"
#include "plans.h"

namespace pkfft {

// Direct DFT butterfly for a compile-time radix (7, 9, 11, 13, 17): y_q = sum_m v_m W_R^{qm}, with
// W_R^e = tw[e * wstep] read from the length-N root table.
template <int R, bool INV>
__device__ __forceinline__ void bf_direct(float2* v, const float2* __restrict__ tw, int wstep) {
    float2 w[R];
#pragma unroll
    for (int e = 0; e < R; e++) {
        w[e] = tw[e * wstep];
        if (INV) w[e].y = -w[e].y;
    }
    float2 out[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
        float2 acc = v[0];
#pragma unroll
        for (int m = 1; m < R; m++) {
            const float2 ww = w[(q * m) % R];
            acc.x += v[m].x * ww.x - v[m].y * ww.y;
            acc.y += v[m].x * ww.y + v[m].y * ww.x;
        }
        out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = out[q];
}

template <int R, int NS, int N, int L, bool LF, bool INV>
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
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[pad(a0 + r * M * ES)];
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
                constexpr int TSTEP = N / (NS * R);
                const int t = k * TSTEP;
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 w = tw[r * t];
                    if (INV) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            if constexpr (R == 2 || R == 3 || R == 4 || R == 5 || R == 8 || R == 16) bfly<R, INV>(v[i]);
            else bf_direct<R, INV>(v[i], tw, N / R);
            const int a0 = l * LS + ((j - k) * R + k) * ES;
#pragma unroll
            for (int r = 0; r < R; r++) buf[pad(a0 + r * NS * ES)] = v[i][r];
        }
    }
    __syncthreads();
}

template <int P, int S, int NS, int L, bool LF, bool INV>
__device__ __forceinline__ void run_plan(float2* buf, const float2* tw, int tid) {
    if constexpr (S < kPlans[P].nst) {
        constexpr int R = kPlans[P].rad[S];
        stage_ct<R, NS, kPlans[P].n, L, LF, INV>(buf, tw, tid);
        run_plan<P, S + 1, NS * R, L, LF, INV>(buf, tw, tid);
    }
}

}  // namespace pkfft
