// Shared-memory FFT engine: mixed-radix Stockham autosort over several lines at once.
//
// A tile of L lines of length n lives in shared memory; element e of line l sits at word
// pad(l*ls + e*es) with pad(a) = a + a/16 (one spare float2 every 16 keeps the stride-R stores of
// the early stages and the strided tiles free of bank conflicts).  Each stage of radix R loads the
// R inputs of every butterfly it owns into registers, barriers, applies the stage twiddles and the
// radix-R DFT, and stores the outputs at their Stockham positions (so no bit reversal pass):
//   in  : j + r*(n/R)            (j < n/R, r < R)
//   out : (j - k)*R + k + r*Ns   (k = j mod Ns, Ns = product of the earlier radices)
//   twiddle of input r: W_{Ns*R}^{r*k}, read from a table of the twN-th roots of unity.
// Radices 2, 3, 4, 5, 8 and 16 have register butterflies; any other factor (7, 11, 13, ...) runs a
// direct DFT stage, so every length works and the 2/3/5/7-smooth ones are fast.
#pragma once
#include "pk_internal.h"

namespace pkfft {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward sign) or +i (inverse sign)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
__device__ __forceinline__ int pad(int a) { return a + (a >> 4); }
__host__ __device__ inline int padded_size(int n) { return n + (n >> 4) + 1; }
// padded_size rounded up to even: what follows the tile starts on a 16-byte boundary
__host__ __device__ inline int padded_size2(int n) { return (padded_size(n) + 1) & ~1; }

template <bool INV>
__device__ __forceinline__ void bf2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void bf4(float2& a0, float2& a1, float2& a2, float2& a3) {
    float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi<INV>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void bf3(float2* v) {
    const float s3 = 0.86602540378443865f;  // sin(2 pi / 3)
    float2 t = cadd(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    float2 d = csub(v[1], v[2]);
    d = mul_mi<INV>(make_float2(s3 * d.x, s3 * d.y));
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, d);
    v[2] = csub(m, d);
}

template <bool INV>
__device__ __forceinline__ void bf5(float2* v) {
    const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;  // cos(2pi/5), cos(4pi/5)
    const float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;   // sin(2pi/5), sin(4pi/5)
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    float2 a0 = v[0];
    float2 r1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
    float2 r2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
    float2 q1 = mul_mi<INV>(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
    float2 q2 = mul_mi<INV>(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
    v[0] = make_float2(a0.x + t1.x + t2.x, a0.y + t1.y + t2.y);
    v[1] = cadd(r1, q1);
    v[4] = csub(r1, q1);
    v[2] = cadd(r2, q2);
    v[3] = csub(r2, q2);
}

template <bool INV>
__device__ __forceinline__ void bf8(float2* v) {
    const float h = 0.70710678118654752f;
    float2 b0 = cadd(v[0], v[4]), c0 = csub(v[0], v[4]);
    float2 b1 = cadd(v[1], v[5]), c1 = csub(v[1], v[5]);
    float2 b2 = cadd(v[2], v[6]), c2 = csub(v[2], v[6]);
    float2 b3 = cadd(v[3], v[7]), c3 = csub(v[3], v[7]);
    c1 = INV ? make_float2(h * (c1.x - c1.y), h * (c1.x + c1.y)) : make_float2(h * (c1.x + c1.y), h * (c1.y - c1.x));
    c2 = mul_mi<INV>(c2);
    c3 = INV ? make_float2(-h * (c3.x + c3.y), h * (c3.x - c3.y)) : make_float2(h * (c3.y - c3.x), -h * (c3.x + c3.y));
    bf4<INV>(b0, b1, b2, b3);
    bf4<INV>(c0, c1, c2, c3);
    v[0] = b0; v[2] = b1; v[4] = b2; v[6] = b3;
    v[1] = c0; v[3] = c1; v[5] = c2; v[7] = c3;
}

template <bool INV>
__device__ __forceinline__ void bf16(float2* v) {
    // n = r + 4s, k = p + 4q:  X[p+4q] = sum_r W4^{rq} W16^{rp} sum_s v[r+4s] W4^{sp}
#pragma unroll
    for (int r = 0; r < 4; r++) bf4<INV>(v[r], v[r + 4], v[r + 8], v[r + 12]);
    // twiddles W16^{r p}: cos/sin(2 pi m / 16) for m = 1, 2, 3, 4, 6, 9
    const float C1 = 0.92387953251128676f, S1 = 0.38268343236508977f;
    const float C2 = 0.70710678118654752f;
    const float sg = INV ? 1.f : -1.f;
    auto tw = [&](float2 a, float c, float s) { return make_float2(a.x * c - a.y * (sg * s), a.x * (sg * s) + a.y * c); };
    v[1 + 4] = tw(v[5], C1, S1);        // r=1 p=1  m=1
    v[1 + 8] = tw(v[9], C2, C2);        // r=1 p=2  m=2
    v[1 + 12] = tw(v[13], S1, C1);      // r=1 p=3  m=3
    v[2 + 4] = tw(v[6], C2, C2);        // r=2 p=1  m=2
    v[2 + 8] = mul_mi<INV>(v[10]);      // r=2 p=2  m=4
    v[2 + 12] = tw(v[14], -C2, C2);     // r=2 p=3  m=6
    v[3 + 4] = tw(v[7], S1, C1);        // r=3 p=1  m=3
    v[3 + 8] = tw(v[11], -C2, C2);      // r=3 p=2  m=6
    v[3 + 12] = tw(v[15], -C1, -S1);    // r=3 p=3  m=9
#pragma unroll
    for (int p = 0; p < 4; p++) bf4<INV>(v[4 * p], v[4 * p + 1], v[4 * p + 2], v[4 * p + 3]);
    // v[4p + q] = X[p + 4q]  -> transpose to natural order
    float2 t[16];
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++) t[p + 4 * q] = v[4 * p + q];
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = t[i];
}

template <int R, bool INV>
__device__ __forceinline__ void bfly(float2* v) {
    if constexpr (R == 2) bf2<INV>(v[0], v[1]);
    else if constexpr (R == 3) bf3<INV>(v);
    else if constexpr (R == 4) bf4<INV>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) bf5<INV>(v);
    else if constexpr (R == 8) bf8<INV>(v);
    else if constexpr (R == 16) bf16<INV>(v);
}

// Element (l, e) -> unpadded word index.
struct TileGeom {
    int L, n, ls, es;
    bool lineFast;  // consecutive butterflies -> consecutive lines (strided tiles) else along a line
};

template <int R, bool INV>
__device__ __forceinline__ void stage(float2* __restrict__ buf, const float2* __restrict__ tw, int twStride,
                                      const TileGeom& g, int Ns, int tid, int nthr) {
    const int m = g.n / R;
    const int B = g.L * m;
    constexpr int MAXB = (PK_PPT + R - 1) / R;
    float2 v[MAXB][R];
    int jj[MAXB], ll[MAXB];
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * nthr;
        if (b < B) {
            int l, j;
            if (g.lineFast) { l = b % g.L; j = b / g.L; }
            else { l = b / m; j = b - l * m; }
            ll[i] = l;
            jj[i] = j;
            const int a0 = l * g.ls + j * g.es;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[pad(a0 + r * m * g.es)];
        }
    }
    __syncthreads();
    const int tstep = (g.n / (Ns * R)) * twStride;
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * nthr;
        if (b < B) {
            const int j = jj[i];
            const int k = j % Ns;
            if (Ns > 1) {
                const int t = k * tstep;
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 w = tw[r * t];
                    if (INV) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            bfly<R, INV>(v[i]);
            const int a0 = ll[i] * g.ls + ((j - k) * R + k) * g.es;
#pragma unroll
            for (int r = 0; r < R; r++) buf[pad(a0 + r * Ns * g.es)] = v[i][r];
        }
    }
    __syncthreads();
}

// Direct DFT stage for any radix R: every output is sum_q in[j + q n/R] W_{Ns R}^{q p}, p = pos mod Ns R.
template <bool INV>
__device__ void stage_generic(float2* __restrict__ buf, const float2* __restrict__ tw, int twStride,
                              const TileGeom& g, int R, int Ns, int tid, int nthr) {
    const int m = g.n / R;
    const int NsR = Ns * R;
    const int tstep = (g.n / NsR) * twStride;
    const int P = g.L * g.n;
    float2 out[PK_PPT];
#pragma unroll
    for (int i = 0; i < PK_PPT; i++) {
        const int o = tid + i * nthr;
        if (o < P) {
            int l, pos;
            if (g.lineFast) { l = o % g.L; pos = o / g.L; }
            else { l = o / g.n; pos = o - l * g.n; }
            const int p = pos % NsR;
            const int k = p % Ns;
            const int j = (pos / NsR) * Ns + k;
            const int a0 = l * g.ls + j * g.es;
            float2 acc = make_float2(0.f, 0.f);
            int e = 0;
            for (int q = 0; q < R; q++) {
                float2 w = tw[e * tstep];
                if (INV) w.y = -w.y;
                const float2 x = buf[pad(a0 + q * m * g.es)];
                acc.x += x.x * w.x - x.y * w.y;
                acc.y += x.x * w.y + x.y * w.x;
                e += p;
                if (e >= NsR) e -= NsR;
            }
            out[i] = acc;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PK_PPT; i++) {
        const int o = tid + i * nthr;
        if (o < P) {
            int l, pos;
            if (g.lineFast) { l = o % g.L; pos = o / g.L; }
            else { l = o / g.n; pos = o - l * g.n; }
            buf[pad(l * g.ls + pos * g.es)] = out[i];
        }
    }
    __syncthreads();
}

// Full transform of the tile's L lines (unnormalised; INV = +i sign).
template <bool INV>
__device__ void fft_lines(float2* buf, const AxisDev& A, const float2* tw, const TileGeom& g, int tid, int nthr) {
    int Ns = 1;
    for (int s = 0; s < A.nst; s++) {
        const int R = A.rad[s];
        switch (R) {
            case 2: stage<2, INV>(buf, tw, A.twStride, g, Ns, tid, nthr); break;
            case 3: stage<3, INV>(buf, tw, A.twStride, g, Ns, tid, nthr); break;
            case 4: stage<4, INV>(buf, tw, A.twStride, g, Ns, tid, nthr); break;
            case 5: stage<5, INV>(buf, tw, A.twStride, g, Ns, tid, nthr); break;
            case 8: stage<8, INV>(buf, tw, A.twStride, g, Ns, tid, nthr); break;
            case 16: stage<16, INV>(buf, tw, A.twStride, g, Ns, tid, nthr); break;
            default: stage_generic<INV>(buf, tw, A.twStride, g, R, Ns, tid, nthr); break;
        }
        Ns *= R;
    }
}

}  // namespace pkfft
