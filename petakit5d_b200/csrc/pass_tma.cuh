// Persistent x / z pass kernels fed by TMA (cp.async.bulk.tensor) for the strided column tiles.
//
// The spectrum S[z][x][k] is a 3-D tensor (k fastest) to the TMA unit; a tile is T adjacent
// k-columns along a whole x (or z) line, i.e. a box {2T floats, n, 1} (x) or {2T floats, 1, n} (z).
// Each CTA is persistent: it walks the tiles g = blockIdx.x, blockIdx.x + gridDim.x, ... and keeps
// two tile buffers, so the TMA load of its next tile is in flight while it transforms the current
// one, and the finished tile leaves as a TMA bulk store that overlaps the next tile's work.  The
// transform runs in place on the dense tile (element (l, e) at e*T + l): with T >= 8 a half-warp
// touches whole 64- or 128-byte rows, so no padding is needed and the rows arrive exactly as the
// TMA box lays them out.  XZ_CONV also brings the OTF tile by TMA (issued at the tile's start, used
// between the forward and the inverse transform).  All tensor maps cover this GPU's own buffers;
// no load uses cluster multicast.
#pragma once
#include <cstdlib>

#include "pass_kernels.cuh"
#include "tma.cuh"

namespace pkpass {

// rows of one TMA box along the transformed axis: the largest divisor of n not above 256 (a box
// dimension is at most 256 elements), so the boxes tile the line exactly
constexpr int tma_box_rows(int n) {
    for (int r = n < 256 ? n : 256; r > 1; r--)
        if (n % r == 0) return r;
    return 1;
}

// plans with a TMA kernel: compile-time plans of >= 2 stages whose column tiles are >= 8 wide
// (lengths 32..512); longer lines keep the register-IO kernels of pass_kernels.cuh
constexpr bool tma_plan(int p) { return p > 0 && kPlans[p].nst >= 2 && kPlans[p].n >= 32 && kPlans[p].n <= 512; }

// shared-memory layout of k_xzt<P, ..., TC, NBUF>: NBUF tile buffers | OTF tile (XZ_CONV) | twiddles |
// barriers, 1024 bytes of slack so the base can be aligned.  TC = columns per tile (0: the plan's
// 4096-point tile width).
template <int P, int TC = 0, int NBUF = 2>
struct XztLayout {
    static constexpr int N = kPlans[P].n;
    static constexpr int T = TC > 0 ? TC : plan_cols_xz(N);
    static constexpr int PTS = T * N;
    static constexpr int ROWS = tma_box_rows(N);
    static constexpr int NBOX = N / ROWS;
    static constexpr size_t BUF = ((size_t)PTS * 8 + 1023) & ~(size_t)1023;
    static constexpr size_t TW = ((size_t)(plan_tw_size(P) > 0 ? plan_tw_size(P) : 1) * 8 + 15) & ~(size_t)15;
    static constexpr size_t bytes(bool conv) { return 1024 + NBUF * BUF + (conv ? BUF : 0) + TW + 64; }
    static_assert(1024 + NBUF * BUF + TW + 64 <= 227 * 1024, "tile buffers exceed shared memory");
};

// CTAs per SM a variant is compiled for (register budget): 3 for 4096-point tiles, 2 for the
// two-buffer convolution (three tile-sized buffers) or one 8192-point buffer, 1 for two 8192-point buffers
constexpr int xzt_min_blocks(int P, int TC, int NBUF, bool conv) {
    return (TC > 0 ? TC : plan_cols_xz(kPlans[P].n)) * kPlans[P].n > 4096 ? (NBUF >= 2 ? 1 : 2)
                                                                           : ((conv && NBUF >= 2) ? 2 : 3);
}

// The TMA kernels run NTH compute threads (NTH / 32 warps) and one producer warp after them that
// issues the TMA loads and stores.  The compute warps synchronise among themselves on named
// barrier 1, so the producer never holds them up and they never wait on a copy they do not need.
template <int NTH>
__device__ __forceinline__ void compute_bar() { asm volatile("bar.sync 1, %0;\n" ::"n"(NTH) : "memory"); }
// every compute thread's `ok`, and-reduced over the compute warps (named barrier 1)
template <int NTH>
__device__ __forceinline__ bool compute_bar_and(bool ok) {
    int r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((unsigned)ok), "n"(NTH)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void mbar_arrive_cta(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(pktma::smem_u32(bar)) : "memory");
}

// ---- dense column-tile stages (element (l, e) at e*L + l, L = T columns)
template <int R, int NS, int N, int L, bool INV, int OFF, int NTH>
__device__ __forceinline__ void dstage(float2* __restrict__ buf, const float2* __restrict__ tw, int tid) {
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = NTH;
    constexpr int MAXB = (B + NT - 1) / NT;
    float2 v[MAXB][R];
    // a thread past the last butterfly reads butterfly 0's elements (in the tile, never used): an
    // unconditional load keeps v's registers out of a predicated region that spills under tight caps
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        const int bb = (B % NT == 0 || b < B) ? b : 0;
        const int l = bb % L, j = bb / L;
#pragma unroll
        for (int r = 0; r < R; r++) v[i][r] = buf[(j + r * M) * L + l];
    }
    compute_bar<NTH>();
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = b % L, j = b / L;
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
            const int a0 = ((j - k) * R + k) * L + l;
#pragma unroll
            for (int r = 0; r < R; r++) buf[a0 + r * NS * L] = v[i][r];
        }
    }
    compute_bar<NTH>();
}

// last stage into registers: v[i][r] = element (j - k) R + k + r NS of column l (b = tid + i NT)
template <int R, int NS, int N, int L, bool INV, int OFF, int NTH>
__device__ __forceinline__ void dstage_s2r(const float2* __restrict__ buf, const float2* __restrict__ tw, int tid,
                                           float2 (&v)[(L * (N / R) + NTH - 1) / NTH][R]) {
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = NTH;
    constexpr int MAXB = (B + NT - 1) / NT;
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = b % L, j = b / L;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = buf[(j + r * M) * L + l];
        }
    }
    compute_bar<NTH>();
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int j = b / L;
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

// first stage from registers: v[i][r] is element j + r (N / R) of column l; butterfly, store
template <int R, int N, int L, bool INV, int NTH>
__device__ __forceinline__ void dstage_r2s(float2* __restrict__ buf, int tid,
                                           float2 (&v)[(L * (N / R) + NTH - 1) / NTH][R]) {
    static_assert(!direct_radix(R), "first stage needs a register butterfly");
    constexpr int M = N / R;
    constexpr int B = L * M;
    constexpr int NT = NTH;
    constexpr int MAXB = (B + NT - 1) / NT;
#pragma unroll
    for (int i = 0; i < MAXB; i++) {
        const int b = tid + i * NT;
        if (B % NT == 0 || b < B) {
            const int l = b % L, j = b / L;
            bfly<R, INV>(v[i]);
            const int a0 = j * R * L + l;
#pragma unroll
            for (int r = 0; r < R; r++) buf[a0 + r * L] = v[i][r];
        }
    }
    compute_bar<NTH>();
}

template <int P, int S, int S1, int NS, int L, bool INV, int NTH>
__device__ __forceinline__ void run_dense(float2* buf, const float2* tw, int tid) {
    if constexpr (S < S1) {
        constexpr int R = kPlans[P].rad[S];
        dstage<R, NS, kPlans[P].n, L, INV, stage_tw_off(P, S), NTH>(buf, tw, tid);
        run_dense<P, S + 1, S1, NS * R, L, INV, NTH>(buf, tw, tid);
    }
}

// One persistent launch of an x (AXIS 1) or z (AXIS 2) pass of plan P over every tile of `nvol`
// volumes (tile prefix in `prefix`).  MODE: XZ_FWD / XZ_INV (x) or XZ_CONV (z: forward, OTF multiply
// -- conjugated when the descriptor says so -- and inverse).  maps[v] holds volume v's tensor maps.
//
// Pipeline per CTA, tile it of the CTA's tiles g = blockIdx.x + it * gridDim.x, buffer s = it % NBUF:
//   producer (warp 8, one lane): once compute has released buffer s (tile it - NBUF done), store that
//     tile by TMA, wait until the store has read the buffer, then load tile it into it (full[s]);
//     for XZ_CONV, once compute has used the previous OTF tile (otf_empty), load tile it's OTF tile;
//   compute (warps 0-7): wait full[s], transform in place (multiply by the OTF tile between the
//     transforms, then release the OTF buffer), then release buffer s (empty[s]).
// With NBUF = 2 (3) the next one (two) tiles' loads are in flight while the current one is transformed.  Every wait
// is bounded; a wait that runs out is recorded in *err and the role that saw it stops.
template <int P, int AXIS, int MODE, int TC = 0, int NBUF = 2, int NTH = PK_THREADS>
__global__ void __launch_bounds__(NTH + 32, xzt_min_blocks(P, TC, NBUF, MODE == XZ_CONV))
    k_xzt(const VolDesc* __restrict__ descs, const XZMaps* __restrict__ maps, const int* __restrict__ prefix, int nvol,
          int* err) {
    static_assert(NBUF >= 1 && NBUF <= 3, "one to three tile buffers (the barrier area holds eight barriers)");
    using Lay = XztLayout<P, TC, NBUF>;
    constexpr int N = Lay::N, T = Lay::T, PTS = Lay::PTS, ROWS = Lay::ROWS, NBOX = Lay::NBOX;
    constexpr int NST = kPlans[P].nst;
    constexpr bool CONV = MODE == XZ_CONV;
    constexpr uint32_t TILE_BYTES = (uint32_t)PTS * 8u;
    constexpr int NT = NTH;
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = smraw + ((1024 - (pktma::smem_u32(smraw) & 1023)) & 1023);
    float2* bufs[NBUF];
    for (int i = 0; i < NBUF; i++) bufs[i] = (float2*)(sm + i * Lay::BUF);
    float2* hb = (float2*)(sm + NBUF * Lay::BUF);
    float2* tw = (float2*)(sm + NBUF * Lay::BUF + (CONV ? Lay::BUF : 0));
    // barriers: full[0..1] (tile landed), empty[0..1] (compute done with the buffer), otf_full, otf_empty
    uint64_t* bars = (uint64_t*)((unsigned char*)tw + Lay::TW);
    uint64_t* full = bars;
    uint64_t* empty = bars + NBUF;
    uint64_t* otf_full = bars + 2 * NBUF;
    uint64_t* otf_empty = bars + 2 * NBUF + 1;
    const int tid = threadIdx.x;
    const int total = prefix[nvol];
    if ((int)blockIdx.x >= total) return;
    if (!PK_SMEM_OK(descs[0], Lay::bytes(CONV), 6)) return;   // uniform over the CTA, before any barrier

    // tile g -> volume and TMA coordinates of its first box (box r adds r*ROWS on the line's axis)
    auto locate = [&](int g, int& vol, int& c0, int& c1, int& c2) {
        vol = find_vol(prefix, nvol, g);
        const int lb = g - prefix[vol];
        const int ctiles = (descs[vol].Py + T - 1) / T;
        const int outer = lb / ctiles;
        c0 = 2 * (lb - outer * ctiles) * T;
        if (AXIS == 1) { c1 = 0; c2 = outer; }
        else { c1 = outer; c2 = 0; }
    };
    auto box_load = [&](const CUtensorMap* map, int c0, int c1, int c2, float2* dst, uint64_t* bar) {
        pktma::mbar_expect_tx(bar, TILE_BYTES);
#pragma unroll
        for (int r = 0; r < NBOX; r++) {
            if (AXIS == 1) pktma::tma_load_3d(dst + r * ROWS * T, map, c0, c1 + r * ROWS, c2, bar);
            else pktma::tma_load_3d(dst + r * ROWS * T, map, c0, c1, c2 + r * ROWS, bar);
        }
    };
    auto box_store = [&](const CUtensorMap* map, int c0, int c1, int c2, const float2* src) {
#pragma unroll
        for (int r = 0; r < NBOX; r++) {
            if (AXIS == 1) pktma::tma_store_3d(map, c0, c1 + r * ROWS, c2, src + r * ROWS * T);
            else pktma::tma_store_3d(map, c0, c1, c2 + r * ROWS, src + r * ROWS * T);
        }
        pktma::bulk_commit();
    };

    if (tid == 0) {
        for (int i = 0; i < 2 * NBUF + 2; i++) pktma::mbar_init(&bars[i], 1);
        pktma::fence_mbar_init();
    }
    // the plan's twiddles, once per CTA (every volume of the launch has this plan)
    {
        const float2* gtw = AXIS == 1 ? descs[0].ax.tw : descs[0].az.tw;
        for (int i = tid; i < plan_tw_size(P); i += NTH + 32) tw[i] = gtw[i];
    }
    __syncthreads();

    if (tid >= NT) {
        // ---------------- producer
        if (tid != NT) return;
        for (int v = 0; v < nvol; v++) {
            pktma::tmap_acquire(&maps[v].s);
            if (CONV) pktma::tmap_acquire(&maps[v].otf);
        }
        int it = 0;
        int pv[NBUF], pc[NBUF][3];   // volume and coordinates of each buffer's tile
        for (int g = blockIdx.x; g < total; g += gridDim.x, it++) {
            const int s = it % NBUF;
            int vol, c0, c1, c2;
            locate(g, vol, c0, c1, c2);
            if (it >= NBUF) {
                // tile it - NBUF is done with buffer s: store it, let the store read the buffer
                if (!pktma::mbar_wait(&empty[s], (uint32_t)(((it / NBUF) - 1) & 1))) {
                    pktma::report_wait_failure(err, 1);
                    break;
                }
                box_store(&maps[pv[s]].s, pc[s][0], pc[s][1], pc[s][2], bufs[s]);
                pktma::bulk_wait_read_all();
            }
            pktma::fence_async_smem();
            box_load(&maps[vol].s, c0, c1, c2, bufs[s], &full[s]);
            pv[s] = vol;
            pc[s][0] = c0; pc[s][1] = c1; pc[s][2] = c2;
            if (CONV) {
                if (it >= 1 && !pktma::mbar_wait(otf_empty, (uint32_t)((it - 1) & 1))) {
                    pktma::report_wait_failure(err, 1);
                    break;
                }
                box_load(&maps[vol].otf, c0, c1, c2, hb, otf_full);
            }
        }
        // the last tiles: store each once compute has released its buffer
        const int n_it = it;
        for (int k = n_it - NBUF < 0 ? 0 : n_it - NBUF; k < n_it; k++) {
            const int s = k % NBUF;
            if (!pktma::mbar_wait(&empty[s], (uint32_t)((k / NBUF) & 1))) {
                pktma::report_wait_failure(err, 1);
                break;
            }
            box_store(&maps[pv[s]].s, pc[s][0], pc[s][1], pc[s][2], bufs[s]);
        }
        pktma::bulk_wait_all();
        return;
    }

    // ---------------- compute (warps 0 .. NTH/32 - 1)
    int it = 0;
    for (int g = blockIdx.x; g < total; g += gridDim.x, it++) {
        const int s = it % NBUF;
        float2* cur = bufs[s];
        const int vol = find_vol(prefix, nvol, g);
        bool ok = pktma::mbar_wait(&full[s], (uint32_t)((it / NBUF) & 1));
        if (!compute_bar_and<NTH>(ok)) {
            if (tid == 0) pktma::report_wait_failure(err, 1);
            return;
        }
        if constexpr (!CONV) {
            run_dense<P, 0, NST, 1, T, MODE == XZ_INV, NTH>(cur, tw, tid);
        } else {
            const bool cj = descs[vol].conj != 0;
            if constexpr (pkpass::same_end_radix(P)) {
                constexpr int R = kPlans[P].rad[0], MS = N / R, MAXB = (T * MS + NT - 1) / NT;
                float2 v[MAXB][R];
                run_dense<P, 0, NST - 1, 1, T, false, NTH>(cur, tw, tid);
                dstage_s2r<R, plan_ns_before(P, NST - 1), N, T, false, stage_tw_off(P, NST - 1), NTH>(cur, tw, tid, v);
                ok = pktma::mbar_wait(otf_full, (uint32_t)(it & 1));
                if (!compute_bar_and<NTH>(ok)) {
                    if (tid == 0) pktma::report_wait_failure(err, 1);
                    return;
                }
#pragma unroll
                for (int i = 0; i < MAXB; i++) {
                    const int b = tid + i * NT;
                    if (MAXB * NT == T * MS || b < T * MS) {
                        const int l = b % T, j = b / T;
#pragma unroll
                        for (int r = 0; r < R; r++) {
                            float2 h = hb[(j + r * MS) * T + l];
                            if (cj) h.y = -h.y;
                            v[i][r] = cmul(v[i][r], h);
                        }
                    }
                }
                compute_bar<NTH>();   // every OTF read done: the producer may refill it
                if (tid == 0) mbar_arrive_cta(otf_empty);
                dstage_r2s<R, N, T, true, NTH>(cur, tid, v);
                run_dense<P, 1, NST, R, T, true, NTH>(cur, tw, tid);
            } else {
                run_dense<P, 0, NST, 1, T, false, NTH>(cur, tw, tid);
                ok = pktma::mbar_wait(otf_full, (uint32_t)(it & 1));
                if (!compute_bar_and<NTH>(ok)) {
                    if (tid == 0) pktma::report_wait_failure(err, 1);
                    return;
                }
                for (int i = tid; i < PTS; i += NT) {
                    float2 h = hb[i];
                    if (cj) h.y = -h.y;
                    cur[i] = cmul(cur[i], h);
                }
                compute_bar<NTH>();
                if (tid == 0) mbar_arrive_cta(otf_empty);
                run_dense<P, 0, NST, 1, T, true, NTH>(cur, tw, tid);
            }
        }
        // the tile leaves by TMA: each thread's writes are ordered before the async proxy's reads,
        // then the buffer is handed to the producer
        pktma::fence_async_smem();
        compute_bar<NTH>();
        if (tid == 0) mbar_arrive_cta(&empty[s]);
    }
}

// The TMA kernels by plan, pass and variant: [p][0] x forward, [p][1] x inverse, [p][2] z convolution;
// variant 0 is the plan's 4096-point tile with two buffers, variants 1 and 2 (where built) are the
// alternatives the autotuner times against it.  With each one's dynamic shared memory, resident CTAs
// per SM (the persistent grid is that times the SMs) and tile width.
enum { TMA_X_FWD = 0, TMA_X_INV = 1, TMA_Z_CONV = 2 };
constexpr int kTmaVariants = 3;
struct TmaTable {
    void (*k[kNumPlans][3][kTmaVariants])(const VolDesc*, const XZMaps*, const int*, int, int*);
    size_t smem[kNumPlans][3][kTmaVariants];
    int per_sm[kNumPlans][3][kTmaVariants];
    int cols[kNumPlans][3][kTmaVariants];    // columns per tile (the tile prefix and the TMA box follow it)
    int nbuf[kNumPlans][3][kTmaVariants];
    int threads[kNumPlans][3][kTmaVariants];   // compute threads + the producer warp
};

template <int P, int IDX, int VAR, int AXIS, int MODE, int TC = 0, int NBUF = 2, int NTH = PK_THREADS>
inline void register_tma_one(TmaTable& t) {
    auto fn = k_xzt<P, AXIS, MODE, TC, NBUF, NTH>;
    t.threads[P][IDX][VAR] = NTH + 32;
    const size_t smem = XztLayout<P, TC, NBUF>::bytes(MODE == XZ_CONV);
    t.k[P][IDX][VAR] = fn;
    t.smem[P][IDX][VAR] = smem;
    t.cols[P][IDX][VAR] = XztLayout<P, TC, NBUF>::T;
    t.nbuf[P][IDX][VAR] = NBUF;
    int n = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, NTH + 32, smem) != cudaSuccess || n < 1) {
        cudaGetLastError();
        t.k[P][IDX][VAR] = nullptr;   // this variant is not offered
        n = 0;
    }
    t.per_sm[P][IDX][VAR] = n;
}

template <int P, int HI>
struct RegisterTma {
    static void fill(TmaTable& t) {
        if constexpr (tma_plan(P)) {
            register_tma_one<P, TMA_X_FWD, 0, 1, XZ_FWD>(t);
            register_tma_one<P, TMA_X_INV, 0, 1, XZ_INV>(t);
            register_tma_one<P, TMA_Z_CONV, 0, 2, XZ_CONV>(t);
            if constexpr (kPlans[P].n == 512) {
                // 8-column tiles (64-byte rows, 3 CTAs per SM) against 16-column tiles (128-byte rows,
                // one CTA per SM, 16 compute warps) with two or three buffers
                register_tma_one<P, TMA_X_FWD, 1, 1, XZ_FWD, 16, 2, 512>(t);
                register_tma_one<P, TMA_X_INV, 1, 1, XZ_INV, 16, 2, 512>(t);
                register_tma_one<P, TMA_X_FWD, 2, 1, XZ_FWD, 16, 3, 512>(t);
                register_tma_one<P, TMA_X_INV, 2, 1, XZ_INV, 16, 3, 512>(t);
            }
            if constexpr (kPlans[P].n == 256) {
                // the convolution with 32-column tiles (256-byte rows, two buffers, 16 compute warps) and
                // with 24-column tiles (three buffers, 12 compute warps), one CTA per SM
                register_tma_one<P, TMA_Z_CONV, 1, 2, XZ_CONV, 32, 2, 512>(t);
                register_tma_one<P, TMA_Z_CONV, 2, 2, XZ_CONV, 24, 3, 384>(t);
            }
            if constexpr (kPlans[P].n > 256 && kPlans[P].n < 512) {
                // lines longer than 256: the 4096-point tile is 8 columns (64-byte rows) or fewer wide;
                // 16-column tiles (128-byte rows), 16 compute warps, three or two buffers, one CTA per SM
                register_tma_one<P, TMA_X_FWD, 1, 1, XZ_FWD, 16, 3, 512>(t);
                register_tma_one<P, TMA_X_INV, 1, 1, XZ_INV, 16, 3, 512>(t);
                register_tma_one<P, TMA_X_FWD, 2, 1, XZ_FWD, 16, 2, 512>(t);
                register_tma_one<P, TMA_X_INV, 2, 1, XZ_INV, 16, 2, 512>(t);
                if constexpr (XztLayout<P, 16, 3>::bytes(true) <= 227 * 1024)
                    register_tma_one<P, TMA_Z_CONV, 1, 2, XZ_CONV, 16, 3, 384>(t);
                register_tma_one<P, TMA_Z_CONV, 2, 2, XZ_CONV, 16, 2, 512>(t);
            }
            if constexpr (kPlans[P].n >= 128 && kPlans[P].n < 256) {
                // 16- or 32-column tiles already: three buffers (x)
                register_tma_one<P, TMA_X_FWD, 1, 1, XZ_FWD, 0, 3>(t);
                register_tma_one<P, TMA_X_INV, 1, 1, XZ_INV, 0, 3>(t);
            }
        }
        RegisterTma<P + 1, HI>::fill(t);
    }
};
template <int HI>
struct RegisterTma<HI, HI> {
    static void fill(TmaTable&) {}
};

}  // namespace pkpass
