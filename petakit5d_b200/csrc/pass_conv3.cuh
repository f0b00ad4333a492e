// Fused convolution pass: x forward, z forward-OTF-inverse and x inverse of one volume in one
// persistent launch, with the spectrum's k-columns flowing through the three stages so that the
// data between stages stays in L2.
//
// The separate passes move 7 Sb per convolution (x: read + write, z: read + OTF + write, x: read +
// write); the ruler is 3 Sb (read S, read the OTF, write S).  Here the k-columns are cut into
// K = ceil(Py / T) column tiles c.  For each c, the work items are the x-line tiles X(c, z) (one per
// z), then the z-line tiles Z(c, x) (one per x) and then the x-line tiles I(c, z), in the sequence
// of c3_locate; the copies carry L2 eviction priorities (intermediate tiles evict-last, data read
// or written for the last time evict-first) so that the intermediates stay in L2 while the
// streaming reads and writes pass through it.
//
// A Z(c, .) item may start once every X(c, .) item is stored, an I(c, .) item once every Z(c, .)
// item is: per-column-tile counters in global memory, raised with release semantics after a tile's
// store has completed and read with acquire semantics before the dependent tile is loaded.  CTAs
// claim items in sequence order from a global counter (an atomic add), so every claimed item is held
// by a running CTA and the lowest unfinished item always has its inputs complete: the launch makes
// progress with any number of its CTAs resident (other kernels may hold SMs).  Two producer threads
// run beside the compute warps: the loader claims the next item, waits for its inputs, prefetches its
// tiles into L2 and loads them when a buffer is free; the storer stores transformed tiles in order,
// frees their buffers and publishes completed stores.  When nothing moves for PK_WAIT_LIMIT_NS either
// records a timeout in the status word and stops; every wait of the compute warps is bounded too.
// The counters (claim counter, then K + K column counters, one 128-byte line each) arrive as zeros
// with the program's descriptors before every launch.
#pragma once
#include "pass_tma.cuh"

namespace pkpass {

enum { C3_X = 0, C3_Z = 1, C3_I = 2 };

// Sequence index -> item: type, column tile c, line o (z for X / I items, x for Z items).  The
// sequence is X(0), X(1), then per column tile b: Z(b), I(b - 1) (b >= 1), X(b + 2) (b + 2 < K), and
// last I(K - 1): a Z block starts about nx + 2 nz items after its X block ended, an I block
// about the same after its Z block, so the items other CTAs still hold (up to NBUF + 1 each) have
// finished by then, while about three column tiles of intermediates are live in L2.
__device__ __forceinline__ void c3_locate(int i, int K, int nx, int nz, int& type, int& c, int& o) {
    const int pro = (K < 2 ? K : 2) * nz;
    if (i < pro) {
        type = C3_X;
        c = i / nz;
        o = i - c * nz;
        return;
    }
    int rem = i - pro;
    const int b0 = nx + (K > 2 ? nz : 0);   // block 0: Z(0), X(2)
    if (rem < b0) {
        if (rem < nx) { type = C3_Z; c = 0; o = rem; }
        else { type = C3_X; c = 2; o = rem - nx; }
        return;
    }
    rem -= b0;
    const int nmid = K > 3 ? K - 3 : 0, B = nx + 2 * nz;   // blocks 1 .. K - 3: Z(b), I(b - 1), X(b + 2)
    if (rem < nmid * B) {
        const int q = rem / B, w = rem - q * B, b = 1 + q;
        if (w < nx) { type = C3_Z; c = b; o = w; }
        else if (w < nx + nz) { type = C3_I; c = b - 1; o = w - nx; }
        else { type = C3_X; c = b + 2; o = w - nx - nz; }
        return;
    }
    rem -= nmid * B;
    for (int b = K - 2 > 1 ? K - 2 : 1; b <= K - 1; b++) {   // the last blocks: Z(b), I(b - 1)
        if (rem < nx) { type = C3_Z; c = b; o = rem; return; }
        rem -= nx;
        if (rem < nz) { type = C3_I; c = b - 1; o = rem; return; }
        rem -= nz;
    }
    type = C3_I;
    c = K - 1;
    o = rem;
}

// The claim counter and the column-tile counters each sit on their own 128-byte line (32 ints), so
// that the claims, the polls and the raises of different counters do not queue on one L2 line.
constexpr int kC3Line = 32;
__host__ __device__ constexpr int c3_counter_ints(int K) { return (1 + 2 * K) * kC3Line; }

// shared memory of k_conv3: NBUF tile buffers | OTF tile | x twiddles | z twiddles | barriers, 1024
// bytes of slack to align the base.  When NBUF buffers of an x tile or a z tile plus its OTF tile
// fit (OIB), a z item's OTF tile travels in its own buffer behind the S tile and there is no
// separate OTF buffer; otherwise each buffer is the larger of an x and a z tile and one OTF buffer
// serves the z items in turn.
template <int PX, int PZ, int T, int NBUF>
struct Conv3Layout {
    static constexpr int NX = kPlans[PX].n, NZ = kPlans[PZ].n;
    static constexpr size_t XB = (size_t)T * NX * 8, ZB = (size_t)T * NZ * 8;
    static constexpr size_t TWX = ((size_t)(plan_tw_size(PX) > 0 ? plan_tw_size(PX) : 1) * 8 + 15) & ~(size_t)15;
    static constexpr size_t TWZ = ((size_t)(plan_tw_size(PZ) > 0 ? plan_tw_size(PZ) : 1) * 8 + 15) & ~(size_t)15;
    static constexpr size_t BUF_OIB = (((XB > 2 * ZB ? XB : 2 * ZB)) + 1023) & ~(size_t)1023;
    static constexpr size_t BARS = (8 * (3 * (size_t)NBUF + 2) + 15) & ~(size_t)15;
    static constexpr bool OIB = 1024 + NBUF * BUF_OIB + TWX + TWZ + BARS <= 227 * 1024;
    static constexpr size_t BUF = OIB ? BUF_OIB : (((XB > ZB ? XB : ZB)) + 1023) & ~(size_t)1023;
    static constexpr size_t OTF = OIB ? 0 : (ZB + 1023) & ~(size_t)1023;
    static constexpr size_t bytes() { return 1024 + NBUF * BUF + OTF + TWX + TWZ + BARS; }
    static_assert(1024 + NBUF * BUF + OTF + TWX + TWZ + BARS <= 227 * 1024, "tiles exceed shared memory");
};

// z convolution of a z tile whose OTF tile is in shared memory already: the forward stages but the
// last in shared memory; the last forward stage, the OTF multiply and the first inverse stage in
// registers, one butterfly column per thread for the first B = T NZ / R threads (whole warps; the
// others only keep the barriers); the remaining inverse stages in shared memory.  The same element
// order, twiddles and operations as dstage_s2r / dstage_r2s with the multiply between them.
template <int PZ, int T, int NTH>
__device__ __forceinline__ void c3_zconv(float2* __restrict__ cur, const float2* __restrict__ twz,
                                         const float2* __restrict__ hb, bool cj, int tid) {
    constexpr int NZ = kPlans[PZ].n, NST = kPlans[PZ].nst, R = kPlans[PZ].rad[0], MS = NZ / R, B = T * MS;
    constexpr int NS = plan_ns_before(PZ, NST - 1), OFF = stage_tw_off(PZ, NST - 1);
    static_assert(same_end_radix(PZ) && !direct_radix(R) && NS == MS, "first and last radix equal, register butterfly");
    static_assert(B <= NTH && B % 32 == 0, "one butterfly column per thread, whole warps");
    run_dense<PZ, 0, NST - 1, 1, T, false, NTH>(cur, twz, tid);
    float2 v[R];
    const int l = tid % T, j = tid / T;
    if (tid < B) {
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = cur[(j + r * MS) * T + l];
    }
    compute_bar<NTH>();   // every element read before the first inverse stage overwrites the tile
    if (tid < B) {
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) v[r] = cmul(v[r], twz[OFF + (r - 1) * NS + j]);
        }
        bfly<R, false>(v);
#pragma unroll
        for (int r = 0; r < R; r++) {
            float2 h = hb[(j + r * MS) * T + l];
            if (cj) h.y = -h.y;
            v[r] = cmul(v[r], h);
        }
        bfly<R, true>(v);
        const int a0 = j * R * T + l;
#pragma unroll
        for (int r = 0; r < R; r++) cur[a0 + r * T] = v[r];
    }
    compute_bar<NTH>();
    run_dense<PZ, 1, NST, R, T, true, NTH>(cur, twz, tid);
}

template <int PX, int PZ, int T, int NBUF, int NTH>
__global__ void __launch_bounds__(NTH + 64, 1)
    k_conv3(const VolDesc* __restrict__ descs, const XZMaps* __restrict__ maps, int* cnt, int* err) {
    static_assert(NBUF >= 1 && NBUF <= 4, "one to four tile buffers");
    using Lay = Conv3Layout<PX, PZ, T, NBUF>;
    constexpr bool OIB = Lay::OIB;
    constexpr int NX = Lay::NX, NZ = Lay::NZ;
    constexpr int ROWSX = tma_box_rows(NX), NBOXX = NX / ROWSX;
    constexpr int ROWSZ = tma_box_rows(NZ), NBOXZ = NZ / ROWSZ;
    constexpr int NSTX = kPlans[PX].nst, NSTZ = kPlans[PZ].nst;
    constexpr uint32_t XBYTES = (uint32_t)Lay::XB, ZBYTES = (uint32_t)Lay::ZB;
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = smraw + ((1024 - (pktma::smem_u32(smraw) & 1023)) & 1023);
    float2* twx = (float2*)(sm + NBUF * Lay::BUF + Lay::OTF);
    float2* twz = (float2*)((unsigned char*)twx + Lay::TWX);
    uint64_t* bars = (uint64_t*)((unsigned char*)twz + Lay::TWZ);
    uint64_t* full = bars;               // a tile has landed (the compute warps wait)
    uint64_t* empty = bars + NBUF;       // a tile is transformed (the storer waits)
    uint64_t* freed = bars + 2 * NBUF;   // a tile's store has read the buffer (the loader waits)
    uint64_t* otf_full = bars + 3 * NBUF;
    uint64_t* otf_empty = bars + 3 * NBUF + 1;
    __shared__ int slot_item[NBUF];   // the item each buffer holds (-1: no more items)
    __shared__ int slot_type[NBUF];   // its type (C3_X / C3_Z / C3_I) for the compute warps
    __shared__ int n_items;           // items this CTA loaded, once the loader has no more (-1 before)
    const int tid = threadIdx.x;
    const VolDesc& d = descs[0];
    const int K = (d.Py + T - 1) / T;
    const int nx = d.nx, nz = d.nz;
    const int total = K * (2 * nz + nx);
    int* next = cnt;   // counter i at cnt[i * kC3Line]: the claim counter, then X and Z counters
    auto cntX = [&](int c) { return cnt + (1 + c) * kC3Line; };
    auto cntZ = [&](int c) { return cnt + (1 + K + c) * kC3Line; };
    if (!PK_SMEM_OK(d, Lay::bytes(), 7) || !PK_IN(d, nx == NX && nz == NZ, 8)) return;   // uniform, before any barrier
    auto buf = [&](int s) { return (float2*)(sm + s * Lay::BUF); };
    // the OTF tile of a z item in buffer s
    auto otf_of = [&](int s) { return OIB ? buf(s) + T * NZ : (float2*)(sm + NBUF * Lay::BUF); };

    if (tid == 0) {
        for (int i = 0; i < 3 * NBUF + 2; i++) pktma::mbar_init(&bars[i], 1);
        pktma::fence_mbar_init();
        n_items = -1;
    }
    for (int i = tid; i < plan_tw_size(PX); i += NTH + 64) twx[i] = d.ax.tw[i];
    for (int i = tid; i < plan_tw_size(PZ); i += NTH + 64) twz[i] = d.az.tw[i];
    __syncthreads();

    if (tid >= NTH) {
        // ---------------- two producer threads: the loader (first lane of warp NTH / 32) claims
        // items, waits for their inputs and a free buffer and loads them; the storer (first lane of
        // the next warp) stores transformed tiles in order, frees their buffers and publishes them
        if (tid != NTH && tid != NTH + 32) return;
        const XZMaps& m = maps[0];
        const uint64_t keep = pktma::l2_evict_last();     // tiles the next stage reads back
        const uint64_t stream = pktma::l2_evict_first();  // first reads of S, OTF tiles, final tiles
        uint64_t t_last = pktma::global_ns();
        bool failed = false;
        if (tid == NTH) {
            pktma::tmap_acquire(&m.s);
            pktma::tmap_acquire(&m.s2);
            pktma::tmap_acquire(&m.otf);
            int k_load = 0, z_loaded = 0;
            int claimed = -1;      // the next item, claimed ahead of its buffer
            bool ready = false;    // its inputs are complete (its tiles are then prefetched into L2)
            bool no_more = false;  // the claim counter is past the last item
            for (;;) {
                bool prog = false;
                if (!no_more && claimed < 0) {
                    claimed = atomicAdd(next, 1);
                    prog = true;
                    if (claimed >= total) {
                        claimed = -1;
                        no_more = true;
                    }
                }
                int type = C3_X, c = 0, o = 0;
                if (claimed >= 0) {
                    c3_locate(claimed, K, nx, nz, type, c, o);
                    if (!ready) {
                        ready = type == C3_X || (type == C3_Z ? pktma::ld_acquire_gpu(cntX(c)) >= nz
                                                              : pktma::ld_acquire_gpu(cntZ(c)) >= nx);
                        prog |= ready;
                        if (!ready) {
                            __nanosleep(128);   // back off: many CTAs poll the same counter
                        } else {
                            // while a buffer frees up, bring the item's tiles from DRAM into L2
                            const int c0 = 2 * c * T;
                            if (type == C3_Z) {
#pragma unroll
                                for (int r = 0; r < NBOXZ; r++) {
                                    pktma::tma_prefetch_3d(&m.s, c0, o, r * ROWSZ);
                                    pktma::tma_prefetch_3d(&m.otf, c0, o, r * ROWSZ);
                                }
                            } else {
#pragma unroll
                                for (int r = 0; r < NBOXX; r++) pktma::tma_prefetch_3d(&m.s2, c0, r * ROWSX, o);
                            }
                        }
                    }
                }
                const int s = k_load % NBUF;
                if ((ready || no_more) &&
                    (k_load < NBUF || pktma::mbar_try(&freed[s], (uint32_t)(((k_load / NBUF) - 1) & 1)))) {
                    if (claimed < 0) {   // an arrival without bytes: no more items
                        slot_item[s] = -1;
                        slot_type[s] = -1;
                        *(volatile int*)&n_items = k_load;
                        mbar_arrive_cta(&full[s]);
                        break;
                    }
                    // a z item without its own OTF space waits until the previous z item has used the OTF tile
                    if (OIB || type != C3_Z || z_loaded == 0 || pktma::mbar_try(otf_empty, (uint32_t)((z_loaded - 1) & 1))) {
                        pktma::fence_async_global();
                        slot_item[s] = claimed;
                        slot_type[s] = type;
                        const int c0 = 2 * c * T;
                        if (type == C3_Z) {
                            uint64_t* ob = OIB ? &full[s] : otf_full;
                            if (OIB) {
                                pktma::mbar_expect_tx(&full[s], 2 * ZBYTES);
                            } else {
                                pktma::mbar_expect_tx(&full[s], ZBYTES);
                                pktma::mbar_expect_tx(otf_full, ZBYTES);
                            }
#pragma unroll
                            for (int r = 0; r < NBOXZ; r++)
                                pktma::tma_load_3d_hint(buf(s) + r * ROWSZ * T, &m.s, c0, o, r * ROWSZ, &full[s], keep);
#pragma unroll
                            for (int r = 0; r < NBOXZ; r++)
                                pktma::tma_load_3d_hint(otf_of(s) + r * ROWSZ * T, &m.otf, c0, o, r * ROWSZ, ob, stream);
                            z_loaded++;
                        } else {
                            pktma::mbar_expect_tx(&full[s], XBYTES);
#pragma unroll
                            for (int r = 0; r < NBOXX; r++)
                                pktma::tma_load_3d_hint(buf(s) + r * ROWSX * T, &m.s2, c0, r * ROWSX, o, &full[s], stream);
                        }
                        k_load++;
                        claimed = -1;
                        ready = false;
                        prog = true;
                    }
                }
                const uint64_t now = pktma::global_ns();
                if (prog) {
                    t_last = now;
                } else if (now - t_last > PK_WAIT_LIMIT_NS) {
                    failed = true;
                    break;
                }
            }
        } else {
            pktma::tmap_acquire(&m.s);
            pktma::tmap_acquire(&m.s2);
            int ring[8];   // items stored and not yet published (at most three)
            int k_store = 0, k_pub = 0;
            // raise the counters of stored items [k_pub, upto): their stores have completed
            auto publish = [&](int upto) {
                pktma::fence_async_global();
                for (; k_pub < upto; k_pub++) {
                    int type, c, o;
                    c3_locate(ring[k_pub & 7], K, nx, nz, type, c, o);
                    if (type == C3_X) pktma::red_release_gpu_add(cntX(c), 1);
                    else if (type == C3_Z) pktma::red_release_gpu_add(cntZ(c), 1);
                }
            };
            for (;;) {
                const int n = *(volatile int*)&n_items;
                if (n >= 0 && k_store == n && k_pub == k_store) break;
                bool prog = false;
                const int s = k_store % NBUF;
                if (pktma::mbar_try(&empty[s], (uint32_t)((k_store / NBUF) & 1))) {
                    const int item = slot_item[s];
                    int type, c, o;
                    c3_locate(item, K, nx, nz, type, c, o);
                    const int c0 = 2 * c * T;
                    if (type == C3_Z) {
#pragma unroll
                        for (int r = 0; r < NBOXZ; r++)
                            pktma::tma_store_3d_hint(&m.s, c0, o, r * ROWSZ, buf(s) + r * ROWSZ * T, keep);
                    } else {
                        const uint64_t pol = type == C3_X ? keep : stream;   // I: the tile's final value
#pragma unroll
                        for (int r = 0; r < NBOXX; r++)
                            pktma::tma_store_3d_hint(&m.s2, c0, r * ROWSX, o, buf(s) + r * ROWSX * T, pol);
                    }
                    pktma::bulk_commit();
                    ring[k_store & 7] = item;
                    k_store++;
                    pktma::bulk_wait_read_all();   // the buffer has been read: the loader may refill it
                    mbar_arrive_cta(&freed[s]);
                    prog = true;
                }
                // stores older than the two newest are complete by now: publish; with nothing else
                // to do, wait for all of them
                if (k_pub < k_store - 2) {
                    asm volatile("cp.async.bulk.wait_group 2;\n" ::: "memory");
                    publish(k_store - 2);
                    prog = true;
                } else if (!prog && k_pub < k_store) {
                    pktma::bulk_wait_all();
                    publish(k_store);
                    prog = true;
                }
                const uint64_t now = pktma::global_ns();
                if (prog) {
                    t_last = now;
                } else if (now - t_last > PK_WAIT_LIMIT_NS) {
                    failed = true;
                    break;
                }
            }
            pktma::bulk_wait_all();
        }
        if (failed) pktma::report_wait_failure(err, 1);
        return;
    }

    // ---------------- compute (warps 0 .. NTH/32 - 1)
    int zc = 0;
    for (int k = 0;; k++) {
        const int s = k % NBUF;
        float2* cur = buf(s);
        bool ok = pktma::mbar_wait(&full[s], (uint32_t)((k / NBUF) & 1));
        if (!compute_bar_and<NTH>(ok)) {
            if (tid == 0) pktma::report_wait_failure(err, 1);
            return;
        }
        const int type = slot_type[s];
        if (type < 0) break;   // no more items
        if (type == C3_X) {
            run_dense<PX, 0, NSTX, 1, T, false, NTH>(cur, twx, tid);
        } else if (type == C3_I) {
            run_dense<PX, 0, NSTX, 1, T, true, NTH>(cur, twx, tid);
        } else {
            const bool cj = d.conj != 0;
            const float2* hb = otf_of(s);
            if constexpr (OIB && same_end_radix(PZ) && T * (NZ / kPlans[PZ].rad[0]) <= NTH &&
                          T * (NZ / kPlans[PZ].rad[0]) % 32 == 0) {
                c3_zconv<PZ, T, NTH>(cur, twz, hb, cj, tid);
            } else if constexpr (same_end_radix(PZ)) {
                constexpr int R = kPlans[PZ].rad[0], MS = NZ / R, MAXB = (T * MS + NTH - 1) / NTH;
                float2 v[MAXB][R];
                run_dense<PZ, 0, NSTZ - 1, 1, T, false, NTH>(cur, twz, tid);
                dstage_s2r<R, plan_ns_before(PZ, NSTZ - 1), NZ, T, false, stage_tw_off(PZ, NSTZ - 1), NTH>(cur, twz, tid, v);
                if (!OIB) {
                    ok = pktma::mbar_wait(otf_full, (uint32_t)(zc & 1));
                    if (!compute_bar_and<NTH>(ok)) {
                        if (tid == 0) pktma::report_wait_failure(err, 1);
                        return;
                    }
                }
#pragma unroll
                for (int i = 0; i < MAXB; i++) {
                    const int bb = tid + i * NTH;
                    if (MAXB * NTH == T * MS || bb < T * MS) {
                        const int l = bb % T, j = bb / T;
#pragma unroll
                        for (int r = 0; r < R; r++) {
                            float2 h = hb[(j + r * MS) * T + l];
                            if (cj) h.y = -h.y;
                            v[i][r] = cmul(v[i][r], h);
                        }
                    }
                }
                if (!OIB) {
                    compute_bar<NTH>();   // every OTF read done: the producer may refill it
                    if (tid == 0) mbar_arrive_cta(otf_empty);
                }
                dstage_r2s<R, NZ, T, true, NTH>(cur, tid, v);
                run_dense<PZ, 1, NSTZ, R, T, true, NTH>(cur, twz, tid);
            } else {
                run_dense<PZ, 0, NSTZ, 1, T, false, NTH>(cur, twz, tid);
                if (!OIB) {
                    ok = pktma::mbar_wait(otf_full, (uint32_t)(zc & 1));
                    if (!compute_bar_and<NTH>(ok)) {
                        if (tid == 0) pktma::report_wait_failure(err, 1);
                        return;
                    }
                }
                for (int i = tid; i < T * NZ; i += NTH) {
                    float2 h = hb[i];
                    if (cj) h.y = -h.y;
                    cur[i] = cmul(cur[i], h);
                }
                compute_bar<NTH>();
                if (!OIB && tid == 0) mbar_arrive_cta(otf_empty);
                run_dense<PZ, 0, NSTZ, 1, T, true, NTH>(cur, twz, tid);
            }
            zc++;
        }
        pktma::fence_async_smem();
        compute_bar<NTH>();
        if (tid == 0) mbar_arrive_cta(&empty[s]);
    }
}

// The fused kernels built, by (x plan, z plan).
struct Conv3Entry {
    int px, pz, cols, threads;
    size_t smem;
    void (*k)(const VolDesc*, const XZMaps*, int*, int*);
};

template <int PX, int PZ, int T, int NBUF, int NTH>
inline Conv3Entry conv3_entry() {
    Conv3Entry e{PX, PZ, T, NTH + 64, Conv3Layout<PX, PZ, T, NBUF>::bytes(), k_conv3<PX, PZ, T, NBUF, NTH>};
    if (cudaFuncSetAttribute(e.k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem) != cudaSuccess) {
        cudaGetLastError();
        e.k = nullptr;
    }
    return e;
}

}  // namespace pkpass
