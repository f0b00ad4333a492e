// Fused convolution pass: x forward, z forward-OTF-inverse and x inverse of one volume in one
// persistent launch, with the spectrum's k-columns flowing through the three stages so that the
// data between stages stays in L2.
//
// The separate passes move 7 Sb per convolution (x: read + write, z: read + OTF + write, x: read +
// write); the ruler is 3 Sb (read S, read the OTF, write S).  Here the k-columns are cut into
// K = ceil(Py / T) column tiles c.  For each c, the work items are the x-line tiles X(c, z) (one per
// z), then the z-line tiles Z(c, x) (one per x) and then the x-line tiles I(c, z); the items run in
// rounds r = 0 .. K + 1 of [X(r), Z(r - 1), I(r - 2)], so while column tile c is in its z stage,
// c + 1 is in its first x stage and c - 1 in its last, and the three column tiles in flight
// (3 x T x nx x nz x 8 bytes, 50 MB for 512 x 256 at T = 16) fit in L2: each stage reads the previous
// stage's output from L2, not from DRAM.
//
// A Z(c, .) item may start once every X(c, .) item is stored, an I(c, .) item once every Z(c, .)
// item is: per-column-tile counters in global memory, raised with release semantics after a tile's
// store has completed and read with acquire semantics before the dependent tile is loaded.  CTAs
// claim items in sequence order from a global counter (an atomic add), so every claimed item is held
// by a running CTA and the lowest unfinished item always has its inputs complete: the launch makes
// progress with any number of its CTAs resident (other kernels may hold SMs).  The producer warp
// runs an event loop: it stores tiles whose transform is done, claims and loads the next item when a
// buffer is free and the item's inputs are complete, and publishes its completed stores; when
// nothing moves for PK_WAIT_LIMIT_NS it records a timeout in the status word and the CTA stops.
// Every wait of the compute warps is bounded too.  The counters (claim counter, then K + K column
// counters) arrive as zeros with the program's descriptors before every launch.
#pragma once
#include "pass_tma.cuh"

namespace pkpass {

enum { C3_X = 0, C3_Z = 1, C3_I = 2 };

// Sequence index -> item: type, column tile c, line o (z for X / I items, x for Z items).
__device__ __forceinline__ void c3_locate(int i, int K, int nx, int nz, int& type, int& c, int& o) {
    int rem = i;
    if (rem < nz) { type = C3_X; c = 0; o = rem; return; }
    rem -= nz;
    if (K > 1) {
        if (rem < nz) { type = C3_X; c = 1; o = rem; return; }
        rem -= nz;
    }
    if (rem < nx) { type = C3_Z; c = 0; o = rem; return; }
    rem -= nx;
    const int B = 2 * nz + nx;
    const int mid = K > 2 ? K - 2 : 0;
    if (rem < mid * B) {
        const int q = rem / B, w = rem - q * B, r = 2 + q;
        if (w < nz) { type = C3_X; c = r; o = w; }
        else if (w < nz + nx) { type = C3_Z; c = r - 1; o = w - nz; }
        else { type = C3_I; c = r - 2; o = w - nz - nx; }
        return;
    }
    rem -= mid * B;
    if (K >= 2) {
        if (rem < nx) { type = C3_Z; c = K - 1; o = rem; return; }
        rem -= nx;
        if (rem < nz) { type = C3_I; c = K - 2; o = rem; return; }
        rem -= nz;
    }
    type = C3_I; c = K - 1; o = rem;
}

// shared memory of k_conv3: NBUF tile buffers (each the larger of an x tile and a z tile) | OTF tile
// | x twiddles | z twiddles | barriers, 1024 bytes of slack to align the base
template <int PX, int PZ, int T, int NBUF>
struct Conv3Layout {
    static constexpr int NX = kPlans[PX].n, NZ = kPlans[PZ].n;
    static constexpr size_t XB = (size_t)T * NX * 8, ZB = (size_t)T * NZ * 8;
    static constexpr size_t BUF = (((XB > ZB ? XB : ZB)) + 1023) & ~(size_t)1023;
    static constexpr size_t OTF = (ZB + 1023) & ~(size_t)1023;
    static constexpr size_t TWX = ((size_t)(plan_tw_size(PX) > 0 ? plan_tw_size(PX) : 1) * 8 + 15) & ~(size_t)15;
    static constexpr size_t TWZ = ((size_t)(plan_tw_size(PZ) > 0 ? plan_tw_size(PZ) : 1) * 8 + 15) & ~(size_t)15;
    static constexpr size_t bytes() { return 1024 + NBUF * BUF + OTF + TWX + TWZ + 64; }
    static_assert(1024 + NBUF * BUF + OTF + TWX + TWZ + 64 <= 227 * 1024, "tiles exceed shared memory");
};

template <int PX, int PZ, int T, int NBUF, int NTH>
__global__ void __launch_bounds__(NTH + 32, 1)
    k_conv3(const VolDesc* __restrict__ descs, const XZMaps* __restrict__ maps, int* cnt, int* err) {
    static_assert(NBUF >= 1 && NBUF <= 3, "one to three tile buffers (the barrier area holds eight barriers)");
    using Lay = Conv3Layout<PX, PZ, T, NBUF>;
    constexpr int NX = Lay::NX, NZ = Lay::NZ;
    constexpr int ROWSX = tma_box_rows(NX), NBOXX = NX / ROWSX;
    constexpr int ROWSZ = tma_box_rows(NZ), NBOXZ = NZ / ROWSZ;
    constexpr int NSTX = kPlans[PX].nst, NSTZ = kPlans[PZ].nst;
    constexpr uint32_t XBYTES = (uint32_t)Lay::XB, ZBYTES = (uint32_t)Lay::ZB;
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = smraw + ((1024 - (pktma::smem_u32(smraw) & 1023)) & 1023);
    float2* hb = (float2*)(sm + NBUF * Lay::BUF);
    float2* twx = (float2*)(sm + NBUF * Lay::BUF + Lay::OTF);
    float2* twz = (float2*)((unsigned char*)twx + Lay::TWX);
    uint64_t* bars = (uint64_t*)((unsigned char*)twz + Lay::TWZ);
    uint64_t* full = bars;
    uint64_t* empty = bars + NBUF;
    uint64_t* otf_full = bars + 2 * NBUF;
    uint64_t* otf_empty = bars + 2 * NBUF + 1;
    __shared__ int slot_item[NBUF];   // the item each buffer holds (-1: no more items)
    const int tid = threadIdx.x;
    const VolDesc& d = descs[0];
    const int K = (d.Py + T - 1) / T;
    const int nx = d.nx, nz = d.nz;
    const int total = K * (2 * nz + nx);
    int* next = cnt;
    int* cntX = cnt + 1;
    int* cntZ = cnt + 1 + K;
    if (!PK_SMEM_OK(d, Lay::bytes(), 7) || !PK_IN(d, nx == NX && nz == NZ, 8)) return;   // uniform, before any barrier
    auto buf = [&](int s) { return (float2*)(sm + s * Lay::BUF); };

    if (tid == 0) {
        for (int i = 0; i < 2 * NBUF + 2; i++) pktma::mbar_init(&bars[i], 1);
        pktma::fence_mbar_init();
    }
    for (int i = tid; i < plan_tw_size(PX); i += NTH + 32) twx[i] = d.ax.tw[i];
    for (int i = tid; i < plan_tw_size(PZ); i += NTH + 32) twz[i] = d.az.tw[i];
    __syncthreads();

    if (tid >= NTH) {
        // ---------------- producer: one thread runs the event loop
        if (tid != NTH) return;
        const XZMaps& m = maps[0];
        pktma::tmap_acquire(&m.s);
        pktma::tmap_acquire(&m.s2);
        pktma::tmap_acquire(&m.otf);
        int ring[8];   // items by local order (loaded - published <= NBUF + 2 < 8)
        int k_load = 0, k_store = 0, k_pub = 0, z_loaded = 0;
        int claimed = -1;        // claimed, waiting for its inputs
        bool exhausted = false;  // no items left: the compute warps have been told
        auto store = [&](int item, int s) {
            int type, c, o;
            c3_locate(item, K, nx, nz, type, c, o);
            const int c0 = 2 * c * T;
            if (type == C3_Z) {
#pragma unroll
                for (int r = 0; r < NBOXZ; r++) pktma::tma_store_3d(&m.s, c0, o, r * ROWSZ, buf(s) + r * ROWSZ * T);
            } else {
#pragma unroll
                for (int r = 0; r < NBOXX; r++) pktma::tma_store_3d(&m.s2, c0, r * ROWSX, o, buf(s) + r * ROWSX * T);
            }
            pktma::bulk_commit();
        };
        // raise the counters of stored items [k_pub, upto): their stores have completed
        auto publish = [&](int upto) {
            pktma::fence_async_global();
            for (; k_pub < upto; k_pub++) {
                int type, c, o;
                c3_locate(ring[k_pub & 7], K, nx, nz, type, c, o);
                if (type == C3_X) pktma::red_release_gpu_add(&cntX[c], 1);
                else if (type == C3_Z) pktma::red_release_gpu_add(&cntZ[c], 1);
            }
        };
        uint64_t t_last = pktma::global_ns();
        bool failed = false;
        while (!(exhausted && k_pub == k_load)) {
            bool prog = false;
            // a) the oldest transformed tile goes out
            if (k_store < k_load && pktma::mbar_try(&empty[k_store % NBUF], (uint32_t)((k_store / NBUF) & 1))) {
                store(ring[k_store & 7], k_store % NBUF);
                k_store++;
                prog = true;
            }
            // b) with a buffer free: claim the next item, load it once its inputs are complete
            if (!exhausted && k_load - k_store < NBUF) {
                const int s = k_load % NBUF;
                if (claimed < 0) {
                    claimed = atomicAdd(next, 1);
                    prog = true;
                    if (claimed >= total) {   // tell the compute warps: an arrival without bytes
                        claimed = -1;
                        exhausted = true;
                        if (k_load >= NBUF) pktma::bulk_wait_read_all();
                        slot_item[s] = -1;
                        mbar_arrive_cta(&full[s]);
                    }
                }
                if (claimed >= 0) {
                    int type, c, o;
                    c3_locate(claimed, K, nx, nz, type, c, o);
                    bool ready = type == C3_X || (type == C3_Z ? pktma::ld_acquire_gpu(&cntX[c]) >= nz
                                                               : pktma::ld_acquire_gpu(&cntZ[c]) >= nx);
                    if (ready && type == C3_Z && z_loaded > 0)   // the previous OTF tile is used up
                        ready = pktma::mbar_try(otf_empty, (uint32_t)((z_loaded - 1) & 1));
                    if (ready) {
                        if (k_load >= NBUF) pktma::bulk_wait_read_all();   // the buffer's last store has read it
                        pktma::fence_async_global();
                        slot_item[s] = claimed;
                        ring[k_load & 7] = claimed;
                        const int c0 = 2 * c * T;
                        if (type == C3_Z) {
                            pktma::mbar_expect_tx(&full[s], ZBYTES);
#pragma unroll
                            for (int r = 0; r < NBOXZ; r++)
                                pktma::tma_load_3d(buf(s) + r * ROWSZ * T, &m.s, c0, o, r * ROWSZ, &full[s]);
                            pktma::mbar_expect_tx(otf_full, ZBYTES);
#pragma unroll
                            for (int r = 0; r < NBOXZ; r++)
                                pktma::tma_load_3d(hb + r * ROWSZ * T, &m.otf, c0, o, r * ROWSZ, otf_full);
                            z_loaded++;
                        } else {
                            pktma::mbar_expect_tx(&full[s], XBYTES);
#pragma unroll
                            for (int r = 0; r < NBOXX; r++)
                                pktma::tma_load_3d(buf(s) + r * ROWSX * T, &m.s2, c0, r * ROWSX, o, &full[s]);
                        }
                        k_load++;
                        claimed = -1;
                        prog = true;
                    }
                }
            }
            // c) stores older than the newest are complete by now (each had a transform's time): publish;
            //    with nothing else to do, wait for all of them
            if (k_pub < k_store - 1) {
                asm volatile("cp.async.bulk.wait_group 1;\n" ::: "memory");
                publish(k_store - 1);
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
        if (failed) pktma::report_wait_failure(err, 1);
        pktma::bulk_wait_all();
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
        const int item = slot_item[s];
        if (item < 0) break;   // no more items
        int type, c, o;
        c3_locate(item, K, nx, nz, type, c, o);
        if (type == C3_X) {
            run_dense<PX, 0, NSTX, 1, T, false, NTH>(cur, twx, tid);
        } else if (type == C3_I) {
            run_dense<PX, 0, NSTX, 1, T, true, NTH>(cur, twx, tid);
        } else {
            const bool cj = d.conj != 0;
            if constexpr (same_end_radix(PZ)) {
                constexpr int R = kPlans[PZ].rad[0], MS = NZ / R, MAXB = (T * MS + NTH - 1) / NTH;
                float2 v[MAXB][R];
                run_dense<PZ, 0, NSTZ - 1, 1, T, false, NTH>(cur, twz, tid);
                dstage_s2r<R, plan_ns_before(PZ, NSTZ - 1), NZ, T, false, stage_tw_off(PZ, NSTZ - 1), NTH>(cur, twz, tid, v);
                ok = pktma::mbar_wait(otf_full, (uint32_t)(zc & 1));
                if (!compute_bar_and<NTH>(ok)) {
                    if (tid == 0) pktma::report_wait_failure(err, 1);
                    return;
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
                compute_bar<NTH>();   // every OTF read done: the producer may refill it
                if (tid == 0) mbar_arrive_cta(otf_empty);
                dstage_r2s<R, NZ, T, true, NTH>(cur, tid, v);
                run_dense<PZ, 1, NSTZ, R, T, true, NTH>(cur, twz, tid);
            } else {
                run_dense<PZ, 0, NSTZ, 1, T, false, NTH>(cur, twz, tid);
                ok = pktma::mbar_wait(otf_full, (uint32_t)(zc & 1));
                if (!compute_bar_and<NTH>(ok)) {
                    if (tid == 0) pktma::report_wait_failure(err, 1);
                    return;
                }
                for (int i = tid; i < T * NZ; i += NTH) {
                    float2 h = hb[i];
                    if (cj) h.y = -h.y;
                    cur[i] = cmul(cur[i], h);
                }
                compute_bar<NTH>();
                if (tid == 0) mbar_arrive_cta(otf_empty);
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
    Conv3Entry e{PX, PZ, T, NTH + 32, Conv3Layout<PX, PZ, T, NBUF>::bytes(), k_conv3<PX, PZ, T, NBUF, NTH>};
    if (cudaFuncSetAttribute(e.k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem) != cudaSuccess) {
        cudaGetLastError();
        e.k = nullptr;
    }
    return e;
}

}  // namespace pkpass
