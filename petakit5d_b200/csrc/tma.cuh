// Tensor-memory-accelerator (TMA) and mbarrier primitives for sm_100a, as inline PTX.
//
// Tiled bulk tensor copies (cp.async.bulk.tensor) move a box of a global tensor into shared memory
// with one instruction and signal an mbarrier with the bytes delivered; stores go the other way as
// bulk groups.  None of these copies uses cluster multicast: every tensor map covers this GPU's own
// buffers.  Waits on an mbarrier are bounded by a deadline on the global timer; a wait that runs out
// reports failure instead of spinning on.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace pktma {

// Deadline of one mbarrier wait: far above any tile's load time (microseconds), far below a hang.
#define PK_WAIT_LIMIT_NS 1000000000ull

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes the barriers' initialisation visible to the async proxy (the TMA unit)
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// orders this thread's generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Waits for the phase of `bar` with the given parity to complete; false when limit_ns passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = PK_WAIT_LIMIT_NS) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// Records that a device wait ran out in the context's page-locked status word (the host reads it).
__device__ __forceinline__ void report_wait_failure(int* err, int code) {
    if (err) {
        *(volatile int*)err = code;
        __threadfence_system();
    }
}

// 3-D tiled load of the box at (c0, c1, c2) (c0 innermost, in elements) into shared memory; the
// delivered bytes complete on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// L2 eviction priorities for the cache-hinted copies below (applied to every line a copy touches)
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}

// tma_load_3d with an L2 eviction priority
__device__ __forceinline__ void tma_load_3d_hint(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar,
                                                 uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, %3, "
        "%4}], [%5], %6;\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}

// Prefetch of the box at (c0, c1, c2) into L2 (no shared memory, no completion to wait for)
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];\n" ::"l"(map), "r"(c0), "r"(c1),
                 "r"(c2)
                 : "memory");
}

// Untiled bulk copy of `bytes` contiguous bytes (both addresses 16-byte aligned, bytes a multiple
// of 16) from global to shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 3-D tiled store of a shared-memory box to (c0, c1, c2); elements outside the tensor are not written.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int c0, int c1, int c2, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(map), "r"(c0),
                 "r"(c1), "r"(c2), "r"(smem_u32(src))
                 : "memory");
}

// tma_store_3d with an L2 eviction priority
__device__ __forceinline__ void tma_store_3d_hint(const CUtensorMap* map, int c0, int c1, int c2, const void* src,
                                                  uint64_t pol) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2, %3}], [%4], %5;\n" ::"l"(
                     map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src)), "l"(pol)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the shared-memory sources of every committed store have been read
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// every committed store has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// orders this thread's generic-proxy global accesses with its async-proxy (bulk copy) ones
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }

// an int in global memory read with gpu-scope acquire / raised with gpu-scope release
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_gpu_add(int* p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// a tensor map that the host wrote to global memory before the launch, made visible to the TMA unit
__device__ __forceinline__ void tmap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
}

}  // namespace pktma
