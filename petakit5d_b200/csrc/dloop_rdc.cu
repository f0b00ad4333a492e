// Dispatcher of the server's device-resident request loop (compiled with relocatable device code:
// it launches graphs from the device).
//
// One thread polls the request ring in page-locked host memory.  Each ready entry is an admitted
// request's whole pass program, instantiated for device launch; the dispatcher launches it
// fire-and-forget, so a request that arrives while others run starts at once and its passes
// overlap theirs on the GPU, and no host round trip sits between requests.  Every wait is bounded:
// the loop polls with a short sleep and returns when the host asks it to stop, when it has
// launched kDlLaunchBudget graphs (the device runtime allows 120 fire-and-forget launches per
// launching graph's execution; the host then starts the next instance), when no entry has come
// for idle_ns (an idle dispatcher would otherwise hold up every device-wide synchronisation of the
// process; the host starts a new instance for the next entry), or when the host's heartbeat has
// not moved for heartbeat_ns (the host side is gone or stalled).  The reason goes to
// ring->exit_code.
#include "pk_internal.h"

namespace {

__device__ __forceinline__ unsigned long long dl_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ long long dl_load_acquire(const volatile long long* p) {
    long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__global__ void k_dispatch(DlRing* ring) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const long long my_epoch = ring->epoch_launched;
    int launched = 0;
    int code = DL_NONE;
    long long hb = ring->heartbeat;
    unsigned long long hb_seen = dl_now();
    const unsigned long long hb_limit = (unsigned long long)ring->heartbeat_ns;
    const unsigned long long idle_limit = (unsigned long long)ring->idle_ns;
    unsigned long long last_entry = hb_seen;
    for (;;) {
        if (ring->stop) {
            code = DL_STOPPED;
            break;
        }
        const long long tail = dl_load_acquire(&ring->tail);   // entries before tail are complete
        const long long head = ring->head;
        if (head < tail) {
            if (launched >= kDlLaunchBudget) {
                code = DL_BUDGET;
                break;
            }
            const int i = (int)(head % kDlRingCap);
            const cudaError_t e = cudaGraphLaunch(ring->graph[i], cudaStreamGraphFireAndForget);
            ring->epoch[i] = (int)my_epoch;
            ring->status[i] = 1 + (int)e;
            __threadfence_system();
            ring->head = head + 1;
            launched++;
            last_entry = dl_now();
            continue;
        }
        const unsigned long long now = dl_now();
        if (idle_limit && now - last_entry > idle_limit) {
            code = DL_IDLE;
            break;
        }
        const long long h = ring->heartbeat;
        if (h != hb) {
            hb = h;
            hb_seen = now;
        } else if (now - hb_seen > hb_limit) {
            code = DL_HEARTBEAT;
            break;
        }
        __nanosleep(2000);
    }
    ring->exit_code = code;
    __threadfence_system();
    ring->epoch_ended = my_epoch;
}

}  // namespace

pk_status pk_dloop_instance(DlRing* d_ring, cudaStream_t st, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    cudaGraphNode_t node = nullptr;
    cudaKernelNodeParams p = {};
    void* args[] = {(void*)&d_ring};
    p.func = (void*)k_dispatch;
    p.gridDim = dim3(1);
    p.blockDim = dim3(32);
    p.kernelParams = args;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e == cudaSuccess) e = cudaGraphAddKernelNode(&node, g, nullptr, 0, &p);
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    if (e == cudaSuccess) e = cudaGraphUpload(*out, st);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return pk_fail(PK_ERR_CUDA, std::string("dispatcher graph: ") + cudaGetErrorString(e));
    }
    return PK_OK;
}
