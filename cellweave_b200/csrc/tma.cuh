// Tensor-memory-accelerator (TMA) copies into shared memory and the
// mbarriers they complete on, shared by the kernels that stage tiles:
// the FP32 sweeps (field32.cu) and the FP64 residual (field.cu).
//
// Every wait is bounded: a copy that has not landed within TMA_WAIT_NS is
// reported to the caller, which records an error and returns instead of
// spinning on.  Loads only, never multicast.  A tiled copy's innermost
// coordinate times the element size must be a multiple of 16 bytes; the
// callers keep x to that rule (x may be negative: the box reads zeros there).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

namespace cw {

constexpr unsigned long long TMA_WAIT_NS = 2000000000ull;  // a copy not landed in 2 s is an error

__device__ __forceinline__ uint32_t sh_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t tma_clock_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Make the barriers' initialisation visible to the async proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// This thread's arrival, announcing `bytes` to come by transaction.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// The phase `parity` of a barrier, waited for `limit_ns` (TMA_WAIT_NS) at most.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity,
                                                  unsigned long long limit_ns = TMA_WAIT_NS) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = tma_clock_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (tma_clock_ns() - t0 > limit_ns) return false;
    }
}

// Generic-proxy accesses of shared memory before the async proxy's next writes.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One box of a 2-D tensor map into shared memory at `dst`, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :
        : "r"(sh_addr(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// The driver's cuTensorMapEncodeTiled, found once; null if the driver has none.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

}  // namespace cw
