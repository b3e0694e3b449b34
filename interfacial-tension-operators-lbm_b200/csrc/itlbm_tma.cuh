// itlbm_tma.cuh -- shared-memory barriers and tensor copies (TMA) of the step kernels, sm_100a.
//
// Every wait is bounded: mbar_wait gives up after one second of %globaltimer and the caller reports
// ITLBM_E_TIMEOUT, so no kernel can spin forever on a copy that does not land.
#pragma once

#include <cuda.h>

namespace itlbm {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bounded wait for the phase of parity `par` to complete: false after 1 s.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned par) {
    const unsigned a = smem_u32(bar);
    const unsigned long long t0 = gtimer();
    for (unsigned it = 0;; ++it) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(par)
            : "memory");
        if (done) return true;
        if ((it & 63) == 63 && gtimer() - t0 > 1000000000ull) return false;
    }
}

// One tiled copy of a 4-D box at coordinates (x, y, z, w) of `map` into shared memory at `dst`
// (128-byte aligned), completing on `bar`.  x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_4d(const CUtensorMap *map, void *dst, int x, int y, int z, int w,
                                            unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

// The tensor map lives in global memory written by the host: order the tensor-map proxy after it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

}  // namespace itlbm
