// vfd_tma.h -- tensor-memory-accelerator (TMA) staging for the axis passes:
// host-side tensor-map encoding and the device-side mbarrier / bulk-tensor
// copy primitives (sm_90+ PTX, used here on sm_100a).
//
// A field is described to the TMA unit as a 3D fp32 tensor {nx, ny, nz}
// (x fastest, strides nx*4 and nx*ny*4 bytes).  A pass copies boxes of it
// into shared memory; positions outside the field (the zero padding of the
// overlap-save windows) are filled with zeros by the hardware.  Every load
// starts at an x coordinate that is a multiple of 4 floats (16 bytes), and
// tensor maps only ever cover this GPU's own field buffers; no copy uses
// cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vfd {

// Whether the driver offers cuTensorMapEncodeTiled (looked up once).
bool tma_available();

// Encodes a tiled map of the fp32 tensor at `base` with dims {d0, d1, d2}
// (d0 contiguous), byte strides s1 (dim 1) and s2 (dim 2), box {b0, b1, b2},
// zero fill out of bounds.  Returns false when the driver rejects it or the
// layout breaks a TMA rule (16-byte aligned base and strides, b0 * 4 a
// multiple of 16, every box dim <= 256).
bool tma_encode_3d(CUtensorMap *m, const float *base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1,
                   uint64_t s2, uint32_t b0, uint32_t b1, uint32_t b2);

#ifdef __CUDACC__
// Cycles after which a wait for a bulk copy gives up (about 1 s at 2 GHz).
constexpr long long kTmaWaitCycles = 2000000000ll;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the barrier initialisation visible to the async proxy (TMA).
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier, at most `limit` cycles; false
// when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit = kTmaWaitCycles)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// Orders this thread's earlier generic-proxy shared-memory accesses (and
// those ordered before them by a warp or CTA barrier) before later
// async-proxy (TMA) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// 3D tiled bulk copy global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}
#endif

}  // namespace vfd
