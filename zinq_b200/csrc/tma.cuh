// tma.cuh -- Tensor Memory Accelerator (TMA) staging for the N-D axis passes (sm_100a).
//
// Device side: mbarrier set-up and bounded waits, tiled tensor copies global -> shared
// (completing on an mbarrier) and shared -> global (bulk groups).  Every copy here reads or
// writes this GPU's own memory and none uses cluster multicast.
// Host side: a tensor map over the wavefunction buffer, encoded through the driver entry point
// that the runtime hands out (no link against libcuda).
#pragma once

#include <cuda.h> // CUtensorMap and its enums (types only)
#include <cuda_runtime.h>
#include <stdint.h>

namespace zqd {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes initialised mbarriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// orders this thread's generic-proxy writes to shared memory before later TMA reads of it
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for phase `parity` of bar to complete, for at most `budget` SM cycles.  Returns false
// when the budget ran out (the caller records the error and stops using the stage).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long budget) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > budget) return false;
    return true;
}

// tiled 3-D load of the tensor map's box at (x, y, z) into shared memory dst; the bytes
// complete on bar (transaction count)
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
// tiled 3-D store of shared memory src to the box at (x, y, z), in the current bulk group
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the bulk groups committed by this thread have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and their writes to global memory are done
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ------------------------------------------------------------ host side
// A 3-D tensor map of 8-byte words over `base`: dims[0] words fastest, then dims[1] rows at
// stride1 bytes, dims[2] planes at stride2 bytes; box[3] words x rows x planes.  l2promo is
// the L2 fill granularity in bytes (0, 64, 128 or 256); swizzle128: the 128-byte shared-memory
// swizzle (box rows of exactly 128 bytes).  Returns a CUDA error code (as int): 0 on success.
int encode_map_3d(CUtensorMap* map, void* base, const uint64_t dims[3], uint64_t stride1, uint64_t stride2,
                  const uint32_t box[3], int l2promo, bool swizzle128 = false);

} // namespace zqd
