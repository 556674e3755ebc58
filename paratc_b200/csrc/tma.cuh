// tma.cuh -- the tensor-memory-accelerator (TMA) and mbarrier operations the
// TMA-fed kernels use, as inline PTX: tiled 2-D / 3-D loads into shared
// memory completing on an mbarrier, tiled stores from shared memory in bulk
// groups, untiled bulk copies of contiguous runs, and bounded waits.  Only this GPU's memory; no cluster multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

namespace ptc {
namespace tma {

// polls of a bounded wait before it gives up
constexpr long long kSpinLimit = 1LL << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* m, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(m)), "r"(bytes) : "memory");
}
// one arrival (release at CTA scope: the arriving thread's shared-memory
// writes are visible to a thread whose wait sees the phase complete)
__device__ __forceinline__ void mbar_arrive(unsigned long long* m) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(m)) : "memory");
}
// polls the pipeline waits of a TMA-fed kernel make before they give up.
// err points at the context's error word; err[1] holds a test setting
// (paratc_set_wait_limit): 0 keeps kSpinLimit, v > 0 allows v - 1 polls, so
// that a test can make a wait run out.  The waits that drain a CTA's own
// copies in flight after a failure always keep kSpinLimit.
__device__ __forceinline__ long long wait_limit(const unsigned int* err) {
    const unsigned v = *(volatile const unsigned int*)(err + 1);
    return v == 0u ? kSpinLimit : (long long)(v - 1u);
}

// true once phase `parity` of the barrier has completed; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* m, unsigned parity, long long limit = kSpinLimit) {
    const unsigned a = smem_addr(m);
    for (long long it = 0; it < limit; it++) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void load_2d(void* dst, const CUtensorMap* tm, int x, int y, unsigned long long* m) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(tm)), "r"(x), "r"(y), "r"(smem_addr(m))
        : "memory");
}
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z, unsigned long long* m) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(m))
        : "memory");
}
__device__ __forceinline__ void store_2d(const CUtensorMap* tm, int x, int y, const void* src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                     reinterpret_cast<unsigned long long>(tm)),
                 "r"(x), "r"(y), "r"(smem_addr(src))
                 : "memory");
}
__device__ __forceinline__ void store_3d(const CUtensorMap* tm, int x, int y, int z, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
                     reinterpret_cast<unsigned long long>(tm)),
                 "r"(x), "r"(y), "r"(z), "r"(smem_addr(src))
                 : "memory");
}
// untiled bulk copies: both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(smem_addr(m))
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(
                     reinterpret_cast<unsigned long long>(dst)),
                 "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

}  // namespace tma

// cuTensorMapEncodeTiled through the runtime's driver entry point (null if
// the driver has none)
PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn();

}  // namespace ptc
