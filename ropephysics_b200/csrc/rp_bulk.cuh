// rp_bulk.cuh -- untiled bulk copies (the TMA unit's 1-D form) between this
// GPU's global memory and a CTA's shared memory, completed on an mbarrier.
//
// A rod's state rows are contiguous in both places (16-byte float4 rows,
// rod-major in global memory, one section per array in shared memory), so
// staging a rod is one bulk copy per array issued by one thread, instead of
// every thread of the team moving rows through registers. Rules the callers
// keep: both addresses 16-byte aligned, sizes multiples of 16 bytes, sources
// in this GPU's own memory (no multicast form is used anywhere).
#pragma once

#include <cstdint>

namespace rp {

__device__ __forceinline__ uint32_t sharedAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One arrival expected (the issuing thread's), plus the copies' bytes.
__device__ __forceinline__ void mbarInit(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sharedAddr(bar)) : "memory");
    // make the initialised barrier visible to the async proxy the copies use
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbarInvalidate(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(sharedAddr(bar)) : "memory");
}

__device__ __forceinline__ void mbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sharedAddr(bar)), "r"(bytes)
                 : "memory");
}

// Order this thread's earlier generic-proxy accesses of shared memory before
// its later async-proxy ones (bulk copies reading or writing that memory).
__device__ __forceinline__ void fenceProxyAsyncShared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// global -> shared, counted on `bar` when the bytes have landed
__device__ __forceinline__ void bulkLoad(void* dstShared, const void* srcGlobal, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sharedAddr(dstShared)),
                 "l"(srcGlobal), "r"(bytes), "r"(sharedAddr(bar))
                 : "memory");
}

// shared -> global in the issuing thread's current bulk group
__device__ __forceinline__ void bulkStore(void* dstGlobal, const void* srcShared, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dstGlobal),
                 "r"(sharedAddr(srcShared)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulkCommit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// this thread's committed stores have finished reading shared memory
__device__ __forceinline__ void bulkWaitRead() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// this thread's committed stores are complete
__device__ __forceinline__ void bulkWaitAll() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(sharedAddr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for phase `parity` of `bar` to complete, at most `tries` polls (each
// poll may itself suspend the thread for a while). False when it gave up.
__device__ __forceinline__ bool mbarWaitBounded(uint64_t* bar, uint32_t parity, int tries) {
    for (int i = 0; i < tries; ++i)
        if (mbarTryWait(bar, parity)) return true;
    return false;
}

}  // namespace rp
