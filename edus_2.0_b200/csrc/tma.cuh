// Tensor-memory-accelerator copies and mbarrier hand-overs used by the
// persistent commutator (comm_ws.cuh) and the persistent plane kernel.
//
// A wait on an mbarrier gives up after a bounded number of polls and reports
// false; the caller then records an error for the host (EDUS_ERR_TIMEOUT)
// instead of spinning without end.
#pragma once
#include <cuda.h>

namespace edus {

// Operand tensor maps of one launch (H, rho, G, y, acc), each describing a
// [B][P][Nk] complex array as the 4-D tensor {2 Nk, nb, nb, B} of doubles.
struct OperandMaps {
    CUtensorMap m[5];
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// true once the phase of parity `parity` has completed; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// every lane polls; the warp agrees on the outcome
__device__ __forceinline__ bool warp_wait(unsigned long long* bar, unsigned parity, int limit) {
    const bool ok = mbar_wait(bar, parity, limit);
    return __all_sync(0xffffffffu, ok);
}
// box at coordinates {x, 0, 0, b} of `map` into shared memory at dst (a
// 128-byte multiple), completion counted in bytes on `bar`
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int b, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(0), "r"(0), "r"(b), "r"(smem_u32(bar))
        : "memory");
}

// Untiled bulk copy global -> shared (no multicast): addresses 16-byte aligned,
// size a multiple of 16 bytes, completion counted in bytes on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Untiled bulk copy shared -> global in the issuing thread's bulk group; the
// thread commits the group and waits for its reads of shared memory (before
// the buffer is reused) or for its completion (before the CTA ends).
__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(
                     reinterpret_cast<unsigned long long>(dst)),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

}  // namespace edus
