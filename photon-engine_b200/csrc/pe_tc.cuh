// pe_tc.cuh — the 5th-generation tensor-core instructions the guiding MLP uses (sm_100a):
// TMEM allocation, tcgen05.mma (kind::f16, one CTA, D in TMEM), commit to an mbarrier, TMEM
// loads, and the shared-memory operand layout the descriptors describe.
//
// Operand layout (K-major, no swizzle): a tile of R rows × K halves is stored as 8×8 "core
// matrices" of 128 contiguous bytes (8 rows × 16 bytes); core matrix (row block rb, k block kb)
// sits at byte ((kb · R/8) + rb) · 128.  In the descriptor the leading byte offset (LBO) is the
// distance between k-adjacent core matrices (R/8 · 128 B) and the stride byte offset (SBO) the
// distance between row-adjacent ones (128 B).  One MMA consumes K = 16 (two k blocks).
#pragma once

#include <cstdint>

namespace pe {

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) in an R-row core-matrix tile.
__host__ __device__ __forceinline__ uint32_t coreOffset(int r, int k, int rows) {
    return static_cast<uint32_t>(((k >> 3) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, LBO and SBO in 16-byte units; version 1
// (Blackwell) at bits 46-47; layout type 0 (no swizzle) at bits 61-63; base offset 0.
__host__ __device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lboBytes, uint32_t sboBytes) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lboBytes >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sboBytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with F16 A and B (both K-major), F32 D, M × N.
__host__ __device__ constexpr uint32_t instrDescF16(int M, int N) {
    return (1u << 4)                                   // D format F32
           | (static_cast<uint32_t>(N >> 3) << 17)     // N / 8
           | (static_cast<uint32_t>(M >> 4) << 24);    // M / 16
}

__device__ __forceinline__ void tmemAlloc(uint32_t* dstSmem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(dstSmem)), "r"(cols));
}
__device__ __forceinline__ void tmemRelinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmemDealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols));
}
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes → visible to the tensor core's async proxy
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] · B[smem]ᵀ, issued by one thread.
__device__ __forceinline__ void tcMma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u;
    const uint32_t z = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Arrives on the mbarrier once every MMA this thread issued before has completed.
__device__ __forceinline__ void tcCommit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbarInit(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(mbar)), "r"(count));
}

__device__ __forceinline__ bool mbarTryWait(uint64_t* mbar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}"
        : "=r"(done)
        : "r"(smemAddr(mbar)), "r"(phase)
        : "memory");
    return done != 0;
}

// Waits for phase `phase` of the mbarrier, at most `limit` polls; false = gave up.
__device__ __forceinline__ bool mbarWait(uint64_t* mbar, uint32_t phase, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbarTryWait(mbar, phase)) return true;
    return false;
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (warp w reads lanes 32w..32w+31).
// The load and its wait share one asm statement, so the registers are defined only after the
// wait and no use can be scheduled before it.
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

} // namespace pe
