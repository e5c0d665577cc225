// tcgen05 / TMEM / mbarrier primitives for sm_100a, as inline PTX.
//
// Used by the surrogate network's convolution kernels (surrogate.cu): the
// fifth-generation tensor core instruction tcgen05.mma reads both operands
// from shared memory through 64-bit matrix descriptors and accumulates into
// tensor memory (TMEM), which the epilogue reads back with tcgen05.ld.
//
// Operand tiles use the no-swizzle ("interleaved") canonical layout: a core
// matrix is 8 rows of 16 bytes stored contiguously (128 bytes).
//   K-major operand  (rows = M or N, 16-byte row = 8 consecutive K values):
//     SBO = byte stride between 8-row groups along M/N,
//     LBO = byte stride between the two 16-byte K chunks of one K=16 step.
//   MN-major operand (16-byte row = 8 consecutive M/N values at one k):
//     SBO = byte stride between groups of 8 along M/N,
//     LBO = byte stride between groups of 8 along K.
// Every wait on an mbarrier is bounded: after kSpinLimit polls the caller
// records an error flag and goes on, so a wrong program cannot hang the GPU.
#pragma once
#include <stdint.h>

namespace tc05 {

constexpr unsigned kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, no swizzle, sm_100 version field = 1.
__device__ __forceinline__ uint64_t desc_noswizzle(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
    // base offset 0, LBO mode 0, layout type 0 = SWIZZLE_NONE (bits 61-63)
    return d;
}

// Instruction descriptor of kind::f16 with bf16 A and B, fp32 accumulator.
// a_mn / b_mn: 1 when the operand is MN-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, int a_mn, int b_mn) {
    return (1u << 4)                     // D format: f32
           | (1u << 7)                   // A format: bf16
           | (1u << 10)                  // B format: bf16
           | ((uint32_t)a_mn << 15)      // A major
           | ((uint32_t)b_mn << 16)      // B major
           | ((uint32_t)(N >> 3) << 17)  // N / 8
           | ((uint32_t)(M >> 4) << 24); // M / 16
}

// ---- TMEM allocation (one full warp) -------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- ordering ----------------------------------------------------------
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes this thread's completed shared-memory writes (st.shared, cp.async)
// visible to the async proxy that tcgen05.mma reads through.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- MMA -----------------------------------------------------------------
// D[tmem] (+)= A[M x K=16] * B[K=16 x N], issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
// The mbarrier receives one arrival when every MMA this thread issued before
// has completed (their shared-memory reads and TMEM writes are done).
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

// ---- TMEM -> registers: 32 lanes x 16 columns of 32 bits per warp ---------
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- mbarrier --------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of the given parity to complete; false when the
// limit ran out (the caller flags an error and carries on).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
    for (unsigned i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

// ---- cp.async 16-byte copies -------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
// Zero-filling variant: copies src_bytes (0 or 16) and fills the rest with zeros.
__device__ __forceinline__ void cp_async16_zfill(void *smem_dst, const void *gsrc, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem_dst)), "l"(gsrc),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace tc05
