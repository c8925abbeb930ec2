// tc_sm100.cuh -- the 5th-generation tensor-core primitives (tcgen05) the
// block solves use, as inline PTX for sm_100a: tensor-memory allocation,
// shared-memory matrix descriptors, kind::tf32 MMA with the accumulator in
// tensor memory, completion through an mbarrier, and tensor-memory loads
// and stores.
//
// Operand layout (both operands K-major, no swizzle): an R x 8 TF32 slab
// (R a multiple of 8) is stored as R/8 groups of two 8-row x 16-byte core
// matrices, 256 bytes per group:
//   byte(r, k) = (r/8)*256 + (k/4)*128 + (r%8)*16 + (k%4)*4,   k in [0, 8)
// i.e. leading-dimension byte offset 128 (between the two K halves of a core
// matrix pair) and stride byte offset 256 (between 8-row groups).  One MMA
// consumes one slab of A (M rows) and one of B (N rows): D[M x N] += A B^T.
//
// The accumulator of an M = 128, cta_group::1 MMA maps row i to tensor-memory
// lane i; warp w of the CTA reads and writes lanes 32*(w%4) .. 32*(w%4)+31.
//
// Every wait is bounded: a wait that runs out returns false and the caller
// records an error instead of hanging.
#pragma once

#include <cstdint>

namespace wind {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (r, k) inside one R x 8 TF32 slab
__device__ __forceinline__ int slab_off(int r, int k) {
    return ((r >> 3) << 8) + ((k >> 2) << 7) + ((r & 7) << 4) + ((k & 3) << 2);
}

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 256 B.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::tf32 with an FP32 accumulator, both
// operands K-major, no negation.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4)                       // D format F32
         | (2u << 7)                       // A format TF32
         | (2u << 10)                      // B format TF32
         | ((uint32_t)(N >> 3) << 17)      // N / 8
         | ((uint32_t)(M >> 4) << 24);     // M / 16
}

// Round to TF32 (round to nearest, ties away), as the tensor core reads it.
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// ---- tensor memory ----------------------------------------------------------
// Allocate `ncols` columns (a power of two >= 32) for the CTA; one full warp
// calls it and the base address lands in *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes visible to the tensor core's reads.
__device__ __forceinline__ void fence_smem_to_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive 32-bit columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        :: "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])),
           "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])),
           "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
           "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
           "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
           "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// ---- MMA and completion -----------------------------------------------------
// D[tmem] (+)= A B^T, one slab each; issued by ONE thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
// Arrive once on the mbarrier when every MMA this thread issued has completed.
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Wait for the phase with parity `parity` to complete; false after
// `max_polls` unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_polls) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < max_polls; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace tc
}  // namespace wind
