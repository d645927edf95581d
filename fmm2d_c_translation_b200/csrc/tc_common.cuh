// tc_common.cuh -- inline PTX helpers for the 5th-generation tensor cores
// (tcgen05) shared by the M2L kernels: shared-memory matrix descriptors,
// the kind::tf32 MMA, commits to mbarriers, bounded barrier waits and
// tensor-memory loads.
//
// Operands use the no-swizzle K-major layout: 8-row x 16-byte core
// matrices, contiguous 128 bytes each; core matrix (row group g, K chunk c)
// at ((c * G + g) * 128) bytes for G = rows / 8.  So SBO (between row
// groups) = 128 bytes and LBO (between K chunks) = G * 128 bytes, and row r
// of a K chunk sits at r * 16 bytes: a descriptor that starts s rows
// further down reads the operand shifted by s rows.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fmm2d {

__device__ __forceinline__ uint32_t smem_u32(const void *ptr) {
    return (uint32_t)__cvta_generic_to_shared(ptr);
}

// Shared-memory matrix descriptor: start, LBO, SBO (bytes, 16-byte units),
// descriptor version 1 (bits 46-47), no swizzle.
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::tf32 with FP32 accumulation, both
// operands K-major: M rows (64 or 128), N columns.
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

// x rounded to TF32 (round to nearest, ties away), kept in an FP32 register.
__device__ __forceinline__ float tc_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

// The barrier's next phase completes once every tcgen05 operation issued
// so far by this thread has completed.
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Arrival that also expects `bytes` of asynchronous copies to complete on
// the barrier's current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(mbar),
        "r"(bytes)
        : "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global to this CTA's shared memory, completing on the barrier.  No
// multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar)
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the completion of the barrier phase with the given
// parity: gives up after `limit_ns` nanoseconds, or early once *abort is
// set by another thread of the block.  Returns false on giving up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity,
                                                  volatile int *abort, uint64_t limit_ns) {
    if (mbar_test(mbar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; it++) {
        if (mbar_test(mbar, parity)) return true;
        if ((it & 31u) == 0) {
            if (*abort) return false;
            if (global_ns() - t0 > limit_ns) return false;
        }
    }
}

// As mbar_wait_bounded, for waits off the critical path: after the first
// polls the thread sleeps between tests, leaving issue slots to the
// block's other warps.
__device__ __forceinline__ bool mbar_wait_backoff(uint32_t mbar, uint32_t parity,
                                                  volatile int *abort, uint64_t limit_ns) {
    if (mbar_test(mbar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1;; it++) {
        if (mbar_test(mbar, parity)) return true;
        if (it > 64) __nanosleep(256);
        if ((it & 15u) == 0) {
            if (*abort) return false;
            if (global_ns() - t0 > limit_ns) return false;
        }
    }
}

__device__ __forceinline__ void tc_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// Element (row, k) of a K-major no-swizzle operand of `rows` rows, as a
// float index.
__host__ __device__ __forceinline__ int tc_fidx(int row, int k, int rows) {
    return (((k >> 2) * (rows >> 3) + (row >> 3)) << 5) + ((row & 7) << 2) + (k & 3);
}

}  // namespace fmm2d
