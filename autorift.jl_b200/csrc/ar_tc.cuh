// sm_100a tensor-core primitives: shared-memory and instruction descriptors for tcgen05.mma,
// Tensor Memory allocation and loads, mbarriers with bounded waits, and the proxy fences
// between them. Inline PTX, one CTA (cta_group::1), no clusters and no multicast.
//
// Operand layout (SWIZZLE_NONE, K-major): the tensor core reads an operand as "core matrices"
// of 8 rows x 16 bytes, each 128 contiguous bytes with rows 16 bytes apart. The descriptor's
// stride byte offset (SBO) is the distance between 8-row groups and its leading byte offset
// (LBO) the distance between the 16-byte K chunks. With SBO = 128 every row sits 16 bytes after
// the previous one, so a descriptor may start at any row of a 16-byte-row array: a matrix whose
// rows are successive 16-byte slices of one array (row m+1 starts 16 bytes after row m) needs
// no copy per row.

#pragma once

#include <cstdint>

namespace ar {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05 "matrix descriptor"): start address, LBO and SBO in
// 16-byte units, descriptor version 1, SWIZZLE_NONE.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes,
                                              uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1u) << 46;  // version
    return d;                              // base offset 0, legacy LBO mode, layout 0 (none)
}

// Instruction descriptor for kind::i8: unsigned 8-bit A and B, signed 32-bit accumulator,
// both operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_u8_s32(int M, int N) {
    return (2u << 4)                                       // D format S32
           | (0u << 7) | (0u << 10)                        // A, B unsigned 8-bit
           | (static_cast<uint32_t>(N >> 3) << 17)         // N / 8
           | (static_cast<uint32_t>(M >> 4) << 24);        // M / 16
}

// Instruction descriptor for kind::f16 with BF16 A and B and an FP32 accumulator, both operands
// K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4)                                       // D format F32
           | (1u << 7) | (1u << 10)                        // A, B BF16
           | (static_cast<uint32_t>(N >> 3) << 17)         // N / 8
           | (static_cast<uint32_t>(M >> 4) << 24);        // M / 16
}

// D (+)= A * B^T for BF16 operands (kind::f16, K = 16 elements), descriptors as 32-bit halves;
// `accumulate` 0 overwrites D.
__device__ __forceinline__ void mma_bf16_halves(uint32_t d_tmem, uint32_t a_lo, uint32_t a_hi,
                                                uint32_t b_lo, uint32_t b_hi, uint32_t idesc,
                                                uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .b64 da, db;\n\t"
        ".reg .pred p;\n\t"
        "mov.b64 da, {%1, %2};\n\t"
        "mov.b64 db, {%3, %4};\n\t"
        "setp.ne.b32 p, %6, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], da, db, %5, {%7, %7, %7, %7}, p;\n\t"
        "}\n"
        :
        : "r"(d_tmem), "r"(a_lo), "r"(a_hi), "r"(b_lo), "r"(b_hi), "r"(idesc), "r"(accumulate),
          "r"(0u)
        : "memory");
}

// D (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void mma_u8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                       uint32_t idesc, bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u;
    const uint32_t zero = 0u;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
        "}\n"
        :
        : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc), "r"(zero)
        : "memory");
}

// D (+)= A * B^T with the descriptors given as 32-bit halves (lo, hi): a caller that advances
// only the start-address field keeps the halves in registers and adds to `lo` alone.
__device__ __forceinline__ void mma_u8_halves(uint32_t d_tmem, uint32_t a_lo, uint32_t a_hi,
                                              uint32_t b_lo, uint32_t b_hi, uint32_t idesc) {
    asm volatile(
        "{\n\t"
        ".reg .b64 da, db;\n\t"
        ".reg .pred p;\n\t"
        "mov.b64 da, {%1, %2};\n\t"
        "mov.b64 db, {%3, %4};\n\t"
        "setp.ne.b32 p, 1, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], da, db, %5, {%6, %6, %6, %6}, p;\n\t"
        "}\n"
        :
        : "r"(d_tmem), "r"(a_lo), "r"(a_hi), "r"(b_lo), "r"(b_hi), "r"(idesc), "r"(0u)
        : "memory");
}

// Arrive on `mbar` once every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
        :
        : "r"(smem_u32(mbar))
        : "memory");
}

// Tensor Memory allocation by one full warp; the column base address is written to `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(taddr), "r"(ncols)
                 : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets lane (base lane + t),
// columns [col, col + 16).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
// 16 lanes x 32 columns (four 16x256b patterns): thread t gets lanes L = t / 4 and L + 8 of
// the warp's lane base, columns 8 k + 2 (t % 4) and 8 k + 2 (t % 4) + 1 for k = 0..3, in
// registers r[4 k + 0] (L, even column), r[4 k + 1] (L, odd), r[4 k + 2] (L + 8, even),
// r[4 k + 3] (L + 8, odd). This is the M = 64 accumulator's half of a lane quarter.
__device__ __forceinline__ void tmem_ld16dp(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x4.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns from registers (the layout of tmem_ld16).
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
        :
        : "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]),
          "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]),
          "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(mbar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 16 bytes global -> shared without registers (cp.async, L2 only); both addresses 16-byte
// aligned. Completion: cp_async_commit() then cp_async_wait_all() by the issuing thread.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Bounded wait for phase `parity` of `mbar` to complete: false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
    for (uint32_t k = 0; k < limit; ++k)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

}  // namespace tc
}  // namespace ar
