// Tensor-core (tcgen05, kind::i8) pieces of the correlation: a self-test of the operand layouts
// the correlation kernel relies on.

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "ar_internal.cuh"
#include "ar_tc.cuh"

namespace ar {
namespace {

struct ProbeArgs {
    const uint8_t* a_img;
    const uint8_t* b_img;
    int a_bytes, b_bytes;      // images copied to shared memory, A at 0, B at b_base
    int b_base;
    int a_off, a_lbo, a_sbo, a_kstep;
    int b_off, b_lbo, b_sbo, b_kstep;
    int M, N, nk, ncols, dstep, dcols, mode;
    int32_t* d_out;            // 128 lanes x dcols columns
    int* status;               // 0 ok, 1 the MMA did not complete in time
};

__global__ void __launch_bounds__(128, 1) k_tc_probe(const ProbeArgs P) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int e = tid; e < P.a_bytes; e += blockDim.x) smem[e] = P.a_img[e];
    for (int e = tid; e < P.b_bytes; e += blockDim.x) smem[P.b_base + e] = P.b_img[e];
    if (warp == 0) {
        tc::tmem_alloc(&tbase, static_cast<uint32_t>(P.ncols));
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_mbar_init();
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = tbase;
    if (P.dstep > 0) {
        // Steps write overlapping column windows: clear the accumulator and always add.
        uint32_t z[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) z[k] = 0u;
        for (int c = 0; c < P.dcols; c += 16)
            tc::tmem_st16(taddr + (static_cast<uint32_t>(32 * warp) << 16) + c, z);
        tc::tmem_wait_st();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // Mode 2 issues no product: nothing arrives on the barrier, so the bounded wait below runs
    // out (a few thousand polls), the kernel reports it in `status` and returns normally.
    if (tid == 0 && P.mode != 2) {
        const uint32_t sa = tc::smem_u32(smem), sb = tc::smem_u32(smem + P.b_base);
        const uint32_t idesc = tc::idesc_u8_s32(P.M, P.N);
        for (int s = 0; s < P.nk; ++s) {
            const uint64_t da = tc::smem_desc(sa + P.a_off + s * P.a_kstep, P.a_lbo, P.a_sbo);
            const uint64_t db = tc::smem_desc(sb + P.b_off + s * P.b_kstep, P.b_lbo, P.b_sbo);
            tc::mma_u8(taddr + static_cast<uint32_t>(s * P.dstep), da, db, idesc,
                       P.dstep > 0 || s > 0);
        }
        tc::mma_commit(&mbar);
    }
    const bool ok = tc::mbar_wait(&mbar, 0, P.mode == 2 ? (1u << 12) : (1u << 24));
    if (!ok && tid == 0) *P.status = 1;
    tc::fence_after_sync();
    if (ok && P.mode == 0) {
        for (int c = 0; c < P.dcols; c += 16) {
            uint32_t r[16];
            tc::tmem_ld16(taddr + (static_cast<uint32_t>(32 * warp) << 16) + c, r);
            tc::tmem_wait_ld();
#pragma unroll
            for (int k = 0; k < 16; ++k)
                P.d_out[(32 * warp + lane) * P.dcols + c + k] = static_cast<int32_t>(r[k]);
        }
    } else if (ok) {
        // The 16x256b pattern: each warp reads the first 16 lanes of its quarter, columns
        // [0, 32); thread t's register k goes to d_out[(32 warp + t) * dcols + k].
        uint32_t r[16];
        tc::tmem_ld16dp(taddr + (static_cast<uint32_t>(32 * warp) << 16), r);
        tc::tmem_wait_ld();
#pragma unroll
        for (int k = 0; k < 16; ++k)
            P.d_out[(32 * warp + lane) * P.dcols + k] = static_cast<int32_t>(r[k]);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, static_cast<uint32_t>(P.ncols));
}

// Highest byte offset a K-major SWIZZLE_NONE operand of `rows` rows reads, plus one, over
// `nk` K-steps.
int64_t operand_extent(int off, int lbo, int sbo, int kstep, int rows, int nk) {
    const int64_t last = static_cast<int64_t>(off) + static_cast<int64_t>(nk - 1) * kstep;
    const int64_t row = static_cast<int64_t>((rows - 1) / 8) * sbo + ((rows - 1) % 8) * 16;
    return last + row + lbo + 16;
}

}  // namespace

cudaError_t tc_probe(const uint8_t* a_img, int a_bytes, const uint8_t* b_img, int b_bytes,
                     const int* params, int32_t* d_out, int* status, cudaStream_t s,
                     std::string* err) {
    ProbeArgs P{};
    P.a_img = a_img;
    P.b_img = b_img;
    P.a_bytes = a_bytes;
    P.b_bytes = b_bytes;
    P.a_off = params[0];
    P.a_lbo = params[1];
    P.a_sbo = params[2];
    P.a_kstep = params[3];
    P.b_off = params[4];
    P.b_lbo = params[5];
    P.b_sbo = params[6];
    P.b_kstep = params[7];
    P.M = params[8];
    P.N = params[9];
    P.nk = params[10];
    P.dstep = params[11];
    P.mode = params[12];
    auto bad = [&](const char* m) {
        if (err) *err = m;
        return cudaErrorInvalidValue;
    };
    if (P.M != 64 && P.M != 128) return bad("M must be 64 or 128");
    if (!(P.N == 8 || (P.N % 16 == 0 && P.N >= 16 && P.N <= 256))) return bad("invalid N");
    if (P.nk < 1 || P.nk > 64) return bad("nk must be in 1..64");
    if (a_bytes <= 0 || b_bytes <= 0 || a_bytes > 96 * 1024 || b_bytes > 96 * 1024)
        return bad("operand images must be 1..96 KiB");
    for (int v : {P.a_off, P.a_lbo, P.a_sbo, P.b_off, P.b_lbo, P.b_sbo, P.a_kstep, P.b_kstep})
        if (v < 0 || (v & 15)) return bad("offsets and strides must be non-negative multiples of 16");
    if (operand_extent(P.a_off, P.a_lbo, P.a_sbo, P.a_kstep, P.M, P.nk) > a_bytes)
        return bad("A descriptor reads past its image");
    if (operand_extent(P.b_off, P.b_lbo, P.b_sbo, P.b_kstep, P.N, P.nk) > b_bytes)
        return bad("B descriptor reads past its image");
    if (P.dstep < 0 || (P.dstep & 15)) return bad("dstep must be a non-negative multiple of 16");
    P.dcols = P.N + (P.nk - 1) * P.dstep;
    if (P.dcols > 512) return bad("the accumulator columns exceed Tensor Memory");
    if (P.mode < 0 || P.mode > 2) return bad("mode must be 0, 1 or 2");
    if (P.mode == 1 && P.dcols < 32) return bad("mode 1 reads 32 columns");
    P.b_base = (a_bytes + 1023) & ~1023;
    int ncols = 32;
    while (ncols < P.dcols) ncols <<= 1;
    P.ncols = ncols;
    P.d_out = d_out;
    P.status = status;
    const int smem = P.b_base + b_bytes;
    if (smem > kDynSmemCap) return bad("operand images exceed shared memory");
    cudaError_t e =
        cudaFuncSetAttribute(k_tc_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, kDynSmemCap);
    if (e != cudaSuccess) return e;
    k_tc_probe<<<1, 128, smem, s>>>(P);
    return cudaGetLastError();
}

}  // namespace ar
