// Pre-correlation filters and UInt8 quantisation on the device: the `_prepare` step of
// AutoRIFT.jl (src/api.jl:305-311) -- preprocess (src/preprocess.jl:149-160, 275-460) then
// quantize (src/preprocess.jl:488-592) -- applied to one image at a time.
//
// Stencils. The mask-aware box mean (src/preprocess.jl:371-399 over src/window.jl:228-439)
// is a shared-memory tile: per-pixel values and "contributes" flags (valid and not NaN) for a
// 32x32 output tile plus its halo, FP64 column sums, then FP64 row sums, divided by the count
// and rounded to Float32. For integer images and for Float32 images of bounded dynamic range
// every partial sum is an exact FP64 value, so the mean equals the reference's banded running
// sum bit for bit. Erosion of the validity mask (src/preprocess.jl:447-460) is the same
// stencil over the mask, and the highpass / Wallis output, the non-finite clean-up and the
// mask update of `_filtered` (src/preprocess.jl:275-288) are fused into the final pass.
//
// Quantisation. The global mean and Bessel-corrected deviation of `_to_uint8` are reduced in
// double-double (TwoSum) with a fixed block order -- deterministic, and within an ulp of the
// exactly rounded sums, which for highpass output of integer imagery equal the reference's
// sequential FP64 sums exactly. Rounding half to even, as Julia's round(UInt8, x).

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "ar_internal.cuh"

namespace ar {
namespace {

constexpr int kTile = 32;
constexpr int kBoxThreads = 256;
constexpr int kMaxWidth = 63;
constexpr int kStatBlocks = 592;
constexpr int kStatThreads = 256;
constexpr unsigned kFullMask = 0xffffffffu;

template <typename T>
__device__ __forceinline__ float as_f32(T v) {
    return static_cast<float>(v);
}

// Which per-pixel quantity a box pass averages.
enum BoxMode { BOX_IMAGE = 0, BOX_DEV2 = 1 };

// Shared-memory layout of one tile with its halo: values, flags, column sums. The window is
// (wx, wy) after the reference's clamp to the image (src/window.jl:632-637), with the extra
// element of an even width on the left (src/window.jl:254-257).
struct BoxSmem {
    float* val;       // Rr x Rc, Rr = kTile + wy - 1, Rc = kTile + wx - 1, column-major
    uint8_t* contr;   // contributes to the mean
    uint8_t* mok;     // mask for erosion (true outside the image)
    double* vs;       // kTile x Rc column sums
    int* vc;          // kTile x Rc counts
    uint8_t* ve;      // kTile x Rc eroded columns
};

// The Wallis deviation of one pixel (src/preprocess.jl:416-430).
__device__ __forceinline__ float dev2_of(float x, bool m, float mean, bool* contributes) {
    if (m && isfinite(mean)) {
        const float d = __fsub_rn(x, mean);
        const float v = __fmul_rn(d, d);
        *contributes = !isnan(v);
        return v;
    }
    *contributes = false;
    return 0.0f;
}

// Tile loop of a box pass: for every output pixel of the tile, the FP64 sum and count of
// contributing neighbours and whether every in-bounds neighbour is valid.
template <typename T, int MODE, typename Out>
__device__ void box_tile(const T* img, const uint8_t* mask, const float* mean, int64_t nr,
                         int64_t nc, int wx, int wy, int64_t r0, int64_t c0, BoxSmem S, Out out) {
    const int ly = wy / 2, lx = wx / 2;
    const int Rr = kTile + wy - 1, Rc = kTile + wx - 1;
    const int tid = threadIdx.x, bd = blockDim.x;
    for (int e = tid; e < Rr * Rc; e += bd) {
        const int r = e % Rr, c = e / Rr;
        const int64_t gr = r0 - ly + r, gc = c0 - lx + c;
        float v = 0.0f;
        uint8_t contrib = 0, mk = 1;
        if (gr >= 0 && gr < nr && gc >= 0 && gc < nc) {
            const int64_t g = gr + gc * nr;
            const bool m = mask[g] != 0;
            mk = m ? 1 : 0;
            const float x = as_f32(img[g]);
            if (MODE == BOX_IMAGE) {
                v = x;
                contrib = (m && !isnan(x)) ? 1 : 0;
            } else {
                bool cb;
                v = dev2_of(x, m, mean[g], &cb);
                contrib = cb ? 1 : 0;
            }
        }
        S.val[e] = contrib ? v : 0.0f;
        S.contr[e] = contrib;
        S.mok[e] = mk;
    }
    __syncthreads();
    // Column sums over wy rows for each output row of the tile.
    for (int e = tid; e < kTile * Rc; e += bd) {
        const int r = e % kTile, c = e / kTile;
        double s = 0.0;
        int cnt = 0;
        uint8_t ok = 1;
        for (int k = 0; k < wy; ++k) {
            const int q = (r + k) + c * Rr;
            s = __dadd_rn(s, static_cast<double>(S.val[q]));
            cnt += S.contr[q];
            ok &= S.mok[q];
        }
        S.vs[e] = s;
        S.vc[e] = cnt;
        S.ve[e] = ok;
    }
    __syncthreads();
    for (int e = tid; e < kTile * kTile; e += bd) {
        const int r = e % kTile, c = e / kTile;
        const int64_t gr = r0 + r, gc = c0 + c;
        if (gr >= nr || gc >= nc) continue;
        double s = 0.0;
        int cnt = 0;
        uint8_t ok = 1;
        for (int k = 0; k < wx; ++k) {
            const int q = r + (c + k) * kTile;
            s = __dadd_rn(s, S.vs[q]);
            cnt += S.vc[q];
            ok &= S.ve[q];
        }
        out(gr + gc * nr, s, cnt, ok != 0);
    }
    __syncthreads();
}

__device__ __forceinline__ float box_mean(double s, int cnt) {
    return cnt > 0 ? __double2float_rn(__ddiv_rn(s, static_cast<double>(cnt))) : __int_as_float(0x7fc00000);
}

__device__ BoxSmem box_smem(unsigned char* base, int wx, int wy) {
    const int Rr = kTile + wy - 1, Rc = kTile + wx - 1;
    BoxSmem S;
    size_t off = 0;
    S.vs = reinterpret_cast<double*>(base + off);
    off += sizeof(double) * kTile * Rc;
    S.val = reinterpret_cast<float*>(base + off);
    off += sizeof(float) * Rr * Rc;
    S.vc = reinterpret_cast<int*>(base + off);
    off += sizeof(int) * kTile * Rc;
    S.contr = base + off;
    off += Rr * Rc;
    S.mok = base + off;
    off += Rr * Rc;
    S.ve = base + off;
    return S;
}

size_t box_smem_bytes(int wx, int wy) {
    const size_t Rr = kTile + wy - 1, Rc = kTile + wx - 1;
    return sizeof(double) * kTile * Rc + sizeof(float) * Rr * Rc + sizeof(int) * kTile * Rc +
           2 * Rr * Rc + kTile * Rc + 64;
}

// Highpass (src/preprocess.jl:304-312) with `_filtered`: out = img - boxmean where valid,
// zero and invalid elsewhere; the mask erodes by the filter width.
template <typename T>
__global__ void __launch_bounds__(kBoxThreads) k_highpass(const T* img, const uint8_t* mask,
                                                          int64_t nr, int64_t nc, int wx, int wy,
                                                          float* out, uint8_t* vout) {
    extern __shared__ __align__(16) unsigned char bsm[];
    const BoxSmem S = box_smem(bsm, wx, wy);
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kTile;
    const int64_t c0 = static_cast<int64_t>(blockIdx.y) * kTile;
    box_tile<T, BOX_IMAGE>(img, mask, nullptr, nr, nc, wx, wy, r0, c0, S,
                           [&](int64_t g, double s, int cnt, bool eroded) {
                               const float mean = box_mean(s, cnt);
                               float o = (mask[g] && isfinite(mean)) ? __fsub_rn(as_f32(img[g]), mean)
                                                                    : __int_as_float(0x7fc00000);
                               bool v = eroded;
                               if (!isfinite(o)) {
                                   o = 0.0f;
                                   v = false;
                               }
                               out[g] = o;
                               vout[g] = v ? 1 : 0;
                           });
}

// Highpass of integer imagery (UInt8, UInt16, Int16): the same stencil as k_highpass with the
// sums carried as exact 32-bit integers (at most 63 x 63 values below 2^16 in magnitude), so
// the mean s / cnt -- an FP64 division of exact integers rounded to Float32 -- is the reference's
// bit for bit. A block stages a tile of TR x kHpCols outputs plus its halo in shared memory
// with 16-byte loads of the column-major image and mask (aligned chunks of each column's linear
// range, element-wise only where a chunk would leave the array), then slides the window down each
// column (value sums, and the contributing and in-image-invalid counts packed in one word:
// erosion is "no in-image neighbour is invalid") and across columns, writing the Float32 output
// and the mask with consecutive threads on consecutive rows.
constexpr int kHpCols = 32;
constexpr int kHpThreads = 256;

// Loads the elements [e0, e1) of `base` (nelem elements) as the aligned 16-byte chunks that
// cover them -- scalars for a chunk that is not entirely inside [base, base + nelem) -- handing
// each element (its index and value) to `put`. Lane `task0` of `stride` lanes takes every
// stride-th chunk.
template <typename T, typename Put>
__device__ __forceinline__ void load_chunks(const T* base, int64_t nelem, int64_t e0, int64_t e1,
                                            int task0, int stride, Put put) {
    constexpr int64_t sz = static_cast<int64_t>(sizeof(T));
    constexpr int per = 16 / static_cast<int>(sizeof(T));
    const int64_t b = static_cast<int64_t>(reinterpret_cast<uintptr_t>(base));
    const int64_t first = (b + e0 * sz) & ~int64_t{15};
    const int64_t end = b + e1 * sz, lim = b + nelem * sz;
    for (int64_t a = first + 16 * task0; a < end; a += 16 * stride) {
        const int64_t ea = (a - b) / sz;  // element at the chunk's first byte (a - b is a multiple of sz)
        if (a >= b && a + 16 <= lim) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(a));
            const T* t = reinterpret_cast<const T*>(&v);
#pragma unroll
            for (int k = 0; k < per; ++k) {
                const int64_t e = ea + k;
                if (e >= e0 && e < e1) put(e, t[k]);
            }
        } else {
            for (int k = 0; k < per; ++k) {
                const int64_t e = ea + k;
                if (e >= e0 && e < e1 && e >= 0 && e < nelem) put(e, base[e]);
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kHpThreads) k_highpass_int(const T* img, const uint8_t* mask,
                                                             int64_t nr, int64_t nc, int wx,
                                                             int wy, int TR, float* out,
                                                             uint8_t* vout) {
    extern __shared__ __align__(16) unsigned char hsm[];
    const int ly = wy / 2, lx = wx / 2;
    const int IR = TR + wy - 1, IC = kHpCols + wx - 1;
    const int IRp = IR | 1;  // odd column stride: a warp's rows of different columns spread banks
    int* sv = reinterpret_cast<int*>(hsm);                      // IC x IRp: value where contributing
    uint32_t* sf = reinterpret_cast<uint32_t*>(sv + IC * IRp);  // 1 contributing | 1 << 16 invalid
    int* vs = reinterpret_cast<int*>(sf + IC * IRp);            // IC x TR: column sums of values
    uint32_t* vf = reinterpret_cast<uint32_t*>(vs + IC * TR);   // IC x TR: column sums of flags
    const int tid = threadIdx.x;
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * TR;
    const int64_t c0 = static_cast<int64_t>(blockIdx.y) * kHpCols;
    const int64_t n = nr * nc;

    // Out-of-image elements: no contribution, not invalid (erosion ignores them).
    for (int e = tid; e < IC * IRp; e += kHpThreads) {
        sv[e] = 0;
        sf[e] = 0u;
    }
    __syncthreads();
    // Column segment cc covers rows [r0 - ly, r0 - ly + IR) of image column c0 - lx + cc; only its
    // in-image rows are loaded. Warps take segments; lanes take 16-byte chunks.
    const int warp = tid >> 5, lane = tid & 31;
    for (int cc = warp; cc < IC; cc += kHpThreads / 32) {
        const int64_t gc = c0 - lx + cc;
        if (gc < 0 || gc >= nc) continue;
        const int64_t rlo = r0 - ly > 0 ? r0 - ly : 0;
        const int64_t rhi = r0 - ly + IR < nr ? r0 - ly + IR : nr;
        if (rhi <= rlo) continue;
        const int64_t e0 = gc * nr + rlo, e1 = gc * nr + rhi;
        const int64_t shift = gc * nr + (r0 - ly);  // linear index of segment row 0
        int* colv = sv + cc * IRp;
        uint32_t* colf = sf + cc * IRp;
        load_chunks(img, n, e0, e1, lane, 32, [&](int64_t e, T v) {
            colv[e - shift] = static_cast<int>(v);
        });
        __syncwarp();
        load_chunks(mask, n, e0, e1, lane, 32, [&](int64_t e, uint8_t m) {
            const int i = static_cast<int>(e - shift);
            if (m) {
                colf[i] = 1u;
            } else {
                colf[i] = 1u << 16;
                colv[i] = 0;
            }
        });
    }
    __syncthreads();
    // Down each column: a task is a column and 16 output rows.
    const int nseg = (TR + 15) >> 4;
    for (int task = tid; task < IC * nseg; task += kHpThreads) {
        const int cc = task / nseg, i0 = 16 * (task - cc * nseg);
        const int* colv = sv + cc * IRp;
        const uint32_t* colf = sf + cc * IRp;
        int a = 0;
        uint32_t f = 0u;
        for (int k = 0; k < wy; ++k) {
            a += colv[i0 + k];
            f += colf[i0 + k];
        }
        const int iend = min(i0 + 16, TR);
        for (int i = i0; i < iend; ++i) {
            vs[cc * TR + i] = a;
            vf[cc * TR + i] = f;
            a += colv[i + wy] - colv[i];
            f += colf[i + wy] - colf[i];
        }
    }
    __syncthreads();
    // Across columns: a thread is an output row and a share of the tile's columns.
    const int r = tid % TR;
    const int parts = kHpThreads / TR;  // TR divides kHpThreads
    const int cw_ = kHpCols / parts;
    const int cb = (tid / TR) * cw_;
    const int64_t gr = r0 + r;
    if (gr >= nr) return;
    int a = 0;
    uint32_t f = 0u;
    for (int k = 0; k < wx; ++k) {
        a += vs[(cb + k) * TR + r];
        f += vf[(cb + k) * TR + r];
    }
    for (int c = cb; c < cb + cw_; ++c) {
        const int64_t gc = c0 + c;
        if (gc >= nc) break;
        const int cnt = static_cast<int>(f & 0xFFFFu);
        const bool eroded = (f >> 16) == 0u;
        const float mean = cnt > 0 ? __double2float_rn(__ddiv_rn(static_cast<double>(a),
                                                                 static_cast<double>(cnt)))
                                   : __int_as_float(0x7fc00000);
        const int ci = (c + lx) * IRp + (r + ly);  // the centre pixel in the staged tile
        const bool m = (sf[ci] & 1u) != 0u;
        float o = (m && isfinite(mean)) ? __fsub_rn(static_cast<float>(sv[ci]), mean)
                                        : __int_as_float(0x7fc00000);
        bool v = eroded;
        if (!isfinite(o)) {
            o = 0.0f;
            v = false;
        }
        const int64_t g = gr + gc * nr;
        out[g] = o;
        vout[g] = v ? 1 : 0;
        if (c + 1 < cb + cw_) {
            a += vs[(c + wx) * TR + r] - vs[c * TR + r];
            f += vf[(c + wx) * TR + r] - vf[c * TR + r];
        }
    }
}

// The same filter for square windows of odd width W <= 9 (the usual highpass widths), without
// shared memory: a warp holds 32 consecutive rows of one column (a lane per row, coalesced loads
// and stores) and walks along its columns, W columns' loads at a time. An element becomes one
// 32-bit word -- its value (offset to be non-negative) in bits 0-19 when it contributes, a
// contributing count of 1 at bit 20 or an in-image-invalid count of 1 at bit 24 -- so the three
// sums down a column of the window are one 32-bit sum across lanes (shuffles); along the row they
// are a sliding sum over a register ring of the last W columns, widened to 64 bits (value in the
// low word, counts at bits 32 and 48). A warp writes the 32 - (W - 1) rows whose whole window it
// holds. The mean is an FP32 division of the exact sum by the count: both are exact in FP32
// (below 2^24) and FP64 has more than 2 x 24 + 2 bits, so it equals the generic kernel's FP64
// quotient rounded to FP32 (double rounding is innocuous there); the output is the generic
// kernel's, bit for bit.
constexpr int kHwCols = 64;     // columns per warp
constexpr int kHwWarps = 8;     // warps (row strips) per block

template <typename T, int W>
__global__ void __launch_bounds__(kHwWarps * 32) k_highpass_w(const T* img, const uint8_t* mask,
                                                              int64_t nr, int64_t nc, float* out,
                                                              uint8_t* vout) {
    constexpr int L = W / 2;
    constexpr int RO = 32 - 2 * L;  // output rows of a strip
    constexpr uint32_t kC32 = 1u << 20, kI32 = 1u << 24;
    constexpr int kBias = std::is_signed<T>::value ? 32768 : 0;
    const int lane = threadIdx.x & 31;
    const int64_t strip = static_cast<int64_t>(blockIdx.x) * kHwWarps + (threadIdx.x >> 5);
    const int64_t r0 = strip * RO;  // first output row of the strip
    if (r0 >= nr) return;
    const int64_t c0 = static_cast<int64_t>(blockIdx.y) * kHwCols;
    const int64_t c1 = c0 + kHwCols < nc ? c0 + kHwCols : nc;
    const int64_t r = r0 - L + lane;
    const bool rin = r >= 0 && r < nr;
    const bool writes = lane >= L && lane < 32 - L && r < nr;
    uint64_t ring_v[W];
    uint32_t ring_p[W];
#pragma unroll
    for (int u = 0; u < W; ++u) {
        ring_v[u] = 0ull;
        ring_p[u] = 0u;
    }
    uint64_t S = 0ull;
    for (int64_t cb = c0 - L; cb < c1 + L; cb += W) {
        uint32_t pv[W];
#pragma unroll
        for (int u = 0; u < W; ++u) {
            const int64_t c = cb + u;
            pv[u] = 0u;
            if (rin && c >= 0 && c < nc) {
                const int64_t g = r + c * nr;
                const uint32_t v = static_cast<uint32_t>(static_cast<int>(img[g]) + kBias);
                pv[u] = mask[g] ? (v | kC32) : kI32;
            }
        }
#pragma unroll
        for (int u = 0; u < W; ++u) {
            const uint32_t p = pv[u];
            uint32_t V = p;
#pragma unroll
            for (int d = 1; d <= L; ++d) V += __shfl_up_sync(kFullMask, p, d) + __shfl_down_sync(kFullMask, p, d);
            const uint64_t V64 = static_cast<uint64_t>(V & (kC32 - 1u)) |
                                 (static_cast<uint64_t>((V >> 20) & 0xFu) << 32) |
                                 (static_cast<uint64_t>(V >> 24) << 48);
            S += V64 - ring_v[u];
            ring_v[u] = V64;
            ring_p[u] = p;
            const int64_t j = cb + u - L;  // the output column whose window ends at column cb + u
            if (writes && j >= c0 && j < c1) {
                const int cnt = static_cast<int>((S >> 32) & 0xFFFFull);
                const int inv = static_cast<int>(S >> 48);
                const int a = static_cast<int>(static_cast<uint32_t>(S)) - kBias * cnt;
                const float mean = cnt > 0 ? __fdiv_rn(static_cast<float>(a), static_cast<float>(cnt))
                                           : __int_as_float(0x7fc00000);
                const uint32_t pc = ring_p[(u - L + W) % W];  // column j's element
                const bool m = (pc & kC32) != 0u;
                const float x = static_cast<float>(static_cast<int>(pc & (kC32 - 1u)) - kBias);
                float o = (m && isfinite(mean)) ? __fsub_rn(x, mean) : __int_as_float(0x7fc00000);
                bool v = inv == 0;
                if (!isfinite(o)) {
                    o = 0.0f;
                    v = false;
                }
                const int64_t g = r + j * nr;
                out[g] = o;
                vout[g] = v ? 1 : 0;
            }
        }
    }
}

size_t highpass_int_smem(int wx, int wy, int TR) {
    const size_t IR = TR + wy - 1, IC = kHpCols + wx - 1, IRp = IR | 1;
    return IC * IRp * 8 + IC * TR * 8;
}

// First Wallis pass: the masked box mean (src/preprocess.jl:336).
template <typename T>
__global__ void __launch_bounds__(kBoxThreads) k_boxmean(const T* img, const uint8_t* mask,
                                                         int64_t nr, int64_t nc, int wx, int wy,
                                                         float* mean) {
    extern __shared__ __align__(16) unsigned char bsm[];
    const BoxSmem S = box_smem(bsm, wx, wy);
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kTile;
    const int64_t c0 = static_cast<int64_t>(blockIdx.y) * kTile;
    box_tile<T, BOX_IMAGE>(img, mask, nullptr, nr, nc, wx, wy, r0, c0, S,
                           [&](int64_t g, double s, int cnt, bool) { mean[g] = box_mean(s, cnt); });
}

// Second Wallis pass (src/preprocess.jl:337-351, 416-438) with `_filtered`.
template <typename T>
__global__ void __launch_bounds__(kBoxThreads) k_wallis(const T* img, const uint8_t* mask,
                                                        const float* mean, int64_t nr,
                                                        int64_t nc, int wx, int wy, float floor_sd,
                                                        float* out, uint8_t* vout) {
    extern __shared__ __align__(16) unsigned char bsm[];
    const BoxSmem S = box_smem(bsm, wx, wy);
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kTile;
    const int64_t c0 = static_cast<int64_t>(blockIdx.y) * kTile;
    box_tile<T, BOX_DEV2>(img, mask, mean, nr, nc, wx, wy, r0, c0, S,
                          [&](int64_t g, double s, int cnt, bool eroded) {
                              float msd = box_mean(s, cnt);
                              // sqrt(max(msd, 0f0)): Julia's max keeps a NaN.
                              if (!isnan(msd)) msd = __fsqrt_rn(fmaxf(msd, 0.0f));
                              const float m = mean[g];
                              float o;
                              if (!mask[g] || !isfinite(m) || !isfinite(msd)) {
                                  o = __int_as_float(0x7fc00000);
                              } else {
                                  const float sd = fmaxf(msd, floor_sd);
                                  o = sd > 0.0f ? __fdiv_rn(__fsub_rn(as_f32(img[g]), m), sd)
                                                : __int_as_float(0x7fc00000);
                              }
                              bool v = eroded;
                              if (!isfinite(o)) {
                                  o = 0.0f;
                                  v = false;
                              }
                              out[g] = o;
                              vout[g] = v ? 1 : 0;
                          });
}

// ---------------------------------------------------------------------------------------------
// Quantisation (src/preprocess.jl:546-592)

}  // namespace

// Double-double accumulator and the quantiser's device-side statistics (declared in
// ar_internal.cuh so the context can size the scratch).
struct DD {
    double hi, lo;
};

__device__ __forceinline__ void dd_add(DD& a, double x) {
    const double s = __dadd_rn(a.hi, x);
    const double bb = __dsub_rn(s, a.hi);
    const double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(x, bb));
    a.hi = s;
    a.lo = __dadd_rn(a.lo, e);
}

__device__ __forceinline__ void dd_merge(DD& a, const DD& b) {
    dd_add(a, b.hi);
    a.lo = __dadd_rn(a.lo, b.lo);
}

struct QuantStats {
    double mean, sd, lo, scale;
    long long n;
    DD part[kStatBlocks];
    long long cnt[kStatBlocks];
};

namespace {

__device__ void block_dd(DD& a, long long& c, DD* sa, long long* sc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD b{__shfl_xor_sync(kFullMask, a.hi, o), __shfl_xor_sync(kFullMask, a.lo, o)};
        dd_merge(a, b);
        c += __shfl_xor_sync(kFullMask, c, o);
    }
    if (lane == 0) {
        sa[warp] = a;
        sc[warp] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < nw; ++k) {
            dd_merge(a, sa[k]);
            c += sc[k];
        }
    }
}

// pass 0: sum and count of the valid finite values; pass 1: sum of squared deviations. A thread
// takes runs of four consecutive elements (one vector load of the image and one of the mask
// where both are aligned) and keeps kQU runs in flight, each feeding its own double-double
// accumulator; the accumulators merge in a fixed order.
constexpr int kQU = 4;

template <typename T>
struct alignas(4 * sizeof(T)) Run4 {
    T x[4];
};
struct alignas(4) Mask4 {
    uint8_t x[4];
};

template <typename T, int PASS>
__global__ void __launch_bounds__(kStatThreads) k_qstats(const T* img, const uint8_t* mask,
                                                         int64_t n, QuantStats* st) {
    __shared__ DD sa[32];
    __shared__ long long sc[32];
    DD acc[kQU];
    long long cc[kQU];
#pragma unroll
    for (int u = 0; u < kQU; ++u) {
        acc[u] = DD{0.0, 0.0};
        cc[u] = 0;
    }
    const double mean = PASS == 1 ? st->mean : 0.0;
    const bool vec = (reinterpret_cast<uintptr_t>(img) % (4 * sizeof(T))) == 0 &&
                     (reinterpret_cast<uintptr_t>(mask) % 4) == 0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;  // in runs of four
    for (int64_t r0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; 4 * r0 < n;
         r0 += kQU * stride) {
        T t[kQU][4];
        uint8_t m[kQU][4];
#pragma unroll
        for (int u = 0; u < kQU; ++u) {
            const int64_t i = 4 * (r0 + u * stride);
            if (vec && i + 4 <= n) {
                const Run4<T> w = *reinterpret_cast<const Run4<T>*>(img + i);
                const Mask4 k = *reinterpret_cast<const Mask4*>(mask + i);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    t[u][e] = w.x[e];
                    m[u][e] = k.x[e];
                }
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const bool in = i + e < n;
                    t[u][e] = in ? img[i + e] : T(0);
                    m[u][e] = in ? mask[i + e] : static_cast<uint8_t>(0);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kQU; ++u) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double v = static_cast<double>(t[u][e]);
                if (!(m[u][e] && isfinite(v))) continue;
                if (PASS == 0) {
                    dd_add(acc[u], v);
                    ++cc[u];
                } else {
                    const double d = __dsub_rn(v, mean);
                    dd_add(acc[u], __dmul_rn(d, d));
                }
            }
        }
    }
    DD a = acc[0];
    long long c = cc[0];
#pragma unroll
    for (int u = 1; u < kQU; ++u) {
        dd_merge(a, acc[u]);
        c += cc[u];
    }
    block_dd(a, c, sa, sc);
    if (threadIdx.x == 0) {
        st->part[blockIdx.x] = a;
        st->cnt[blockIdx.x] = c;
    }
}

// Fixed-order combination of the block partials: the block stages them in shared memory with
// coalesced loads, then one thread merges them in block order (the merge chain is sequential,
// so its operands must not wait on global memory).
template <int PASS>
__global__ void k_qfinal(QuantStats* st, int nblocks) {
    __shared__ DD s_part[kStatBlocks];
    __shared__ long long s_cnt[kStatBlocks];
    if (blockIdx.x != 0) return;
    for (int k = threadIdx.x; k < nblocks; k += blockDim.x) {
        s_part[k] = st->part[k];
        s_cnt[k] = st->cnt[k];
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    DD a{0.0, 0.0};
    long long c = 0;
    for (int k = 0; k < nblocks; ++k) {
        dd_merge(a, s_part[k]);
        c += s_cnt[k];
    }
    const double s = __dadd_rn(a.hi, a.lo);
    if (PASS == 0) {
        st->n = c;
        st->mean = c > 0 ? __ddiv_rn(s, static_cast<double>(c)) : 0.0;
    } else {
        const long long nn = st->n;
        const double sd = nn > 1 ? __dsqrt_rn(__ddiv_rn(s, static_cast<double>(nn - 1))) : 0.0;
        st->sd = sd;
        st->lo = __dsub_rn(st->mean, __dmul_rn(3.0, sd));
        st->scale = sd != 0.0 ? __ddiv_rn(255.0, __dmul_rn(6.0, sd)) : 0.0;
    }
}

// kQV consecutive pixels per thread as runs of four: one vector load of the image and one of the
// mask per run where aligned (the filtered Float32 scratch and the masks always are), one 4-byte
// store of the output per run.
constexpr int kQV = 8;

template <typename T>
__global__ void k_quantize(const T* img, const uint8_t* mask, int64_t n, const QuantStats* st,
                           uint8_t* out) {
    const int64_t i0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) * kQV;
    if (i0 >= n) return;
    const long long cnt = st->n;
    const double sd = st->sd, lo = st->lo, scale = st->scale;
    const bool vec = (reinterpret_cast<uintptr_t>(img) % (4 * sizeof(T))) == 0 &&
                     (reinterpret_cast<uintptr_t>(mask) % 4) == 0 &&
                     (reinterpret_cast<uintptr_t>(out) % 4) == 0;
    T vals[kQV];
    uint8_t ms[kQV];
#pragma unroll
    for (int r = 0; r < kQV; r += 4) {
        const int64_t i = i0 + r;
        if (vec && i + 4 <= n) {
            const Run4<T> w = *reinterpret_cast<const Run4<T>*>(img + i);
            const Mask4 k = *reinterpret_cast<const Mask4*>(mask + i);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                vals[r + e] = w.x[e];
                ms[r + e] = k.x[e];
            }
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const bool in = i + e < n;
                vals[r + e] = in ? img[i + e] : T(0);
                ms[r + e] = in ? mask[i + e] : static_cast<uint8_t>(0);
            }
        }
    }
    uint8_t o[kQV];
#pragma unroll
    for (int u = 0; u < kQV; ++u) {
        const bool m = ms[u] != 0;
        const double v = static_cast<double>(vals[u]);
        if (cnt == 0) {
            o[u] = 0;
        } else if (sd == 0.0) {
            o[u] = m ? 0x80 : 0x00;
        } else if (!m || !isfinite(v)) {
            o[u] = 0;
        } else {
            double x = __dmul_rn(__dsub_rn(v, lo), scale);
            x = x < 0.0 ? 0.0 : (x > 255.0 ? 255.0 : x);
            o[u] = static_cast<uint8_t>(__double2uint_rn(x));
        }
    }
#pragma unroll
    for (int r = 0; r < kQV; r += 4) {
        const int64_t i = i0 + r;
        if (vec && i + 4 <= n) {
            *reinterpret_cast<uchar4*>(out + i) = make_uchar4(o[r], o[r + 1], o[r + 2], o[r + 3]);
        } else {
            for (int e = 0; e < 4; ++e)
                if (i + e < n) out[i + e] = o[r + e];
        }
    }
}

// NoQuantize of a float image: non-finite values become zero, the mask is kept
// (src/preprocess.jl:495-507).
template <typename T>
__global__ void k_finite_copy(const T* img, int64_t n, T* out) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const T v = img[i];
    out[i] = isfinite(static_cast<double>(v)) ? v : T(0);
}

template <typename T>
cudaError_t quantize_u8(const T* img, const uint8_t* mask, int64_t n, QuantStats* st,
                        uint8_t* out, cudaStream_t s, long long* launches) {
    k_qstats<T, 0><<<kStatBlocks, kStatThreads, 0, s>>>(img, mask, n, st);
    k_qfinal<0><<<1, 256, 0, s>>>(st, kStatBlocks);
    k_qstats<T, 1><<<kStatBlocks, kStatThreads, 0, s>>>(img, mask, n, st);
    k_qfinal<1><<<1, 256, 0, s>>>(st, kStatBlocks);
    const int threads = 256;
    const int64_t per_block = static_cast<int64_t>(threads) * kQV;
    k_quantize<T><<<static_cast<unsigned>((n + per_block - 1) / per_block), threads, 0, s>>>(
        img, mask, n, st, out);
    *launches += 5;
    return cudaGetLastError();
}

template <typename T>
cudaError_t prepare_t(const PrepareJob& J, cudaStream_t s, long long* launches) {
    const T* img = static_cast<const T*>(J.img);
    const int64_t n = J.nrows * J.ncols;
    if (J.preprocess == 0) {
        cudaError_t e = cudaMemcpyAsync(J.vout, J.mask, n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
        if (J.quantize == 1)
            return quantize_u8(img, J.mask, n, J.stats, static_cast<uint8_t*>(J.out), s, launches);
        const int threads = 256;
        k_finite_copy<T><<<static_cast<unsigned>((n + threads - 1) / threads), threads, 0, s>>>(
            img, n, static_cast<T*>(J.out));
        *launches += 1;
        return cudaGetLastError();
    }
    const dim3 grid(static_cast<unsigned>((J.nrows + kTile - 1) / kTile),
                    static_cast<unsigned>((J.ncols + kTile - 1) / kTile));
    // The window clamped to the image (src/window.jl:632-637).
    const int wx = static_cast<int>(std::min<int64_t>(J.width, J.ncols));
    const int wy = static_cast<int>(std::min<int64_t>(J.width, J.nrows));
    const size_t smem = box_smem_bytes(wx, wy);
    float* filt = J.quantize == 1 ? J.ftmp : static_cast<float*>(J.out);
    cudaError_t e;
    if (smem > static_cast<size_t>(kDynSmemCap)) return cudaErrorInvalidValue;
    if (J.preprocess == 1 && !std::is_same<T, float>::value && wx == wy && (wx & 1) && wx <= 9) {
        // Integer imagery, square odd window up to 9: the shared-memory-free kernel.
        constexpr int RO_of[10] = {0, 32, 0, 30, 0, 28, 0, 26, 0, 24};
        const int RO = RO_of[wx];
        const int64_t strips = (J.nrows + RO - 1) / RO;
        const dim3 wgrid(static_cast<unsigned>((strips + kHwWarps - 1) / kHwWarps),
                         static_cast<unsigned>((J.ncols + kHwCols - 1) / kHwCols));
        switch (wx) {
            case 1: k_highpass_w<T, 1><<<wgrid, kHwWarps * 32, 0, s>>>(img, J.mask, J.nrows, J.ncols, filt, J.vout); break;
            case 3: k_highpass_w<T, 3><<<wgrid, kHwWarps * 32, 0, s>>>(img, J.mask, J.nrows, J.ncols, filt, J.vout); break;
            case 5: k_highpass_w<T, 5><<<wgrid, kHwWarps * 32, 0, s>>>(img, J.mask, J.nrows, J.ncols, filt, J.vout); break;
            case 7: k_highpass_w<T, 7><<<wgrid, kHwWarps * 32, 0, s>>>(img, J.mask, J.nrows, J.ncols, filt, J.vout); break;
            default: k_highpass_w<T, 9><<<wgrid, kHwWarps * 32, 0, s>>>(img, J.mask, J.nrows, J.ncols, filt, J.vout); break;
        }
        *launches += 1;
    } else if (J.preprocess == 1 && !std::is_same<T, float>::value) {
        // Integer imagery: exact 32-bit sums, the tallest tile whose staging fits.
        int TR = 128;
        while (TR > 32 && highpass_int_smem(wx, wy, TR) > static_cast<size_t>(kDynSmemCap)) TR /= 2;
        const size_t hsm = highpass_int_smem(wx, wy, TR);
        if (hsm > static_cast<size_t>(kDynSmemCap)) return cudaErrorInvalidValue;
        e = cudaFuncSetAttribute(k_highpass_int<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kDynSmemCap);
        if (e != cudaSuccess) return e;
        const dim3 hgrid(static_cast<unsigned>((J.nrows + TR - 1) / TR),
                         static_cast<unsigned>((J.ncols + kHpCols - 1) / kHpCols));
        k_highpass_int<T><<<hgrid, kHpThreads, hsm, s>>>(img, J.mask, J.nrows, J.ncols, wx, wy, TR,
                                                         filt, J.vout);
        *launches += 1;
    } else if (J.preprocess == 1) {
        e = cudaFuncSetAttribute(k_highpass<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kDynSmemCap);
        if (e != cudaSuccess) return e;
        k_highpass<T><<<grid, kBoxThreads, smem, s>>>(img, J.mask, J.nrows, J.ncols, wx, wy, filt, J.vout);
        *launches += 1;
    } else {
        e = cudaFuncSetAttribute(k_boxmean<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kDynSmemCap);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_wallis<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kDynSmemCap);
        if (e != cudaSuccess) return e;
        k_boxmean<T><<<grid, kBoxThreads, smem, s>>>(img, J.mask, J.nrows, J.ncols, wx, wy, J.mtmp);
        k_wallis<T><<<grid, kBoxThreads, smem, s>>>(img, J.mask, J.mtmp, J.nrows, J.ncols, wx, wy,
                                                    static_cast<float>(J.min_std), filt, J.vout);
        *launches += 2;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess || J.quantize != 1) return e;
    return quantize_u8(filt, J.vout, n, J.stats, static_cast<uint8_t*>(J.out), s, launches);
}

}  // namespace

size_t quant_stats_bytes() { return sizeof(QuantStats); }

int max_filter_width() { return kMaxWidth; }

cudaError_t launch_prepare(const PrepareJob& J, cudaStream_t s, long long* launches) {
    if (J.width > kMaxWidth && J.preprocess != 0) return cudaErrorInvalidValue;
    switch (J.dtype) {
        case AR_U8: return prepare_t<uint8_t>(J, s, launches);
        case AR_U16: return prepare_t<uint16_t>(J, s, launches);
        case AR_I16: return prepare_t<int16_t>(J, s, launches);
        case AR_F32: return prepare_t<float>(J, s, launches);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ar
