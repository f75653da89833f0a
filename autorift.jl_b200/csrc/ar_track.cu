// The track pass on sm_100a: one CTA per search point computes the ZNCC surface in shared
// memory, its row-major argmax and the 5x5 refinement patch; a second kernel runs the pyrUp
// cascade on the patches. The surface never leaves shared memory.
//
// Reference (AutoRIFT.jl): src/track.jl:103-152, 249-305 (the grid loop), src/points.jl:358-395
// (chip and window bounds), src/correlate.jl:423-453 (prepare_chip!), 575-630 (ZNCC / NCC
// normalisation), 785-848 (numerator), src/integral.jl:141-170, 244-247 (per-window sums),
// src/peak.jl:32-61, 102-106, 196-324, 456-522 (peak and sub-pixel cascade).
//
// Numerics.
//  * Numerator: FP32 products accumulated in FP32 over a few chip columns, then flushed into
//    an FP64 accumulator. For UInt8 imagery the chip and window are staged as raw integers
//    and the flush interval keeps every FP32 partial below 2^24, so the numerator
//    sum(T*W) - mean(T)*sum(W) is exact -- the value the reference's FP32 FFT approximates.
//    Other element types stage the mean-removed chip and a centred window (W - c).
//  * Denominator: window box sums from per-window prefix tables built by warp scans in
//    shared memory -- exact integers (uint32) for UInt8, FP64 otherwise -- and
//    wvar = max(s2 - s1*s1/n, 0), den = cnorm*sqrt(wvar), surface = Float32(num/den), each
//    operation an explicitly rounded FP64 intrinsic, as in src/correlate.jl:591-600.
//  * Cascade: every pyrUp sample is fl(fl(0.75*b) + fl(0.125*fl(a+c))) or
//    fl(0.5*fl(b+c)) with __fmul_rn/__fadd_rn, so no step is fused into an FMA and the result
//    is bit-identical to the reference's Float32 arithmetic on the same patch.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <type_traits>

#include "ar_internal.cuh"
#include "ar_tc.cuh"

namespace ar {
namespace {

constexpr int kMI = 10;        // surface rows per thread item
constexpr int kUA = 16;        // chip rows per inner step
constexpr int kCorrThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

template <typename T>
struct Traits;
template <>
struct Traits<uint8_t> {
    static constexpr bool raw = true;  // exact integer numerator
    static constexpr bool integer = true;
    typedef uint32_t ph_t;
};
template <>
struct Traits<uint16_t> {
    static constexpr bool raw = false;
    static constexpr bool integer = true;
    typedef double ph_t;
};
template <>
struct Traits<int16_t> {
    static constexpr bool raw = false;
    static constexpr bool integer = true;
    typedef double ph_t;
};
template <>
struct Traits<float> {
    static constexpr bool raw = false;
    static constexpr bool integer = false;
    typedef double ph_t;
};

// ----------------------------------------------------------------------------------------------
// Reductions

// Key for a row-major first strict maximum (src/peak.jl:32-61): the larger value wins, and
// among equal values the smaller row-major index. NaN never wins; -0 equals +0.
__device__ __forceinline__ unsigned long long argmax_key(float v, unsigned rowmajor) {
    if (v != v) return 0ull;
    if (v == 0.0f) v = 0.0f;
    unsigned u = __float_as_uint(v);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return (static_cast<unsigned long long>(u) << 32) | (0xffffffffu - rowmajor);
}

__device__ __forceinline__ float key_value(unsigned long long key) {
    unsigned u = static_cast<unsigned>(key >> 32);
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return __uint_as_float(u);
}

// Decode to (row-major index, value); the reference returns (1,1) when nothing beats -Inf.
__device__ __forceinline__ bool key_decode(unsigned long long key, unsigned* rowmajor,
                                          float* value) {
    if (key == 0ull) return false;
    const float v = key_value(key);
    if (v == -INFINITY) return false;
    *rowmajor = 0xffffffffu - static_cast<unsigned>(key & 0xffffffffull);
    *value = v;
    return true;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(kFull, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Block-wide max; every thread gets the result. `red` holds >= 32 entries.
__device__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_max_u64(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    unsigned long long r = lane < nw ? red[lane] : 0ull;
    r = warp_max_u64(r);
    return r;
}

__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// Block-wide sum of up to three doubles; every thread gets the results.
template <int N>
__device__ void block_sum_f64(double (&v)[N], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = warp_sum_f64(v[q]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < N; ++q) red[q * 32 + warp] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; ++q) {
        double r = lane < nw ? red[q * 32 + lane] : 0.0;
        v[q] = warp_sum_f64(r);
    }
}

template <typename V>
__device__ __forceinline__ V warp_inclusive_scan(V v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const V w = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v = v + w;
    }
    return v;
}

// ----------------------------------------------------------------------------------------------
// pyrUp arithmetic

// One pyrUp sample in the reference's operation order (src/peak.jl:266-292).
__device__ __forceinline__ float pyr_sample(int nt, float a, float b, float c) {
    return nt == 3 ? __fadd_rn(__fmul_rn(0.75f, b), __fmul_rn(0.125f, __fadd_rn(a, c)))
                   : __fmul_rn(0.5f, __fadd_rn(b, c));
}

// ----------------------------------------------------------------------------------------------
// Correlation kernel

struct CorrArgs {
    const void* ref;
    const void* sec;
    const uint8_t* valid;
    int64_t nrows, ncols;
    DevPoints pts;
    int64_t padx, pady;
    int up, measure;
    int TI, TJ;   // surface tile; TI a multiple of kMI and (TI/kMI)*TJ <= blockDim
    int CHP;      // chip smem stride (rows), >= every point's ch rounded up to 16
    int CWM;      // largest chip width
    int BC;       // chip columns staged at a time (== CWM: the whole chip once per point)
    int WS;       // window smem stride (floats): even, WS/2 odd, >= TI + CHP
    int PHS;      // prefix-table stride (entries), >= TI + largest ch
    int NRS;      // surface smem stride (rows), >= largest nr
    int NCM;      // largest nc
    unsigned off_win, off_ph1, off_ph2, off_surf, off_red;  // byte offsets, chip at 0
    DevOutputs out;
    int* sub_count;
    int64_t* sub_point;
    int32_t* sub_origin;
    float* sub_patch;
    float* surf_out;  // optional: each point's surface, NRS x NCM floats per point
    unsigned long long* flops;  // optional: algorithmic FLOPs of the surfaces computed
    unsigned off_surf2;  // rotation search: the best surface so far (NRS x NCM floats)
    Rotation rot;        // rotation search angles (k_corr<T, true> only)
};
static_assert(sizeof(CorrArgs) <= 4096, "k_corr's arguments must fit the 4 KB parameter space");

template <typename T>
__device__ __forceinline__ double pixel(const T* img, int64_t nrows, int64_t ncols, int64_t r,
                                        int64_t c) {
    if (r < 0 || r >= nrows || c < 0 || c >= ncols) return 0.0;
    return static_cast<double>(img[r + c * nrows]);
}

template <typename PH>
__device__ __forceinline__ PH ph_of(float w);
template <>
__device__ __forceinline__ uint32_t ph_of<uint32_t>(float w) {
    return static_cast<uint32_t>(w);
}

// _rotate_chip (src/track.jl:377-409) at 0-based chip element (a, b) of a ch x cw chip whose
// first element is image element (chip_r, chip_c): the source point by the inverse rotation
// about the chip centre ((ch + 1) / 2, (cw + 1) / 2, 1-based), FP64 bilinear from its four
// neighbours, zero when one of them falls outside the chip, rounded to Float32. Each
// operation is rounded separately, in the reference's order (no contraction).
template <typename T>
__device__ __forceinline__ float rotated_sample(const T* sec, int64_t nrows, int64_t ncols,
                                                int64_t chip_r, int64_t chip_c, int ch, int cw,
                                                int a, int b, double sn, double cs) {
    const double yc = static_cast<double>(ch + 1) * 0.5, xc = static_cast<double>(cw + 1) * 0.5;
    const double dy = static_cast<double>(a + 1) - yc, dx = static_cast<double>(b + 1) - xc;
    const double sy = __dadd_rn(__dadd_rn(yc, __dmul_rn(cs, dy)), __dmul_rn(sn, dx));
    const double sx = __dadd_rn(__dsub_rn(xc, __dmul_rn(sn, dy)), __dmul_rn(cs, dx));
    const double fi = floor(sy), fj = floor(sx);
    if (!(fi >= 1.0 && fj >= 1.0 && fi + 1.0 <= static_cast<double>(ch) &&
          fj + 1.0 <= static_cast<double>(cw)))
        return 0.0f;
    const int i0 = static_cast<int>(fi), j0 = static_cast<int>(fj);  // 1-based
    const double fy = __dsub_rn(sy, fi), fx = __dsub_rn(sx, fj);
    const double v00 = pixel(sec, nrows, ncols, chip_r + i0 - 1, chip_c + j0 - 1);
    const double v10 = pixel(sec, nrows, ncols, chip_r + i0, chip_c + j0 - 1);
    const double v01 = pixel(sec, nrows, ncols, chip_r + i0 - 1, chip_c + j0);
    const double v11 = pixel(sec, nrows, ncols, chip_r + i0, chip_c + j0);
    const double gx = __dsub_rn(1.0, fx), gy = __dsub_rn(1.0, fy);
    const double top = __dadd_rn(__dmul_rn(gx, v00), __dmul_rn(fx, v01));
    const double bot = __dadd_rn(__dmul_rn(gx, v10), __dmul_rn(fx, v11));
    return __double2float_rn(__dadd_rn(__dmul_rn(gy, top), __dmul_rn(fy, bot)));
}

// ROT: the rotation search. Its chips are Float32 (turned chips are resampled), so the
// numerator takes the FP32/FP64 branch and the box sums are FP64 for every element type.
template <typename T, bool ROT>
__global__ void __launch_bounds__(kCorrThreads, 2) k_corr(const CorrArgs A) {
    typedef Traits<T> Tr;
    constexpr bool RAW = Tr::raw && !ROT;
    typedef typename std::conditional<ROT, double, typename Tr::ph_t>::type PH;
    extern __shared__ __align__(16) unsigned char smem[];
    float* s_chip = reinterpret_cast<float*>(smem);
    float* s_win = reinterpret_cast<float*>(smem + A.off_win);
    PH* s_ph1 = reinterpret_cast<PH*>(smem + A.off_ph1);
    PH* s_ph2 = reinterpret_cast<PH*>(smem + A.off_ph2);
    float* s_surf = reinterpret_cast<float*>(smem + A.off_surf);
    float* s_surf2 = reinterpret_cast<float*>(smem + A.off_surf2);
    double* s_red = reinterpret_cast<double*>(smem + A.off_red);
    __shared__ int s_slot;

    const int tid = threadIdx.x, bd = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = bd >> 5;
    const T* ref = static_cast<const T*>(A.ref);
    const T* sec = static_cast<const T*>(A.sec);
    const int64_t NR = A.nrows + 2 * A.pady, NC = A.ncols + 2 * A.padx;
    const double shx = static_cast<double>(A.padx) + 0.5;
    const double shy = static_cast<double>(A.pady) + 0.5;

    for (int64_t k = blockIdx.x; k < A.pts.n; k += gridDim.x) {
        __syncthreads();  // shared buffers of the previous point are no longer read
        const int64_t prx = A.pts.rx[k], pry = A.pts.ry[k];
        if (!(prx > 0 && pry > 0)) continue;  // issearchable (src/points.jl:116-117)

        // Geometry in padded 1-based coordinates (src/track.jl:207-210, src/points.jl:358-395).
        const double xs = A.pts.x[k] + shx, ys = A.pts.y[k] + shy;
        const int64_t hx = A.pts.csx[k] / 2, hy = A.pts.csy[k] / 2;
        const int64_t ccx = static_cast<int64_t>(floor(__dsub_rn(xs, A.pts.dx0[k])));
        const int64_t ccy = static_cast<int64_t>(floor(__dsub_rn(ys, A.pts.dy0[k])));
        const int64_t wcx = static_cast<int64_t>(floor(xs)), wcy = static_cast<int64_t>(floor(ys));
        const int64_t cr0 = ccy - hy, cr1 = ccy + hy - 1, cc0 = ccx - hx, cc1 = ccx + hx - 1;
        const int64_t wr0 = wcy - hy - pry, wr1 = wcy + hy + pry - 2;
        const int64_t wc0 = wcx - hx - prx, wc1 = wcx + hx + prx - 2;
        // checkbounds (src/track.jl:271-272): an empty range is always in bounds.
        const bool chip_in = (cr1 < cr0 || cc1 < cc0) ||
                             (cr0 >= 1 && cr1 <= NR && cc0 >= 1 && cc1 <= NC);
        const bool win_in = (wr1 < wr0 || wc1 < wc0) ||
                            (wr0 >= 1 && wr1 <= NR && wc0 >= 1 && wc1 <= NC);
        if (!chip_in || !win_in) continue;
        const int ch = static_cast<int>(2 * hy), cw = static_cast<int>(2 * hx);
        const int nr = static_cast<int>(2 * pry), nc = static_cast<int>(2 * prx);
        if (ch <= 0 || cw <= 0) continue;  // an empty chip has no valid pixel
        if (ch > A.CHP || cw > A.CWM || nr > A.NRS || nc > A.NCM) continue;  // not sized for
        const int64_t chip_r = cr0 - 1 - A.pady, chip_c = cc0 - 1 - A.padx;
        const int64_t win_r = wr0 - 1 - A.pady, win_c = wc0 - 1 - A.padx;

        // _any_valid over the chip (src/track.jl:416-421).
        int any = 0;
        for (int e = tid; e < ch * cw; e += bd) {
            const int64_t r = chip_r + e % ch, c = chip_c + e / ch;
            if (r >= 0 && r < A.nrows && c >= 0 && c < A.ncols && A.valid[r + c * A.nrows])
                any = 1;
        }
        if (!__syncthreads_or(any)) continue;
        if (tid == 0) A.out.searched[k] = 1;

        // One correlation, or with the rotation search one per angle with the best surface kept
        // (_correlate_rotations!, src/track.jl:313-350): an angle whose turned chip is
        // degenerate is skipped, and a surface replaces the best so far only if its maximum is
        // strictly larger. s_cur receives each surface; s_best is the best one so far.
        const int nang = ROT ? A.rot.count : 1;
        float* s_cur = s_surf;
        float* s_best = s_surf2;
        float bestpk = -INFINITY;
        unsigned long long best = 0ull;
        bool found = false;
        for (int ia = 0; ia < nang; ++ia) {
            const bool turn = ROT && A.rot.turn[ia];
            const double rsn = ROT ? A.rot.sn[ia] : 0.0, rcs = ROT ? A.rot.cs[ia] : 1.0;

            // prepare_chip! (src/correlate.jl:423-453): FP64 mean, then the mean-removed
            // Float32 copy, its FP64 sum of squares, and the FP64 sum of the rounded copy. With
            // the rotation search the chip (turned, or itself at angle 0) is first staged as
            // Float32 values.
            double st[1] = {0.0};
            for (int e = tid; e < ch * cw; e += bd) {
                const int a = e % ch, b = e / ch;
                double v;
                if (turn) {
                    v = static_cast<double>(rotated_sample(sec, A.nrows, A.ncols, chip_r,
                                                           chip_c, ch, cw, a, b, rsn, rcs));
                } else {
                    v = pixel(sec, A.nrows, A.ncols, chip_r + a, chip_c + b);
                }
                if (ROT) s_chip[b * A.CHP + a] = static_cast<float>(v);
                st[0] = __dadd_rn(st[0], v);
            }
            block_sum_f64<1>(st, s_red);
            const double nn = static_cast<double>(ch * cw);
            const double mean = __ddiv_rn(st[0], nn);
            const int chp = (ch + kUA - 1) & ~(kUA - 1);
            double acc2[2] = {0.0, 0.0};
            for (int e = tid; e < chp * cw; e += bd) {
                const int a = e % chp, b = e / chp;
                float staged = 0.0f;
                if (a < ch) {
                    const double v = ROT ? static_cast<double>(s_chip[b * A.CHP + a])
                                         : pixel(sec, A.nrows, A.ncols, chip_r + a, chip_c + b);
                    const double d = __dsub_rn(v, mean);
                    const float df = __double2float_rn(d);
                    acc2[0] = __dadd_rn(acc2[0], __dmul_rn(d, d));
                    acc2[1] = __dadd_rn(acc2[1], static_cast<double>(df));
                    staged = RAW ? static_cast<float>(v) : df;
                }
                if (A.BC >= cw) s_chip[b * A.CHP + a] = staged;
            }
            block_sum_f64<2>(acc2, s_red);
            const double sq = acc2[0], sumd = acc2[1];
            if (!(sq > __dmul_rn(__dmul_rn(DBL_EPSILON, static_cast<double>(ch)),
                                 static_cast<double>(cw))))
                continue;  // degenerate chip: no surface at this angle (src/track.jl:286, 326)
            const double cnorm = __dsqrt_rn(sq);
            // Centring constant for the window of non-raw element types.
            double cshift = 0.0;
            if (!RAW) cshift = Tr::integer ? rint(mean) : static_cast<double>(__double2float_rn(mean));

            const int F = RAW ? max(1, 16777216 / (chp * 65025)) : 2;
            for (int ti = 0; ti < nr; ti += A.TI) {
                const int trows = min(A.TI, nr - ti);
                const int trows_p = (trows + kMI - 1) / kMI * kMI;
                const int srows = trows_p + chp;  // staged window rows (<= WS)
                const int wrows = trows + ch - 1; // rows the box sums use
                for (int tj = 0; tj < nc; tj += A.TJ) {
                    const int tcols = min(A.TJ, nc - tj);
                    // Numerator item = (row group, column), kMI surface rows per thread; its
                    // partial sums run across the chip-column chunks.
                    const int ig = tid / A.TJ, jl = tid % A.TJ;
                    const bool item = ig * kMI < trows && jl < tcols;
                    const int il = ig * kMI;
                    float acc[kMI];
                    double acc64[kMI];
    #pragma unroll
                    for (int m = 0; m < kMI; ++m) { acc[m] = 0.0f; acc64[m] = 0.0; }
                    int fc = 0;
                    for (int b0 = 0; b0 < cw; b0 += A.BC) {
                        const int bc = min(A.BC, cw - b0);
                        const int xcols = tcols + bc - 1;
                        __syncthreads();
                        if (!ROT && A.BC < cw) {
                            // This chunk of chip columns, staged as in the unchunked case.
                            for (int e = tid; e < chp * bc; e += bd) {
                                const int a = e % chp, bl = e / chp;
                                float staged = 0.0f;
                                if (a < ch) {
                                    const double v = pixel(sec, A.nrows, A.ncols, chip_r + a, chip_c + b0 + bl);
                                    staged = RAW ? static_cast<float>(v)
                                                     : __double2float_rn(__dsub_rn(v, mean));
                                }
                                s_chip[bl * A.CHP + a] = staged;
                            }
                        }
                        // Stage the window block column-major, zero outside the image and below
                        // the window's last row.
                        for (int e = tid; e < xcols * srows; e += bd) {
                            const int r = e % srows, x = e / srows;
                            float v = 0.0f;
                            if (r < wrows) {
                                const double pv =
                                    pixel(ref, A.nrows, A.ncols, win_r + ti + r, win_c + tj + b0 + x);
                                v = RAW ? static_cast<float>(pv)
                                            : __double2float_rn(__dsub_rn(pv, cshift));
                            }
                            s_win[x * A.WS + r] = v;
                        }
                        __syncthreads();
                        // Per-window sums of W and W^2 over the chunk's columns for every row the
                        // tile uses (integral_both!, src/integral.jl:141-170), added at slot r + 1.
                        // They sum the image values themselves: a non-raw staged window is shifted
                        // by cshift for the numerator's FP32 products, and adding the shift back
                        // restores the image value (exactly for zero padding, within one Float32
                        // rounding otherwise). A window without variance -- all zero padding, or
                        // flat integer data -- then sums to exactly zero variance, as the
                        // reference's FP64 integral images do; expanding shifted sums instead
                        // leaves a rounding residue that the numerator's FP32 error turns into
                        // arbitrary correlation values.
                        auto wv = [&](int idx) -> PH {
                            if constexpr (RAW) {
                                return ph_of<PH>(s_win[idx]);
                            } else {
                                return static_cast<PH>(
                                    __dadd_rn(static_cast<double>(s_win[idx]), cshift));
                            }
                        };
                        const int nseg = (tcols + 15) >> 4;
                        for (int task = tid; task < wrows * nseg; task += bd) {
                            const int r = task % wrows, seg = task / wrows;
                            const int j0s = seg << 4, j1s = min(j0s + 16, tcols);
                            PH h1 = 0, h2 = 0;
                            for (int b = 0; b < bc; ++b) {
                                const PH w = wv((j0s + b) * A.WS + r);
                                h1 = h1 + w;
                                h2 = h2 + w * w;
                            }
                            for (int jj = j0s; jj < j1s; ++jj) {
                                if (jj > j0s) {
                                    const PH wo = wv((jj - 1) * A.WS + r);
                                    const PH wn = wv((jj - 1 + bc) * A.WS + r);
                                    h1 = h1 + wn - wo;
                                    h2 = h2 + wn * wn - wo * wo;
                                }
                                PH* p1 = &s_ph1[jj * A.PHS + r + 1];
                                PH* p2 = &s_ph2[jj * A.PHS + r + 1];
                                *p1 = b0 == 0 ? h1 : *p1 + h1;
                                *p2 = b0 == 0 ? h2 : *p2 + h2;
                            }
                        }
                        // The chunk's share of the numerator.
                        if (item) {
                            const float* wbase = s_win + jl * A.WS + il;
                            for (int b = 0; b < bc; ++b) {
                                const float* wc = wbase + b * A.WS;
                                const float* cc = s_chip + b * A.CHP;
                                for (int a0 = 0; a0 < chp; a0 += kUA) {
                                    float c[kUA];
                                    float w[kUA + kMI];
    #pragma unroll
                                    for (int q = 0; q < kUA / 4; ++q) {
                                        const float4 v = *reinterpret_cast<const float4*>(cc + a0 + 4 * q);
                                        c[4 * q] = v.x; c[4 * q + 1] = v.y; c[4 * q + 2] = v.z; c[4 * q + 3] = v.w;
                                    }
    #pragma unroll
                                    for (int q = 0; q < (kUA + kMI) / 2; ++q) {
                                        const float2 v = *reinterpret_cast<const float2*>(wc + a0 + 2 * q);
                                        w[2 * q] = v.x; w[2 * q + 1] = v.y;
                                    }
    #pragma unroll
                                    for (int a = 0; a < kUA; ++a)
    #pragma unroll
                                        for (int m = 0; m < kMI; ++m) acc[m] = fmaf(c[a], w[m + a], acc[m]);
                                }
                                if (++fc == F) {
    #pragma unroll
                                    for (int m = 0; m < kMI; ++m) {
                                        acc64[m] = __dadd_rn(acc64[m], static_cast<double>(acc[m]));
                                        acc[m] = 0.0f;
                                    }
                                    fc = 0;
                                }
                            }
                        }
                    }
                    __syncthreads();
                    // Exclusive prefix down each column by warp scans: ph[jl][q] = sum_{r<q} H[r].
                    for (int jw = warp; jw < tcols; jw += nwarps) {
                        PH c1 = 0, c2 = 0;
                        for (int q = 1; q <= wrows; q += 32) {
                            const int idx = q + lane;
                            PH v1 = idx <= wrows ? s_ph1[jw * A.PHS + idx] : PH(0);
                            PH v2 = idx <= wrows ? s_ph2[jw * A.PHS + idx] : PH(0);
                            v1 = warp_inclusive_scan(v1) + c1;
                            v2 = warp_inclusive_scan(v2) + c2;
                            if (idx <= wrows) {
                                s_ph1[jw * A.PHS + idx] = v1;
                                s_ph2[jw * A.PHS + idx] = v2;
                            }
                            c1 = __shfl_sync(kFull, v1, 31);
                            c2 = __shfl_sync(kFull, v2, 31);
                        }
                        if (lane == 0) {
                            s_ph1[jw * A.PHS] = PH(0);
                            s_ph2[jw * A.PHS] = PH(0);
                        }
                    }
                    __syncthreads();

                    if (item) {
    #pragma unroll
                        for (int m = 0; m < kMI; ++m)
                            acc64[m] = __dadd_rn(acc64[m], static_cast<double>(acc[m]));

                        // Normalisation (src/correlate.jl:591-600, 624-628).
    #pragma unroll
                        for (int m = 0; m < kMI; ++m) {
                            const int ir = il + m;
                            if (ir < trows) {
                                const PH p1 = s_ph1[jl * A.PHS + ir + ch] - s_ph1[jl * A.PHS + ir];
                                const PH p2 = s_ph2[jl * A.PHS + ir + ch] - s_ph2[jl * A.PHS + ir];
                                const double s1 = static_cast<double>(p1);
                                const double s2 = static_cast<double>(p2);
                                const double num =
                                    RAW ? __dsub_rn(acc64[m], __dmul_rn(mean, s1))
                                        : __dadd_rn(acc64[m], __dmul_rn(cshift, sumd));
                                double den;
                                if (A.measure == AR_NCC) {
                                    den = __dmul_rn(cnorm, __dsqrt_rn(s2 > 0.0 ? s2 : 0.0));
                                } else {
                                    double wvar = __dsub_rn(s2, __ddiv_rn(__dmul_rn(s1, s1), nn));
                                    if (!(wvar > 0.0)) wvar = 0.0;
                                    den = __dmul_rn(cnorm, __dsqrt_rn(wvar));
                                }
                                const float sv = den > 0.0 ? __double2float_rn(__ddiv_rn(num, den)) : 0.0f;
                                s_cur[(ti + ir) + (tj + jl) * A.NRS] = sv;
                            }
                        }
                    }
                }
            }
            __syncthreads();
            if (A.flops && tid == 0)
                atomicAdd(A.flops, 2ull * static_cast<unsigned long long>(ch) * cw * nr * nc);

            // Integer peak (src/peak.jl:32-61), and the angle's maximum (src/track.jl:327-328).
            unsigned long long key = 0ull;
            for (int e = tid; e < nr * nc; e += bd) {
                const int i = e % nr, j = e / nr;
                const unsigned long long kk =
                    argmax_key(s_cur[i + j * A.NRS], static_cast<unsigned>(i * nc + j));
                key = kk > key ? kk : key;
            }
            key = block_max_u64(key, reinterpret_cast<unsigned long long*>(s_red));
            const float pk = key == 0ull ? NAN : key_value(key);
            if (!ROT || pk > bestpk) {
                bestpk = pk;
                best = key;
                float* t = s_best;
                s_best = s_cur;
                s_cur = t;
                found = true;
            }
        }
        if (!found) continue;  // every angle degenerate: searched, no measurement
        if (A.surf_out) {
            float* so = A.surf_out + k * static_cast<int64_t>(A.NRS) * A.NCM;
            for (int e = tid; e < nr * nc; e += bd) so[e] = s_best[(e % nr) + (e / nr) * A.NRS];
        }

        unsigned rm = 0;
        float pv = 0.0f;
        int pi = 0, pj = 0;
        if (key_decode(best, &rm, &pv)) {
            pi = static_cast<int>(rm / nc);
            pj = static_cast<int>(rm % nc);
        }
        if (A.up == 1 || nr < 5 || nc < 5) {
            // peak_offset (src/peak.jl:102-106) and the output write (src/track.jl:293-295).
            if (tid == 0) {
                const float v = s_best[pi + pj * A.NRS];
                A.out.dx[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pj - static_cast<int>(prx)), A.pts.dx0[k]));
                A.out.dy[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pi - static_cast<int>(pry)), A.pts.dy0[k]));
                A.out.corr[k] = v;
            }
        } else {
            // The clamped 5x5 patch of subpixel_peak (src/peak.jl:473-482), queued.
            const int pi0 = min(max(pi - 2, 0), max(nr - 5, 0));
            const int pj0 = min(max(pj - 2, 0), max(nc - 5, 0));
            if (tid == 0) s_slot = atomicAdd(A.sub_count, 1);
            __syncthreads();
            const int slot = s_slot;
            if (tid < 25) {
                const int a = tid % 5, b = tid / 5;
                A.sub_patch[static_cast<int64_t>(slot) * 25 + tid] =
                    s_best[(pi0 + a) + (pj0 + b) * A.NRS];
            }
            if (tid == 0) {
                A.sub_point[slot] = k;
                A.sub_origin[2 * slot] = pi0;
                A.sub_origin[2 * slot + 1] = pj0;
            }
        }
    }
}

// ----------------------------------------------------------------------------------------------
// Tensor-core correlation for UInt8 imagery (tcgen05.mma kind::i8, exact 32-bit accumulation).
//
// The numerator S[i, j] = sum_{a,b} C[a, b] W[i + a, j + b] (C the chip, W the window, i the
// surface row, j the surface column) is a sum of products D[j, i] += sum_k A[j, k] B[i, k] over
// K = (16-row block q of the window, chip column b, row r within the block):
//   A[j, (q, b, r)] = W'[16 q + r, j + b]     the window as 16-byte blocks s_W[q][x][r]; row j
//                                             of A starts 16 bytes after row j - 1, so A is
//                                             read in place;
//   B[i, (q, b, r)] = E_b[i - 16 q][r]        with E_b[u][r] = C[r - u - delta, b], the chip as
//                                             16-byte rows per column b, built once per point.
// W' starts at the 16-aligned image row `delta` rows above the window's first row, so each
// 16-byte block of a column-major image with 16-aligned columns is one aligned load. The chip
// rows a block q can meet are surface rows i in [16 q + 16 - NB, 16 q + 16), i.e. the same
// NB = 16 * ceil((ch + 30) / 16) rows u = i - 16 q of E for every q: each block's product
// (M = 64 surface columns, N = NB, K = 32: two chip columns) adds into accumulator columns
// [16 q, 16 q + NB), surface row i living in column i + NB - 16 of a cleared accumulator. The
// products are exact (u8 x u8 summed below 2^31), so the numerator equals the CUDA-core
// kernel's and every surface value, the peak and the patch are bit-identical to it.
//
// Normalising all 2ry x 2rx values in FP64 would cost as much as the products, and only the
// peak and its 5 x 5 patch are read. So each value is first estimated in FP32 together with a
// rigorous bound on its distance from the FP32 surface value; only values whose bound reaches
// the largest estimate, and the patch, get the reference's exact FP64 normalisation.

constexpr int kTcThreads = 256;
constexpr int kTc2Issuers = 3;  // k_corr_tc2: threads issuing a point's products
constexpr int kPadL = 32;            // zero bytes before each staged chip column
constexpr uint32_t kTcWaitPolls = 1u << 22;

struct TcArgs {
    const uint8_t* ref;
    const uint8_t* sec;
    const uint8_t* valid;
    int64_t nrows, ncols;
    DevPoints pts;
    int64_t padx, pady;
    int up, measure;
    int NB, QM, QS, PS, PC, XS, XT, NRS, NRM, NCM, CHM, CWM;
    int BC;                          // chip columns per chunk of the chip operand (even)
    int MT;                          // MMA M: 64 or 128 surface columns
    int big;                         // 1: box sums before the products, chunks reuse their space
    unsigned off_E, off_W, off_T, off_P, off_V, off_S1, off_S2, off_num, off_est, off_red;
    int XV;                          // k_corr_tc2: row stride (words) of the column sums V1, V2
    int acc1_col;                    // stride between the accumulators (first column of the
                                     // second one)
    int issuers;                     // k_corr_tc: threads issuing the products, 2 or 4
    uint32_t tmem_cols;
    DevOutputs out;
    int* sub_count;
    int64_t* sub_point;
    int32_t* sub_origin;
    float* sub_patch;
    float* surf_out;
    unsigned long long* flops;
    int* status;                     // set to 1 when a tensor-core wait ran out
};

// The reference's normalisation of one value from its exact integer numerator and box sums
// (the raw-numerator branch of k_corr).
__device__ __forceinline__ float tc_exact(uint32_t D, uint32_t S1, uint32_t S2, double mean,
                                          double nn, double cnorm, int measure) {
    const double s1 = static_cast<double>(S1), s2 = static_cast<double>(S2);
    const double num = __dsub_rn(static_cast<double>(D), __dmul_rn(mean, s1));
    double den;
    if (measure == AR_NCC) {
        den = __dmul_rn(cnorm, __dsqrt_rn(s2 > 0.0 ? s2 : 0.0));
    } else {
        double wvar = __dsub_rn(s2, __ddiv_rn(__dmul_rn(s1, s1), nn));
        if (!(wvar > 0.0)) wvar = 0.0;
        den = __dmul_rn(cnorm, __dsqrt_rn(wvar));
    }
    return den > 0.0 ? __double2float_rn(__ddiv_rn(num, den)) : 0.0f;
}

// FP32 estimate of one surface value and a bound on its distance from the value tc_exact
// returns. With nn, C = sum(chip), s1, s2, D exact integers, the value is
//   ZNCC: (nn D - C s1) / (cnorm sqrt(nn) sqrt(nn s2 - s1^2)),  NCC: (nn D - C s1) / (cnorm nn sqrt(s2)).
// D and s2 are converted with one rounding each (s1 < 2^24 and C are exact). The numerator and
// the variance are then formed with three roundings of relative size u = 2^-24 on terms no
// larger than `tn` and `tv`, so their absolute errors are below 3u tn and 3u tv; rsqrt (2 ulp),
// the scale `k` and two products add < 6u relative, and the final Float32 rounding of the
// reference 1u. 1/vx is taken as r^2 (within 9u of it). The bound returned covers all of it
// with more than 3x slack; NaN marks a value whose variance is too small for the bound
// (evaluated exactly). `k7` is 7u k.
__device__ __forceinline__ float tc_estimate(uint32_t D, uint32_t S1, uint32_t S2, float nnf,
                                             float csum, float k, float k7, int measure,
                                             float* bound) {
    const float d = __uint2float_rn(D), s1 = __uint2float_rn(S1), s2 = __uint2float_rn(S2);
    const float p = __fmul_rn(csum, s1);
    const float nx = __fmaf_rn(nnf, d, -p);
    const float tn = __fmaf_rn(nnf, d, p);  // |nn D| + |C s1| (both non-negative)
    float vx, tv;
    if (measure == AR_NCC) {
        vx = s2;
        tv = s2;
    } else {
        const float q = __fmul_rn(s1, s1);
        vx = __fmaf_rn(nnf, s2, -q);
        tv = __fmaf_rn(nnf, s2, q);
    }
    const float ev = 3.5762786865234375e-07f * tv;  // 6u tv
    if (!(vx > 64.0f * ev)) {
        *bound = 0.0f;
        return __int_as_float(0x7fc00000);
    }
    const float r = rsqrtf(vx);
    const float est = __fmul_rn(__fmul_rn(nx, r), k);
    // |err| <= |est| (8u + ev / vx) + 3.5u tn r k  (u = 2^-24), doubled for slack.
    const float rel = __fmaf_rn(ev, __fmul_rn(r, r), 9.5367431640625e-07f);  // 16u + ev/vx
    *bound = __fmaf_rn(fabsf(est), 2.0f * rel, __fmul_rn(__fmul_rn(tn, r), k7)) + 1e-30f;
    return est;
}

// tc_estimate for two values at once on packed FP32 pairs: every operation rounds each lane as
// the scalar form does, so the estimates and bounds are the scalar ones bit for bit.
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 tc_estimate2(uint32_t D0, uint32_t D1, uint32_t S10,
                                               uint32_t S11, uint32_t S20, uint32_t S21,
                                               float nnf, float csum, float k, float k7,
                                               int measure, float2* bound) {
    const float2 d = make_float2(__uint2float_rn(D0), __uint2float_rn(D1));
    const float2 s1 = make_float2(__uint2float_rn(S10), __uint2float_rn(S11));
    const float2 s2 = make_float2(__uint2float_rn(S20), __uint2float_rn(S21));
    const float2 nn2 = make_float2(nnf, nnf);
    const float2 p = __fmul2_rn(make_float2(csum, csum), s1);
    const float2 nx = __ffma2_rn(nn2, d, neg2(p));
    const float2 tn = __ffma2_rn(nn2, d, p);
    float2 vx, tv;
    if (measure == AR_NCC) {
        vx = s2;
        tv = s2;
    } else {
        const float2 q = __fmul2_rn(s1, s1);
        vx = __ffma2_rn(nn2, s2, neg2(q));
        tv = __ffma2_rn(nn2, s2, q);
    }
    const float2 ev = __fmul2_rn(make_float2(3.5762786865234375e-07f, 3.5762786865234375e-07f), tv);
    const float2 ev64 = __fmul2_rn(make_float2(64.0f, 64.0f), ev);
    const bool ok0 = vx.x > ev64.x, ok1 = vx.y > ev64.y;
    const float2 r = make_float2(rsqrtf(ok0 ? vx.x : 1.0f), rsqrtf(ok1 ? vx.y : 1.0f));
    const float2 est = __fmul2_rn(__fmul2_rn(nx, r), make_float2(k, k));
    const float2 rel = __ffma2_rn(ev, __fmul2_rn(r, r),
                                  make_float2(9.5367431640625e-07f, 9.5367431640625e-07f));
    const float2 b = __fadd2_rn(
        __ffma2_rn(make_float2(fabsf(est.x), fabsf(est.y)), __fmul2_rn(make_float2(2.0f, 2.0f), rel),
                   __fmul2_rn(__fmul2_rn(tn, r), make_float2(k7, k7))),
        make_float2(1e-30f, 1e-30f));
    const float qn = __int_as_float(0x7fc00000);
    *bound = make_float2(ok0 ? b.x : 0.0f, ok1 ? b.y : 0.0f);
    return make_float2(ok0 ? est.x : qn, ok1 ? est.y : qn);
}

// Rows of the chip operand that block q's product needs: operand row e holds offset
// u = e - NB + 16 (surface row i = 16 q + u), and only surface rows 0 <= i < nr are read, so
// e runs over [max(0, NB - 16 - 16 q), min(NB, NB - 16 + nr - 16 q)). Returned as a 16-aligned
// start `elo` and a multiple of 16 `n` (elo + n <= NB); false when the block reaches no
// surface row.
__device__ __forceinline__ bool block_rows(int q, int NB, int nr, int* elo, int* n) {
    const int lo = max(0, NB - 16 - 16 * q);
    const int hi = min(NB, NB - 16 + nr - 16 * q);
    if (hi <= lo) return false;
    *elo = lo & ~15;
    *n = (hi - *elo + 15) & ~15;
    return true;
}

// Sixteen bytes of column `c` from row r0 (zero outside the image), in two steps so that a
// thread can have several in flight: col16_issue starts the loads -- two aligned 16-byte loads
// when they stay inside the image, else byte by byte -- and col16_finish shifts the bytes into
// place.
struct Col16 {
    uint4 lo, hi;
    uint32_t s;  // byte offset of row r0 in `lo` (0: `lo` is the result)
};

__device__ __forceinline__ Col16 col16_issue(const uint8_t* img, const uint8_t* img_end,
                                             int64_t nrows, int64_t ncols, int64_t c, int64_t r0) {
    Col16 L;
    L.s = 0;
    L.lo = L.hi = make_uint4(0, 0, 0, 0);
    if (c < 0 || c >= ncols) return L;
    const uint8_t* p = img + c * nrows + r0;
    if (r0 >= 0 && r0 + 16 <= nrows) {
        const uintptr_t pa = reinterpret_cast<uintptr_t>(p);
        const uint32_t s = static_cast<uint32_t>(pa & 15);
        const uint4* a = reinterpret_cast<const uint4*>(pa - s);
        if (s == 0) {
            L.lo = __ldg(a);
            return L;
        }
        if (reinterpret_cast<const uint8_t*>(a) + 32 <= img_end) {
            L.lo = __ldg(a);
            L.hi = __ldg(a + 1);
            L.s = s;
            return L;
        }
    }
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int t = 0; t < 16; ++t) {
        const int64_t r = r0 + t;
        const uint32_t bb = (r >= 0 && r < nrows) ? p[t] : 0u;
        w[t >> 2] |= bb << (8 * (t & 3));
    }
    L.lo = make_uint4(w[0], w[1], w[2], w[3]);
    return L;
}

__device__ __forceinline__ uint4 col16_finish(const Col16& L) {
    const uint32_t s = L.s;
    if (s == 0) return L.lo;
    const uint32_t w[8] = {L.lo.x, L.lo.y, L.lo.z, L.lo.w, L.hi.x, L.hi.y, L.hi.z, L.hi.w};
    uint32_t u[6], v[5];
#pragma unroll
    for (int k = 0; k < 6; ++k) u[k] = (s & 8) ? w[k + 2] : w[k];
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = (s & 4) ? u[k + 1] : u[k];
    const uint32_t sh = (s & 3) * 8u;
    return make_uint4(__funnelshift_r(v[0], v[1], sh), __funnelshift_r(v[1], v[2], sh),
                      __funnelshift_r(v[2], v[3], sh), __funnelshift_r(v[3], v[4], sh));
}

// prepare_chip! statistics (src/correlate.jl:423-453) of a UInt8 chip staged as zero-padded
// byte columns (row a of column b at s_P[b * PC + kPadL + a]; rows outside the image are 0, as
// `pixel` reads them), with the CUDA-core kernel's FP64 results bit for bit: thread t takes
// elements t, t + bd, ... of the column-major chip (rows padded to a multiple of kUA) and the
// per-thread partial sums go through the same block sum.
//   One pass gives each thread the count m, sum P and sum of squares Q of its elements (exact
// integers; the sum of C is exact in any order). When the area nn is a power of two the mean
// S/nn is exact, so is every deviation d = N/nn (N = nn C - S) and its square, and a thread's
// FP64 running sum of squares is exactly K/nn^2 with K = sum N^2 = nn^2 Q - 2 nn S P + m S^2
// while K stays below 2^53 -- guaranteed when (its terms) x (255 nn)^2 is: then the partial is
// that integer scaled by 1/nn^2, the double the FP64 loop produces. Other areas take the FP64
// loop over the staged chip.
__device__ __forceinline__ void staged_chip_stats(const uint8_t* s_P, int PC, int ch, int cw, int tid,
                                                  int bd, double* s_red, double* csum, double* mean,
                                                  double* sq) {
    const int chp = (ch + kUA - 1) & ~(kUA - 1);
    const int ne = chp * cw;
    const int db = bd / chp, da = bd - db * chp;
    const int b0 = tid / chp, a0 = tid - b0 * chp;
    auto step = [&](int& a, int& b) {
        a += da;
        b += db;
        if (a >= chp) {
            a -= chp;
            ++b;
        }
    };
    uint32_t P = 0u, Q = 0u, m = 0u;
    {
        int a = a0, b = b0;
        for (int e = tid; e < ne; e += 4 * bd) {
            int o[4];
            bool in[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                in[u] = e + u * bd < ne && a < ch;
                o[u] = b * PC + kPadL + a;
                step(a, b);
            }
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = in[u] ? s_P[o[u]] : 0u;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                P += v[u];
                Q += v[u] * v[u];
                m += in[u] ? 1u : 0u;
            }
        }
    }
    double st[1] = {static_cast<double>(P)};
    block_sum_f64<1>(st, s_red);
    *csum = st[0];
    const int nn = ch * cw;
    const double mn = __ddiv_rn(st[0], static_cast<double>(nn));
    *mean = mn;
    const int terms = (ne + bd - 1) / bd;
    const double span = 255.0 * static_cast<double>(nn);
    const bool exact = (nn & (nn - 1)) == 0 && static_cast<double>(terms) * span * span < 9007199254740992.0;
    double acc2[1] = {0.0};
    if (exact) {
        const long long S = static_cast<long long>(st[0]), N2 = static_cast<long long>(nn);
        const long long K = N2 * N2 * static_cast<long long>(Q) - 2 * N2 * S * static_cast<long long>(P) +
                            static_cast<long long>(m) * S * S;
        const double inv = 1.0 / (static_cast<double>(nn) * static_cast<double>(nn));  // 2^-2k
        acc2[0] = static_cast<double>(K) * inv;
    } else {
        int a = a0, b = b0;
        for (int e = tid; e < ne; e += bd) {
            if (a < ch) {
                const double d = __dsub_rn(static_cast<double>(s_P[b * PC + kPadL + a]), mn);
                acc2[0] = __dadd_rn(acc2[0], __dmul_rn(d, d));
            }
            step(a, b);
        }
    }
    block_sum_f64<1>(acc2, s_red);
    *sq = acc2[0];
}

// Optional phase timer (compiled in with -DAR_TC_PHASES, for profiling builds only): thread 0
// of each CTA accumulates clock64() cycles between the marks below, per phase, and adds them to
// g_tc_phase at exit; entry 15 counts the points that reached the output phase.
#ifdef AR_TC_PHASES
__device__ unsigned long long g_tc_phase[16];
#define TC_PHASE_INIT unsigned long long tcp_t = clock64(), tcp_acc[12] = {}, tcp_n = 0;
#define TC_PHASE(n)                              \
    if (tid == 0) {                              \
        const unsigned long long t_ = clock64(); \
        tcp_acc[n] += t_ - tcp_t;                \
        tcp_t = t_;                              \
    }
#define TC_PHASE_POINT \
    if (tid == 0) ++tcp_n;
#define TC_PHASE_FLUSH                                                           \
    if (tid == 0) {                                                              \
        for (int n_ = 0; n_ < 12; ++n_) atomicAdd(&g_tc_phase[n_], tcp_acc[n_]); \
        atomicAdd(&g_tc_phase[15], tcp_n);                                       \
    }
#else
#define TC_PHASE_INIT
#define TC_PHASE(n)
#define TC_PHASE_POINT
#define TC_PHASE_FLUSH
#endif

// REG: every surface of the pass has at most 64 rows and 64 columns (M = 64), so one 16x256b
// read per warp covers it and each thread keeps its 16 numerators and upper bounds in
// registers through both passes. Otherwise the numerators go to shared memory and both passes
// run over the surface in flattened order, four values per thread and step, so that every warp
// has work even when the surface's columns fill only two or three of the M = 128 accumulator's
// lane quarters.
template <bool REG>
__global__ void __launch_bounds__(kTcThreads, 2) k_corr_tc(const TcArgs A) {
    extern __shared__ __align__(1024) unsigned char smem_tc[];
    __shared__ uint64_t s_mbar;
    __shared__ uint32_t s_taddr;
    __shared__ int s_slot;
    __shared__ int s_ncand;
    __shared__ uint32_t s_pd[25];
    __shared__ float s_fmax[kTcThreads / 32];
    __shared__ unsigned long long s_isum[2][2];
    uint8_t* s_E = smem_tc + A.off_E;
    uint8_t* s_W = smem_tc + A.off_W;
    uint8_t* s_T = smem_tc + A.off_T;
    uint8_t* s_P = smem_tc + A.off_P;
    uint32_t* s_V1 = reinterpret_cast<uint32_t*>(smem_tc + A.off_V);
    uint32_t* s_S1 = reinterpret_cast<uint32_t*>(smem_tc + A.off_S1);
    uint32_t* s_S2 = reinterpret_cast<uint32_t*>(smem_tc + A.off_S2);
    uint32_t* s_num = reinterpret_cast<uint32_t*>(smem_tc + A.off_num);
    float* s_est = reinterpret_cast<float*>(smem_tc + A.off_est);
    double* s_red = reinterpret_cast<double*>(smem_tc + A.off_red);

    const int tid = threadIdx.x, bd = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = bd >> 5;
    // Threads issuing the products (only plans of the register epilogue take four).
    const int NI = REG ? A.issuers : 2;
    const int64_t NR = A.nrows + 2 * A.pady, NC = A.ncols + 2 * A.padx;
    const double shx = static_cast<double>(A.padx) + 0.5;
    const double shy = static_cast<double>(A.pady) + 0.5;
    const uint8_t* ref_end = A.ref + A.nrows * A.ncols;
    const uint8_t* sec_end = A.sec + A.nrows * A.ncols;
    const uint8_t* valid_end = A.valid + A.nrows * A.ncols;

    if (warp == 0) {
        tc::tmem_alloc(&s_taddr, A.tmem_cols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&s_mbar, NI);  // one commit per issuing thread
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = s_taddr;
    const uint32_t acc1 = static_cast<uint32_t>(A.acc1_col);  // second accumulator's first column
    uint32_t phase = 0;
    bool failed = false;
    if (tid < 4) s_isum[tid >> 1][tid & 1] = 0ull;
    for (int e = tid; e < A.CWM * A.PC; e += bd) s_P[e] = 0;
    int iter = 0;
    int dirty_ch = 0;
    TC_PHASE_INIT

    // Each CTA takes a contiguous run of points: consecutive points of a grid column have the
    // same window columns one grid step lower, so most of their box sums carry over. s_S1 / s_S2
    // are rings of NRS rows per column: surface row i of the held point is stored at row
    // (i + rbase) mod NRS, and carrying the sums down by `sh` rows advances rbase.
    const int64_t per = (A.pts.n + gridDim.x - 1) / gridDim.x;
    const int64_t kbeg = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t kend = min(A.pts.n, kbeg + per);
    bool held = false;  // s_S1 / s_S2 hold the sums of the geometry h_*
    int64_t h_wr = 0, h_wc = 0;
    int h_ch = 0, h_cw = 0, h_nr = 0, h_nc = 0;
    int rbase = 0;
    auto ring = [&](int i) {
        const int r = i + rbase;
        return r >= A.NRS ? r - A.NRS : r;
    };

    for (int64_t k = kbeg; k < kend; ++k, ++iter) {
        tc::fence_before_sync();
        __syncthreads();  // the previous point's buffers and accumulator are no longer read
        tc::fence_after_sync();
        TC_PHASE(0)
        // The chip sums of this iteration go to s_isum[ib]; the other buffer, last read
        // before the barrier above, is cleared for the next iteration.
        const int ib = iter & 1;
        if (tid < 2) s_isum[ib ^ 1][tid] = 0ull;
        const int64_t prx = A.pts.rx[k], pry = A.pts.ry[k];
        if (!(prx > 0 && pry > 0)) continue;
        const double xs = A.pts.x[k] + shx, ys = A.pts.y[k] + shy;
        const int64_t hx = A.pts.csx[k] / 2, hy = A.pts.csy[k] / 2;
        const int64_t ccx = static_cast<int64_t>(floor(__dsub_rn(xs, A.pts.dx0[k])));
        const int64_t ccy = static_cast<int64_t>(floor(__dsub_rn(ys, A.pts.dy0[k])));
        const int64_t wcx = static_cast<int64_t>(floor(xs)), wcy = static_cast<int64_t>(floor(ys));
        const int64_t cr0 = ccy - hy, cr1 = ccy + hy - 1, cc0 = ccx - hx, cc1 = ccx + hx - 1;
        const int64_t wr0 = wcy - hy - pry, wr1 = wcy + hy + pry - 2;
        const int64_t wc0 = wcx - hx - prx, wc1 = wcx + hx + prx - 2;
        const bool chip_in = (cr1 < cr0 || cc1 < cc0) ||
                             (cr0 >= 1 && cr1 <= NR && cc0 >= 1 && cc1 <= NC);
        const bool win_in = (wr1 < wr0 || wc1 < wc0) ||
                            (wr0 >= 1 && wr1 <= NR && wc0 >= 1 && wc1 <= NC);
        if (!chip_in || !win_in) continue;
        const int ch = static_cast<int>(2 * hy), cw = static_cast<int>(2 * hx);
        const int nr = static_cast<int>(2 * pry), nc = static_cast<int>(2 * prx);
        if (ch <= 0 || cw <= 0) continue;
        if (ch > A.CHM || cw > A.CWM || nr > A.NRM || nc > A.NCM || nc > A.MT) continue;
        TC_PHASE(1)
        const int64_t chip_r = cr0 - 1 - A.pady, chip_c = cc0 - 1 - A.padx;
        const int64_t win_r = wr0 - 1 - A.pady, win_c = wc0 - 1 - A.padx;
        const long long nnl = static_cast<long long>(ch) * cw;
        // Power-of-two areas up to 4096: every term of the reference's FP64 chip sums is exact.
        const bool pow2 = (nnl & (nnl - 1)) == 0 && nnl <= 4096;

        // The chip as zero-padded byte columns, _any_valid over it (src/track.jl:416-421) and,
        // for power-of-two areas, its exact integer sums: warps over chip columns, lanes over
        // rows, all loads of a lane issued before their uses. Rows a taller chip left behind
        // are cleared (the padding itself is never written).
        // Invariant: chip rows at or beyond `dirty_ch` are zero in every column.
        if (ch < dirty_ch)
            for (int b = warp; b < A.CWM; b += nwarps)
                for (int a = ch + lane; a < dirty_ch; a += 32) s_P[b * A.PC + kPadL + a] = 0;
        dirty_ch = ch;
        // A task is 16 rows of one chip column: a 16-byte block of the image and of its mask
        // (col16_issue: aligned loads and a byte shift, zero outside the image), rows beyond ch
        // zeroed. Each thread starts the loads of two tasks before using them.
        int any = 0;
        unsigned long long isum = 0ull, isq = 0ull;
        {
            const int nb16 = (ch + 15) >> 4, ntask = nb16 * cw;
            uint32_t s1 = 0u, s2 = 0u;
            for (int t0 = tid; t0 < ntask; t0 += 2 * bd) {
                Col16 Lv[2], Lm[2];
                int tb[2], tj[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int t = t0 + u * bd;
                    tb[u] = t / nb16;
                    tj[u] = t - tb[u] * nb16;
                    const int64_t c = t < ntask ? chip_c + tb[u] : -1;
                    Lv[u] = col16_issue(A.sec, sec_end, A.nrows, A.ncols, c, chip_r + 16 * tj[u]);
                    Lm[u] = col16_issue(A.valid, valid_end, A.nrows, A.ncols, c, chip_r + 16 * tj[u]);
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (t0 + u * bd >= ntask) continue;
                    const uint4 v = col16_finish(Lv[u]), mk = col16_finish(Lm[u]);
                    const int keep = ch - 16 * tj[u];
                    uint32_t w[4] = {v.x, v.y, v.z, v.w}, mw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int kb = keep - 4 * i;
                        const uint32_t m = kb >= 4 ? 0xffffffffu : kb <= 0 ? 0u : (1u << (8 * kb)) - 1u;
                        w[i] &= m;
                        any |= (mw[i] & m) != 0u;
                        s1 = __dp4a(w[i], 0x01010101u, s1);
                        s2 = __dp4a(w[i], w[i], s2);
                    }
                    *reinterpret_cast<uint4*>(s_P + tb[u] * A.PC + kPadL + 16 * tj[u]) =
                        make_uint4(w[0], w[1], w[2], w[3]);
                }
            }
            isum = s1;
            isq = s2;
        }
        if (pow2) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                isum += __shfl_xor_sync(kFull, isum, o);
                isq += __shfl_xor_sync(kFull, isq, o);
            }
            if (lane == 0) {
                atomicAdd(&s_isum[ib][0], isum);
                atomicAdd(&s_isum[ib][1], isq);
            }
        }
        if (!__syncthreads_or(any)) continue;
        TC_PHASE(2)
        if (tid == 0) A.out.searched[k] = 1;

        // prepare_chip! statistics. Power-of-two areas: every term of the reference's FP64
        // sums is exact, so mean = sum/nn and sq = (nn sum(C^2) - sum(C)^2)/nn exactly;
        // otherwise the CUDA-core kernel's FP64 loops, in its order (bit-identical sums).
        double mean, sq, csum_d;
        if (pow2) {
            const long long cs = static_cast<long long>(s_isum[ib][0]);
            const long long c2 = static_cast<long long>(s_isum[ib][1]);
            csum_d = static_cast<double>(cs);
            mean = __ddiv_rn(csum_d, static_cast<double>(nnl));
            sq = __ddiv_rn(static_cast<double>(nnl * c2 - cs * cs), static_cast<double>(nnl));
        } else {
            staged_chip_stats(s_P, A.PC, ch, cw, tid, bd, s_red, &csum_d, &mean, &sq);
        }
        if (!(sq > __dmul_rn(__dmul_rn(DBL_EPSILON, static_cast<double>(ch)), static_cast<double>(cw))))
            continue;  // degenerate chip: searched, no measurement (src/track.jl:286)
        TC_PHASE(3)
        const double cnorm = __dsqrt_rn(sq);
        // The point is measured: its refinement slot is taken now, read after later barriers.
        if (tid == 0 && !(A.up == 1 || nr < 5 || nc < 5)) s_slot = atomicAdd(A.sub_count, 1);
        const double nn = static_cast<double>(nnl);

        // Box sums carried from the held point: same window columns and shape, `sh` rows
        // higher; only surface rows iA .. nr - 1 are computed (iA = 0: all of them).
        const int64_t sh64 = win_r - h_wr;
        const bool carry = held && win_c == h_wc && ch == h_ch && cw == h_cw && nr == h_nr &&
                           nc == h_nc && sh64 > 0 && sh64 < nr;
        int iA = 0;
        if (carry) {
            iA = nr - static_cast<int>(sh64);
            rbase += static_cast<int>(sh64);
            if (rbase >= A.NRS) rbase -= A.NRS;
        } else {
            rbase = 0;
        }
        held = true;
        h_wr = win_r;
        h_wc = win_c;
        h_ch = ch;
        h_cw = cw;
        h_nr = nr;
        h_nc = nc;
#ifdef AR_TC_PHASES
        if (tid == 0 && carry) atomicAdd(&g_tc_phase[14], 1ull);
#endif

        // Window blocks W'[16 q + r][x] (x < XS) from 16 image rows at base_r + 16 q, and the
        // same window transposed, s_T[row][x], for the box sums (the blocks from the one that
        // holds window row iA: the rows the box sums read).
        const int64_t delta = ((win_r % 16) + 16) % 16;
        const int64_t base_r = win_r - delta;
        const int Q = static_cast<int>((delta + ch + nr - 1 + 15) / 16);
        const int XW = cw + nc - 1;
        const int qT = static_cast<int>((delta + iA) >> 4);
        // A block is one aligned 16-byte load when the image's columns are 16-byte aligned (row
        // counts divisible by 16), otherwise two aligned loads and a byte shift.
        // A task is block q of column x (consecutive threads on consecutive columns); each thread
        // starts the loads of three tasks before using them.
        {
            const int ntask = Q * A.XS;
            for (int t0 = tid; t0 < ntask; t0 += 3 * bd) {
                Col16 L[3];
                int tq[3], tx[3];
#pragma unroll
                for (int u = 0; u < 3; ++u) {
                    const int t = t0 + u * bd;
                    tq[u] = t / A.XS;
                    tx[u] = t - tq[u] * A.XS;
                    const int64_t c = t < ntask ? win_c + tx[u] : -1;
                    L[u] = col16_issue(A.ref, ref_end, A.nrows, A.ncols, c, base_r + 16 * tq[u]);
                }
#pragma unroll
                for (int u = 0; u < 3; ++u) {
                    if (t0 + u * bd >= ntask) continue;
                    const int q = tq[u], x = tx[u];
                    const uint4 v = col16_finish(L[u]);
                    *reinterpret_cast<uint4*>(s_W + q * A.QS + x * 16) = v;
                    if (x < XW && q >= qT) {
                        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                        for (int t = 0; t < 16; ++t)
                            s_T[(16 * q + t) * A.XT + x] = static_cast<uint8_t>(w[t >> 2] >> (8 * (t & 3)));
                    }
                }
            }
        }
        __syncthreads();  // s_P, s_W, s_T complete
        TC_PHASE(4)

        // Box sums of W and W^2 (integral_both!, boxsum, src/integral.jl:141-170, 244-247) as
        // exact integers: V[i][x] sums ch rows down column x, S[j][i] sums cw columns of V.
        // They run while the tensor core works on the first chunk, or, when the chip operand
        // comes in several chunks that reuse their space, before it. Only surface rows
        // iA .. nr - 1 are computed (the others carried over), into ring rows.
        // Threads 0 .. kBT - 1 (named barrier 1): the warps below the issuing ones.
        auto box_sums = [&](const int kBT) {
            uint32_t* s_V2 = s_V1 + A.NRM * XW;
            const int nrw = nr - iA;
            // V: one round of tasks (column x, a run of rows), each an unrolled first sum with
            // independent partials and a sliding update with the next values loaded ahead.
            const int nseg = max(1, min((nrw + 7) / 8, kBT / XW));
            const int seglen = (nrw + nseg - 1) / nseg;
            for (int task = tid; task < XW * nseg; task += kBT) {
                const int x = task % XW, seg = task / XW;
                const int i0 = iA + seg * seglen, i1 = min(i0 + seglen, nr);
                if (i0 >= i1) continue;
                const uint8_t* col = s_T + static_cast<int>(delta) * A.XT + x;
                uint32_t p1[4] = {0, 0, 0, 0}, p2[4] = {0, 0, 0, 0};
                int a = 0;
                for (; a + 4 <= ch; a += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t w = col[(i0 + a + u) * A.XT];
                        p1[u] += w;
                        p2[u] += w * w;
                    }
                }
                for (; a < ch; ++a) {
                    const uint32_t w = col[(i0 + a) * A.XT];
                    p1[0] += w;
                    p2[0] += w * w;
                }
                uint32_t h1 = (p1[0] + p1[1]) + (p1[2] + p1[3]);
                uint32_t h2 = (p2[0] + p2[1]) + (p2[2] + p2[3]);
                uint32_t wo = col[i0 * A.XT], wn = col[(i0 + ch) * A.XT];
                for (int i = i0; i < i1; ++i) {
                    s_V1[i * XW + x] = h1;
                    s_V2[i * XW + x] = h2;
                    if (i + 1 < i1) {
                        const uint32_t wo2 = col[(i + 1) * A.XT], wn2 = col[(i + 1 + ch) * A.XT];
                        h1 = h1 + wn - wo;
                        h2 = h2 + wn * wn - wo * wo;
                        wo = wo2;
                        wn = wn2;
                    }
                }
            }
            asm volatile("bar.sync 1, %0;" ::"r"(kBT) : "memory");
            // S: tasks (surface row i, a run of 16 columns), the same pattern along V's rows.
            const int jseg = (nc + 15) >> 4;
            for (int task = tid; task < nrw * jseg; task += kBT) {
                const int i = iA + task % nrw, seg = task / nrw;
                const int ri = ring(i);
                const int j0 = seg << 4, j1 = min(j0 + 16, nc);
                const uint32_t* v1 = s_V1 + i * XW;
                const uint32_t* v2 = s_V2 + i * XW;
                uint32_t q1[4] = {0, 0, 0, 0}, q2[4] = {0, 0, 0, 0};
                int b = 0;
                for (; b + 4 <= cw; b += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        q1[u] += v1[j0 + b + u];
                        q2[u] += v2[j0 + b + u];
                    }
                }
                for (; b < cw; ++b) {
                    q1[0] += v1[j0 + b];
                    q2[0] += v2[j0 + b];
                }
                uint32_t g1 = (q1[0] + q1[1]) + (q1[2] + q1[3]);
                uint32_t g2 = (q2[0] + q2[1]) + (q2[2] + q2[3]);
                for (int j = j0; j < j1; ++j) {
                    s_S1[j * A.NRS + ri] = g1;
                    s_S2[j * A.NRS + ri] = g2;
                    if (j + 1 < j1) {
                        g1 = g1 + v1[j + cw] - v1[j];
                        g2 = g2 + v2[j + cw] - v2[j];
                    }
                }
            }
        };
        if (A.big) {
            if (warp < nwarps - NI) box_sums(kTcThreads - 32 * NI);
            __syncthreads();  // the chip chunks overwrite s_T and s_V
        }

        const int nchunk = (cw + A.BC - 1) / A.BC;
        bool ok = true;
        for (int cc = 0; cc < nchunk; ++cc) {
            const int b0 = cc * A.BC, b1 = min(cw, b0 + A.BC);
            if (cc > 0) {
                // The previous chunk's products must be done before its rows are replaced.
                ok = tc::mbar_wait(&s_mbar, phase, kTcWaitPolls);
                phase ^= 1u;
                if (__syncthreads_or(!ok)) break;
                tc::fence_after_sync();
            }
            // E: NB rows u = 16 - NB ... 15 per chip column, row u at e = u - 16 + NB: 16 bytes
            // from chip row -u - delta. Consecutive threads take consecutive rows.
            {
                const int nrow = (b1 - b0) * A.NB;
                int bl = tid / A.NB, e = tid - bl * A.NB;
                const int sbl = bd / A.NB, se = bd - sbl * A.NB;
                for (int t = tid; t < nrow; t += bd) {
                    const int src = (b0 + bl) * A.PC + kPadL - 16 + A.NB - static_cast<int>(delta) - e;
                    const uint32_t* w = reinterpret_cast<const uint32_t*>(s_P + (src & ~3));
                    const uint32_t sh = static_cast<uint32_t>(src & 3) * 8u;
                    uint4 o;
                    o.x = __funnelshift_r(w[0], w[1], sh);
                    o.y = __funnelshift_r(w[1], w[2], sh);
                    o.z = __funnelshift_r(w[2], w[3], sh);
                    o.w = __funnelshift_r(w[3], w[4], sh);
                    *reinterpret_cast<uint4*>(s_E + bl * A.PS + e * 16) = o;
                    bl += sbl;
                    e += se;
                    if (e >= A.NB) {
                        e -= A.NB;
                        ++bl;
                    }
                }
            }
            if (cc == 0 && warp < 4) {
                // Clear the accumulator columns the products add into (one lane quarter each).
                uint32_t z[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) z[t] = 0u;
                // Products land in columns [NB - 16, NB + nr) of block coordinates (their rows are
                // trimmed to the surface rows), stored from column 0 of each accumulator.
                const int zc = (nr + 16 + 15) & ~15;
                const uint32_t lq = taddr + (static_cast<uint32_t>(32 * warp) << 16);
                for (int s = 0; s < NI; ++s)
                    for (int c = 0; c < zc; c += 16)
                        tc::tmem_st16(lq + static_cast<uint32_t>(s) * acc1 + static_cast<uint32_t>(c), z);
                tc::tmem_wait_st();
            }
            tc::fence_proxy_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            TC_PHASE(5)
            // Lane 0 of each of the last NI warps issues the products of a share of the
            // chunk's chip column pairs into its own accumulator (one thread's MMAs run one after
            // another, so the products of one point are spread over two or four threads).
            if (REG ? (lane == 0 && warp >= nwarps - NI)
                    : (tid == kTcThreads - 32 || tid == kTcThreads - 64)) {
                const int stream = REG ? nwarps - 1 - warp : (tid == kTcThreads - 32 ? 0 : 1);
                tc::fence_after_sync();
                const uint32_t sW = tc::smem_u32(s_W), sE = tc::smem_u32(s_E);
                const int p0 = b0 / 2, p1 = b1 / 2;
                const int tb = p0 + (p1 - p0) * stream / NI;
                const int te = p0 + (p1 - p0) * (stream + 1) / NI;
                const uint32_t dacc = taddr + static_cast<uint32_t>(stream) * acc1;
                for (int q = 0; q < Q; ++q) {
                    // Only the operand rows e in [elo, elo + n) of block q reach surface rows;
                    // their accumulator columns start at NB - 16 in block coordinates.
                    int elo, n;
                    if (!block_rows(q, A.NB, nr, &elo, &n)) continue;
                    const uint32_t idesc = tc::idesc_u8_s32(A.MT, n);
                    const uint32_t dcol = static_cast<uint32_t>(16 * q + elo - (A.NB - 16));
                    for (int t = tb; t < te; ++t) {
                        const uint64_t da = tc::smem_desc(sW + q * A.QS + 32 * t, 16, 128);
                        const uint64_t db =
                            tc::smem_desc(sE + (2 * t - b0) * A.PS + 16 * elo, A.PS, 128);
                        tc::mma_u8(dacc + dcol, da, db, idesc, true);
                    }
                }
                tc::mma_commit(&s_mbar);
            }
            if (cc == 0 && !A.big && warp < nwarps - NI) box_sums(kTcThreads - 32 * NI);
            TC_PHASE(6)
        }
        if (ok) {
            // Wait for the last chunk's products (bounded; every thread polls the same phase).
            ok = tc::mbar_wait(&s_mbar, phase, kTcWaitPolls);
            phase ^= 1u;
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(A.status, 1);
            failed = true;
            break;
        }
        tc::fence_after_sync();
        TC_PHASE(7)

        // Pass 1: numerators out of Tensor Memory, estimates and bounds, the largest lower bound.
        // Surface column j is accumulator row j (lane (j % 16) + 32 (j / 16) of the M = 64
        // layout); surface row i is column i of each accumulator (their sum). Warp w reads its quarter's
        // 16 lanes (16x256b: thread t gets rows 16 q + t/4 and + 8, columns 2 (t % 4) + {0, 1}
        // + 8 k), columns from 32 (w / 4) in steps of 64.
        const float kk = __double2float_rn(
            A.measure == AR_NCC ? __drcp_rn(__dmul_rn(cnorm, nn))
                                : __drcp_rn(__dmul_rn(cnorm, __dsqrt_rn(nn))));
        const float kk7 = 4.172325134277344e-07f * kk;  // 7u k
        const float nnf = static_cast<float>(nnl);
        const float csf = static_cast<float>(csum_d);
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t col0 = 0u;
        float lmax = -INFINITY;
        if constexpr (REG) {
            // One read per warp: value v of this thread is surface row
            // i = 32 half + 8 (v / 4) + 2 (lane % 4) + v % 2, column j = 16 quarter + lane / 4
            // (+ 8 when v % 4 >= 2). Registers keep its numerator and its upper bound.
            const int ib0 = 32 * half + 2 * (lane & 3);
            const int jb0 = 16 * quarter + (lane >> 2);
            uint32_t dv[16];
            float upb[16];
            uint32_t vm = 0u;  // values of this thread inside the surface
            if (32 * half < nr) {
                const uint32_t base = taddr + (static_cast<uint32_t>(32 * quarter) << 16) + col0 +
                                      static_cast<uint32_t>(32 * half);
                uint32_t dv1[16];
                tc::tmem_ld16dp(base, dv);
                tc::tmem_ld16dp(base + acc1, dv1);
                tc::tmem_wait_ld();
#pragma unroll
                for (int v = 0; v < 16; ++v) dv[v] += dv1[v];
                for (int s = 2; s < NI; ++s) {
                    tc::tmem_ld16dp(base + static_cast<uint32_t>(s) * acc1, dv1);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int v = 0; v < 16; ++v) dv[v] += dv1[v];
                }
#pragma unroll
                for (int v = 0; v < 16; ++v) {
                    const int i = ib0 + 8 * (v >> 2) + (v & 1), j = jb0 + ((v & 2) ? 8 : 0);
                    upb[v] = -INFINITY;
                    if (i < nr && j < nc) {
                        vm |= 1u << v;
                        const int o = j * A.NRS + ring(i);
                        float bnd;
                        const float est = tc_estimate(dv[v], s_S1[o], s_S2[o], nnf, csf, kk, kk7,
                                                      A.measure, &bnd);
                        upb[v] = est + bnd;
                        lmax = fmaxf(lmax, est - bnd);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(kFull, lmax, o));
            if (lane == 0) s_fmax[warp] = lmax;
            if (tid == 0) s_ncand = 0;
            __syncthreads();
            TC_PHASE(8)
            float M = s_fmax[0];
            for (int w = 1; w < kTcThreads / 32; ++w) M = fmaxf(M, s_fmax[w]);
            // Pass 2: values whose upper bound reaches M (or whose estimate was not made) go to a
            // list -- numerator and (row, column) -- and are normalised exactly, one per thread.
            uint32_t* s_cD = s_num;
            uint32_t* s_cI = reinterpret_cast<uint32_t*>(s_est);
#pragma unroll
            for (int v = 0; v < 16; ++v) {
                if (((vm >> v) & 1u) && (upb[v] >= M || isnan(upb[v]))) {
                    const int c = atomicAdd(&s_ncand, 1);
                    s_cD[c] = dv[v];
                    s_cI[c] = (static_cast<uint32_t>(ib0 + 8 * (v >> 2) + (v & 1)) << 16) |
                              static_cast<uint32_t>(jb0 + ((v & 2) ? 8 : 0));
                }
            }
            __syncthreads();
            const int ncand = s_ncand;
            unsigned long long best = 0ull;
            for (int c = tid; c < ncand; c += bd) {
                const int i = static_cast<int>(s_cI[c] >> 16), j = static_cast<int>(s_cI[c] & 0xFFFFu);
                const int o = j * A.NRS + ring(i);
                const float x = tc_exact(s_cD[c], s_S1[o], s_S2[o], mean, nn, cnorm, A.measure);
                const unsigned long long key = argmax_key(x, static_cast<unsigned>(i * nc + j));
                best = key > best ? key : best;
            }
            best = block_max_u64(best, reinterpret_cast<unsigned long long*>(s_red));
            TC_PHASE(9)
            if (A.flops && tid == 0)
                atomicAdd(A.flops, 2ull * static_cast<unsigned long long>(ch) * cw * nr * nc);
            if (A.surf_out) {
                // Every value exactly (diagnostic surfaces): numerators to shared memory first.
#pragma unroll
                for (int v = 0; v < 16; ++v)
                    if ((vm >> v) & 1u)
                        s_num[(jb0 + ((v & 2) ? 8 : 0)) * A.NRS + ib0 + 8 * (v >> 2) + (v & 1)] = dv[v];
                __syncthreads();
                float* so = A.surf_out + k * static_cast<int64_t>(A.NRM) * A.NCM;
                for (int e = tid; e < nr * nc; e += bd) {
                    const int o = (e / nr) * A.NRS + (e % nr);
                    const int os = (e / nr) * A.NRS + ring(e % nr);
                    so[e] = tc_exact(s_num[o], s_S1[os], s_S2[os], mean, nn, cnorm, A.measure);
                }
            }
            unsigned rm = 0;
            float pv = 0.0f;
            int pi = 0, pj = 0;
            if (key_decode(best, &rm, &pv)) {
                pi = static_cast<int>(rm / nc);
                pj = static_cast<int>(rm % nc);
            }
            const bool single = A.up == 1 || nr < 5 || nc < 5;
            // The numerators of the output: the peak, or the 5 x 5 patch (all inside the surface).
            const int pi0 = single ? pi : min(max(pi - 2, 0), max(nr - 5, 0));
            const int pj0 = single ? pj : min(max(pj - 2, 0), max(nc - 5, 0));
            const int span = single ? 1 : 5;
#pragma unroll
            for (int v = 0; v < 16; ++v) {
                const int a = ib0 + 8 * (v >> 2) + (v & 1) - pi0, b = jb0 + ((v & 2) ? 8 : 0) - pj0;
                if (a >= 0 && a < span && b >= 0 && b < span && ((vm >> v) & 1u)) s_pd[b * 5 + a] = dv[v];
            }
            __syncthreads();
            if (single) {
                if (tid == 0) {
                    const int o = pj * A.NRS + ring(pi);
                    A.out.dx[k] = __double2float_rn(
                        __dadd_rn(static_cast<double>(pj - static_cast<int>(prx)), A.pts.dx0[k]));
                    A.out.dy[k] = __double2float_rn(
                        __dadd_rn(static_cast<double>(pi - static_cast<int>(pry)), A.pts.dy0[k]));
                    A.out.corr[k] = tc_exact(s_pd[0], s_S1[o], s_S2[o], mean, nn, cnorm, A.measure);
                }
            } else {
                const int slot = s_slot;
                if (tid < 25) {
                    const int a = tid % 5, b = tid / 5;
                    const int o = (pj0 + b) * A.NRS + ring(pi0 + a);
                    A.sub_patch[static_cast<int64_t>(slot) * 25 + tid] =
                        tc_exact(s_pd[tid], s_S1[o], s_S2[o], mean, nn, cnorm, A.measure);
                }
                if (tid == 0) {
                    A.sub_point[slot] = k;
                    A.sub_origin[2 * slot] = pi0;
                    A.sub_origin[2 * slot + 1] = pj0;
                }
            }
            TC_PHASE(10)
            TC_PHASE_POINT
            continue;
        }
        // The surface's values in flattened order e = i + nr j: thread t starts at e = t and
        // steps by kTcThreads (row and column advanced without a division).
        const int ne = nr * nc;
        const int fj0 = tid / nr, fi0 = tid - fj0 * nr;
        const int fdj = kTcThreads / nr, fdi = kTcThreads - fdj * nr;
        auto fstep = [&](int& i, int& j) {
            i += fdi;
            j += fdj;
            if (i >= nr) {
                i -= nr;
                ++j;
            }
        };
        auto take = [&](uint32_t d, int i, int j) {
            if (j < nc && i < nr) {
                const int o = j * A.NRS + i;
                const int os = j * A.NRS + ring(i);
                float bnd;
                const float est = tc_estimate(d, s_S1[os], s_S2[os], nnf, csf, kk, kk7, A.measure, &bnd);
                s_num[o] = d;
                s_est[o] = est;
                s_est[o + A.NCM * A.NRS] = bnd;
                lmax = fmaxf(lmax, est - bnd);
            }
        };
        if (A.MT == 64) {
            for (int i0 = 32 * half; i0 < nr; i0 += 64) {
                uint32_t r[16], r1[16];
                const uint32_t base = taddr + (static_cast<uint32_t>(32 * quarter) << 16) + col0 +
                                      static_cast<uint32_t>(i0);
                tc::tmem_ld16dp(base, r);
                tc::tmem_ld16dp(base + acc1, r1);
                tc::tmem_wait_ld();
#pragma unroll
                for (int v = 0; v < 16; ++v) r[v] += r1[v];
                for (int s = 2; s < NI; ++s) {
                    tc::tmem_ld16dp(base + static_cast<uint32_t>(s) * acc1, r1);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int v = 0; v < 16; ++v) r[v] += r1[v];
                }
#pragma unroll
                for (int v = 0; v < 16; ++v)
                    take(r[v], i0 + 8 * (v >> 2) + 2 * (lane & 3) + (v & 1),
                         16 * quarter + (lane >> 2) + ((v & 2) ? 8 : 0));
            }
        } else {
            // M = 128: accumulator row j is lane j; thread = row 32 q + lane, 16 columns. Only
            // the lane quarters below nc hold surface columns (for nc <= 96, two or three of
            // the four), so their warps move the numerators to shared memory and the estimates
            // are spread over all warps: warp w takes columns w, w + 8, ..., lanes the rows.
            if (32 * quarter < nc) {
                const int j = 32 * quarter + lane;
                for (int i0 = 16 * half; i0 < nr; i0 += 32) {
                    uint32_t r[16], r1[16];
                    const uint32_t base = taddr + (static_cast<uint32_t>(32 * quarter) << 16) +
                                          col0 + static_cast<uint32_t>(i0);
                    tc::tmem_ld16(base, r);
                    tc::tmem_ld16(base + acc1, r1);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int m = 0; m < 16; ++m) r[m] += r1[m];
                    for (int s = 2; s < NI; ++s) {
                        tc::tmem_ld16(base + static_cast<uint32_t>(s) * acc1, r1);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int m = 0; m < 16; ++m) r[m] += r1[m];
                    }
                    if (j < nc) {
#pragma unroll
                        for (int m = 0; m < 16; ++m)
                            if (i0 + m < nr) s_num[j * A.NRS + i0 + m] = r[m];
                    }
                }
            }
            __syncthreads();
            // Four values per thread and step, their loads issued before the (paired) arithmetic.
            int fi = fi0, fj = fj0;
            for (int e = tid; e < ne; e += 4 * kTcThreads) {
                int o[4], os[4];
                bool in[4];
                uint32_t d[4], s1[4], s2[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    in[u] = e + u * kTcThreads < ne;
                    o[u] = fj * A.NRS + fi;
                    os[u] = fj * A.NRS + ring(fi);
                    fstep(fi, fj);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    d[u] = in[u] ? s_num[o[u]] : 0u;
                    s1[u] = in[u] ? s_S1[os[u]] : 0u;
                    s2[u] = in[u] ? s_S2[os[u]] : 0u;
                }
                float2 b01, b23;
                const float2 e01 = tc_estimate2(d[0], d[1], s1[0], s1[1], s2[0], s2[1], nnf, csf,
                                                kk, kk7, A.measure, &b01);
                const float2 e23 = tc_estimate2(d[2], d[3], s1[2], s1[3], s2[2], s2[3], nnf, csf,
                                                kk, kk7, A.measure, &b23);
                const float ev[4] = {e01.x, e01.y, e23.x, e23.y};
                const float bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (in[u]) {
                        s_est[o[u]] = ev[u];
                        s_est[o[u] + A.NCM * A.NRS] = bv[u];
                        lmax = fmaxf(lmax, ev[u] - bv[u]);
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(kFull, lmax, o));
        if (lane == 0) s_fmax[warp] = lmax;
        __syncthreads();
        TC_PHASE(8)
        float M = s_fmax[0];
        for (int w = 1; w < kTcThreads / 32; ++w) M = fmaxf(M, s_fmax[w]);
        // M: the largest lower bound of any value. A value whose upper bound is below it is
        // strictly below some other value: it cannot be the (first) maximum.

        // Pass 2: exact values where the upper bound reaches M; the peak key. The same flattened
        // order, four values per thread and step.
        unsigned long long best = 0ull;
        {
            int fi = fi0, fj = fj0;
            for (int e = tid; e < ne; e += 4 * kTcThreads) {
                int o[4], ii[4], jj[4];
                bool in[4];
                float est[4], bnd[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    in[u] = e + u * kTcThreads < ne;
                    ii[u] = fi;
                    jj[u] = fj;
                    o[u] = fj * A.NRS + fi;
                    fstep(fi, fj);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    est[u] = in[u] ? s_est[o[u]] : 0.0f;
                    bnd[u] = in[u] ? s_est[o[u] + A.NCM * A.NRS] : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (!in[u] || (!(est[u] + bnd[u] >= M) && !isnan(est[u]))) continue;
                    const int os = jj[u] * A.NRS + ring(ii[u]);
                    const float v =
                        tc_exact(s_num[o[u]], s_S1[os], s_S2[os], mean, nn, cnorm, A.measure);
                    const unsigned long long key =
                        argmax_key(v, static_cast<unsigned>(ii[u] * nc + jj[u]));
                    best = key > best ? key : best;
                }
            }
        }
        best = block_max_u64(best, reinterpret_cast<unsigned long long*>(s_red));
        TC_PHASE(9)
        if (A.flops && tid == 0)
            atomicAdd(A.flops, 2ull * static_cast<unsigned long long>(ch) * cw * nr * nc);
        if (A.surf_out) {
            float* so = A.surf_out + k * static_cast<int64_t>(A.NRM) * A.NCM;
            for (int e = tid; e < nr * nc; e += bd) {
                const int o = (e / nr) * A.NRS + (e % nr);
                const int os = (e / nr) * A.NRS + ring(e % nr);
                so[e] = tc_exact(s_num[o], s_S1[os], s_S2[os], mean, nn, cnorm, A.measure);
            }
        }
        unsigned rm = 0;
        float pv = 0.0f;
        int pi = 0, pj = 0;
        if (key_decode(best, &rm, &pv)) {
            pi = static_cast<int>(rm / nc);
            pj = static_cast<int>(rm % nc);
        }
        if (A.up == 1 || nr < 5 || nc < 5) {
            if (tid == 0) {
                const int o = pj * A.NRS + pi;
                const int os = pj * A.NRS + ring(pi);
                const float v = tc_exact(s_num[o], s_S1[os], s_S2[os], mean, nn, cnorm, A.measure);
                A.out.dx[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pj - static_cast<int>(prx)), A.pts.dx0[k]));
                A.out.dy[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pi - static_cast<int>(pry)), A.pts.dy0[k]));
                A.out.corr[k] = v;
            }
        } else {
            const int pi0 = min(max(pi - 2, 0), max(nr - 5, 0));
            const int pj0 = min(max(pj - 2, 0), max(nc - 5, 0));
            const int slot = s_slot;
            if (tid < 25) {
                const int a = tid % 5, b = tid / 5;
                const int o = (pj0 + b) * A.NRS + (pi0 + a);
                const int os = (pj0 + b) * A.NRS + ring(pi0 + a);
                A.sub_patch[static_cast<int64_t>(slot) * 25 + tid] =
                    tc_exact(s_num[o], s_S1[os], s_S2[os], mean, nn, cnorm, A.measure);
            }
            if (tid == 0) {
                A.sub_point[slot] = k;
                A.sub_origin[2 * slot] = pi0;
                A.sub_origin[2 * slot + 1] = pj0;
            }
        }
        TC_PHASE(10)
        TC_PHASE_POINT
    }
    TC_PHASE_FLUSH
    if (failed) {
        // Products may still be in flight: give them a bounded time before freeing the
        // accumulator.
        tc::mbar_wait(&s_mbar, phase ^ 1u, kTcWaitPolls);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, A.tmem_cols);
}

// ----------------------------------------------------------------------------------------------
// Tensor-core correlation, surfaces up to 64 x 64 with the chip operand whole (k_corr_tc2).
//
// The window is staged from its first row (no alignment offset; each 16-byte block of a column
// is realigned from the aligned 16-byte chunks cp.async copied into shared memory, or from two
// aligned global loads), so block q of 16 rows meets surface rows i in [16 q - ch + 1,
// 16 q + 15]: NB = 16 * ceil((ch + 15) / 16) rows of the chip operand E_b[u][r] = C[r - u, b]
// (u = 16 - NB ... 15). A block's product lands at accumulator column 16 q + e - (NB - 16) for
// its operand row e, so surface row i is column i and the products of three issuing threads
// write three accumulators of round16(nr) columns. The box sums come from the 16-byte window
// blocks: column sums V down ch rows per 16-row block of surface rows (dp4a for the first, a
// sliding update for the rest), then row sums of V with 16-byte loads. Estimates stay in
// registers; candidates and the patch get the reference's FP64 normalisation.

// A point's chip and window placement (src/points.jl:358-395 with the pass's padding and the
// +0.5 shift, src/track.jl:128-138, 207-220) and whether it is searched at all.
struct PtGeo {
    long long k, chip_r, chip_c, win_r, win_c;
    int ch, cw, nr, nc, prx, pry, ok;
};

__device__ __forceinline__ void pt_geometry(const TcArgs& A, int64_t k, PtGeo& g) {
    // All eight fields are loaded before any is used.
    const int64_t prx = A.pts.rx[k], pry = A.pts.ry[k];
    const double x = A.pts.x[k], y = A.pts.y[k], dx0 = A.pts.dx0[k], dy0 = A.pts.dy0[k];
    const int64_t csx = A.pts.csx[k], csy = A.pts.csy[k];
    const int64_t NR = A.nrows + 2 * A.pady, NC = A.ncols + 2 * A.padx;
    g.k = k;
    g.ok = 0;
    if (!(prx > 0 && pry > 0)) return;
    const double xs = x + (static_cast<double>(A.padx) + 0.5);
    const double ys = y + (static_cast<double>(A.pady) + 0.5);
    const int64_t hx = csx / 2, hy = csy / 2;
    const int64_t ccx = static_cast<int64_t>(floor(__dsub_rn(xs, dx0)));
    const int64_t ccy = static_cast<int64_t>(floor(__dsub_rn(ys, dy0)));
    const int64_t wcx = static_cast<int64_t>(floor(xs)), wcy = static_cast<int64_t>(floor(ys));
    const int64_t cr0 = ccy - hy, cr1 = ccy + hy - 1, cc0 = ccx - hx, cc1 = ccx + hx - 1;
    const int64_t wr0 = wcy - hy - pry, wr1 = wcy + hy + pry - 2;
    const int64_t wc0 = wcx - hx - prx, wc1 = wcx + hx + prx - 2;
    const bool chip_in = (cr1 < cr0 || cc1 < cc0) ||
                         (cr0 >= 1 && cr1 <= NR && cc0 >= 1 && cc1 <= NC);
    const bool win_in = (wr1 < wr0 || wc1 < wc0) ||
                        (wr0 >= 1 && wr1 <= NR && wc0 >= 1 && wc1 <= NC);
    if (!chip_in || !win_in) return;
    g.ch = static_cast<int>(2 * hy);
    g.cw = static_cast<int>(2 * hx);
    g.nr = static_cast<int>(2 * pry);
    g.nc = static_cast<int>(2 * prx);
    g.prx = static_cast<int>(prx);
    g.pry = static_cast<int>(pry);
    if (g.ch <= 0 || g.cw <= 0) return;
    if (g.ch > A.CHM || g.cw > A.CWM || g.nr > A.NRM || g.nc > A.NCM) return;
    g.chip_r = cr0 - 1 - A.pady;
    g.chip_c = cc0 - 1 - A.padx;
    g.win_r = wr0 - 1 - A.pady;
    g.win_c = wc0 - 1 - A.padx;
    g.ok = 1;
}

__global__ void __launch_bounds__(kTcThreads, 2) k_corr_tc2(const TcArgs A) {
    extern __shared__ __align__(1024) unsigned char smem_tc[];
    __shared__ uint64_t s_mbar;
    __shared__ uint32_t s_taddr;
    __shared__ int s_slot;
    __shared__ int s_ncand;
    __shared__ uint32_t s_pd[25];
    __shared__ float s_fmax[kTcThreads / 32];
    __shared__ unsigned long long s_isum[2][2];
    __shared__ PtGeo s_geo[2];  // by iteration parity: a point's geometry, computed ahead
    uint8_t* s_E = smem_tc + A.off_E;
    uint8_t* s_W = smem_tc + A.off_W;
    uint8_t* s_P = smem_tc + A.off_P;
    uint32_t* s_V1 = reinterpret_cast<uint32_t*>(smem_tc + A.off_V);
    uint32_t* s_V2 = s_V1 + A.NRM * A.XV + 16;
    uint32_t* s_S1 = reinterpret_cast<uint32_t*>(smem_tc + A.off_S1);
    uint32_t* s_S2 = reinterpret_cast<uint32_t*>(smem_tc + A.off_S2);
    uint32_t* s_num = reinterpret_cast<uint32_t*>(smem_tc + A.off_num);
    uint32_t* s_cI = reinterpret_cast<uint32_t*>(smem_tc + A.off_est);
    double* s_red = reinterpret_cast<double*>(smem_tc + A.off_red);

    const int tid = threadIdx.x, bd = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = bd >> 5;
    const uint8_t* ref_end = A.ref + A.nrows * A.ncols;

    if (tid < 2) s_geo[tid].k = -1;
    if (warp == 0) {
        tc::tmem_alloc(&s_taddr, A.tmem_cols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&s_mbar, kTc2Issuers);  // one commit per issuing thread
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = s_taddr;
    const uint32_t acc1 = static_cast<uint32_t>(A.acc1_col);  // stride between accumulators
    uint32_t phase = 0;
    bool failed = false;
    if (tid < 4) s_isum[tid >> 1][tid & 1] = 0ull;
    for (int e = tid; e < A.CWM * A.PC; e += bd) s_P[e] = 0;
    int iter = 0;
    int dirty_ch = 0;
    TC_PHASE_INIT
#ifdef AR_TC_PHASES
    unsigned long long tmi_issue = 0, tmi_done = 0;
#endif

    // Each CTA takes a contiguous run of points: consecutive points of a grid column have the
    // same window columns one grid step lower, so most of their box sums carry over.
    const int64_t per = (A.pts.n + gridDim.x - 1) / gridDim.x;
    const int64_t kbeg = static_cast<int64_t>(blockIdx.x) * per;
    const int64_t kend = min(A.pts.n, kbeg + per);
    // The point whose box sums s_S1 / s_S2 hold (held = false: none).
    bool held = false;
    int64_t h_wr = 0, h_wc = 0;
    // s_S1 / s_S2 are rings of NRS rows per column: surface row i of the held point is stored at
    // row (i + rbase) mod NRS, so carrying the sums down by `sh` rows advances rbase instead of
    // moving them.
    int rbase = 0;
    auto ring = [&](int i) {
        const int r = i + rbase;
        return r >= A.NRS ? r - A.NRS : r;
    };
    int h_ch = 0, h_cw = 0, h_nr = 0, h_nc = 0;
    for (int64_t k = kbeg; k < kend; ++k, ++iter) {
        tc::cp_async_wait_all();  // no copy of a skipped point is still landing
        tc::fence_before_sync();
        __syncthreads();  // the previous point's buffers and accumulators are no longer read
        tc::fence_after_sync();
        TC_PHASE(0)
        const int ib = iter & 1;
        if (tid < 2) s_isum[ib ^ 1][tid] = 0ull;
        // The geometry: computed ahead by the previous iteration when it reached its products.
        PtGeo g;
        if (s_geo[ib].k == k) {
            g = s_geo[ib];
        } else {
            pt_geometry(A, k, g);
        }
        if (!g.ok) continue;
        const int ch = g.ch, cw = g.cw, nr = g.nr, nc = g.nc, prx = g.prx, pry = g.pry;
        TC_PHASE(1)
        const int64_t chip_r = g.chip_r, chip_c = g.chip_c, win_r = g.win_r, win_c = g.win_c;
        const long long nnl = static_cast<long long>(ch) * cw;
        const bool pow2 = (nnl & (nnl - 1)) == 0 && nnl <= 4096;

        // The window's columns as aligned 16-byte chunks, copied asynchronously (cp.async) into
        // the column-sum buffer -- free until the box sums -- while the chip is staged: when
        // every row of the window lies in the image, a column takes the Q + 1 chunks from the
        // aligned address at or below its first row (columns whose chunks would leave the array,
        // and windows that reach outside the image's rows, are staged from global memory below).
        const int Q = (ch + nr - 1 + 15) / 16;
        const int RQ = Q + 1;
        uint8_t* s_Wraw = reinterpret_cast<uint8_t*>(s_V1);
        const bool rows_in = win_r >= 0 && win_r + 16 * Q <= A.nrows;
        auto raw_col = [&](int x, const uint8_t** first) {
            // Column x's aligned first chunk when all its chunks are inside the array, else null.
            const int64_t c = win_c + x;
            if (!rows_in || c < 0 || c >= A.ncols) return false;
            const uint8_t* p = A.ref + c * A.nrows + win_r;
            const uint8_t* a0 = reinterpret_cast<const uint8_t*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(15));
            if (a0 < A.ref || a0 + 16 * RQ > ref_end) return false;
            *first = a0;
            return true;
        };
        if (rows_in) {
            for (int it = tid; it < A.XS * RQ; it += bd) {
                const int x = it / RQ, kq = it - x * RQ;
                const uint8_t* a0;
                if (raw_col(x, &a0)) tc::cp_async16(s_Wraw + static_cast<size_t>(it) * 16, a0 + 16 * kq);
            }
        }
        tc::cp_async_commit();

        // The chip as zero-padded byte columns, _any_valid over it (src/track.jl:416-421) and,
        // for power-of-two areas, its exact integer sums (as in k_corr_tc).
        int any = 0;
        unsigned long long isum = 0ull, isq = 0ull;
        if (ch < dirty_ch)
            for (int b = warp; b < A.CWM; b += nwarps)
                for (int a = ch + lane; a < dirty_ch; a += 32) s_P[b * A.PC + kPadL + a] = 0;
        dirty_ch = ch;
        for (int a0 = 0; a0 < ch; a0 += 32) {
            const int a = a0 + lane;
            const int64_t r = chip_r + a;
            const bool rin = a < ch && r >= 0 && r < A.nrows;
            constexpr int kU = 4;
            for (int b0 = warp; b0 < cw; b0 += kU * nwarps) {
                uint32_t v[kU], m[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int b = b0 + u * nwarps;
                    const int64_t c = chip_c + b;
                    const bool in = rin && b < cw && c >= 0 && c < A.ncols;
                    v[u] = in ? A.sec[r + c * A.nrows] : 0u;
                    m[u] = in ? A.valid[r + c * A.nrows] : 0u;
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int b = b0 + u * nwarps;
                    if (a < ch && b < cw) {
                        s_P[b * A.PC + kPadL + a] = static_cast<uint8_t>(v[u]);
                        any |= m[u];
                        isum += v[u];
                        isq += v[u] * v[u];
                    }
                }
            }
        }
        if (pow2) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                isum += __shfl_xor_sync(kFull, isum, o);
                isq += __shfl_xor_sync(kFull, isq, o);
            }
            if (lane == 0) {
                atomicAdd(&s_isum[ib][0], isum);
                atomicAdd(&s_isum[ib][1], isq);
            }
        }
        tc::cp_async_wait_all();  // this thread's window chunks have landed (visible after the barrier)
        if (!__syncthreads_or(any)) continue;
        TC_PHASE(2)
        if (tid == 0) A.out.searched[k] = 1;

        double mean, sq, csum_d;
        if (pow2) {
            const long long cs = static_cast<long long>(s_isum[ib][0]);
            const long long c2 = static_cast<long long>(s_isum[ib][1]);
            csum_d = static_cast<double>(cs);
            mean = __ddiv_rn(csum_d, static_cast<double>(nnl));
            sq = __ddiv_rn(static_cast<double>(nnl * c2 - cs * cs), static_cast<double>(nnl));
        } else {
            staged_chip_stats(s_P, A.PC, ch, cw, tid, bd, s_red, &csum_d, &mean, &sq);
        }
        if (!(sq > __dmul_rn(__dmul_rn(DBL_EPSILON, static_cast<double>(ch)), static_cast<double>(cw))))
            continue;  // degenerate chip: searched, no measurement (src/track.jl:286)
        TC_PHASE(3)
        const double cnorm = __dsqrt_rn(sq);
        if (tid == 0 && !(A.up == 1 || nr < 5 || nc < 5)) s_slot = atomicAdd(A.sub_count, 1);
        const double nn = static_cast<double>(nnl);

        // Window blocks W[16 q + r][x] (x < XS) from the window's first row: from the chunks in
        // shared memory, or from global memory for the columns that have none.
        const int XW = cw + nc - 1;
        for (int q = warp; q < Q; q += nwarps)
            for (int x = lane; x < A.XS; x += 32) {
                const uint8_t* a0;
                Col16 L;
                if (raw_col(x, &a0)) {
                    const uint4* rc = reinterpret_cast<const uint4*>(s_Wraw + static_cast<size_t>(x * RQ + q) * 16);
                    L.lo = rc[0];
                    L.hi = rc[1];
                    L.s = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(A.ref + (win_c + x) * A.nrows + win_r) & 15);
                } else {
                    L = col16_issue(A.ref, ref_end, A.nrows, A.ncols, win_c + x, win_r + 16 * q);
                }
                *reinterpret_cast<uint4*>(s_W + q * A.QS + x * 16) = col16_finish(L);
            }
        // E: NB rows per chip column, row e (u = e - NB + 16) = 16 bytes from chip row -u.
        {
            const int nrow = cw * A.NB;
            int bl = tid / A.NB, e = tid - bl * A.NB;
            const int sbl = bd / A.NB, se = bd - sbl * A.NB;
            for (int t = tid; t < nrow; t += bd) {
                const int src = bl * A.PC + kPadL - 16 + A.NB - e;
                const uint32_t* w = reinterpret_cast<const uint32_t*>(s_P + (src & ~3));
                const uint32_t sh = static_cast<uint32_t>(src & 3) * 8u;
                uint4 o;
                o.x = __funnelshift_r(w[0], w[1], sh);
                o.y = __funnelshift_r(w[1], w[2], sh);
                o.z = __funnelshift_r(w[2], w[3], sh);
                o.w = __funnelshift_r(w[3], w[4], sh);
                *reinterpret_cast<uint4*>(s_E + bl * A.PS + e * 16) = o;
                bl += sbl;
                e += se;
                if (e >= A.NB) {
                    e -= A.NB;
                    ++bl;
                }
            }
        }
        // The products add into accumulator columns [0, round16(nr)): surface row i is column i.
        const int dcols = (nr + 15) & ~15;
        if (warp < 4) {
            // Clear the columns the products add into (one lane quarter per warp).
            uint32_t z[16];
#pragma unroll
            for (int t = 0; t < 16; ++t) z[t] = 0u;
            const uint32_t lq = taddr + (static_cast<uint32_t>(32 * warp) << 16);
            for (int c = 0; c < dcols; c += 16)
#pragma unroll
                for (int t = 0; t < kTc2Issuers; ++t)
                    tc::tmem_st16(lq + static_cast<uint32_t>(t) * acc1 + static_cast<uint32_t>(c), z);
            tc::tmem_wait_st();
        }
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();  // s_P, s_W, s_E complete; accumulator cleared
        TC_PHASE(4)
        // Lane 0 of the last kTc2Issuers warps issue the products, each for a share of the chip
        // column pairs into its own accumulator (one thread issues an MMA about every 120
        // cycles; several issuers interleave theirs).
        if (lane == 0 && warp >= nwarps - kTc2Issuers) {
            const int stream = nwarps - 1 - warp;
            tc::fence_after_sync();
#ifdef AR_TC_PHASES
            const unsigned long long tmi0 = clock64();
#endif
            // Descriptors advance by adding to their start-address field, the low bits of the
            // low word (16-byte units; shared addresses stay below 2^18, so nothing carries):
            // a product costs the issuing thread two 32-bit adds and the MMA itself.
            const uint64_t da0 = tc::smem_desc(tc::smem_u32(s_W), 16, 128);
            const uint64_t db0 = tc::smem_desc(tc::smem_u32(s_E), A.PS, 128);
            const uint32_t a_hi = static_cast<uint32_t>(da0 >> 32);
            const uint32_t b_hi = static_cast<uint32_t>(db0 >> 32);
            const uint32_t bstep = static_cast<uint32_t>(2 * A.PS) >> 4;
            const int pairs = cw / 2;
            const int t_begin = pairs * stream / kTc2Issuers;
            const int npairs = pairs * (stream + 1) / kTc2Issuers - t_begin;
            for (int q = 0; q < Q; ++q) {
                // Only the operand rows e in [elo, elo + n) of block q reach surface rows.
                int elo, n;
                if (!block_rows(q, A.NB, nr, &elo, &n)) continue;
                const uint32_t idesc = tc::idesc_u8_s32(64, n);
                uint32_t a_lo = static_cast<uint32_t>(da0) +
                                static_cast<uint32_t>(q * A.QS >> 4) + 2u * static_cast<uint32_t>(t_begin);
                uint32_t b_lo = static_cast<uint32_t>(db0) + static_cast<uint32_t>(elo) +
                                bstep * static_cast<uint32_t>(t_begin);
                const uint32_t dn = taddr + static_cast<uint32_t>(stream) * acc1 +
                                    static_cast<uint32_t>(16 * q + elo - (A.NB - 16));
                int t = 0;
                for (; t + 4 <= npairs; t += 4) {
                    tc::mma_u8_halves(dn, a_lo, a_hi, b_lo, b_hi, idesc);
                    tc::mma_u8_halves(dn, a_lo + 2, a_hi, b_lo + bstep, b_hi, idesc);
                    tc::mma_u8_halves(dn, a_lo + 4, a_hi, b_lo + 2 * bstep, b_hi, idesc);
                    tc::mma_u8_halves(dn, a_lo + 6, a_hi, b_lo + 3 * bstep, b_hi, idesc);
                    a_lo += 8;
                    b_lo += 4 * bstep;
                }
                for (; t < npairs; ++t) {
                    tc::mma_u8_halves(dn, a_lo, a_hi, b_lo, b_hi, idesc);
                    a_lo += 2;
                    b_lo += bstep;
                }
            }
            tc::mma_commit(&s_mbar);
#ifdef AR_TC_PHASES
            // Profiling builds: time to issue the products, then until they complete.
            const unsigned long long tmi1 = clock64();
            if (stream == 0) {
                tc::mbar_wait(&s_mbar, phase, kTcWaitPolls);
                tmi_issue += tmi1 - tmi0;
                tmi_done += clock64() - tmi1;
            }
#endif
            // The next point's geometry, read after the next loop-top barrier.
            const int64_t kn = k + 1;
            if (stream == 0 && kn < kend) pt_geometry(A, kn, s_geo[ib ^ 1]);
        }
        TC_PHASE(5)
        // S[j][i] = sums of V[i][j .. j + cw - 1] for rows i in [i_lo, i_lo + ni): a task is a
        // row i and 16 columns j (the warps that do not issue products).
        auto box_rows = [&](int i_lo, int ni) {
            constexpr int kBT = kTcThreads - 32 * kTc2Issuers;
            const int jseg = (nc + 15) >> 4;
            const bool vec = (cw & 3) == 0;
            for (int task = tid; task < ni * jseg; task += kBT) {
                const int sg = task / ni, i = i_lo + (task - sg * ni);
                const int j0 = 16 * sg;
                const uint32_t* r1 = s_V1 + i * A.XV;
                const uint32_t* r2 = s_V2 + i * A.XV;
                uint32_t g1 = 0, g2 = 0;
                int bb = 0;
                for (; bb + 4 <= cw; bb += 4) {
                    const uint4 v = *reinterpret_cast<const uint4*>(r1 + j0 + bb);
                    const uint4 w = *reinterpret_cast<const uint4*>(r2 + j0 + bb);
                    g1 += (v.x + v.y) + (v.z + v.w);
                    g2 += (w.x + w.y) + (w.z + w.w);
                }
                for (; bb < cw; ++bb) {
                    g1 += r1[j0 + bb];
                    g2 += r2[j0 + bb];
                }
#pragma unroll
                for (int u4 = 0; u4 < 16; u4 += 4) {
                    const uint4 o1 = *reinterpret_cast<const uint4*>(r1 + j0 + u4);
                    const uint4 o2 = *reinterpret_cast<const uint4*>(r2 + j0 + u4);
                    uint4 i1, i2;
                    if (vec) {
                        i1 = *reinterpret_cast<const uint4*>(r1 + j0 + u4 + cw);
                        i2 = *reinterpret_cast<const uint4*>(r2 + j0 + u4 + cw);
                    } else {
                        const uint32_t* p1 = r1 + j0 + u4 + cw;
                        const uint32_t* p2 = r2 + j0 + u4 + cw;
                        i1 = make_uint4(p1[0], p1[1], p1[2], p1[3]);
                        i2 = make_uint4(p2[0], p2[1], p2[2], p2[3]);
                    }
                    const uint32_t oo1[4] = {o1.x, o1.y, o1.z, o1.w}, ii1[4] = {i1.x, i1.y, i1.z, i1.w};
                    const uint32_t oo2[4] = {o2.x, o2.y, o2.z, o2.w}, ii2[4] = {i2.x, i2.y, i2.z, i2.w};
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const int j = j0 + u4 + m;
                        if (j < nc) {
                            s_S1[j * A.NRS + i] = g1;
                            s_S2[j * A.NRS + i] = g2;
                            g1 = g1 + ii1[m] - oo1[m];
                            g2 = g2 + ii2[m] - oo2[m];
                        }
                    }
                }
            }
        };
        // Box sums of W and W^2 (integral_both!, boxsum, src/integral.jl:141-170, 244-247) as
        // exact integers, warps 0-4 (named barrier 1) while warps 5-7 issue the products. When
        // the held sums belong to the same window geometry `sh` rows higher, the ring's base
        // advances by `sh` (the held rows become rows 0 .. nr - sh - 1) and only the last `sh`
        // rows are computed.
        const int64_t sh64 = win_r - h_wr;
        const bool carry = held && win_c == h_wc && ch == h_ch && cw == h_cw && nr == h_nr &&
                           nc == h_nc && sh64 > 0 && sh64 < nr;
        if (carry) {
            rbase += static_cast<int>(sh64);
            if (rbase >= A.NRS) rbase -= A.NRS;
        } else {
            rbase = 0;
        }
#ifdef AR_TC_PHASES
        if (tid == 0 && carry) atomicAdd(&g_tc_phase[14], 1ull);
#endif
        if (warp < nwarps - kTc2Issuers) {
            constexpr int kBT = kTcThreads - 32 * kTc2Issuers;
            if (carry) {
                const int sh = static_cast<int>(sh64);
                // Column sums of the new rows i in [nr - sh, nr): an item is a window column and
                // up to 4 consecutive rows; its first sum from 4-byte groups (dp4a), then a
                // sliding update. The row groups of a column are adjacent lanes: their words lie
                // in different banks of the column's 16-byte block.
                const int i0 = nr - sh;
                const int nparts = (sh + 3) >> 2;
                for (int item = tid; item < XW * nparts; item += kBT) {
                    const int x = item / nparts, pt = item - x * nparts;
                    const int ia = i0 + 4 * pt, ie = min(ia + 4, nr);
                    const uint8_t* colx = s_W + x * 16;
                    // Rows r .. r + 3 of column x as one word (a group may cross a block).
                    auto word = [&](int r) {
                        const int rb = r >> 4, o = r & 15, ow = o & ~3;
                        const uint32_t lo = *reinterpret_cast<const uint32_t*>(colx + rb * A.QS + ow);
                        if ((o & 3) == 0) return lo;
                        const int nb = ow + 4 < 16 ? rb : rb + 1, no = ow + 4 < 16 ? ow + 4 : 0;
                        const uint32_t hi = nb < Q ? *reinterpret_cast<const uint32_t*>(colx + nb * A.QS + no) : 0u;
                        return __funnelshift_r(lo, hi, 8u * static_cast<uint32_t>(o & 3));
                    };
                    uint32_t h1 = 0, h2 = 0;
                    int a = 0;
                    for (; a + 4 <= ch; a += 4) {
                        const uint32_t w = word(ia + a);
                        h1 = __dp4a(w, 0x01010101u, h1);
                        h2 = __dp4a(w, w, h2);
                    }
                    if (a < ch) {
                        const uint32_t mk = (1u << (8 * (ch - a))) - 1u;
                        const uint32_t w = word(ia + a) & mk;
                        h1 = __dp4a(w, 0x01010101u, h1);
                        h2 = __dp4a(w, w, h2);
                    }
                    for (int i = ia; i < ie; ++i) {
                        s_V1[i * A.XV + x] = h1;
                        s_V2[i * A.XV + x] = h2;
                        if (i + 1 < ie) {
                            const uint32_t o = colx[(i >> 4) * A.QS + (i & 15)];
                            const int R = i + ch;
                            const uint32_t n = colx[(R >> 4) * A.QS + (R & 15)];
                            h1 = h1 + n - o;
                            h2 = h2 + n * n - o * o;
                        }
                    }
                }
                asm volatile("bar.sync 1, %0;" ::"r"(kBT) : "memory");
                // Row sums of the new rows: a task is a row and 4 consecutive columns j.
                const int ng = (nc + 3) >> 2;
                for (int task = tid; task < sh * ng; task += kBT) {
                    const int g = task / sh, i = i0 + (task - g * sh);
                    const int j0 = 4 * g;
                    const uint32_t* r1 = s_V1 + i * A.XV;
                    const uint32_t* r2 = s_V2 + i * A.XV;
                    uint32_t g1 = 0, g2 = 0;
                    int bb = 0;
                    for (; bb + 4 <= cw; bb += 4) {
                        const uint4 v = *reinterpret_cast<const uint4*>(r1 + j0 + bb);
                        const uint4 w = *reinterpret_cast<const uint4*>(r2 + j0 + bb);
                        g1 += (v.x + v.y) + (v.z + v.w);
                        g2 += (w.x + w.y) + (w.z + w.w);
                    }
                    for (; bb < cw; ++bb) {
                        g1 += r1[j0 + bb];
                        g2 += r2[j0 + bb];
                    }
                    // Outgoing and incoming columns as 16-byte loads (rows stay inside XV).
                    const uint4 o1 = *reinterpret_cast<const uint4*>(r1 + j0);
                    const uint4 o2 = *reinterpret_cast<const uint4*>(r2 + j0);
                    uint4 i1, i2;
                    if ((cw & 3) == 0) {
                        i1 = *reinterpret_cast<const uint4*>(r1 + j0 + cw);
                        i2 = *reinterpret_cast<const uint4*>(r2 + j0 + cw);
                    } else {
                        const uint32_t* p1 = r1 + j0 + cw;
                        const uint32_t* p2 = r2 + j0 + cw;
                        i1 = make_uint4(p1[0], p1[1], p1[2], p1[3]);
                        i2 = make_uint4(p2[0], p2[1], p2[2], p2[3]);
                    }
                    const uint32_t oo1[4] = {o1.x, o1.y, o1.z, o1.w}, ii1[4] = {i1.x, i1.y, i1.z, i1.w};
                    const uint32_t oo2[4] = {o2.x, o2.y, o2.z, o2.w}, ii2[4] = {i2.x, i2.y, i2.z, i2.w};
                    const int ri = ring(i);
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        const int j = j0 + m;
                        if (j < nc) {
                            s_S1[j * A.NRS + ri] = g1;
                            s_S2[j * A.NRS + ri] = g2;
                            g1 = g1 + ii1[m] - oo1[m];
                            g2 = g2 + ii2[m] - oo2[m];
                        }
                    }
                }
            } else {
                // V[i][x] = sums over rows i .. i + ch - 1 of column x: a task is a column and the 16
                // rows i of one block; its outgoing rows are that block, its incoming rows start ch
                // rows lower.
                const int nseg = (nr + 15) >> 4;
                const int chb = ch >> 4, chr = ch & 15;
                for (int task = tid; task < XW * nseg; task += kBT) {
                    const int sgi = task / XW, x = task - sgi * XW;
                    const int i0 = 16 * sgi;
                    const uint8_t* colx = s_W + x * 16;
                    const uint4 bo = *reinterpret_cast<const uint4*>(colx + sgi * A.QS);
                    uint32_t h1 = 0, h2 = 0;
                    for (int bb = 0; bb < chb; ++bb) {
                        const uint4 w = *reinterpret_cast<const uint4*>(colx + (sgi + bb) * A.QS);
                        h1 = __dp4a(w.x, 0x01010101u, h1);
                        h1 = __dp4a(w.y, 0x01010101u, h1);
                        h1 = __dp4a(w.z, 0x01010101u, h1);
                        h1 = __dp4a(w.w, 0x01010101u, h1);
                        h2 = __dp4a(w.x, w.x, h2);
                        h2 = __dp4a(w.y, w.y, h2);
                        h2 = __dp4a(w.z, w.z, h2);
                        h2 = __dp4a(w.w, w.w, h2);
                    }
                    const uint4 bi = *reinterpret_cast<const uint4*>(colx + (sgi + chb) * A.QS);
                    if (chr) {
                        const uint32_t wv[4] = {bi.x, bi.y, bi.z, bi.w};
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            const int keep = min(max(chr - 4 * m, 0), 4);
                            const uint32_t mk = keep == 4 ? 0xffffffffu : ((1u << (8 * keep)) - 1u);
                            h1 = __dp4a(wv[m] & mk, 0x01010101u, h1);
                            h2 = __dp4a(wv[m] & mk, wv[m], h2);
                        }
                    }
                    const uint32_t wo[4] = {bo.x, bo.y, bo.z, bo.w};
                    const uint32_t wi[4] = {bi.x, bi.y, bi.z, bi.w};
                    uint32_t* v1o = s_V1 + i0 * A.XV + x;
                    uint32_t* v2o = s_V2 + i0 * A.XV + x;
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        if (i0 + u < nr) {
                            v1o[u * A.XV] = h1;
                            v2o[u * A.XV] = h2;
                            const uint32_t o = (wo[u >> 2] >> (8 * (u & 3))) & 0xffu;
                            uint32_t in;
                            if (chr == 0) {
                                in = (wi[u >> 2] >> (8 * (u & 3))) & 0xffu;
                            } else {
                                const int R = i0 + u + ch;
                                in = colx[(R >> 4) * A.QS + (R & 15)];
                            }
                            h1 = h1 + in - o;
                            h2 = h2 + in * in - o * o;
                        }
                    }
                }
                asm volatile("bar.sync 1, %0;" ::"r"(kBT) : "memory");
                box_rows(0, nr);
            }
        }
        held = true;
        h_wr = win_r;
        h_wc = win_c;
        h_ch = ch;
        h_cw = cw;
        h_nr = nr;
        h_nc = nc;
        TC_PHASE(6)
        bool ok = tc::mbar_wait(&s_mbar, phase, kTcWaitPolls);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(A.status, 1);
            failed = true;
            break;
        }
        tc::fence_after_sync();
        TC_PHASE(7)

        // Pass 1: numerators out of Tensor Memory (one 16x256b read per warp), box sums from
        // shared memory; estimates and upper bounds stay in registers. Value v
        // of a thread is surface row i = 32 half + 8 (v / 4) + 2 (lane % 4) + v % 2, column
        // j = 16 quarter + lane / 4 (+ 8 when v % 4 >= 2).
        const float kk = __double2float_rn(
            A.measure == AR_NCC ? __drcp_rn(__dmul_rn(cnorm, nn))
                                : __drcp_rn(__dmul_rn(cnorm, __dsqrt_rn(nn))));
        const float kk7 = 4.172325134277344e-07f * kk;  // 7u k
        const float nnf = static_cast<float>(nnl);
        const float csf = static_cast<float>(csum_d);
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t col0 = 0u;  // surface row i is accumulator column i
        const int ib0 = 32 * half + 2 * (lane & 3);
        const int jb0 = 16 * quarter + (lane >> 2);
        uint32_t dv[16];
        float upb[16];
        uint32_t vm = 0u;
        float lmax = -INFINITY;
        if (32 * half < nr) {
            const uint32_t base = taddr + (static_cast<uint32_t>(32 * quarter) << 16) + col0 +
                                  static_cast<uint32_t>(32 * half);
            uint32_t dv1[kTc2Issuers - 1][16];
            tc::tmem_ld16dp(base, dv);
#pragma unroll
            for (int t = 1; t < kTc2Issuers; ++t) tc::tmem_ld16dp(base + static_cast<uint32_t>(t) * acc1, dv1[t - 1]);
            tc::tmem_wait_ld();
#pragma unroll
            for (int t = 1; t < kTc2Issuers; ++t)
#pragma unroll
                for (int v = 0; v < 16; ++v) dv[v] += dv1[t - 1][v];  // the issuers' shares
            // Values v and v + 1 are surface rows i and i + 1 of one column: estimated as a pair.
#pragma unroll
            for (int v = 0; v < 16; v += 2) {
                const int i = ib0 + 8 * (v >> 2), j = jb0 + ((v & 2) ? 8 : 0);
                upb[v] = upb[v + 1] = -INFINITY;
                if (j < nc && i < nr) {
                    const bool two = i + 1 < nr;
                    vm |= (two ? 3u : 1u) << v;
                    const int o = j * A.NRS + ring(i), o1 = j * A.NRS + ring(i + 1);
                    const uint32_t b1 = two ? s_S1[o1] : 0u, b2 = two ? s_S2[o1] : 0u;
                    float2 bnd;
                    const float2 est = tc_estimate2(dv[v], dv[v + 1], s_S1[o], b1, s_S2[o], b2,
                                                    nnf, csf, kk, kk7, A.measure, &bnd);
                    upb[v] = est.x + bnd.x;
                    lmax = fmaxf(lmax, est.x - bnd.x);
                    if (two) {
                        upb[v + 1] = est.y + bnd.y;
                        lmax = fmaxf(lmax, est.y - bnd.y);
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(kFull, lmax, o));
        if (lane == 0) s_fmax[warp] = lmax;
        if (tid == 0) s_ncand = 0;
        __syncthreads();
        TC_PHASE(8)
        float M = s_fmax[0];
        for (int w = 1; w < kTcThreads / 32; ++w) M = fmaxf(M, s_fmax[w]);
        // Pass 2: values whose upper bound reaches M (or whose estimate was not made) go to a
        // list and are normalised exactly, one per thread.
#pragma unroll
        for (int v = 0; v < 16; ++v) {
            if (((vm >> v) & 1u) && (upb[v] >= M || isnan(upb[v]))) {
                const int c = atomicAdd(&s_ncand, 1);
                s_num[c] = dv[v];
                s_cI[c] = (static_cast<uint32_t>(ib0 + 8 * (v >> 2) + (v & 1)) << 16) |
                          static_cast<uint32_t>(jb0 + ((v & 2) ? 8 : 0));
            }
        }
        __syncthreads();
        const int ncand = s_ncand;
        unsigned rm = 0;
        float pv = 0.0f;
        int pi = 0, pj = 0;
        if (ncand == 1 && M > -INFINITY) {
            // M is finite, so the value whose lower bound is M is in the list; when it is the
            // only entry, every other FP32 surface value is at most its upper bound, below M,
            // and this one is at least M: it is the strict (so the first) maximum.
            pi = static_cast<int>(s_cI[0] >> 16);
            pj = static_cast<int>(s_cI[0] & 0xFFFFu);
        } else {
            unsigned long long best = 0ull;
            for (int c = tid; c < ncand; c += bd) {
                const int i = static_cast<int>(s_cI[c] >> 16), j = static_cast<int>(s_cI[c] & 0xFFFFu);
                const int o = j * A.NRS + ring(i);
                const float x = tc_exact(s_num[c], s_S1[o], s_S2[o], mean, nn, cnorm, A.measure);
                const unsigned long long key = argmax_key(x, static_cast<unsigned>(i * nc + j));
                best = key > best ? key : best;
            }
            best = block_max_u64(best, reinterpret_cast<unsigned long long*>(s_red));
            if (key_decode(best, &rm, &pv)) {
                pi = static_cast<int>(rm / nc);
                pj = static_cast<int>(rm % nc);
            }
        }
        TC_PHASE(9)
        if (A.flops && tid == 0)
            atomicAdd(A.flops, 2ull * static_cast<unsigned long long>(ch) * cw * nr * nc);
        if (A.surf_out) {
            // Every value exactly (diagnostic surfaces): numerators to shared memory first.
#pragma unroll
            for (int v = 0; v < 16; ++v)
                if ((vm >> v) & 1u)
                    s_num[(jb0 + ((v & 2) ? 8 : 0)) * A.NRS + ib0 + 8 * (v >> 2) + (v & 1)] = dv[v];
            __syncthreads();
            float* so = A.surf_out + k * static_cast<int64_t>(A.NRM) * A.NCM;
            for (int e = tid; e < nr * nc; e += bd) {
                const int o = (e / nr) * A.NRS + (e % nr), os = (e / nr) * A.NRS + ring(e % nr);
                so[e] = tc_exact(s_num[o], s_S1[os], s_S2[os], mean, nn, cnorm, A.measure);
            }
        }
        const bool single = A.up == 1 || nr < 5 || nc < 5;
        const int pi0 = single ? pi : min(max(pi - 2, 0), max(nr - 5, 0));
        const int pj0 = single ? pj : min(max(pj - 2, 0), max(nc - 5, 0));
        const int span = single ? 1 : 5;
#pragma unroll
        for (int v = 0; v < 16; ++v) {
            const int a = ib0 + 8 * (v >> 2) + (v & 1) - pi0, b = jb0 + ((v & 2) ? 8 : 0) - pj0;
            if (a >= 0 && a < span && b >= 0 && b < span && ((vm >> v) & 1u)) s_pd[b * 5 + a] = dv[v];
        }
        __syncthreads();
        if (single) {
            if (tid == 0) {
                A.out.dx[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pj - static_cast<int>(prx)), A.pts.dx0[k]));
                A.out.dy[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pi - static_cast<int>(pry)), A.pts.dy0[k]));
                const int o = pj * A.NRS + ring(pi);
                A.out.corr[k] = tc_exact(s_pd[0], s_S1[o], s_S2[o], mean, nn, cnorm, A.measure);
            }
        } else {
            const int slot = s_slot;
            if (tid < 25) {
                const int a = tid % 5, b = tid / 5;
                const int o = (pj0 + b) * A.NRS + ring(pi0 + a);
                A.sub_patch[static_cast<int64_t>(slot) * 25 + tid] =
                    tc_exact(s_pd[tid], s_S1[o], s_S2[o], mean, nn, cnorm, A.measure);
            }
            if (tid == 0) {
                A.sub_point[slot] = k;
                A.sub_origin[2 * slot] = pi0;
                A.sub_origin[2 * slot + 1] = pj0;
            }
        }
        TC_PHASE(10)
        TC_PHASE_POINT
    }
    TC_PHASE_FLUSH
#ifdef AR_TC_PHASES
    if (tid == kTcThreads - 32) {
        atomicAdd(&g_tc_phase[12], tmi_issue);
        atomicAdd(&g_tc_phase[13], tmi_done);
    }
#endif
    if (failed) tc::mbar_wait(&s_mbar, phase ^ 1u, kTcWaitPolls);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, A.tmem_cols);
}

// ----------------------------------------------------------------------------------------------
// Split-BF16 tensor-core correlation for UInt16, Int16 and Float32 imagery (k_corr_bf).
//
// The numerator of the CUDA-core kernel, sum_{a,b} C'[a, b] W'[i + a, j + b], with C' the chip of
// prepare_chip! (src/correlate.jl:423-453: Float32(x - mean)) and W' the window shifted by a
// centring constant (W' = Float32(w - cshift), cshift the chip mean rounded to an integer for
// integer imagery and to Float32 otherwise; num = sum C' W' + cshift sum C'), as products on the
// tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32 accumulators in Tensor Memory). Each
// operand is split into three BF16 limbs, v = v0 + v1 + v2 with v0 = bf16(v), v1 = bf16(v - v0),
// v2 = bf16(v - v0 - v1) (24 significant bits: a Float32 value exactly), and the numerator is the
// sum of the six products whose order is at least 2^-16 -- c0 w0, c0 w1, c1 w0, c1 w1, c2 w0,
// c0 w2 -- which recovers FP32 accuracy. The integer windows of UInt16 and Int16 imagery are
// exactly w0 + w1 (an integer below 2^16 in magnitude is the sum of two BF16 values), so their
// c0 w2 product is skipped.
//
// Layout (as the UInt8 kernels, with 2-byte elements and one chip column per product):
//   A[j, (q, b, r)] = W'[16 q + r, j + b]    r < 16, stored as two 8-row halves h:
//                                            s_W[limb][q][h][x] (16 bytes), row j of A 16 bytes
//                                            after row j - 1, the halves LW x 16 bytes apart;
//   B[i, (q, b, r)] = E_b[i - 16 q][r]       E_b[u][r] = C'[r - u, b], stored s_E[limb][b][h][e].
// Block q meets surface rows [16 q - ch + 1, 16 q + 15]: NB = 16 ceil((ch + 15) / 16) operand rows,
// surface row i in accumulator column i (rows trimmed to 0 <= i < nr in steps of 16).
//
// Per point: the chip's statistics; the window's box sums (integral_both!, boxsum,
// src/integral.jl:141-170, 244-247) in FP64 from the image values, a stripe of window columns
// at a time in shared memory -- column sums of ch rows, then a running sum along each surface
// row whose differences cw columns apart are the box sums -- and from them each surface value's
// FP64 denominator (src/correlate.jl:575-630); then the window's limbs for as many chip columns
// as shared memory holds (all of them up to 64-px chips), and the products chunk by chunk of BC
// chip columns. Four threads issue a chunk's products, each into an accumulator of its own (one
// thread issues an MMA about every 120 cycles, so the small M = 64 products need several issuers
// to keep the tensor core busy). Two sets of four accumulators take alternate chunks: while the
// tensor core runs chunk c, the threads build chunk c + 1's chip operand and add chunk c - 1's
// accumulators into FP64 sums they keep in registers (the tensor core's FP32 accumulation does
// not round to nearest, so a long chain of products into one accumulator drifts: ~1e-4 of the
// numerator over the ~1,000 products per accumulator of a 192-px chip; a chunk's chain is kept
// near kBfChain). Surfaces up to 64 x 64.

constexpr int kBfThreads = 256;
constexpr int kBfLimbs = 3;        // BF16 limbs per operand
constexpr int kBfPadL = 16;        // zero elements before each staged chip column
constexpr int kBfChain = 24;       // accumulating products per accumulator element per chunk
constexpr int kBfIssuers = 4;      // issuing threads (and accumulators) per set
constexpr int kBfPre = 4;          // staged chip elements per thread and chunk
constexpr int kBfBatch = 8;        // global loads a thread issues before using them

struct BfArgs {
    const void* ref;
    const void* sec;
    const uint8_t* valid;
    int64_t nrows, ncols;
    DevPoints pts;
    int64_t padx, pady;
    int up, measure;
    int CHM, CWM, NRM, NCM;
    int NB;                          // chip operand rows per column (multiple of 16)
    int BC;                          // chip columns per chunk
    int OB;                          // chip columns per window staging (multiple of BC)
    int LW;                          // window columns staged (OB + 63)
    int PC;                          // staged chip column length (elements, even)
    int NRS;                         // surface, box-sum and denominator row stride
    int AC;                          // columns per accumulator (multiple of 16)
    int RS;                          // row stride of a box-sum stripe's window columns (odd)
    int VS;                          // row stride of a stripe's column sums (nr + 1)
    int XS;                          // window columns per box-sum stripe
    unsigned off_S2, off_raw, off_V; // box-sum phase (S1 at 0)
    unsigned off_den, off_E, off_P, off_red;
    unsigned Eb, Pb;                 // bytes per chip-operand / staged-chip buffer
    uint32_t tmem_cols;
    DevOutputs out;
    int* sub_count;
    int64_t* sub_point;
    int32_t* sub_origin;
    float* sub_patch;
    float* surf_out;
    unsigned long long* flops;
    int* status;
};

// The three BF16 limbs of v, as raw 16-bit patterns: l[0] = bf16(v), l[1] = bf16(v - l[0]),
// l[2] = bf16(v - l[0] - l[1]). Each difference is exact in FP32 (its operands are within a
// factor of two of each other), and the last remainder has at most 8 significant bits, so
// v = l[0] + l[1] + l[2] for every normal v.
__device__ __forceinline__ void bf16_split3(float v, uint32_t (&l)[kBfLimbs]) {
    float r = v;
#pragma unroll
    for (int t = 0; t < kBfLimbs; ++t) {
        const __nv_bfloat16 h = __float2bfloat16_rn(r);
        l[t] = static_cast<uint32_t>(__bfloat16_as_ushort(h));
        r = __fsub_rn(r, __bfloat162float(h));
    }
}

template <typename T>
__global__ void __launch_bounds__(kBfThreads, 1) k_corr_bf(const BfArgs A) {
    typedef Traits<T> Tr;
    extern __shared__ __align__(1024) unsigned char smem_bf[];
    __shared__ uint64_t s_mbar[2];
    __shared__ uint32_t s_taddr;
    __shared__ int s_slot;
    const int tid = threadIdx.x, bd = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const T* ref = static_cast<const T*>(A.ref);
    const T* sec = static_cast<const T*>(A.sec);
    // Window limbs [limb][q][h][x] (16 bytes each) from offset 0, where the box-sum phase keeps
    // S1 and S2 [j][NRS] (FP64) and the epilogue the surface; the stripe buffers of the box sums
    // reach into the region of the denominators [j][NRS] (FP64), the two chip-operand buffers
    // [limb][b][h][e] and the two staged-chip buffers [limb][b][PC] (raw BF16 bits).
    unsigned char* s_W = smem_bf;
    double* s_S1 = reinterpret_cast<double*>(smem_bf);
    double* s_S2 = reinterpret_cast<double*>(smem_bf + A.off_S2);
    float* s_raw = reinterpret_cast<float*>(smem_bf + A.off_raw);
    double* s_V = reinterpret_cast<double*>(smem_bf + A.off_V);
    double* s_den = reinterpret_cast<double*>(smem_bf + A.off_den);
    unsigned char* s_E = smem_bf + A.off_E;
    unsigned char* s_Pb = smem_bf + A.off_P;
    double* s_red = reinterpret_cast<double*>(smem_bf + A.off_red);
    float* s_surf = reinterpret_cast<float*>(smem_bf);
    const size_t wlimb = static_cast<size_t>((A.CHM + A.NRM - 1 + 15) / 16) * 2 * A.LW * 16;
    const size_t elimb = static_cast<size_t>(A.BC) * 2 * A.NB * 16;
    const int plimb = A.BC * A.PC;
    const int64_t NR = A.nrows + 2 * A.pady, NC = A.ncols + 2 * A.padx;
    const double shx = static_cast<double>(A.padx) + 0.5;
    const double shy = static_cast<double>(A.pady) + 0.5;

    if (warp == 0) {
        tc::tmem_alloc(&s_taddr, A.tmem_cols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&s_mbar[0], kBfIssuers);  // one commit per issuer and chunk
        tc::mbar_init(&s_mbar[1], kBfIssuers);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = s_taddr;
    uint32_t ph[2] = {0u, 0u};
    bool pend[2] = {false, false};
    bool failed = false;
    TC_PHASE_INIT

    // Accumulator values of a thread after a chunk: value v is surface row
    // i = 32 half + 8 (v / 4) + 2 (lane % 4) + v % 2, column j = 16 quarter + lane / 4 (+ 8 when
    // v % 4 >= 2) -- the 16x256b read pattern of its lane quarter's half.
    const int quarter = warp & 3, half = warp >> 2;
    const uint32_t qbase = taddr + (static_cast<uint32_t>(32 * quarter) << 16) +
                           static_cast<uint32_t>(32 * half);
    // Zeros into this warp's lane quarter and half of the columns of set s's accumulators
    // (columns [32 half, 32 half + 32) of each, as far as the accumulator reaches): the warps
    // of the two halves together clear the set, each after reading its own values.
    auto clear_half = [&](int s) {
        uint32_t z[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) z[t] = 0u;
        const int c1 = min(32 * (half + 1), A.AC);
        for (int t = 0; t < kBfIssuers; ++t) {
            const uint32_t a0 = qbase - static_cast<uint32_t>(32 * half) +
                                static_cast<uint32_t>((kBfIssuers * s + t) * A.AC);
            for (int c = 32 * half; c < c1; c += 16) tc::tmem_st16(a0 + static_cast<uint32_t>(c), z);
        }
        tc::tmem_wait_st();
    };
    // Bounded wait for set s's products; on success the set is no longer pending.
    auto wait_set = [&](int s) -> bool {
        const bool ok = tc::mbar_wait(&s_mbar[s], ph[s], kTcWaitPolls);
        if (ok) {
            ph[s] ^= 1u;
            pend[s] = false;
        }
        return ok;
    };

    for (int64_t k = blockIdx.x; k < A.pts.n && !failed; k += gridDim.x) {
        tc::fence_before_sync();
        __syncthreads();  // the previous point's buffers and accumulators are no longer read
        tc::fence_after_sync();
        TC_PHASE(0)
        const int64_t prx = A.pts.rx[k], pry = A.pts.ry[k];
        if (!(prx > 0 && pry > 0)) continue;
        const double xs = A.pts.x[k] + shx, ys = A.pts.y[k] + shy;
        const int64_t hx = A.pts.csx[k] / 2, hy = A.pts.csy[k] / 2;
        const int64_t ccx = static_cast<int64_t>(floor(__dsub_rn(xs, A.pts.dx0[k])));
        const int64_t ccy = static_cast<int64_t>(floor(__dsub_rn(ys, A.pts.dy0[k])));
        const int64_t wcx = static_cast<int64_t>(floor(xs)), wcy = static_cast<int64_t>(floor(ys));
        const int64_t cr0 = ccy - hy, cr1 = ccy + hy - 1, cc0 = ccx - hx, cc1 = ccx + hx - 1;
        const int64_t wr0 = wcy - hy - pry, wr1 = wcy + hy + pry - 2;
        const int64_t wc0 = wcx - hx - prx, wc1 = wcx + hx + prx - 2;
        const bool chip_in = (cr1 < cr0 || cc1 < cc0) ||
                             (cr0 >= 1 && cr1 <= NR && cc0 >= 1 && cc1 <= NC);
        const bool win_in = (wr1 < wr0 || wc1 < wc0) ||
                            (wr0 >= 1 && wr1 <= NR && wc0 >= 1 && wc1 <= NC);
        if (!chip_in || !win_in) continue;
        const int ch = static_cast<int>(2 * hy), cw = static_cast<int>(2 * hx);
        const int nr = static_cast<int>(2 * pry), nc = static_cast<int>(2 * prx);
        if (ch <= 0 || cw <= 0) continue;
        if (ch > A.CHM || cw > A.CWM || nr > A.NRM || nc > A.NCM || nr > 64 || nc > 64) continue;
        const int64_t chip_r = cr0 - 1 - A.pady, chip_c = cc0 - 1 - A.padx;
        const int64_t win_r = wr0 - 1 - A.pady, win_c = wc0 - 1 - A.padx;
        const int nn_i = ch * cw;

        // _any_valid over the chip (src/track.jl:416-421).
        int any = 0;
        for (int e0 = tid; e0 < nn_i && !any; e0 += kBfBatch * bd) {
            uint8_t v[kBfBatch];
#pragma unroll
            for (int u = 0; u < kBfBatch; ++u) {
                const int e = e0 + u * bd;
                const int64_t r = chip_r + e % ch, c = chip_c + e / ch;
                v[u] = (e < nn_i && r >= 0 && r < A.nrows && c >= 0 && c < A.ncols)
                           ? A.valid[r + c * A.nrows] : static_cast<uint8_t>(0);
            }
#pragma unroll
            for (int u = 0; u < kBfBatch; ++u) any |= v[u] ? 1 : 0;
        }
        if (!__syncthreads_or(any)) continue;
        if (tid == 0) A.out.searched[k] = 1;
        TC_PHASE(1)

        // prepare_chip! as the CUDA-core kernel (the same per-thread order): FP64 mean, FP64 sum
        // of squares of the deviations, FP64 sum of the Float32-rounded deviations.
        double st[1] = {0.0};
        for (int e0 = tid; e0 < nn_i; e0 += kBfBatch * bd) {
            double v[kBfBatch];
#pragma unroll
            for (int u = 0; u < kBfBatch; ++u) {
                const int e = e0 + u * bd;
                v[u] = e < nn_i ? pixel(sec, A.nrows, A.ncols, chip_r + e % ch, chip_c + e / ch) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBfBatch; ++u)
                if (e0 + u * bd < nn_i) st[0] = __dadd_rn(st[0], v[u]);
        }
        block_sum_f64<1>(st, s_red);
        const double nn = static_cast<double>(nn_i);
        const double mean = __ddiv_rn(st[0], nn);
        const int chp = (ch + kUA - 1) & ~(kUA - 1);
        double acc2[2] = {0.0, 0.0};
        for (int e0 = tid; e0 < chp * cw; e0 += kBfBatch * bd) {
            double v[kBfBatch];
#pragma unroll
            for (int u = 0; u < kBfBatch; ++u) {
                const int e = e0 + u * bd, a = e % chp, b = e / chp;
                v[u] = (e < chp * cw && a < ch) ? pixel(sec, A.nrows, A.ncols, chip_r + a, chip_c + b) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBfBatch; ++u) {
                const int e = e0 + u * bd;
                if (e < chp * cw && e % chp < ch) {
                    const double d = __dsub_rn(v[u], mean);
                    acc2[0] = __dadd_rn(acc2[0], __dmul_rn(d, d));
                    acc2[1] = __dadd_rn(acc2[1], static_cast<double>(__double2float_rn(d)));
                }
            }
        }
        block_sum_f64<2>(acc2, s_red);
        const double sq = acc2[0], sumd = acc2[1];
        if (!(sq > __dmul_rn(__dmul_rn(DBL_EPSILON, static_cast<double>(ch)), static_cast<double>(cw))))
            continue;  // degenerate chip: searched, no measurement (src/track.jl:286)
        const double cnorm = __dsqrt_rn(sq);
        const double cshift = Tr::integer ? rint(mean) : static_cast<double>(__double2float_rn(mean));
        const float csf = static_cast<float>(cshift);
        if (tid == 0 && !(A.up == 1 || nr < 5 || nc < 5)) s_slot = atomicAdd(A.sub_count, 1);
        TC_PHASE(2)

        // Box sums in FP64, a stripe of window columns at a time: the stripe's image values
        // (exact in FP32 for every element type), its column sums V(i, x) of ch rows, then the
        // running sum Q along each surface row i (a thread per row and sum): the box sum at column
        // j is Q after window column j + cw - 1 less Q before column j.
        const int RW = ch + nr - 1, XW = cw + nc - 1;
        double qrun = 0.0;
        for (int x0 = 0; x0 < XW; x0 += A.XS) {
            const int xn = min(A.XS, XW - x0);
            for (int e0 = tid; e0 < xn * RW; e0 += kBfBatch * bd) {
                double v[kBfBatch];
#pragma unroll
                for (int u = 0; u < kBfBatch; ++u) {
                    const int e = e0 + u * bd;
                    v[u] = e < xn * RW ? pixel(ref, A.nrows, A.ncols, win_r + e % RW, win_c + x0 + e / RW) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kBfBatch; ++u) {
                    const int e = e0 + u * bd;
                    if (e < xn * RW) s_raw[(e / RW) * A.RS + e % RW] = static_cast<float>(v[u]);
                }
            }
            __syncthreads();
            TC_PHASE(3)
            {
                const int segs = max(1, min(nr, bd / xn));
                const int len = (nr + segs - 1) / segs;
                for (int t = tid; t < xn * segs; t += bd) {
                    const int x = t % xn, i0 = (t / xn) * len, i1 = min(nr, i0 + len);
                    if (i0 >= i1) continue;
                    const float* col = s_raw + x * A.RS;
                    double h1 = 0.0, h2 = 0.0;
                    for (int a = i0; a < i0 + ch; ++a) {
                        const double w = static_cast<double>(col[a]);
                        h1 = __dadd_rn(h1, w);
                        h2 = __dadd_rn(h2, __dmul_rn(w, w));
                    }
                    for (int i = i0; i < i1; ++i) {
                        s_V[2 * (x * A.VS + i)] = h1;
                        s_V[2 * (x * A.VS + i) + 1] = h2;
                        if (i + 1 < i1) {
                            const double wo = static_cast<double>(col[i]);
                            const double wn = static_cast<double>(col[i + ch]);
                            h1 = __dadd_rn(__dsub_rn(h1, wo), wn);
                            h2 = __dadd_rn(__dsub_rn(h2, __dmul_rn(wo, wo)), __dmul_rn(wn, wn));
                        }
                    }
                }
            }
            __syncthreads();
            TC_PHASE(4)
            if (tid < 2 * nr) {
                const int i = tid >> 1, comp = tid & 1;
                double* S = comp ? s_S2 : s_S1;
                for (int x = 0; x < xn; ++x) {
                    const int xg = x0 + x;
                    if (xg < nc) S[xg * A.NRS + i] = qrun;
                    qrun = __dadd_rn(qrun, s_V[2 * (x * A.VS + i) + comp]);
                    const int j = xg - cw + 1;
                    if (j >= 0 && j < nc) S[j * A.NRS + i] = __dsub_rn(qrun, S[j * A.NRS + i]);
                }
            }
            __syncthreads();
            TC_PHASE(5)
        }
        TC_PHASE(5)
        // FP64 denominators (src/correlate.jl:591-600, 624-628).
        for (int e = tid; e < nr * nc; e += bd) {
            const int i = e % nr, j = e / nr;
            const double s1 = s_S1[j * A.NRS + i], s2 = s_S2[j * A.NRS + i];
            double den;
            if (A.measure == AR_NCC) {
                den = __dmul_rn(cnorm, __dsqrt_rn(s2 > 0.0 ? s2 : 0.0));
            } else {
                double wvar = __dsub_rn(s2, __ddiv_rn(__dmul_rn(s1, s1), nn));
                if (!(wvar > 0.0)) wvar = 0.0;
                den = __dmul_rn(cnorm, __dsqrt_rn(wvar));
            }
            s_den[j * A.NRS + i] = den;
        }
        clear_half(0);
        clear_half(1);
        __syncthreads();  // S1 and S2 read before the window limbs replace them
        TC_PHASE(6)

        double accd[16];
#pragma unroll
        for (int v = 0; v < 16; ++v) accd[v] = 0.0;
        auto flush_set = [&](int s) {
            if (32 * half < nr) {
                uint32_t r[kBfIssuers][16];
#pragma unroll
                for (int t = 0; t < kBfIssuers; ++t)
                    tc::tmem_ld16dp(qbase + static_cast<uint32_t>((kBfIssuers * s + t) * A.AC), r[t]);
                tc::tmem_wait_ld();
#pragma unroll
                for (int v = 0; v < 16; ++v)
#pragma unroll
                    for (int t = 0; t < kBfIssuers; ++t)
                        accd[v] = __dadd_rn(accd[v], static_cast<double>(__uint_as_float(r[t][v])));
            }
        };
        // A chunk's chip columns C'[a, b0 + bl] as BF16 limbs, zero-padded: the loads first
        // (into registers), the conversion after other work.
        auto p_load = [&](int b0, int bcn, double (&pr)[kBfPre], int t0, int nt) {
#pragma unroll
            for (int u = 0; u < kBfPre; ++u) {
                const int e = (tid - t0) + u * nt;
                const int bl = e / A.PC, a = e - bl * A.PC - kBfPadL;
                pr[u] = (e < plimb && bl < bcn && a >= 0 && a < ch)
                            ? pixel(sec, A.nrows, A.ncols, chip_r + a, chip_c + b0 + bl) : 0.0;
            }
        };
        auto p_store = [&](int buf, int bcn, const double (&pr)[kBfPre], int t0, int nt) {
            uint16_t* P = reinterpret_cast<uint16_t*>(s_Pb + buf * A.Pb);
#pragma unroll
            for (int u = 0; u < kBfPre; ++u) {
                const int e = (tid - t0) + u * nt;
                if (e < plimb) {
                    const int bl = e / A.PC, a = e - bl * A.PC - kBfPadL;
                    uint32_t l[kBfLimbs] = {0u, 0u, 0u};
                    if (bl < bcn && a >= 0 && a < ch) bf16_split3(__double2float_rn(__dsub_rn(pr[u], mean)), l);
#pragma unroll
                    for (int limb = 0; limb < kBfLimbs; ++limb) P[limb * plimb + e] = static_cast<uint16_t>(l[limb]);
                }
            }
        };

        const int QBp = (ch + nr - 1 + 15) / 16;
        const int gp = 2 * QBp;  // 8-row groups per window column
        bool ok = true;
        for (int ob0 = 0; ob0 < cw && ok; ob0 += A.OB) {
            const int obn = min(A.OB, cw - ob0);
            const int xneed = obn + nc - 1;
            // Window limbs of columns ob0 .. ob0 + LW - 1 (zero past the columns and rows the
            // valid surface values read): item (x, q, h) = 8 consecutive rows of column x,
            // consecutive threads on consecutive row groups of one column; two items' loads at once.
            const int items = A.LW * gp;
            for (int it0 = tid; it0 < items; it0 += 2 * bd) {
                float wv[2][8];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int it = it0 + u * bd;
                    const int x = it / gp, g = it - x * gp;
                    const int r0 = 8 * g;  // 16 q + 8 h
#pragma unroll
                    for (int t = 0; t < 8; ++t)
                        wv[u][t] = (it < items && x < xneed && r0 + t < RW)
                                       ? static_cast<float>(pixel(ref, A.nrows, A.ncols, win_r + r0 + t, win_c + ob0 + x))
                                       : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int it = it0 + u * bd;
                    if (it < items) {
                        const int x = it / gp, g = it - x * gp;
                        const int r0 = 8 * g;
                        uint32_t lw[kBfLimbs][4] = {};
#pragma unroll
                        for (int t = 0; t < 8; ++t) {
                            uint32_t l[kBfLimbs] = {0u, 0u, 0u};
                            if (x < xneed && r0 + t < RW) bf16_split3(__fsub_rn(wv[u][t], csf), l);
#pragma unroll
                            for (int limb = 0; limb < kBfLimbs; ++limb) lw[limb][t >> 1] |= l[limb] << (16 * (t & 1));
                        }
                        const size_t o = (static_cast<size_t>(g) * A.LW + x) * 16;
#pragma unroll
                        for (int limb = 0; limb < kBfLimbs; ++limb)
                            *reinterpret_cast<uint4*>(s_W + limb * wlimb + o) =
                                make_uint4(lw[limb][0], lw[limb][1], lw[limb][2], lw[limb][3]);
                    }
                }
            }
            // Chip operand rows for the chunk in buffer `buf` (threads [t0, t0 + nt)):
            // E_b[h][e] = 8 elements of the staged column from element kBfPadL + 8 h - e + NB - 16
            // (C'[r - u, b] with u = e - NB + 16, r = 8 h + t).
            auto build_E = [&](int buf, int t0, int nt) {
                const uint16_t* P = reinterpret_cast<const uint16_t*>(s_Pb + buf * A.Pb);
                unsigned char* E = s_E + buf * A.Eb;
                for (int it = tid - t0; it < A.BC * 2 * A.NB; it += nt) {
                    const int bl = it / (2 * A.NB), rem = it - bl * 2 * A.NB;
                    const int h = rem / A.NB, e = rem - h * A.NB;
                    const int src = kBfPadL + 8 * h - e + A.NB - 16;  // element index, >= 1
                    const size_t o = (static_cast<size_t>(bl * 2 + h) * A.NB + e) * 16;
#pragma unroll
                    for (int limb = 0; limb < kBfLimbs; ++limb) {
                        const uint16_t* col = P + limb * plimb + bl * A.PC;
                        const uint32_t* w = reinterpret_cast<const uint32_t*>(col + (src & ~1));
                        const uint32_t sh = (src & 1) ? 16u : 0u;
                        uint4 v;
                        v.x = __funnelshift_r(w[0], w[1], sh);
                        v.y = __funnelshift_r(w[1], w[2], sh);
                        v.z = __funnelshift_r(w[2], w[3], sh);
                        v.w = __funnelshift_r(w[3], w[4], sh);
                        *reinterpret_cast<uint4*>(E + limb * elimb + o) = v;
                    }
                }
            };
            const int nch = (obn + A.BC - 1) / A.BC;
            auto chunk_b0 = [&](int c) { return ob0 + c * A.BC; };
            auto chunk_n = [&](int c) { return min(A.BC, ob0 + obn - chunk_b0(c)); };
            // Chunk 0's chip columns and operand, chunk 1's chip columns, by every thread.
            {
                double pr[kBfPre];
                p_load(chunk_b0(0), chunk_n(0), pr, 0, bd);
                p_store(0, chunk_n(0), pr, 0, bd);
                __syncthreads();
                build_E(0, 0, bd);
                if (nch > 1) {
                    p_load(chunk_b0(1), chunk_n(1), pr, 0, bd);
                    p_store(1, chunk_n(1), pr, 0, bd);
                }
            }
            tc::fence_proxy_async_smem();
            tc::fence_before_sync();
            __syncthreads();  // limbs, chunk 0's operand and chunk 1's chip columns complete
            TC_PHASE(7)

            // Chunk c: lane 0 of warps 0-3 issue its products into set c & 1 while warps 4-7 take
            // chunk c - 1's values out of set c & 1 ^ 1 (their half of the columns), build chunk
            // c + 1's operand into the buffer chunk c - 1 used and stage chunk c + 2's chip
            // columns; warps 0-3 then take their half of chunk c - 1's values. One barrier per
            // chunk: set c & 1 ^ 1 is clear and chunk c + 1's operand complete after it.
            for (int c = 0; c < nch && ok; ++c) {
                const int s = c & 1;
                const int b0 = chunk_b0(c), bcn = chunk_n(c);
                bool okc = true;
                if (warp < kBfIssuers) {
                    // Lane 0 of warps 0-3 issue the chunk's products, each into an accumulator of
                    // its own (one thread issues a product about every 120 cycles; four keep the
                    // tensor core busy): issuer t takes the window blocks q of parity t & 1 and
                    // the limb pairs (chip, window) (0,0), (1,1), (2,0) when t < 2, else (0,1),
                    // (1,0), (0,2) (integer windows have no third limb).
                    if (lane == 0) {
                        tc::fence_after_sync();
                        const uint32_t wb = tc::smem_u32(s_W);
                        const uint32_t eb = tc::smem_u32(s_E) + static_cast<uint32_t>(s * A.Eb);
                        const int par = warp & 1;
                        const uint32_t dacc = taddr + static_cast<uint32_t>((kBfIssuers * s + warp) * A.AC);
#pragma unroll 1
                        for (int pp = 0; pp < 3; ++pp) {
                            const int cl = warp < 2 ? pp : (pp == 1 ? 1 : 0);
                            const int wl = warp < 2 ? (pp == 1 ? 1 : 0) : (pp == 0 ? 1 : pp == 2 ? 2 : 0);
                            if (Tr::integer && wl == 2) continue;
                            const uint64_t da0 = tc::smem_desc(wb + static_cast<uint32_t>(wl * wlimb),
                                                               static_cast<uint32_t>(A.LW * 16), 128);
                            const uint64_t db0 = tc::smem_desc(eb + static_cast<uint32_t>(cl * elimb),
                                                               static_cast<uint32_t>(A.NB * 16), 128);
                            const uint32_t a_hi = static_cast<uint32_t>(da0 >> 32);
                            const uint32_t b_hi = static_cast<uint32_t>(db0 >> 32);
                            for (int q = par; q < QBp; q += 2) {
                                int elo, n;
                                if (!block_rows(q, A.NB, nr, &elo, &n)) continue;
                                const uint32_t idesc = tc::idesc_bf16_f32(64, n);
                                const uint32_t dcol = static_cast<uint32_t>(16 * q + elo - (A.NB - 16));
                                for (int bl = 0; bl < bcn; ++bl) {
                                    // A: block q, first half, window column x = b0 - ob0 + bl.
                                    const uint32_t a_lo = static_cast<uint32_t>(da0) +
                                                          static_cast<uint32_t>((q * 2) * A.LW + (b0 - ob0) + bl);
                                    const uint32_t b_lo = static_cast<uint32_t>(db0) +
                                                          static_cast<uint32_t>((bl * 2) * A.NB + elo);
                                    tc::mma_bf16_halves(dacc + dcol, a_lo, a_hi, b_lo, b_hi, idesc, 1u);
                                }
                            }
                        }
                        tc::mma_commit(&s_mbar[s]);
                    }
                    __syncwarp();
                    TC_PHASE(9)
                    if (c >= 1) {
                        okc = tc::mbar_wait(&s_mbar[s ^ 1], ph[s ^ 1], kTcWaitPolls);
                        if (okc) {
                            tc::fence_after_sync();
                            flush_set(s ^ 1);
                            clear_half(s ^ 1);
                        }
                    }
                } else {
                    // Chunk c + 2's chip columns are loaded first and converted last, so the
                    // loads are in flight through the wait, the flush and the operand build.
                    const bool stage = c + 2 < nch;
                    double pr[kBfPre];
                    if (stage) p_load(chunk_b0(c + 2), chunk_n(c + 2), pr, 32 * kBfIssuers, bd - 32 * kBfIssuers);
                    if (c >= 1) {
                        okc = tc::mbar_wait(&s_mbar[s ^ 1], ph[s ^ 1], kTcWaitPolls);
                        if (okc) {
                            tc::fence_after_sync();
                            flush_set(s ^ 1);
                            clear_half(s ^ 1);
                        }
                    }
                    if (okc && c + 1 < nch) build_E(s ^ 1, 32 * kBfIssuers, bd - 32 * kBfIssuers);
                    if (okc && stage) p_store(s, chunk_n(c + 2), pr, 32 * kBfIssuers, bd - 32 * kBfIssuers);
                }
                pend[s] = true;
                tc::fence_proxy_async_smem();
                tc::fence_before_sync();
                if (__syncthreads_or(!okc)) {
                    ok = false;
                    break;
                }
                if (c >= 1) {
                    ph[s ^ 1] ^= 1u;
                    pend[s ^ 1] = false;
                }
                TC_PHASE(8)
            }
            if (ok) {
                // The last chunk's values; each warp clears its half of the set.
                const int sl = (nch - 1) & 1;
                ok = wait_set(sl);
                if (__syncthreads_or(!ok)) {
                    ok = false;
                } else {
                    tc::fence_after_sync();
                    flush_set(sl);
                    clear_half(sl);
                    tc::fence_before_sync();
                    __syncthreads();  // the window limbs are replaced next
                }
            }
            TC_PHASE(8)
        }
        if (!ok) {
            if (tid == 0) atomicExch(A.status, 1);
            failed = true;
            break;
        }

        // Epilogue: every value normalised in FP64 into the surface in shared memory.
        {
            const int ib0 = 32 * half + 2 * (lane & 3);
            const int jb0 = 16 * quarter + (lane >> 2);
            if (32 * half < nr) {
#pragma unroll
                for (int v = 0; v < 16; ++v) {
                    const int i = ib0 + 8 * (v >> 2) + (v & 1), j = jb0 + ((v & 2) ? 8 : 0);
                    if (i < nr && j < nc) {
                        const double num = __dadd_rn(accd[v], __dmul_rn(cshift, sumd));
                        const double den = s_den[j * A.NRS + i];
                        s_surf[j * A.NRS + i] = den > 0.0 ? __double2float_rn(__ddiv_rn(num, den)) : 0.0f;
                    }
                }
            }
        }
        __syncthreads();
        TC_PHASE(10)
        if (A.flops && tid == 0)
            atomicAdd(A.flops, 2ull * static_cast<unsigned long long>(ch) * cw * nr * nc);
        // Integer peak (src/peak.jl:32-61).
        unsigned long long key = 0ull;
        for (int e = tid; e < nr * nc; e += bd) {
            const int i = e % nr, j = e / nr;
            const unsigned long long kk = argmax_key(s_surf[j * A.NRS + i], static_cast<unsigned>(i * nc + j));
            key = kk > key ? kk : key;
        }
        key = block_max_u64(key, reinterpret_cast<unsigned long long*>(s_red));
        if (A.surf_out) {
            float* so = A.surf_out + k * static_cast<int64_t>(A.NRM) * A.NCM;
            for (int e = tid; e < nr * nc; e += bd) so[e] = s_surf[(e / nr) * A.NRS + (e % nr)];
        }
        unsigned rm = 0;
        float pv = 0.0f;
        int pi = 0, pj = 0;
        if (key_decode(key, &rm, &pv)) {
            pi = static_cast<int>(rm / nc);
            pj = static_cast<int>(rm % nc);
        }
        if (A.up == 1 || nr < 5 || nc < 5) {
            if (tid == 0) {
                A.out.dx[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pj - static_cast<int>(prx)), A.pts.dx0[k]));
                A.out.dy[k] = __double2float_rn(
                    __dadd_rn(static_cast<double>(pi - static_cast<int>(pry)), A.pts.dy0[k]));
                A.out.corr[k] = s_surf[pj * A.NRS + pi];
            }
        } else {
            const int pi0 = min(max(pi - 2, 0), max(nr - 5, 0));
            const int pj0 = min(max(pj - 2, 0), max(nc - 5, 0));
            const int slot = s_slot;
            if (tid < 25) {
                const int a = tid % 5, b = tid / 5;
                A.sub_patch[static_cast<int64_t>(slot) * 25 + tid] = s_surf[(pj0 + b) * A.NRS + (pi0 + a)];
            }
            if (tid == 0) {
                A.sub_point[slot] = k;
                A.sub_origin[2 * slot] = pi0;
                A.sub_origin[2 * slot + 1] = pj0;
            }
        }
        TC_PHASE(11)
        TC_PHASE_POINT
    }
    TC_PHASE_FLUSH
    // Products still in flight after a failed wait finish before their columns are freed.
    for (int s = 0; s < 2; ++s)
        if (pend[s]) tc::mbar_wait(&s_mbar[s], ph[s], kTcWaitPolls);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, A.tmem_cols);
}

// ----------------------------------------------------------------------------------------------
// Sub-pixel cascade kernel (src/peak.jl:456-522 from the patch onward), one warp per patch.
//
// Levels 1 and 2 of the cascade (10^2, 20^2) are materialised in the warp's shared memory. Up to
// 8x the final level is materialised too. Beyond, the final level is cut into 16 x 16 blocks and
// a block's samples are computed through its dependency cone only: the rows and columns of each
// coarser level its taps reach, down to level 2. Every pyrUp sample is a rounded convex
// combination of its taps, so no sample of a block exceeds the largest level-2 sample of its
// cone by more than the accumulated rounding (bounded by k * 2^-20 * max|level 2| over k
// levels). Blocks are visited in decreasing order of that bound; a visited block is first
// carried to level L - 2, where the largest cone sample gives a tighter two-level bound, and is
// finished only if that bound still reaches the best value found. The search ends when the best
// remaining bound is strictly below the best value, so the result (value and row-major-first
// position) is exactly the full cascade's: each computed sample is the same function of the same
// inputs as in the full cascade.

constexpr int kRefineWarps = 8;
constexpr int kFB = 16;  // final-level block side

struct RefineArgs {
    const int* count;       // device count of queued items (or null: use n_items)
    int64_t n_items;
    const int64_t* point;   // point index per item (null for bare patches)
    const int32_t* origin;  // patch origin per item (null for bare patches)
    const float* patch;     // 25 floats per item
    DevPoints pts;
    DevOutputs out;
    int32_t* orow;          // bare-patch outputs (when point is null)
    int32_t* ocol;
    float* oval;
    int levels;             // log2(upsampling) >= 1
    int warp_floats;        // shared floats per warp
};

// Taps of output position p on an axis whose source has n >= 2 samples: the closed form of
// src/peak.jl:312-324 (reflection in upsampled space only ever folds the first sample's minus
// tap onto sample 1 and the last samples' plus tap onto sample n-1).
__device__ __forceinline__ int taps(int p, int n, int& m, int& c, int& q) {
    c = p >> 1;
    q = min(c + 1, n - 1);
    if (p & 1) {
        m = c;
        return 2;
    }
    m = c == 0 ? 1 : c - 1;
    return 3;
}

// Source index range [lo, hi] the taps of outputs [p0, p1] read (source size n).
__device__ __forceinline__ void tap_range(int p0, int p1, int n, int& lo, int& hi) {
    lo = (p0 & 1) ? (p0 >> 1) : max((p0 >> 1) - 1, 0);
    hi = min((p1 >> 1) + 1, n - 1);
}

// One full pyrUp step by a warp: src (S x S, column-major) -> dst (2S x 2S) via tmp (2S x S).
// Vertical then horizontal, as src/peak.jl:261-292. Outputs 2c and 2c + 1 of an axis read the
// same source samples (c - 1, or 1 at the edge; c; c + 1, clamped), so each lane produces such a
// pair from three loads: `taps` in closed form, with the same rounded operations per sample.
// `tmp` must be 8-byte aligned.
template <int S>
__device__ void pyrup_warp(const float* src, float* dst, float* tmp) {
    const int lane = threadIdx.x & 31;
    constexpr int D = 2 * S;
    for (int e = lane; e < S * S; e += 32) {
        const int c = e % S, j = e / S;
        const int m = c == 0 ? 1 : c - 1, q = min(c + 1, S - 1);
        const float* s = src + j * S;
        const float a = s[m], b = s[c], d = s[q];
        float2 v;
        v.x = pyr_sample(3, a, b, d);
        v.y = pyr_sample(2, b, b, d);
        *reinterpret_cast<float2*>(tmp + 2 * c + j * D) = v;
    }
    __syncwarp();
    for (int e = lane; e < D * S; e += 32) {
        const int i = e % D, c = e / D;
        const int m = c == 0 ? 1 : c - 1, q = min(c + 1, S - 1);
        const float a = tmp[i + m * D], b = tmp[i + c * D], d = tmp[i + q * D];
        dst[i + 2 * c * D] = pyr_sample(3, a, b, d);
        dst[i + (2 * c + 1) * D] = pyr_sample(2, b, b, d);
    }
    __syncwarp();
}

// (value, row-major index) pairs: larger value wins, equal values go to the smaller index;
// NaN never wins.
__device__ __forceinline__ void best_update(float v, int idx, float& bv, int& bi) {
    if (v > bv || (v == bv && idx < bi)) {
        bv = v;
        bi = idx;
    }
}

__device__ __forceinline__ void warp_best(float& bv, int& bi) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(kFull, bv, o);
        const int i2 = __shfl_xor_sync(kFull, bi, o);
        best_update(v2, i2, bv, bi);
    }
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// A cone level: rows [r0, r1] and columns [c0, c1] of a level of size n.
struct ConeLevel {
    int r0, r1, c0, c1;
};

// Level region `dst` (rows d.r0..d.r1, columns d.c0..d.c1) of a level computed from the source
// region `s` of the level below (size n), stored column-major from its first element with
// leading dimension lds; tmp holds the vertical pass (dst rows x source columns). Regions have
// at most 16 rows: the warp splits into 32 / rows groups of `rows` lanes, each group taking
// every (32 / rows)-th column.
__device__ void cone_step(const float* src, int lds, const ConeLevel& s, int n,
                          const ConeLevel& d, float* tmp, float* dst) {
    const int lane = threadIdx.x & 31;
    const int rows = d.r1 - d.r0 + 1, scols = s.c1 - s.c0 + 1;
    const int groups = 32 / rows;
    const int cpar = lane / rows, r = lane - cpar * rows;
    const bool active = cpar < groups;
    if (active) {
        int m, c, q;
        const int nt = taps(d.r0 + r, n, m, c, q);
        m -= s.r0;
        c -= s.r0;
        q -= s.r0;
        for (int cc = cpar; cc < scols; cc += groups) {
            const float* col = src + cc * lds;
            tmp[r + cc * rows] = pyr_sample(nt, col[m], col[c], col[q]);
        }
    }
    __syncwarp();
    if (active) {
        for (int cc = cpar; cc <= d.c1 - d.c0; cc += groups) {
            int m, c, q;
            const int nt = taps(d.c0 + cc, n, m, c, q);
            dst[r + cc * rows] = pyr_sample(nt, tmp[r + (m - s.c0) * rows],
                                            tmp[r + (c - s.c0) * rows], tmp[r + (q - s.c0) * rows]);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kRefineWarps * 32) k_refine(const RefineArgs A) {
    extern __shared__ __align__(16) float rsm[];
    // Level-3 rows (or columns) each final block row (or column) reaches, shared by the CTA.
    __shared__ int s_rlo[64], s_rhi[64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const int L = A.levels;
    float* W = rsm + warp * A.warp_floats;
    // Per-warp layout. Up to 8x: the patch, levels 1 and 2, then the pyrUp scratch and level 3.
    // Beyond: level 3 (1600 floats), then a scratch that first holds the patch, levels 1 and 2
    // and the pyrUp temporaries, and after level 3 is built the block bounds, the level-3 row
    // maxima and the cone buffers (regions that are never live at the same time overlap).
    float *P0, *L1, *L2, *WK, *T5, *T10, *T20, *L3, *B;
    if (L <= 3) {
        P0 = W;
        L1 = W + 32;
        L2 = L1 + 100;
        WK = L2 + 400;
        T5 = T10 = T20 = WK;
        L3 = WK + 800;
        B = nullptr;
    } else {
        L3 = W;
        B = W + 1600;
        L2 = B;          // [0, 400)
        T20 = B + 400;   // [400, 1200): the 40 x 20 vertical pass of level 3
        T10 = B + 400;   // [400, 600)
        L1 = B + 1000;   // [1000, 1100)
        P0 = B + 1100;   // [1100, 1125)
        T5 = B + 400;    // [400, 450)
        WK = nullptr;
        const int nb = (5 << L) / kFB;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            int lo = b * kFB, hi = lo + kFB - 1;
            for (int lev = L - 1; lev >= 3; --lev) {
                int a2, b2;
                tap_range(lo, hi, 5 << lev, a2, b2);
                lo = a2;
                hi = b2;
            }
            s_rlo[b] = lo;
            s_rhi[b] = hi;
        }
        __syncthreads();
    }
    const int64_t count = A.count ? static_cast<int64_t>(*A.count) : A.n_items;
    for (int64_t item = static_cast<int64_t>(blockIdx.x) * warps + warp; item < count;
         item += static_cast<int64_t>(gridDim.x) * warps) {
        if (lane < 25) P0[lane] = A.patch[item * 25 + lane];
        __syncwarp();
        float bv = -INFINITY;
        int bi = INT_MAX;
        int nfinal = 5 << L;
        float v0 = 0.0f;  // the final level's first sample, reported when nothing beats -Inf
        if (L <= 3) {
            // Materialise every level; argmax of the last.
            const float* fin;
            if (L == 1) {
                pyrup_warp<5>(P0, L1, T5);
                fin = L1;
            } else {
                pyrup_warp<5>(P0, L1, T5);
                pyrup_warp<10>(L1, L2, T10);
                fin = L2;
                if (L == 3) {
                    pyrup_warp<20>(L2, L3, T20);
                    fin = L3;
                }
            }
            for (int e = lane; e < nfinal * nfinal; e += 32) {
                const int i = e % nfinal, j = e / nfinal;
                best_update(fin[e], i * nfinal + j, bv, bi);
            }
            warp_best(bv, bi);
            v0 = fin[0];
        } else {
            // Levels 1-3 materialised (level 3 is 40 x 40), then the block search above them.
            const int nb = nfinal / kFB;      // blocks per side
            float* BND = B;                   // nb * nb bounds (over level 2, once it is read)
            float* CB = BND + nb * nb;        // row maxima, then cone buffers
            float* RM = CB;                   // level-3 row maxima per block column (40 * nb)
            pyrup_warp<5>(P0, L1, T5);
            pyrup_warp<10>(L1, L2, T10);
            pyrup_warp<20>(L2, L3, T20);
            // Scale of the rounding slack: the largest magnitude of level 2 bounds every later
            // level's (up to the growth of rounding itself, covered by the factor 2).
            float amax = 0.0f;
            for (int e = lane; e < 400; e += 32) amax = fmaxf(amax, fabsf(L2[e]));
            amax = warp_max(amax);
            const float ulp_scale = amax * 9.5367431640625e-07f;  // 2^-20 * max|level 2|
            auto slack = [&](int k) { return k * ulp_scale + k * 2.3509887e-38f; };
            // Cone buffer offsets per level distance d = L - level (regions <= 16, 10, 7, 6 rows
            // for d = 0 .. L - 4, the levels above the materialised level 3).
            const int cap[6] = {16, 10, 7, 6, 5, 5};
            int roff[6], toff[6], off = 0;
            for (int d = 0; d <= L - 4; ++d) {
                roff[d] = off;
                off += cap[d] * cap[d];
                toff[d] = off;
                off += cap[d] * cap[d + 1];
            }
            __syncwarp();  // level 2 is read; its space takes the bounds
            // Loose bound of every final block: its level-3 cone maximum plus L - 3 levels of
            // slack, as row maxima over each block column's range (s_rlo/s_rhi), then maxima
            // over row ranges.
            for (int e = lane; e < 40 * nb; e += 32) {
                const int i = e % 40, bj_ = e / 40;
                const int c0 = s_rlo[bj_], c1 = s_rhi[bj_];
                float mx = -INFINITY;
                for (int j = c0; j <= c1; ++j) mx = fmaxf(mx, L3[i + j * 40]);
                RM[e] = mx;
            }
            __syncwarp();
            {
                int bi_ = lane % nb, bj_ = lane / nb;  // block lane + 32 t, column-major
                const int di = 32 % nb, dj = 32 / nb;
                for (int blk = lane; blk < nb * nb; blk += 32) {
                    const int r0 = s_rlo[bi_], r1 = s_rhi[bi_];
                    float mx = -INFINITY;
                    for (int i = r0; i <= r1; ++i) mx = fmaxf(mx, RM[i + bj_ * 40]);
                    BND[blk] = mx + slack(L - 3);
                    bi_ += di;
                    bj_ += dj;
                    if (bi_ >= nb) {
                        bi_ -= nb;
                        ++bj_;
                    }
                }
            }
            __syncwarp();
            while (true) {
                // The unvisited block with the largest bound (lowest index on ties).
                float m = -INFINITY;
                int sel = INT_MAX;
                for (int b = lane; b < nb * nb; b += 32) {
                    const float v = BND[b];
                    if (v > m || (v == m && b < sel)) {
                        m = v;
                        sel = b;
                    }
                }
                warp_best(m, sel);
                if (sel == INT_MAX || m == -INFINITY || m < bv) break;
                __syncwarp();
                if (lane == 0) BND[sel] = -INFINITY;
                // The block's cone, from the final level down to level 3.
                ConeLevel cl[8];
                {
                    const int bi_ = sel % nb, bj_ = sel / nb;
                    cl[0] = {bi_ * kFB, bi_ * kFB + kFB - 1, bj_ * kFB, bj_ * kFB + kFB - 1};
                    for (int d = 1; d <= L - 3; ++d) {
                        const int n = 5 << (L - d);
                        tap_range(cl[d - 1].r0, cl[d - 1].r1, n, cl[d].r0, cl[d].r1);
                        tap_range(cl[d - 1].c0, cl[d - 1].c1, n, cl[d].c0, cl[d].c1);
                    }
                }
                // Levels 4 .. L - 1 (d = L - 4 .. 1) into the cone buffers; at level L - 2 (when
                // it is above level 3) the tighter two-level bound.
                ConeLevel sreg = cl[L - 3];
                const float* src = L3 + sreg.r0 + sreg.c0 * 40;
                int lds = 40;
                bool pruned = false;
                for (int d = L - 4; d >= 1; --d) {
                    const int n = 5 << (L - d - 1);  // source level size
                    float* dst = CB + roff[d];
                    cone_step(src, lds, sreg, n, cl[d], CB + toff[d], dst);
                    src = dst;
                    sreg = cl[d];
                    lds = cl[d].r1 - cl[d].r0 + 1;
                    if (d == 2) {
                        const int cnt = (cl[2].r1 - cl[2].r0 + 1) * (cl[2].c1 - cl[2].c0 + 1);
                        float mx = -INFINITY;
                        for (int e = lane; e < cnt; e += 32) mx = fmaxf(mx, dst[e]);
                        mx = warp_max(mx);
                        if (mx + slack(2) < bv) {
                            pruned = true;
                            break;
                        }
                    }
                }
                if (pruned) continue;
                // The final level: vertical pass, then each sample into the running best.
                {
                    const int n = 5 << (L - 1);
                    const ConeLevel& dl = cl[0];
                    float* tmp = CB + toff[0];
                    const int r = lane & 15, cpar = lane >> 4;
                    const int scols = sreg.c1 - sreg.c0 + 1;
                    {
                        int m2, c2, q2;
                        const int nt = taps(dl.r0 + r, n, m2, c2, q2);
                        m2 -= sreg.r0;
                        c2 -= sreg.r0;
                        q2 -= sreg.r0;
                        for (int cc = cpar; cc < scols; cc += 2) {
                            const float* col = src + cc * lds;
                            tmp[r + cc * kFB] = pyr_sample(nt, col[m2], col[c2], col[q2]);
                        }
                    }
                    __syncwarp();
                    float lv = -INFINITY;
                    int li = INT_MAX;
                    for (int cc = cpar; cc < kFB; cc += 2) {
                        int m2, c2, q2;
                        const int col = dl.c0 + cc;
                        const int nt = taps(col, n, m2, c2, q2);
                        const float v = pyr_sample(nt, tmp[r + (m2 - sreg.c0) * kFB],
                                                   tmp[r + (c2 - sreg.c0) * kFB],
                                                   tmp[r + (q2 - sreg.c0) * kFB]);
                        best_update(v, (dl.r0 + r) * nfinal + col, lv, li);
                    }
                    warp_best(lv, li);
                    best_update(lv, li, bv, bi);
                    __syncwarp();
                }
            }
            v0 = NAN;
        }
        if (lane == 0) {
            int si = 0, sj = 0;
            float v = bv;
            if (bi != INT_MAX && bv != -INFINITY) {
                si = bi / nfinal;
                sj = bi - si * nfinal;
            } else {
                v = v0;  // nothing above -Inf: the reference reports (1,1)
            }
            if (A.point) {
                const int64_t k = A.point[item];
                const int i0 = A.origin[2 * item], j0 = A.origin[2 * item + 1];
                const double factor = static_cast<double>(1 << L);
                const double row = __dadd_rn(__ddiv_rn(static_cast<double>(si), factor), static_cast<double>(i0));
                const double col = __dadd_rn(__ddiv_rn(static_cast<double>(sj), factor), static_cast<double>(j0));
                const double dx = __dsub_rn(col, static_cast<double>(A.pts.rx[k]));
                const double dy = __dsub_rn(row, static_cast<double>(A.pts.ry[k]));
                A.out.dx[k] = __double2float_rn(__dadd_rn(dx, A.pts.dx0[k]));
                A.out.dy[k] = __double2float_rn(__dadd_rn(dy, A.pts.dy0[k]));
                A.out.corr[k] = v;
            } else {
                A.orow[item] = si;
                A.ocol[item] = sj;
                A.oval[item] = v;
            }
        }
        __syncwarp();
    }
}

// ----------------------------------------------------------------------------------------------
// Small helpers

__global__ void k_init_outputs(DevOutputs out, int64_t n, int* sub_count) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i == 0 && sub_count) *sub_count = 0;
    if (i < n) {
        out.dx[i] = __int_as_float(0x7fc00000);
        out.dy[i] = __int_as_float(0x7fc00000);
        out.corr[i] = __int_as_float(0x7fc00000);
        out.searched[i] = 0;
    }
}

// geom: [0] max ch, [1] max cw, [2] max nr, [3] max nc, [4] max px term, [5] max py term,
// [6] 1 while every window fits, [7] searchable count. Warp reductions, one atomic per warp.
__global__ void k_pass_geometry(DevPoints p, int64_t nrows, int64_t ncols, long long* geom) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    long long v[6] = {0, 0, 0, 0, 0, 0};
    int fits = 1, cnt = 0;
    if (k < p.n) {
        const int64_t rx = p.rx[k], ry = p.ry[k];
        if (rx > 0 && ry > 0) {
            const int64_t hx = p.csx[k] / 2, hy = p.csy[k] / 2;
            v[0] = 2 * hy;
            v[1] = 2 * hx;
            v[2] = 2 * ry;
            v[3] = 2 * rx;
            v[4] = hx + rx + static_cast<int64_t>(ceil(fabs(p.dx0[k])));
            v[5] = hy + ry + static_cast<int64_t>(ceil(fabs(p.dy0[k])));
            const int64_t wcx = static_cast<int64_t>(floor(p.x[k]));
            const int64_t wcy = static_cast<int64_t>(floor(p.y[k]));
            fits = (wcy - hy - ry) >= 1 && (wcy + hy + ry - 2) <= nrows &&
                   (wcx - hx - rx) >= 1 && (wcx + hx + rx - 2) <= ncols;
            cnt = 1;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 6; ++q) v[q] = max(v[q], __shfl_xor_sync(kFull, v[q], o));
        fits &= __shfl_xor_sync(kFull, fits, o);
        cnt += __shfl_xor_sync(kFull, cnt, o);
    }
    if ((threadIdx.x & 31) == 0 && cnt > 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) atomicMax(&geom[q], v[q]);
        if (!fits) atomicMin(&geom[6], 0ll);
        atomicAdd(reinterpret_cast<unsigned long long*>(&geom[7]), static_cast<unsigned long long>(cnt));
    }
}

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Window stride: even with an odd half, so that 16 lanes reading float2 at consecutive
// columns hit 16 distinct 8-byte bank pairs.
inline int window_stride(int rows) {
    int s = round_up(rows, 2);
    if ((s / 2) % 2 == 0) s += 2;
    return s;
}

struct CorrPlan {
    int TI, TJ, CHP, CWM, WS, PHS, NRS, NCM, BC;
    unsigned off_win, off_ph1, off_ph2, off_surf, off_red, off_surf2;
    size_t smem;
};

// `rot`: the rotation search, which stages the whole chip (it is resampled once per angle) and
// holds a second surface, the best one so far.
bool plan_corr(const PassGeometry& g, size_t ph_bytes, size_t smem_cap, CorrPlan* P,
               bool rot = false) {
    const int ch = static_cast<int>(g.max_ch), cw = static_cast<int>(g.max_cw);
    const int nr = static_cast<int>(g.max_nr), nc = static_cast<int>(g.max_nc);
    P->CHP = round_up(std::max(ch, 1), kUA);
    P->CWM = std::max(cw, 1);
    P->NRS = std::max(nr, 1);
    P->NCM = std::max(nc, 1);
    // The whole chip staged once per point if it fits, otherwise chunks of BC chip columns
    // (even, so FP32 partial flushes fall where they would unchunked). Within that, columns
    // per tile: as many as fit one thread each with at least one row group, rows to fill the
    // block; shrink until the shared-memory budget is met.
    const int bcs[] = {P->CWM, 64, 32, 16, 8, 4, 2};
    for (int bc : bcs) {
        if (bc > P->CWM || (bc < P->CWM && (bc & 1)) || (rot && bc < P->CWM)) continue;
        for (int TJ = std::min(nc, kCorrThreads); TJ >= 1; TJ = (TJ > 8 ? TJ - 8 : TJ - 1)) {
            const int groups = std::max(1, kCorrThreads / TJ);
            for (int TI = std::min(round_up(nr, kMI), groups * kMI); TI >= kMI; TI -= kMI) {
                const int WS = window_stride(TI + P->CHP);
                const int PHS = TI + ch + 1;
                size_t off = static_cast<size_t>(P->CHP) * bc * 4;
                off = (off + 15) & ~size_t(15);
                const unsigned off_win = static_cast<unsigned>(off);
                off += static_cast<size_t>(WS) * (TJ + bc - 1) * 4;
                off = (off + 15) & ~size_t(15);
                const unsigned off_ph1 = static_cast<unsigned>(off);
                off += static_cast<size_t>(PHS) * TJ * ph_bytes;
                off = (off + 15) & ~size_t(15);
                const unsigned off_ph2 = static_cast<unsigned>(off);
                off += static_cast<size_t>(PHS) * TJ * ph_bytes;
                off = (off + 15) & ~size_t(15);
                const unsigned off_surf = static_cast<unsigned>(off);
                off += static_cast<size_t>(P->NRS) * P->NCM * 4;
                off = (off + 15) & ~size_t(15);
                const unsigned off_red = static_cast<unsigned>(off);
                off += 3 * 32 * 8;
                off = (off + 15) & ~size_t(15);
                unsigned off_surf2 = off_surf;
                if (rot) {
                    off_surf2 = static_cast<unsigned>(off);
                    off += static_cast<size_t>(P->NRS) * P->NCM * 4;
                }
                if (off <= smem_cap) {
                    P->TI = TI;
                    P->TJ = TJ;
                    P->WS = WS;
                    P->PHS = PHS;
                    P->BC = bc;
                    P->off_win = off_win;
                    P->off_ph1 = off_ph1;
                    P->off_ph2 = off_ph2;
                    P->off_surf = off_surf;
                    P->off_red = off_red;
                    P->off_surf2 = off_surf2;
                    P->smem = off;
                    return true;
                }
            }
            if (TJ == 1) break;
        }
    }
    return false;
}

int ilog2_exact(int up) {
    int L = 0;
    while ((1 << L) < up) ++L;
    return (1 << L) == up ? L : -1;
}

struct RefinePlan {
    int levels, warp_floats;
    int warps;    // warps per CTA
    int per_sm;   // CTAs per SM
    size_t smem;
};

// Shared floats per warp of k_refine: patch, levels 1 and 2, then either the level-3
// materialisation (up <= 8) or level 3 with the block bounds and cone buffers.
RefinePlan plan_refine(int up) {
    RefinePlan R{};
    R.levels = ilog2_exact(up);
    const int L = R.levels;
    if (L <= 3) {
        // The patch, levels 1 and 2, the pyrUp scratch (40 x 20) and level 3.
        R.warp_floats = 32 + 100 + 400 + 800 + 1600;
    } else {
        // Level 3, then a scratch of the larger of the build phase (level 2 and the 40 x 20
        // vertical pass, with the patch and level 1 inside) and the search phase (the block
        // bounds, then the larger of the level-3 row maxima and the cone buffers of levels
        // 4 .. L).
        const int nb = (5 << L) / kFB;
        const int cap[7] = {16, 10, 7, 6, 5, 5, 5};
        int cone = 0;
        for (int d = 0; d <= L - 4; ++d) cone += cap[d] * cap[d] + cap[d] * cap[d + 1];
        R.warp_floats = 1600 + std::max(1200, nb * nb + std::max(40 * nb, cone));
    }
    // Warps per CTA for the most resident warps per SM (228 KB of shared memory, 1 KB charged
    // per CTA): the kernel is issue-bound on dependent shared-memory arithmetic, so resident
    // warps, not CTA size, hide its latencies.
    const size_t per_warp = static_cast<size_t>(R.warp_floats) * sizeof(float);
    int best_w = 1, best_sm = 0;
    for (int w = 1; w <= kRefineWarps; ++w) {
        const size_t cta = w * per_warp + 1024 + 2 * 64 * sizeof(int);
        if (w * per_warp > static_cast<size_t>(kDynSmemCap)) break;
        const int ctas = static_cast<int>(std::min<size_t>(32, (228 * 1024) / cta));
        if (ctas * w >= best_w * best_sm) {
            best_w = w;
            best_sm = ctas;
        }
    }
    R.warps = best_w;
    R.per_sm = std::max(1, best_sm);
    R.smem = static_cast<size_t>(R.warps) * per_warp;
    return R;
}

// Dynamic shared memory a CTA holding `cols` Tensor Memory columns reserves, for a kernel with
// `static_smem` bytes of static shared memory (see the launch below): with the 1 KB the SM
// charges each CTA, its footprint is at least cols/512 of the SM's 228 KB.
size_t tmem_smem_floor(uint32_t cols, size_t static_smem) {
    const size_t share = static_cast<size_t>(cols) * (228 * 1024) / 512;
    return share > 1024 + static_smem ? share - 1024 - static_smem : 0;
}

struct TcPlan {
    int NB, QM, QS, PS, PC, XS, XT, NRS, NRM, NCM, CHM, CWM, BC, big, MT;
    unsigned off_E, off_W, off_T, off_P, off_V, off_S1, off_S2, off_num, off_est, off_red;
    int XV = 0, acc1_col = 0, issuers = 2;
    uint32_t tmem_cols;
    size_t smem;
};

// Shared-memory and Tensor Memory plan of k_corr_tc2 for a pass's largest geometry; false when
// the pass does not fit it (surfaces beyond 64 x 64, chip operand larger than shared memory,
// accumulator beyond 512 columns).
bool plan_corr_tc2(const PassGeometry& g, size_t smem_cap, TcPlan* P) {
    const int ch = static_cast<int>(g.max_ch), cw = static_cast<int>(g.max_cw);
    const int nr = static_cast<int>(g.max_nr), nc = static_cast<int>(g.max_nc);
    if (nc > 64 || nr > 64 || nr < 1 || nc < 1 || cw < 2 || ch < 2 || (cw & 1)) return false;
    P->CHM = ch;
    P->CWM = cw;
    P->NRM = nr;
    P->NCM = nc;
    P->MT = 64;
    P->NB = round_up(ch + 15, 16);
    if (P->NB > 256) return false;
    P->QM = (ch + nr - 1 + 15) / 16;
    P->PS = P->NB * 16;
    P->XS = 64 + cw;
    P->QS = P->XS * 16;
    P->XT = 0;
    P->PC = round_up(kPadL + P->NB + 20, 16);
    P->NRS = nr | 1;
    P->XV = round_up(cw + nc - 1, 32) + 4;
    // kTc2Issuers accumulators whose column i is surface row i (the products write columns below
    // round16(nr), the epilogue reads 32 columns per half of the surface rows).
    const int stride = nr > 32 ? 64 : 32;
    uint32_t t1 = 32;
    while (static_cast<int>(t1) < kTc2Issuers * stride) t1 <<= 1;
    P->acc1_col = stride;
    P->tmem_cols = t1;
    auto a16 = [](size_t v) { return (v + 15) & ~size_t(15); };
    const size_t Eb = static_cast<size_t>(cw) * P->PS;
    const size_t Wb = static_cast<size_t>(P->QM) * P->QS;
    const size_t Pb = a16(static_cast<size_t>(cw) * P->PC);
    const size_t Vb = a16(2 * (static_cast<size_t>(nr) * P->XV + 16) * 4);
    const size_t nbytes = a16(static_cast<size_t>(nc) * P->NRS * 4);
    // [E][W][P][V1, V2 | candidate numerators and indices][S1][S2][red]
    size_t off = 0;
    P->off_E = 0;
    off += Eb;
    P->off_W = static_cast<unsigned>(off);
    off += Wb;
    P->off_P = static_cast<unsigned>(off);
    off += Pb;
    P->off_V = static_cast<unsigned>(off);
    P->off_num = P->off_V;
    P->off_est = static_cast<unsigned>(off + nbytes);
    // The region also takes the window's raw 16-byte chunks before the box sums.
    const size_t rawb = static_cast<size_t>(P->XS) * (P->QM + 1) * 16;
    off += std::max(std::max(Vb, 2 * nbytes), rawb);
    P->off_S1 = static_cast<unsigned>(off);
    off += nbytes;
    P->off_S2 = static_cast<unsigned>(off);
    off += nbytes;
    P->off_red = static_cast<unsigned>(off);
    off += 3 * 32 * 8;
    P->off_T = 0;
    P->BC = cw;
    P->big = 0;
    P->smem = off;
    return off <= smem_cap;
}

// Plan of k_corr_bf: the chunk of chip columns whose products keep each accumulator element's
// chain near kBfChain, the widest window staging that fits `smem_cap` beside the chip operand
// buffers and the denominators, and the box-sum stripes in the space of both; false when the
// pass's surfaces exceed 64 x 64 or its chips 240 px.
struct BfPlan {
    int NB, QB, BC, OB, LW, PC, NRS, AC, RS, VS, XS;
    unsigned off_S2, off_raw, off_V, off_den, off_E, off_P, off_red, Eb, Pb;
    uint32_t tmem_cols;
    size_t smem;
};

bool plan_corr_bf(const PassGeometry& g, size_t smem_cap, BfPlan* P) {
    const int ch = static_cast<int>(g.max_ch), cw = static_cast<int>(g.max_cw);
    const int nr = static_cast<int>(g.max_nr), nc = static_cast<int>(g.max_nc);
    if (nr < 1 || nc < 1 || nr > 64 || nc > 64 || ch < 2 || cw < 2) return false;
    P->NB = round_up(ch + 15, 16);
    if (P->NB > 256) return false;
    P->QB = (ch + nr - 1 + 15) / 16;
    P->PC = round_up(kBfPadL + P->NB + 26, 8);
    P->NRS = nr | 1;
    // A block's products write accumulator columns [16 q + elo - NB + 16, + n), all below
    // round16(nr) (block_rows: elo, NB multiples of 16, the rows' end at most NB - 16 + nr - 16 q).
    P->AC = round_up(nr, 16);
    if (2 * kBfIssuers * P->AC > 512) return false;  // two sets of kBfIssuers accumulators
    P->tmem_cols = 512;
    P->RS = (ch + nr - 1) | 1;
    P->VS = nr + 1;
    // Window blocks meeting one surface row: (ch + 15) / 16 + 1, half of them (one parity) into
    // an accumulator, with three limb pairs each: 1.5 blocks accumulating steps per chip column.
    const int blocks = (ch + 15) / 16 + 1;
    int bc = std::max(1, 2 * kBfChain / (3 * blocks));
    bc = std::min(bc, cw);
    // The staged chip columns of a chunk: kBfPre elements per thread of warps 4-7.
    const int stagers = kBfThreads - 32 * kBfIssuers;
    while (bc > 1 && bc * P->PC > kBfPre * stagers) --bc;
    if (bc * P->PC > kBfPre * stagers) return false;
    P->BC = bc;
    auto a16 = [](size_t v) { return (v + 15) & ~size_t(15); };
    const size_t Sb = a16(static_cast<size_t>(nc) * P->NRS * 8);
    const size_t Eb = static_cast<size_t>(kBfLimbs) * bc * 2 * P->NB * 16;
    const size_t Pb = a16(static_cast<size_t>(kBfLimbs) * bc * P->PC * 2);
    const size_t red = 3 * 32 * 8;
    const size_t X = Sb + 2 * Eb + 2 * Pb + red;
    const size_t colb = static_cast<size_t>(kBfLimbs) * P->QB * 2 * 16;  // limb bytes per column
    const size_t minL = std::max(2 * Sb, a16(static_cast<size_t>(nc) * P->NRS * 4));
    auto Lof = [&](int ob) { return std::max(minL, static_cast<size_t>(ob + 63) * colb); };
    if (X >= smem_cap) return false;
    int OB = round_up(cw, bc);
    if (Lof(OB) + X > smem_cap) {
        const int lw = static_cast<int>((smem_cap - X) / colb);
        const int ob = (lw - 63) / bc * bc;
        if (ob < bc) return false;
        const int nout = (cw + ob - 1) / ob;
        OB = round_up((cw + nout - 1) / nout, bc);
    }
    P->OB = OB;
    P->LW = OB + 63;
    const size_t L = Lof(OB);
    if (L + X > smem_cap) return false;
    // Box-sum stripes after S1 and S2, up to the reduction scratch.
    const int XW = cw + nc - 1;
    const size_t avail = L + X - red - 2 * Sb;
    const size_t per_col = static_cast<size_t>(P->RS) * 4 + static_cast<size_t>(P->VS) * 16;
    if (avail < per_col + 16) return false;
    P->XS = static_cast<int>(std::min<size_t>(XW, (avail - 16) / per_col));
    P->off_S2 = static_cast<unsigned>(Sb);
    P->off_raw = static_cast<unsigned>(2 * Sb);
    P->off_V = static_cast<unsigned>(a16(2 * Sb + static_cast<size_t>(P->XS) * P->RS * 4));
    if (P->off_V + static_cast<size_t>(P->XS) * P->VS * 16 > L + X - red) return false;
    P->off_den = static_cast<unsigned>(L);
    P->off_E = static_cast<unsigned>(L + Sb);
    P->off_P = static_cast<unsigned>(L + Sb + 2 * Eb);
    P->off_red = static_cast<unsigned>(L + Sb + 2 * Eb + 2 * Pb);
    P->Eb = static_cast<unsigned>(Eb);
    P->Pb = static_cast<unsigned>(Pb);
    P->smem = L + X;
    return true;
}

// A k_corr_tc plan whose shared memory leaves room for one CTA per SM anyway has the SM's 512
// Tensor Memory columns to itself: with M = 64 products (surfaces up to 64 x 64: the chip-128
// levels), which one thread issues only about every 120 cycles, it issues them from four threads
// into four accumulators. M = 128 products are bound by the tensor pipe and keep two.
void four_issuers(TcPlan* P) {
    const bool one_per_sm = 2 * (P->smem + 2048) > 228 * 1024;
    if (one_per_sm && P->MT == 64 && P->NRM <= 64 && 4 * P->acc1_col <= 512) {
        P->issuers = 4;
        P->tmem_cols = static_cast<uint32_t>(4 * P->acc1_col);
    }
}

// Shared-memory plan of k_corr_tc for a pass's largest geometry; false when the pass does not
// fit the kernel (surface wider than 64 columns, more than 256 rows, chips taller than 226).
// The whole chip operand and separate box-sum buffers when they fit ("overlap": the box sums
// run beside the products); otherwise the box sums first and the chip operand in chunks of BC
// columns in the space they used.
bool plan_corr_tc(const PassGeometry& g, size_t smem_cap, TcPlan* P) {
    const int ch = static_cast<int>(g.max_ch), cw = static_cast<int>(g.max_cw);
    const int nr = static_cast<int>(g.max_nr), nc = static_cast<int>(g.max_nc);
    if (nc > 128 || nr > 256 || nr < 1 || nc < 1 || cw < 2 || ch < 2 || (cw & 1)) return false;
    P->CHM = ch;
    P->CWM = cw;
    P->NRM = nr;
    P->NCM = nc;
    P->MT = nc <= 64 ? 64 : 128;
    P->NB = round_up(ch + 30, 16);
    if (P->NB > 256) return false;
    P->QM = (15 + ch + nr - 1 + 15) / 16;
    P->PS = P->NB * 16;
    P->XS = P->MT + cw;
    P->QS = P->XS * 16;
    P->XT = round_up(cw + nc - 1, 4) + 4;
    P->PC = round_up(kPadL + P->NB + 20, 16);
    P->NRS = nr | 1;
    // Two accumulators, each holding the columns of surface rows 0 .. nr + 15 (the products'
    // rows are trimmed to the surface rows) and whatever the epilogue's reads reach.
    const int used = (nr + 16 + 15) & ~15;
    const int reads = P->MT == 64 ? 32 * ((nr + 31) / 32) : 16 * ((nr + 15) / 16);
    uint32_t cols = 32;
    while (static_cast<int>(cols) < std::max(used, reads)) cols <<= 1;
    if (2 * cols > 512) return false;
    P->acc1_col = static_cast<int>(cols);
    P->tmem_cols = 2 * cols;
    auto a16 = [](size_t v) { return (v + 15) & ~size_t(15); };
    const size_t Eb = static_cast<size_t>(cw) * P->PS;
    const size_t Wb = static_cast<size_t>(P->QM) * P->QS;
    const size_t Tb = a16(static_cast<size_t>(16 * P->QM) * P->XT);
    const size_t Pb = a16(static_cast<size_t>(cw) * P->PC);
    const size_t Vb = a16(2ull * nr * (cw + nc - 1) * 4);
    const size_t nbytes = a16(static_cast<size_t>(nc) * P->NRS * 4);
    const size_t red = 3 * 32 * 8;
    // Overlap layout: [E][W][T][P][V | num, est, bound][S1][S2][red].
    {
        size_t off = 0;
        P->off_E = 0;
        off += Eb;
        P->off_W = static_cast<unsigned>(off);
        off += Wb;
        P->off_T = static_cast<unsigned>(off);
        off += Tb;
        P->off_P = static_cast<unsigned>(off);
        off += Pb;
        P->off_V = static_cast<unsigned>(off);
        P->off_num = P->off_V;
        P->off_est = static_cast<unsigned>(off + nbytes);
        off += std::max(Vb, 3 * nbytes);
        P->off_S1 = static_cast<unsigned>(off);
        off += nbytes;
        P->off_S2 = static_cast<unsigned>(off);
        off += nbytes;
        P->off_red = static_cast<unsigned>(off);
        off += red;
        if (off <= smem_cap) {
            P->smem = off;
            P->BC = cw;
            P->big = 0;
            four_issuers(P);
            return true;
        }
    }
    // Chunked layout: [W][P][S1][S2][red][zone], the zone holding T and V for the box sums,
    // then the chunks of the chip operand, then num, estimates and bounds.
    size_t off = 0;
    P->off_W = 0;
    off += Wb;
    P->off_P = static_cast<unsigned>(off);
    off += Pb;
    P->off_S1 = static_cast<unsigned>(off);
    off += nbytes;
    P->off_S2 = static_cast<unsigned>(off);
    off += nbytes;
    P->off_red = static_cast<unsigned>(off);
    off += red;
    off = a16(off);
    const size_t zone_min = std::max(Tb + Vb, 3 * nbytes);
    if (off + std::max(zone_min, 2 * static_cast<size_t>(P->PS)) > smem_cap) return false;
    const size_t avail = smem_cap - off;
    int bc = static_cast<int>(std::min<size_t>(cw, avail / P->PS)) & ~1;
    if (bc < 2) return false;
    P->BC = bc;
    P->big = 1;
    P->off_E = P->off_T = P->off_num = static_cast<unsigned>(off);
    P->off_V = static_cast<unsigned>(off + Tb);
    P->off_est = static_cast<unsigned>(off + nbytes);
    P->smem = off + std::max(zone_min, static_cast<size_t>(bc) * P->PS);
    four_issuers(P);
    return true;
}

template <typename T>
cudaError_t launch_corr_t(const CorrArgs& A, const CorrPlan& P, int grid, cudaStream_t stream) {
    if (P.smem > static_cast<size_t>(kDynSmemCap)) return cudaErrorInvalidValue;
    auto kern = A.rot.count > 0 ? k_corr<T, true> : k_corr<T, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kDynSmemCap);
    if (e != cudaSuccess) return e;
    kern<<<grid, kCorrThreads, P.smem, stream>>>(A);
    return cudaGetLastError();
}


std::atomic<long long> g_scratch_allocs{0};

cudaError_t ensure_scratch(TrackScratch& s, int64_t n, cudaStream_t stream) {
    if (s.fixed) {
        // Caller-provided buffers: never allocate; a pass beyond them is an error.
        if (!s.geom || !s.sub_count || !s.status || !s.sub_point || !s.sub_origin || !s.sub_patch)
            return cudaErrorInvalidValue;
        return s.capacity >= n ? cudaSuccess : cudaErrorMemoryAllocation;
    }
    if (!s.geom) {
        cudaError_t e = cudaMalloc(&s.geom, 8 * sizeof(int64_t));
        if (e != cudaSuccess) return e;
        ++g_scratch_allocs;
    }
    if (!s.sub_count) {
        cudaError_t e = cudaMalloc(&s.sub_count, sizeof(int));
        if (e != cudaSuccess) return e;
        ++g_scratch_allocs;
    }
    if (!s.status) {
        cudaError_t e = cudaMalloc(&s.status, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(s.status, 0, sizeof(int));
        if (e != cudaSuccess) return e;
        ++g_scratch_allocs;
    }
    if (s.capacity >= n) return cudaSuccess;
    const int64_t cap = std::max<int64_t>(n, 1024);
    cudaError_t e = cudaSuccess;
    g_scratch_allocs += 3;
    if (s.pool) {
        // Stream-ordered: the old queue is released after the work already on `stream`.
        if (s.sub_point) cudaFreeAsync(s.sub_point, stream);
        if (s.sub_origin) cudaFreeAsync(s.sub_origin, stream);
        if (s.sub_patch) cudaFreeAsync(s.sub_patch, stream);
        s.sub_point = nullptr;
        s.sub_origin = nullptr;
        s.sub_patch = nullptr;
        s.capacity = 0;
        void* a = nullptr;
        void* b = nullptr;
        void* c = nullptr;
        e = cudaMallocFromPoolAsync(&a, cap * sizeof(int64_t), s.pool, stream);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&b, cap * 2 * sizeof(int32_t), s.pool, stream);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&c, cap * 25 * sizeof(float), s.pool, stream);
        s.sub_point = static_cast<int64_t*>(a);
        s.sub_origin = static_cast<int32_t*>(b);
        s.sub_patch = static_cast<float*>(c);
    } else {
        cudaFree(s.sub_point);
        cudaFree(s.sub_origin);
        cudaFree(s.sub_patch);
        s.sub_point = nullptr;
        s.sub_origin = nullptr;
        s.sub_patch = nullptr;
        s.capacity = 0;
        e = cudaMalloc(&s.sub_point, cap * sizeof(int64_t));
        if (e == cudaSuccess) e = cudaMalloc(&s.sub_origin, cap * 2 * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc(&s.sub_patch, cap * 25 * sizeof(float));
    }
    if (e != cudaSuccess) return e;
    s.capacity = cap;
    return cudaSuccess;
}

}  // namespace

bool make_rotation(const double* deg, int count, Rotation* out, std::string* err) {
    if (count < 1 || count > kMaxAngles) {
        if (err) *err = "the rotation search needs 1 to " + std::to_string(kMaxAngles) + " angles";
        return false;
    }
    if (!deg) {
        if (err) *err = "null rotation angles";
        return false;
    }
    for (int i = 0; i < count; ++i) {
        if (!std::isfinite(deg[i])) {
            if (err) *err = "rotation angles must be finite";
            return false;
        }
        for (int j = 0; j < i; ++j)
            if (deg[j] == deg[i]) {
                if (err) *err = "rotation angles must be distinct";
                return false;
            }
    }
    out->count = count;
    for (int i = 0; i < count; ++i) {
        // deg2rad (deg * (pi / 180)), then the C library's sin and cos.
        const double r = deg[i] * (M_PI / 180.0);
        out->sn[i] = std::sin(r);
        out->cs[i] = std::cos(r);
        out->turn[i] = deg[i] != 0.0 ? 1 : 0;
    }
    for (int i = count; i < kMaxAngles; ++i) {
        out->sn[i] = 0.0;
        out->cs[i] = 1.0;
        out->turn[i] = 0;
    }
    return true;
}

cudaEvent_t KernelTimer::get() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

PassGeometry pass_geometry_host(const ar_points& p, int64_t nrows, int64_t ncols) {
    PassGeometry g;
    bool fits = true;
    int64_t px = 0, py = 0;
    for (int64_t k = 0; k < p.n; ++k) {
        const int64_t rx = p.radius_x[k], ry = p.radius_y[k];
        if (!(rx > 0 && ry > 0)) continue;
        const int64_t hx = p.chip_size_x[k] / 2, hy = p.chip_size_y[k] / 2;
        g.max_ch = std::max(g.max_ch, 2 * hy);
        g.max_cw = std::max(g.max_cw, 2 * hx);
        g.max_nr = std::max(g.max_nr, 2 * ry);
        g.max_nc = std::max(g.max_nc, 2 * rx);
        px = std::max(px, hx + rx + static_cast<int64_t>(std::ceil(std::fabs(p.dx_prior[k]))));
        py = std::max(py, hy + ry + static_cast<int64_t>(std::ceil(std::fabs(p.dy_prior[k]))));
        const int64_t wcx = static_cast<int64_t>(std::floor(p.x[k]));
        const int64_t wcy = static_cast<int64_t>(std::floor(p.y[k]));
        fits = fits && (wcy - hy - ry) >= 1 && (wcy + hy + ry - 2) <= nrows &&
               (wcx - hx - rx) >= 1 && (wcx + hx + rx - 2) <= ncols;
        ++g.searchable;
    }
    g.padx = fits ? 0 : px + 2;
    g.pady = fits ? 0 : py + 2;
    return g;
}

cudaError_t scratch_acquire(TrackScratch& s, cudaStream_t stream);

cudaError_t read_status(TrackScratch& scratch, cudaStream_t stream, int* status) {
    *status = 0;
    if (!scratch.status) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(status, scratch.status, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && *status) e = cudaMemsetAsync(scratch.status, 0, sizeof(int), stream);
    return e;
}

cudaError_t pass_geometry_device(const DevPoints& pts, int64_t nrows, int64_t ncols,
                                 TrackScratch& scratch, cudaStream_t stream, PassGeometry* out) {
    cudaError_t e = scratch_acquire(scratch, stream);
    if (e != cudaSuccess) return e;
    e = ensure_scratch(scratch, 0, stream);
    if (e != cudaSuccess) return e;
    long long init[8] = {0, 0, 0, 0, 0, 0, 1, 0};
    e = cudaMemcpyAsync(scratch.geom, init, sizeof(init), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    if (pts.n > 0) {
        const int threads = 256;
        const int64_t blocks = (pts.n + threads - 1) / threads;
        k_pass_geometry<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(
            pts, nrows, ncols, reinterpret_cast<long long*>(scratch.geom));
        scratch.timer.launches += 1;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    long long g[8];
    e = cudaMemcpyAsync(g, scratch.geom, sizeof(g), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    out->max_ch = g[0];
    out->max_cw = g[1];
    out->max_nr = g[2];
    out->max_nc = g[3];
    const bool fits = g[6] != 0;
    out->padx = fits ? 0 : g[4] + 2;
    out->pady = fits ? 0 : g[5] + 2;
    out->searchable = g[7];
    return cudaSuccess;
}

// The scratch buffers are shared by the passes of a context; a pass on one stream waits for
// the last pass that used them, whichever stream that ran on.
cudaError_t scratch_acquire(TrackScratch& s, cudaStream_t stream) {
    if (!s.done) {
        if (s.fixed) return cudaSuccess;  // no event is created for a caller-provided view
        ++g_scratch_allocs;
        return cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    }
    return cudaStreamWaitEvent(stream, s.done, 0);
}

long long scratch_allocations() { return g_scratch_allocs.load(); }

// Passes of at least kTuneMinPoints points are tuned: the tensor-core kernels on their first
// kTuneSample points, the CUDA-core kernel on the first kTuneSampleDirect.
constexpr int64_t kTuneMinPoints = 8192;
constexpr int64_t kTuneSample = 32768;
constexpr int64_t kTuneSampleDirect = 4096;

// Times each candidate kernel (2 k_corr_tc2, 1 k_corr_tc, 0 k_corr) on a sample of the pass --
// consecutive points from its middle, written to their own output slots, without refinement
// (the pass itself then writes the same values there) -- each launched twice and the second
// timed, and returns in `kind` the one with the least time per point (a tie keeps the earlier
// candidate). The tensor-core kernels' sample is large enough that each CTA takes a run of
// consecutive points, as in the full pass: both carry box sums from one point of a run to the
// next, and on a sample of 4096 points (one or two points per CTA) k_corr_tc2 lost that and the
// tuner could pick k_corr_tc, 25 % slower on the full pass. The sample comes from the middle
// because a pass's first points (its first grid columns) lie at the image's edge, where more
// points are skipped or clipped than elsewhere: on a 4096 x 4096 scene the first 32 768 points of
// the chip-32 / radius-25 pass made k_corr_tc look faster, and on the whole pass it is 29 %
// slower (12.9 against 10.0 ms). With diagnostic
// surfaces (`at_start`) the sample is the pass's first points, whose rows they are.
template <typename Launch>
cudaError_t autotune_u8(TrackScratch& scratch, cudaStream_t stream, const DevPoints& pts,
                        const DevOutputs& out, bool at_start, bool fit2, bool fit1, int* kind,
                        Launch launch) {
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i)
        if (!scratch.tune_ev[i]) {
            e = cudaEventCreate(&scratch.tune_ev[i]);
            ++g_scratch_allocs;
        }
    if (e != cudaSuccess) return e;
    float best = INFINITY;
    int chosen = fit2 ? 2 : 1;
    const int cand[3] = {2, 1, 0};
    for (int c : cand) {
        if ((c == 2 && !fit2) || (c == 1 && !fit1)) continue;
        const int64_t m = std::min<int64_t>(pts.n, c == 0 ? kTuneSampleDirect : kTuneSample);
        const int64_t off = at_start ? 0 : (pts.n - m) / 2;
        DevPoints ds = pts;
        ds.x += off;
        ds.y += off;
        ds.rx += off;
        ds.ry += off;
        ds.dx0 += off;
        ds.dy0 += off;
        ds.csx += off;
        ds.csy += off;
        ds.n = m;
        DevOutputs dout = out;
        dout.dx += off;
        dout.dy += off;
        dout.corr += off;
        dout.searched += off;
        e = launch(c, ds, dout);
        if (e == cudaSuccess) e = cudaEventRecord(scratch.tune_ev[0], stream);
        if (e == cudaSuccess) e = launch(c, ds, dout);
        if (e == cudaSuccess) e = cudaEventRecord(scratch.tune_ev[1], stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(scratch.tune_ev[1]);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, scratch.tune_ev[0], scratch.tune_ev[1]);
        if (e != cudaSuccess) return e;
        scratch.timer.launches += 2;
        const float per_point = ms / static_cast<float>(ds.n);
        if (per_point < best) {
            best = per_point;
            chosen = c;
        }
    }
    *kind = chosen;
    return cudaSuccess;
}

cudaError_t launch_track_impl(int dtype, const void* ref, const void* sec, const uint8_t* valid,
                              int64_t nrows, int64_t ncols, const DevPoints& pts,
                              const PassGeometry& geom, int up, int measure,
                              const DevOutputs& out, TrackScratch& scratch, int num_sms,
                              cudaStream_t stream, std::string* err, float* surf_out,
                              const Rotation* rot) {
    cudaError_t e = ensure_scratch(scratch, pts.n, stream);
    if (e != cudaSuccess) return e;
    if (pts.n > 0) {
        const int threads = 256;
        k_init_outputs<<<static_cast<unsigned>((pts.n + threads - 1) / threads), threads, 0, stream>>>(
            out, pts.n, scratch.sub_count);
        scratch.timer.launches += 1;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (geom.searchable == 0 || geom.max_cw == 0 || geom.max_ch == 0) return cudaSuccess;

    const bool rotating = rot && rot->count > 0;
    const size_t ph_bytes = dtype == AR_U8 && !rotating ? 4 : 8;
    CorrPlan P{};
    if (!plan_corr(geom, ph_bytes, 220 * 1024, &P, rotating)) {
        if (err) *err = rotating ? "chip and search geometry too large for shared memory with "
                                   "the rotation search"
                                 : "chip and search geometry too large for shared memory";
        return cudaErrorInvalidValue;
    }
    CorrArgs A{};
    if (rotating) A.rot = *rot;
    A.off_surf2 = P.off_surf2;
    A.ref = ref;
    A.sec = sec;
    A.valid = valid;
    A.nrows = nrows;
    A.ncols = ncols;
    A.pts = pts;
    A.padx = geom.padx;
    A.pady = geom.pady;
    A.up = up;
    A.measure = measure;
    A.TI = P.TI;
    A.TJ = P.TJ;
    A.CHP = P.CHP;
    A.CWM = P.CWM;
    A.BC = P.BC;
    A.WS = P.WS;
    A.PHS = P.PHS;
    A.NRS = P.NRS;
    A.NCM = P.NCM;
    A.off_win = P.off_win;
    A.off_ph1 = P.off_ph1;
    A.off_ph2 = P.off_ph2;
    A.off_surf = P.off_surf;
    A.off_red = P.off_red;
    A.out = out;
    A.sub_count = scratch.sub_count;
    A.sub_point = scratch.sub_point;
    A.sub_origin = scratch.sub_origin;
    A.sub_patch = scratch.sub_patch;
    A.surf_out = surf_out;
    A.flops = scratch.timer.enabled ? scratch.timer.flops : nullptr;

    KernelTimer& T = scratch.timer;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    if (T.enabled) {
        ev0 = T.get();
        ev1 = T.get();
        ev2 = T.get();
        cudaEventRecord(ev0, stream);
    }
    // The UInt8 tensor-core kernels: k_corr_tc2 (`tc2`, surfaces up to 64 x 64 with the chip
    // operand whole) or k_corr_tc (surfaces up to 128 columns), planned by `TP`.
    auto launch_tc = [&](bool tc2, const TcPlan& TP, const DevPoints& pts, int up,
                         const DevOutputs& out, unsigned long long* flops) -> cudaError_t {
        TcArgs B{};
        B.ref = static_cast<const uint8_t*>(ref);
        B.sec = static_cast<const uint8_t*>(sec);
        B.valid = valid;
        B.nrows = nrows;
        B.ncols = ncols;
        B.pts = pts;
        B.padx = geom.padx;
        B.pady = geom.pady;
        B.up = up;
        B.measure = measure;
        B.NB = TP.NB;
        B.QM = TP.QM;
        B.QS = TP.QS;
        B.PS = TP.PS;
        B.PC = TP.PC;
        B.XS = TP.XS;
        B.XT = TP.XT;
        B.NRS = TP.NRS;
        B.NRM = TP.NRM;
        B.NCM = TP.NCM;
        B.CHM = TP.CHM;
        B.CWM = TP.CWM;
        B.BC = TP.BC;
        B.big = TP.big;
        B.MT = TP.MT;
        B.off_E = TP.off_E;
        B.off_W = TP.off_W;
        B.off_T = TP.off_T;
        B.off_P = TP.off_P;
        B.off_V = TP.off_V;
        B.off_S1 = TP.off_S1;
        B.off_S2 = TP.off_S2;
        B.off_num = TP.off_num;
        B.off_est = TP.off_est;
        B.off_red = TP.off_red;
        B.XV = TP.XV;
        B.acc1_col = TP.acc1_col;
        B.issuers = TP.issuers;
        B.tmem_cols = TP.tmem_cols;
        B.out = out;
        B.sub_count = scratch.sub_count;
        B.sub_point = scratch.sub_point;
        B.sub_origin = scratch.sub_origin;
        B.sub_patch = scratch.sub_patch;
        B.surf_out = surf_out;
        B.flops = flops;
        B.status = scratch.status;
        // Each CTA holds its Tensor Memory columns for its lifetime, so the CTAs one SM holds
        // must fit its 512 columns together -- including CTAs of other launches running
        // concurrently (other streams, the request loop's slots), or an allocation would wait
        // for a whole persistent launch to end. A CTA of T columns therefore reserves at least
        // T/512 of the SM's 228 KB of shared memory (less the 1 KB each CTA is charged): any set
        // of CTAs that fits an SM's shared memory fits its Tensor Memory.
        const bool reg = TP.MT == 64 && TP.NRM <= 64;
        auto kern = tc2 ? k_corr_tc2 : reg ? k_corr_tc<true> : k_corr_tc<false>;
        cudaFuncAttributes fa{};
        e = cudaFuncGetAttributes(&fa, kern);
        if (e != cudaSuccess) return e;
        // The per-block limit (227 KB, static included) is this kernel's fixed attribute value.
        const size_t dyn_max = 232448 - fa.sharedSizeBytes;
        const size_t tc_smem = std::max<size_t>(TP.smem, tmem_smem_floor(TP.tmem_cols, fa.sharedSizeBytes));
        const int per_sm_tc = static_cast<int>(std::max<size_t>(
            1, std::min<size_t>(2, (228 * 1024) / (tc_smem + fa.sharedSizeBytes + 1024))));
        if (tc_smem > dyn_max) return cudaErrorInvalidValue;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(dyn_max));
        if (e != cudaSuccess) return e;
        const int grid = static_cast<int>(
            std::max<int64_t>(1, std::min<int64_t>(pts.n, static_cast<int64_t>(num_sms) * per_sm_tc)));
        kern<<<grid, kTcThreads, tc_smem, stream>>>(B);
        e = cudaGetLastError();
            return e;
    };
    // The CUDA-core kernel (the plain method) for any element type.
    auto launch_direct = [&](const DevPoints& pts_, int up_, const DevOutputs& out_,
                             unsigned long long* flops_) -> cudaError_t {
        CorrArgs A2 = A;
        A2.pts = pts_;
        A2.up = up_;
        A2.out = out_;
        A2.flops = flops_;
        const int per_sm = P.smem <= 100 * 1024 ? 2 : 1;
        const int64_t want = static_cast<int64_t>(num_sms) * per_sm * 8;
        const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(pts_.n, want)));
        switch (dtype) {
            case AR_U8: return launch_corr_t<uint8_t>(A2, P, grid, stream);
            case AR_U16: return launch_corr_t<uint16_t>(A2, P, grid, stream);
            case AR_I16: return launch_corr_t<int16_t>(A2, P, grid, stream);
            case AR_F32: return launch_corr_t<float>(A2, P, grid, stream);
            default: return cudaErrorInvalidValue;
        }
    };
    if (dtype != AR_U8 && dtype != AR_U16 && dtype != AR_I16 && dtype != AR_F32) {
        if (err) *err = "unsupported element type";
        return cudaErrorInvalidValue;
    }
    // The rotation search correlates Float32 (resampled) chips: CUDA cores for every type.
    const bool tc_ok = dtype == AR_U8 && scratch.tensor_cores && !rotating;
    // Split-BF16 tensor-core products for the other element types (by default for chips of
    // 64 px and up, where the products are a dense contraction worth the limb splitting).
    bool bf_done = false;
    const bool bf_ok = (dtype == AR_U16 || dtype == AR_I16 || dtype == AR_F32) &&
                       scratch.tensor_cores && !rotating && scratch.split_bf16 != 0 &&
                       (scratch.split_bf16 == 2 || (geom.max_ch >= 64 && geom.max_cw >= 64));
    if (bf_ok) {
        auto kern = dtype == AR_U16 ? k_corr_bf<uint16_t> : dtype == AR_I16 ? k_corr_bf<int16_t>
                                                                             : k_corr_bf<float>;
        cudaFuncAttributes fa{};
        e = cudaFuncGetAttributes(&fa, kern);
        if (e != cudaSuccess) return e;
        const size_t dyn_max = 232448 - fa.sharedSizeBytes;
        BfPlan BPl{};
        if (plan_corr_bf(geom, dyn_max, &BPl)) {
            BfArgs B{};
            B.ref = ref;
            B.sec = sec;
            B.valid = valid;
            B.nrows = nrows;
            B.ncols = ncols;
            B.pts = pts;
            B.padx = geom.padx;
            B.pady = geom.pady;
            B.up = up;
            B.measure = measure;
            B.CHM = static_cast<int>(geom.max_ch);
            B.CWM = static_cast<int>(geom.max_cw);
            B.NRM = static_cast<int>(geom.max_nr);
            B.NCM = static_cast<int>(geom.max_nc);
            B.NB = BPl.NB;
            B.BC = BPl.BC;
            B.OB = BPl.OB;
            B.LW = BPl.LW;
            B.PC = BPl.PC;
            B.NRS = BPl.NRS;
            B.AC = BPl.AC;
            B.RS = BPl.RS;
            B.VS = BPl.VS;
            B.XS = BPl.XS;
            B.off_S2 = BPl.off_S2;
            B.off_raw = BPl.off_raw;
            B.off_V = BPl.off_V;
            B.off_den = BPl.off_den;
            B.off_E = BPl.off_E;
            B.off_P = BPl.off_P;
            B.off_red = BPl.off_red;
            B.Eb = BPl.Eb;
            B.Pb = BPl.Pb;
            B.tmem_cols = BPl.tmem_cols;
            B.out = out;
            B.sub_count = scratch.sub_count;
            B.sub_point = scratch.sub_point;
            B.sub_origin = scratch.sub_origin;
            B.sub_patch = scratch.sub_patch;
            B.surf_out = surf_out;
            B.flops = A.flops;
            B.status = scratch.status;
            // 512 Tensor Memory columns: one CTA per SM, which its shared memory reserves too
            // (no CTA of another launch can wait on this one's columns).
            const size_t bf_smem = std::max<size_t>(BPl.smem, tmem_smem_floor(BPl.tmem_cols, fa.sharedSizeBytes));
            if (bf_smem > dyn_max) return cudaErrorInvalidValue;
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(dyn_max));
            if (e != cudaSuccess) return e;
            const int bgrid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(pts.n, num_sms)));
            kern<<<bgrid, kBfThreads, bf_smem, stream>>>(B);
            e = cudaGetLastError();
            bf_done = true;
        }
    }
    if (!bf_done) {
        // UInt8: the three kernels are exact and give identical results, so the one to run is
        // a matter of speed -- by default the tensor-core kernel whose plan fits (k_corr_tc2
        // first); for large passes the autotuner times the candidates once per geometry on a
        // sample of the pass and the context keeps the fastest.
        TcPlan TP2{}, TP1{};
        const bool fit2 = tc_ok && plan_corr_tc2(geom, 220 * 1024, &TP2);
        const bool fit1 = tc_ok && plan_corr_tc(geom, 220 * 1024, &TP1);
        int kind = fit2 ? 2 : fit1 ? 1 : 0;
        const int force = scratch.uint8_kernel;
        if (force == 0 || (force == 1 && fit1) || (force == 2 && fit2)) kind = force;
        if (force < 0 && (fit2 || fit1) && scratch.autotune && !scratch.fixed &&
            pts.n >= kTuneMinPoints) {
            const uint64_t key = (static_cast<uint64_t>(geom.max_ch) << 48) |
                                 (static_cast<uint64_t>(geom.max_cw) << 32) |
                                 (static_cast<uint64_t>(geom.max_nr) << 16) |
                                 static_cast<uint64_t>(geom.max_nc);
            auto it = scratch.tuned.find(key);
            if (it != scratch.tuned.end()) {
                kind = it->second;
            } else {
                e = autotune_u8(scratch, stream, pts, out, surf_out != nullptr, fit2, fit1, &kind,
                                [&](int kk, const DevPoints& ds, const DevOutputs& dout) -> cudaError_t {
                                    if (kk == 2) return launch_tc(true, TP2, ds, 1, dout, nullptr);
                                    if (kk == 1) return launch_tc(false, TP1, ds, 1, dout, nullptr);
                                    return launch_direct(ds, 1, dout, nullptr);
                                });
                if (e != cudaSuccess) return e;
                scratch.tuned[key] = kind;
            }
        }
        if (kind == 2) {
            e = launch_tc(true, TP2, pts, up, out, A.flops);
        } else if (kind == 1) {
            e = launch_tc(false, TP1, pts, up, out, A.flops);
        } else {
            e = launch_direct(pts, up, out, A.flops);
        }
    }
    if (e != cudaSuccess) return e;
    T.launches += 1;
    if (T.enabled) cudaEventRecord(ev1, stream);
    if (up == 1) {
        if (T.enabled) {
            cudaEventRecord(ev2, stream);
            T.recs.push_back({ev0, ev1, ev2});
        }
        return cudaSuccess;
    }

    const RefinePlan R = plan_refine(up);
    RefineArgs B{};
    B.count = scratch.sub_count;
    B.n_items = 0;
    B.point = scratch.sub_point;
    B.origin = scratch.sub_origin;
    B.patch = scratch.sub_patch;
    B.pts = pts;
    B.out = out;
    B.levels = R.levels;
    B.warp_floats = R.warp_floats;
    if (R.smem > static_cast<size_t>(kDynSmemCap)) return cudaErrorInvalidValue;
    e = cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, kDynSmemCap);
    if (e != cudaSuccess) return e;
    const int rgrid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((pts.n + R.warps - 1) / R.warps,
                             static_cast<int64_t>(num_sms) * R.per_sm)));
    k_refine<<<rgrid, R.warps * 32, R.smem, stream>>>(B);
    e = cudaGetLastError();
    T.launches += 1;
    if (T.enabled) {
        cudaEventRecord(ev2, stream);
        T.recs.push_back({ev0, ev1, ev2});
    }
    return e;
}

cudaError_t launch_track(int dtype, const void* ref, const void* sec, const uint8_t* valid,
                         int64_t nrows, int64_t ncols, const DevPoints& pts,
                         const PassGeometry& geom, int up, int measure, const DevOutputs& out,
                         TrackScratch& scratch, int num_sms, cudaStream_t stream,
                         std::string* err, float* surf_out, const Rotation* rot) {
    cudaError_t e = scratch_acquire(scratch, stream);
    if (e != cudaSuccess) return e;
    e = launch_track_impl(dtype, ref, sec, valid, nrows, ncols, pts, geom, up, measure, out,
                          scratch, num_sms, stream, err, surf_out, rot);
    const cudaError_t r = scratch.done ? cudaEventRecord(scratch.done, stream) : cudaSuccess;
    return e != cudaSuccess ? e : r;
}

cudaError_t launch_refine_patches(const float* patches, int64_t count, int up, int32_t* row,
                                  int32_t* col, float* value, int num_sms, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const RefinePlan R = plan_refine(up);
    RefineArgs B{};
    B.count = nullptr;
    B.n_items = count;
    B.point = nullptr;
    B.origin = nullptr;
    B.patch = patches;
    B.orow = row;
    B.ocol = col;
    B.oval = value;
    B.levels = R.levels;
    B.warp_floats = R.warp_floats;
    if (R.smem > static_cast<size_t>(kDynSmemCap)) return cudaErrorInvalidValue;
    cudaError_t e =
        cudaFuncSetAttribute(k_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, kDynSmemCap);
    if (e != cudaSuccess) return e;
    const int grid = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((count + R.warps - 1) / R.warps,
                             static_cast<int64_t>(num_sms) * R.per_sm)));
    k_refine<<<grid, R.warps * 32, R.smem, stream>>>(B);
    return cudaGetLastError();
}

}  // namespace ar

// ---------------------------------------------------------------------------------------------
// Allocation-free track entry point.
//
// Some callers cannot allocate device memory at the time they correlate: a host that owns the
// whole device pool and hands out only the buffers it planned (an embedded or real-time
// service with a fixed memory budget), code running under another framework's allocator, or
// a caller that must not trigger cudaMalloc's implicit device synchronisation in the middle
// of a pipeline. For them the track pass can run with its scratch -- the refinement queue and
// the pass-geometry words -- in a fixed array in this file instead of context-owned buffers.
//
// The array is sized for kStaticMaxPoints points per call (about 3.8 MB, held by every GPU
// that loads the library until the process exits). Calls share it and it keeps the last
// call's contents; the queue counter and the geometry words are reset by every call before
// use, and so is the status word a bounded tensor-core wait sets when it runs out. Two calls
// that overlap on the GPU (different streams, or different host threads) race on it and must
// not be issued.

namespace ar {
namespace {

constexpr int64_t kStaticMaxPoints = 32768;
constexpr size_t kStaticGeomOff = 0;                                   // 8 x int64
constexpr size_t kStaticCountOff = 64;                                 // int
constexpr size_t kStaticStatusOff = 128;                               // int
constexpr size_t kStaticPointOff = 256;                                // int64 per point
constexpr size_t kStaticOriginOff = kStaticPointOff + 8 * kStaticMaxPoints;   // 2 x int32
constexpr size_t kStaticPatchOff = kStaticOriginOff + 8 * kStaticMaxPoints;   // 25 x float
constexpr size_t kStaticBytes = kStaticPatchOff + 100 * kStaticMaxPoints;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
unsigned char* g_static_addr[kStaticMaxDevices] = {};

// The device address of g_static_scratch on the current device, looked up once per device.
cudaError_t static_scratch(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kStaticMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_static_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_static_addr[dev];
    return cudaSuccess;
}

void static_message(char* buf, size_t size, const char* msg) {
    if (!buf || size == 0) return;
    size_t n = 0;
    while (msg[n] && n + 1 < size) {
        buf[n] = msg[n];
        ++n;
    }
    buf[n] = '\0';
}

}  // namespace
}  // namespace ar

extern "C" int ar_track_device_static(const void* ref, const void* sec, const uint8_t* valid,
                                      int64_t nrows, int64_t ncols, int dtype,
                                      const ar_points* pts, int upsampling, int measure,
                                      float* dx, float* dy, float* correlation,
                                      uint8_t* searched, void* stream, char* err,
                                      size_t err_size) {
    using namespace ar;
    if (!ref || !sec || !valid || !pts || nrows <= 0 || ncols <= 0) {
        static_message(err, err_size, "null or empty input");
        return AR_ERR_ARG;
    }
    if (pts->n < 0 || pts->n > kStaticMaxPoints) {
        static_message(err, err_size,
                       "point count outside [0, 32768], the capacity of the static scratch; "
                       "split the point set or use ar_track_device");
        return AR_ERR_SIZE;
    }
    if (pts->n > 0 && (!dx || !dy || !correlation || !searched || !pts->x || !pts->y ||
                       !pts->radius_x || !pts->radius_y || !pts->dx_prior || !pts->dy_prior ||
                       !pts->chip_size_x || !pts->chip_size_y)) {
        static_message(err, err_size, "null point-set field or output");
        return AR_ERR_ARG;
    }
    if (upsampling < 1 || upsampling > 128 || (upsampling & (upsampling - 1))) {
        static_message(err, err_size, "`upsampling` must be 1 or a power of 2 up to 128");
        return AR_ERR_ARG;
    }
    if (measure != AR_ZNCC && measure != AR_NCC) {
        static_message(err, err_size, "unknown measure");
        return AR_ERR_ARG;
    }
    if (dtype != AR_U8 && dtype != AR_U16 && dtype != AR_I16 && dtype != AR_F32) {
        static_message(err, err_size, "unsupported element type");
        return AR_ERR_UNSUPPORTED;
    }
    if (pts->n == 0) return AR_OK;
    unsigned char* base = nullptr;
    cudaError_t e = static_scratch(&base);
    if (e != cudaSuccess) {
        static_message(err, err_size, cudaGetErrorString(e));
        return AR_ERR_CUDA;
    }
    // A view of the static array in the scratch layout the track launch expects. Its capacity
    // covers the call, so the launch allocates nothing; timing stays off (no events).
    TrackScratch view;
    view.geom = reinterpret_cast<int64_t*>(base + kStaticGeomOff);
    view.sub_count = reinterpret_cast<int*>(base + kStaticCountOff);
    view.sub_point = reinterpret_cast<int64_t*>(base + kStaticPointOff);
    view.sub_origin = reinterpret_cast<int32_t*>(base + kStaticOriginOff);
    view.sub_patch = reinterpret_cast<float*>(base + kStaticPatchOff);
    view.status = reinterpret_cast<int*>(base + kStaticStatusOff);
    view.capacity = kStaticMaxPoints;
    view.fixed = true;  // the launch helpers then neither allocate nor create events
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(view.status, 0, sizeof(int), s);
    if (e != cudaSuccess) {
        static_message(err, err_size, cudaGetErrorString(e));
        return AR_ERR_CUDA;
    }
    DevPoints dp{pts->x, pts->y, pts->radius_x, pts->radius_y, pts->dx_prior, pts->dy_prior,
                 pts->chip_size_x, pts->chip_size_y, pts->n};
    PassGeometry geom;
    e = pass_geometry_device(dp, nrows, ncols, view, s, &geom);
    int num_sms = 148;
    int dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    std::string msg;
    DevOutputs out{dx, dy, correlation, searched};
    if (e == cudaSuccess)
        e = launch_track(dtype, ref, sec, valid, nrows, ncols, dp, geom, upsampling, measure, out,
                         view, num_sms, s, &msg);
    if (e != cudaSuccess) {
        static_message(err, err_size, msg.empty() ? cudaGetErrorString(e) : msg.c_str());
        return msg.empty() ? AR_ERR_CUDA : AR_ERR_UNSUPPORTED;
    }
    // Wait for the pass and read its status word: a bounded tensor-core wait that ran out
    // leaves the outputs incomplete, which the caller must learn of.
    int status = 0;
    e = cudaMemcpyAsync(&status, view.status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        static_message(err, err_size, cudaGetErrorString(e));
        return AR_ERR_CUDA;
    }
    if (status) {
        static_message(err, err_size, "a device wait ran out; results incomplete");
        return AR_ERR_TIMEOUT;
    }
    return AR_OK;
}

extern "C" int ar_scratch_allocations(int64_t* count) {
    if (!count) return AR_ERR_ARG;
    *count = ar::scratch_allocations();
    return AR_OK;
}

#ifdef AR_TC_PHASES
// Profiling builds only: the phase counters of k_corr_tc (16 entries), then cleared.
extern "C" int ar_tc_phase_read(unsigned long long* out) {
    cudaDeviceSynchronize();
    if (cudaMemcpyFromSymbol(out, ar::g_tc_phase, 16 * sizeof(unsigned long long)) != cudaSuccess)
        return 1;
    const unsigned long long z[16] = {};
    return cudaMemcpyToSymbol(ar::g_tc_phase, z, sizeof(z)) == cudaSuccess ? 0 : 1;
}
#endif
