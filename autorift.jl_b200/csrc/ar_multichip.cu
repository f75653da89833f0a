// The multi-chip-size search on the device: correlate_multichip (src/multichip.jl:106-422).
//
// Each chip-size level is a sequence of passes over the point grid, all on the device: the
// level's radii (src/multichip.jl:193-213 with sanitize!, src/points.jl:332-346), the coarse
// pass (decimation with the cell-maximum radius, an integer-peak track, the relaxed Gardner
// filter, the coverage gate, Euclidean dilation and nearest resampling back to the grid,
// src/multichip.jl:224-306), the fine track, outlier rejection and three passes of median hole
// filling (src/multichip.jl:318-390), and the merge into the result (src/multichip.jl:401-422).
// The host only reads a handful of counters per level to take the reference's early exits.
//
// The grid reductions follow src/window.jl:474-637 and src/outliers.jl:90-172 operation for
// operation in Float32 (normalised displacements, agreement counts, insertion-sorted medians
// and MADs) and Float64 (the tolerance floors), so a grid pass is bit-identical to the
// reference's on the same inputs.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "ar_internal.cuh"

namespace ar {
namespace {

constexpr int kT = 256;
constexpr int kMaxWin = 9;  // largest outlier / fill window handled (81 gathered values)

inline unsigned blocks(int64_t n) { return static_cast<unsigned>((n + kT - 1) / kT); }

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fc00000); }

// _level_points + sanitize!: the level's radii, zero where a finer level already owns a point.
__global__ void k_level_points(const int64_t* grx, const int64_t* gry, const uint16_t* rcs,
                               int64_t n, int64_t min_r, int64_t* rx, int64_t* ry,
                               unsigned long long* count) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int c = 0;
    if (i < n) {
        int64_t a = rcs[i] == 0 ? grx[i] : 0, b = rcs[i] == 0 ? gry[i] : 0;
        if (a <= 0 || b <= 0) {
            a = 0;
            b = 0;
        } else {
            a = max(a, min_r);
            b = max(b, min_r);
            c = 1;
        }
        rx[i] = a;
        ry[i] = b;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

__global__ void k_fill_i64(int64_t* a, int64_t n, int64_t v) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) a[i] = v;
}

// pts[rows, cols] with rows = stride:stride:gr, and the cell-maximum radius
// (src/multichip.jl:247-251, 292-306).
__global__ void k_coarse_points(const double* gx, const double* gy, const double* gdx0,
                                const double* gdy0, const int64_t* rx, const int64_t* ry,
                                int64_t gr, int64_t gc, int64_t st, int64_t cr, int64_t cc,
                                int64_t csx, int64_t csy, double* cx, double* cy, double* cdx0,
                                double* cdy0, int64_t* crx, int64_t* cry, int64_t* ccsx,
                                int64_t* ccsy, unsigned long long* count) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int c = 0;
    if (k < cr * cc) {
        const int64_t io = k % cr, jo = k / cr;
        const int64_t i = (io + 1) * st - 1, j = (jo + 1) * st - 1;
        const int64_t f = i + j * gr;
        cx[k] = gx[f];
        cy[k] = gy[f];
        cdx0[k] = gdx0[f];
        cdy0[k] = gdy0[f];
        const int64_t lo = st / 2, hi = st - 1 - lo;
        int64_t mx = 0, my = 0;
        for (int64_t jj = max(j - lo, int64_t(0)); jj <= min(j + hi, gc - 1); ++jj)
            for (int64_t ii = max(i - lo, int64_t(0)); ii <= min(i + hi, gr - 1); ++ii) {
                mx = max(mx, rx[ii + jj * gr]);
                my = max(my, ry[ii + jj * gr]);
            }
        crx[k] = mx;
        cry[k] = my;
        ccsx[k] = csx;
        ccsy[k] = csy;
        c = (mx > 0 && my > 0) ? 1 : 0;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

// measured = !isnan(dx), counted.
__global__ void k_measured(const float* dx, int64_t n, uint8_t* measured,
                           unsigned long long* count) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int c = 0;
    if (i < n) {
        const uint8_t m = isnan(dx[i]) ? 0 : 1;
        measured[i] = m;
        c = m;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

// Normalised displacements (src/outliers.jl:98-106) and keep = valid.
__global__ void k_normalize(const float* dx, const float* dy, const int64_t* rx, const int64_t* ry,
                            const uint8_t* valid, int64_t n, float* nx, float* ny, uint8_t* keep) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    nx[i] = rx[i] > 0 ? __fdiv_rn(dx[i], static_cast<float>(rx[i])) : qnan();
    ny[i] = ry[i] > 0 ? __fdiv_rn(dy[i], static_cast<float>(ry[i])) : qnan();
    keep[i] = valid[i];
}

// _mask_to_nan! (src/outliers.jl:165-172).
__global__ void k_mask_nan(const uint8_t* keep, int64_t n, float* nx, float* ny) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n && !keep[i]) {
        nx[i] = qnan();
        ny[i] = qnan();
    }
}

struct Win {
    int lx, ly, rx, ry;
};

// The window clamped to the grid, extra element of an even width on the left
// (src/window.jl:254-257, 632-637).
inline Win window_of(int64_t w, int64_t nr, int64_t nc) {
    const int wx = static_cast<int>(std::min(w, nc)), wy = static_cast<int>(std::min(w, nr));
    return {wx / 2, wy / 2, wx - 1 - wx / 2, wy - 1 - wy / 2};
}

__device__ int count_agree(const float* A, int64_t nr, int64_t nc, int64_t i, int64_t j, Win W,
                           float t) {
    const float c = A[i + j * nr];
    if (isnan(c)) return 0;
    int n = 0;
    for (int64_t jj = max(j - W.lx, int64_t(0)); jj <= min(j + W.rx, nc - 1); ++jj)
        for (int64_t ii = max(i - W.ly, int64_t(0)); ii <= min(i + W.ry, nr - 1); ++ii)
            if (fabsf(__fsub_rn(A[ii + jj * nr], c)) < t) ++n;
    return n;
}

// Stage 1 of the Gardner filter (src/outliers.jl:118-127, count_agreeing src/window.jl:594-619).
__global__ void k_agree(const float* nx, const float* ny, int64_t nr, int64_t nc, Win W, float t,
                        float needed, uint8_t* keep) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nr * nc) return;
    const int64_t i = k % nr, j = k / nr;
    const float ax = static_cast<float>(count_agree(nx, nr, nc, i, j, W, t));
    const float ay = static_cast<float>(count_agree(ny, nr, nc, i, j, W, t));
    keep[k] = (ax >= needed && ay >= needed) ? 1 : 0;
}

__device__ void isort(float* b, int n) {
    for (int k = 1; k < n; ++k) {
        const float v = b[k];
        int m = k - 1;
        while (m >= 0 && b[m] > v) {
            b[m + 1] = b[m];
            --m;
        }
        b[m + 1] = v;
    }
}

__device__ __forceinline__ float smedian(const float* b, int n) {
    return (n & 1) ? b[(n + 1) / 2 - 1] : __fdiv_rn(__fadd_rn(b[n / 2 - 1], b[n / 2]), 2.0f);
}

// Median and MAD of the non-NaN window values (src/window.jl:513-563); false when empty.
__device__ bool medmad(const float* A, int64_t nr, int64_t nc, int64_t i, int64_t j, Win W,
                       float* med, float* mad) {
    float b[kMaxWin * kMaxWin];
    int n = 0;
    for (int64_t jj = max(j - W.lx, int64_t(0)); jj <= min(j + W.rx, nc - 1); ++jj)
        for (int64_t ii = max(i - W.ly, int64_t(0)); ii <= min(i + W.ry, nr - 1); ++ii) {
            const float v = A[ii + jj * nr];
            if (!isnan(v)) b[n++] = v;
        }
    if (n == 0) return false;
    isort(b, n);
    const float m = smedian(b, n);
    for (int k = 0; k < n; ++k) b[k] = fabsf(__fsub_rn(b[k], m));
    isort(b, n);
    *med = m;
    *mad = smedian(b, n);
    return true;
}

// Bitonic sort of 32 register values, ascending (every index is a compile-time constant once
// the loops unroll, so the array stays in registers).
__device__ __forceinline__ void bitonic32(float (&v)[32]) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const float a = v[i], b = v[l];
                    const bool up = (i & k) == 0;
                    v[i] = up ? fminf(a, b) : fmaxf(a, b);
                    v[l] = up ? fmaxf(a, b) : fminf(a, b);
                }
            }
}

// smedian of the first n of 32 sorted register values (n >= 1), selected without indexing.
__device__ __forceinline__ float smedian32(const float (&v)[32], int n) {
    const int k0 = (n & 1) ? (n + 1) / 2 - 1 : n / 2 - 1, k1 = (n & 1) ? k0 : n / 2;
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int t = 0; t < 25; ++t) {
        if (t == k0) a = v[t];
        if (t == k1) b = v[t];
    }
    return (n & 1) ? a : __fdiv_rn(__fadd_rn(a, b), 2.0f);
}

// medmad for windows of at most 5 x 5: the values in registers, NaN and absent entries as +Inf
// (they sort after every value, and only the first n are read), sorted by a network instead of
// an insertion sort in local memory. Same median and MAD: both are order statistics of the
// same multiset, and signed zeros only ever enter through differences and magnitudes.
__device__ bool medmad25(const float* A, int64_t nr, int64_t nc, int64_t i, int64_t j, Win W,
                         float* med, float* mad) {
    float v[32];
    int n = 0;
#pragma unroll
    for (int dj = 0; dj < 5; ++dj)
#pragma unroll
        for (int di = 0; di < 5; ++di) {
            const int64_t jj = j - W.lx + dj, ii = i - W.ly + di;
            const bool in = dj <= W.lx + W.rx && di <= W.ly + W.ry && jj >= 0 && jj < nc &&
                            ii >= 0 && ii < nr;
            const float x = in ? A[ii + jj * nr] : __int_as_float(0x7fc00000);
            const bool ok = !isnan(x);
            v[dj * 5 + di] = ok ? x : INFINITY;
            n += ok ? 1 : 0;
        }
#pragma unroll
    for (int t = 25; t < 32; ++t) v[t] = INFINITY;
    if (n == 0) return false;
    bitonic32(v);
    const float m = smedian32(v, n);
#pragma unroll
    for (int t = 0; t < 32; ++t) v[t] = t < n ? fabsf(__fsub_rn(v[t], m)) : INFINITY;
    bitonic32(v);
    *med = m;
    *mad = smedian32(v, n);
    return true;
}

// Stage 2 of the Gardner filter (src/outliers.jl:139-158).
__global__ void k_madtest(const float* nx, const float* ny, const int64_t* rx, const int64_t* ry,
                          int64_t nr, int64_t nc, Win W, int up, double scale, uint8_t* keep) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nr * nc || !keep[k]) return;
    const int64_t i = k % nr, j = k / nr;
    float mx = qnan(), sx = qnan(), my = qnan(), sy = qnan();
    const bool small = W.lx + W.rx < 5 && W.ly + W.ry < 5;
    const bool okx = small ? medmad25(nx, nr, nc, i, j, W, &mx, &sx)
                           : medmad(nx, nr, nc, i, j, W, &mx, &sx);
    const bool oky = small ? medmad25(ny, nr, nc, i, j, W, &my, &sy)
                           : medmad(ny, nr, nc, i, j, W, &my, &sy);
    const double fx = rx[k] > 0 ? __ddiv_rn(2.0, static_cast<double>(up * rx[k])) : INFINITY;
    const double fy = ry[k] > 0 ? __ddiv_rn(2.0, static_cast<double>(up * ry[k])) : INFINITY;
    const double tolx = fmax(__dmul_rn(scale, static_cast<double>(sx)), fx);
    const double toly = fmax(__dmul_rn(scale, static_cast<double>(sy)), fy);
    // A NaN median (no valid neighbour) fails the comparison: the point is dropped.
    const bool kx = okx && static_cast<double>(fabsf(__fsub_rn(nx[k], mx))) <= tolx;
    const bool ky = oky && static_cast<double>(fabsf(__fsub_rn(ny[k], my))) <= toly;
    keep[k] = (kx && ky) ? 1 : 0;
}

// keep &= measured, and the coverage gate's counts (src/multichip.jl:265-278).
__global__ void k_gate(uint8_t* keep, const uint8_t* measured, const int64_t* crx, int64_t n,
                       unsigned long long* counts) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int d = 0, m = 0;
    if (k < n) {
        if (!measured[k]) keep[k] = 0;
        if (crx[k] > 0 && measured[k]) {
            d = 1;
            m = keep[k] ? 1 : 0;
        }
    }
    d = __reduce_add_sync(0xffffffffu, d);
    m = __reduce_add_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) {
        if (d) atomicAdd(&counts[0], static_cast<unsigned long long>(d));
        if (m) atomicAdd(&counts[1], static_cast<unsigned long long>(m));
    }
}

// dilate_within (src/resample.jl:190-325): true within Euclidean `radius` of a true, tested
// directly over the disc (the same predicate as the squared-distance transform's d2 <= r^2).
__global__ void k_dilate(const uint8_t* m, int64_t nr, int64_t nc, int64_t radius, uint8_t* out) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nr * nc) return;
    const int64_t i = k % nr, j = k / nr, r2 = radius * radius;
    uint8_t v = 0;
    for (int64_t dj = -radius; dj <= radius && !v; ++dj) {
        const int64_t jj = j + dj;
        if (jj < 0 || jj >= nc) continue;
        for (int64_t di = -radius; di <= radius; ++di) {
            const int64_t ii = i + di;
            if (di * di + dj * dj > r2 || ii < 0 || ii >= nr) continue;
            if (m[ii + jj * nr]) {
                v = 1;
                break;
            }
        }
    }
    out[k] = v;
}

// resample(grown, (gr, gc), Nearest()) .> 0.5 (src/resample.jl:56-71) applied to the level's
// radii (src/multichip.jl:174-179), and the searchable count.
__global__ void k_apply_coarse(const uint8_t* grown, int64_t cr, int64_t cc, int64_t gr, int64_t gc,
                               int64_t* rx, int64_t* ry, unsigned long long* count) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int c = 0;
    if (k < gr * gc) {
        const int64_t i = k % gr + 1, j = k / gr + 1;
        const double ys = __ddiv_rn(static_cast<double>(cr), static_cast<double>(gr));
        const double xs = __ddiv_rn(static_cast<double>(cc), static_cast<double>(gc));
        int64_t si = static_cast<int64_t>(floor(__dmul_rn(static_cast<double>(i) - 0.5, ys))) + 1;
        int64_t sj = static_cast<int64_t>(floor(__dmul_rn(static_cast<double>(j) - 0.5, xs))) + 1;
        si = min(max(si, int64_t(1)), cr);
        sj = min(max(sj, int64_t(1)), cc);
        if (!grown[(si - 1) + (sj - 1) * cr]) {
            rx[k] = 0;
            ry[k] = 0;
        }
        c = (rx[k] > 0 && ry[k] > 0) ? 1 : 0;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

__global__ void k_apply_reject(const uint8_t* keep, int64_t n, float* dx, float* dy, float* corr) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n && !keep[k]) {
        dx[k] = qnan();
        dy[k] = qnan();
        corr[k] = qnan();
    }
}

// One pass of _fill_holes! (src/multichip.jl:347-390): reads the pass-start field (ix, iy),
// writes the filled field (ox, oy); every point sees the same input, as the reference's
// two-phase pass.
__global__ void k_fill(const float* ix, const float* iy, int64_t nr, int64_t nc, int w,
                       float* ox, float* oy, uint8_t* filled) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nr * nc) return;
    float vx = ix[k], vy = iy[k];
    if (isnan(vx)) {
        const int64_t i = k % nr, j = k / nr;
        const int lo = w / 2, hi = w - 1 - lo, needed = 2 * w * w / 3;
        float bx[kMaxWin * kMaxWin], by[kMaxWin * kMaxWin];
        int n = 0;
        for (int64_t jj = max(j - lo, int64_t(0)); jj <= min(j + hi, nc - 1); ++jj)
            for (int64_t ii = max(i - lo, int64_t(0)); ii <= min(i + hi, nr - 1); ++ii) {
                const float v = ix[ii + jj * nr];
                if (isnan(v)) continue;
                bx[n] = v;
                by[n] = iy[ii + jj * nr];
                ++n;
            }
        if (n >= needed) {
            isort(bx, n);
            isort(by, n);
            vx = smedian(bx, n);
            vy = smedian(by, n);
            filled[k] = 1;
        }
    }
    ox[k] = vx;
    oy[k] = vy;
}

// _merge_level! (src/multichip.jl:401-422).
__global__ void k_merge(const float* ldx, const float* ldy, const float* lc, const uint8_t* filled,
                        int64_t n, uint16_t cs, float* rdx, float* rdy, float* rc, uint16_t* rcs,
                        uint8_t* rint, unsigned long long* unresolved) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int u = 0;
    if (k < n) {
        if (rcs[k] == 0 && !isnan(ldx[k])) {
            rdx[k] = ldx[k];
            rdy[k] = ldy[k];
            rc[k] = lc[k];
            rcs[k] = cs;
            rint[k] = filled[k];
        }
        u = rcs[k] == 0 ? 1 : 0;
    }
    u = __reduce_add_sync(0xffffffffu, u);
    if ((threadIdx.x & 31) == 0 && u) atomicAdd(unresolved, static_cast<unsigned long long>(u));
}

__global__ void k_init_result(int64_t n, float* dx, float* dy, float* c, uint16_t* cs, uint8_t* in) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) {
        dx[k] = qnan();
        dy[k] = qnan();
        c[k] = qnan();
        cs[k] = 0;
        in[k] = 0;
    }
}

// Shape bin of a point: -1 not searchable, 0 a surface of at most 64 x 64 (every tensor-core
// kernel and the split-BF16 kernel take it), 1 a larger one. A pass whose points fall in both
// bins runs each bin as its own launch, planned for that bin's largest surface, so a few wide
// searches do not put the whole pass on the wide-surface kernels.
__device__ __forceinline__ int shape_bin(int64_t rx, int64_t ry) {
    if (!(rx > 0 && ry > 0)) return -1;
    return (2 * rx <= 64 && 2 * ry <= 64) ? 0 : 1;
}

// Points per shape bin (count[0], count[1]), one atomic per warp and bin.
__global__ void k_count_bins(const int64_t* rx, const int64_t* ry, int64_t n,
                             unsigned long long* count) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int b = k < n ? shape_bin(rx[k], ry[k]) : -1;
    const unsigned m0 = __ballot_sync(0xffffffffu, b == 0), m1 = __ballot_sync(0xffffffffu, b == 1);
    if ((threadIdx.x & 31) == 0) {
        if (m0) atomicAdd(&count[0], static_cast<unsigned long long>(__popc(m0)));
        if (m1) atomicAdd(&count[1], static_cast<unsigned long long>(__popc(m1)));
    }
}

// Compaction of a pass to its searchable points of shape bin `bin` (-1: every searchable
// point, both radii > 0): the other points of a level are skipped by the track kernels anyway,
// but each would still cost a CTA a loop iteration.
__global__ void k_compact(const int64_t* rx, const int64_t* ry, int64_t n, int bin, int64_t* idx,
                          unsigned long long* count) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int b = k < n ? shape_bin(rx[k], ry[k]) : -1;
    const bool take = b >= 0 && (bin < 0 || b == bin);
    const unsigned m = __ballot_sync(0xffffffffu, take);
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == 0 && m) base = atomicAdd(count, static_cast<unsigned long long>(__popc(m)));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (take) idx[base + __popc(m & ((1u << lane) - 1u))] = k;
}

__global__ void k_gather_points(const int64_t* idx, int64_t ns, DevPoints P, double* x, double* y,
                                int64_t* rx, int64_t* ry, double* dx0, double* dy0, int64_t* csx,
                                int64_t* csy) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= ns) return;
    const int64_t k = idx[i];
    x[i] = P.x[k];
    y[i] = P.y[k];
    rx[i] = P.rx[k];
    ry[i] = P.ry[k];
    dx0[i] = P.dx0[k];
    dy0[i] = P.dy0[k];
    csx[i] = P.csx[k];
    csy[i] = P.csy[k];
}

// Unmeasured outputs everywhere (src/track.jl:58-62), then the compacted results in place.
__global__ void k_unmeasured(DevOutputs O, int64_t n) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k < n) {
        O.dx[k] = qnan();
        O.dy[k] = qnan();
        O.corr[k] = qnan();
        O.searched[k] = 0;
    }
}

__global__ void k_scatter_outputs(const int64_t* idx, int64_t ns, DevOutputs C, DevOutputs O) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= ns) return;
    const int64_t k = idx[i];
    O.dx[k] = C.dx[i];
    O.dy[k] = C.dy[i];
    O.corr[k] = C.corr[i];
    O.searched[k] = C.searched[i];
}

// A bump allocator over one device block.
struct Arena {
    unsigned char* base;
    size_t size, off;
    template <typename T>
    T* take(int64_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += static_cast<size_t>(count) * sizeof(T);
        return p;
    }
};

struct Counter {
    unsigned long long* dev;
    cudaStream_t s;
    cudaError_t* err;
    void zero(int k = 1) {
        if (*err == cudaSuccess) *err = cudaMemsetAsync(dev, 0, 8 * k, s);
    }
    // Counter values 0..k-1 after the stream drains (zero on an earlier error).
    void read(unsigned long long* h, int k = 1) {
        for (int q = 0; q < k; ++q) h[q] = 0;
        if (*err == cudaSuccess) *err = cudaMemcpyAsync(h, dev, 8 * k, cudaMemcpyDeviceToHost, s);
        if (*err == cudaSuccess) *err = cudaStreamSynchronize(s);
    }
    unsigned long long read1() {
        unsigned long long h = 0;
        read(&h, 1);
        return h;
    }
};

}  // namespace

size_t multichip_arena_bytes(int64_t gr, int64_t gc) {
    const int64_t n = gr * gc;
    // Level radii and chip sizes (4 x i64), fine outputs (3 f32 + u8), Gardner scratch
    // (2 f32 + 2 u8), fill ping-pong (2 f32 + u8), coarse copies (<= n of 8 fields + outputs),
    // the compacted pass (index, 8 fields, outputs), counters and alignment slack.
    return static_cast<size_t>(n) * (4 * 8 + 13 + 10 + 9 + 8 * 8 + 13 + 4 + 4 + 8 + 8 * 8 + 13) +
           80 * 256 + 4096;
}

cudaError_t run_multichip(const MultichipJob& J, TrackScratch& scratch, int num_sms,
                          cudaStream_t s, std::string* errmsg) {
    const int64_t gr = J.gr, gc = J.gc, n = gr * gc;
    cudaError_t err = cudaSuccess;
    Arena A{static_cast<unsigned char*>(J.arena), J.arena_bytes, 0};
    Counter C{A.take<unsigned long long>(4), s, &err};
    int64_t* rx = A.take<int64_t>(n);
    int64_t* ry = A.take<int64_t>(n);
    int64_t* csx = A.take<int64_t>(n);
    int64_t* csy = A.take<int64_t>(n);
    float* fdx = A.take<float>(n);
    float* fdy = A.take<float>(n);
    float* fc = A.take<float>(n);
    uint8_t* fs = A.take<uint8_t>(n);
    float* nx = A.take<float>(n);
    float* ny = A.take<float>(n);
    uint8_t* measured = A.take<uint8_t>(n);
    uint8_t* keep = A.take<uint8_t>(n);
    float* gx2 = A.take<float>(n);
    float* gy2 = A.take<float>(n);
    uint8_t* filled = A.take<uint8_t>(n);
    const int64_t st = J.P.stride;
    const int64_t cr = gr / st, cc = gc / st, m = cr * cc;
    double* cx = A.take<double>(m);
    double* cy = A.take<double>(m);
    double* cdx0 = A.take<double>(m);
    double* cdy0 = A.take<double>(m);
    int64_t* crx = A.take<int64_t>(m);
    int64_t* cry = A.take<int64_t>(m);
    int64_t* ccsx = A.take<int64_t>(m);
    int64_t* ccsy = A.take<int64_t>(m);
    float* cdx = A.take<float>(m);
    float* cdy = A.take<float>(m);
    float* ccor = A.take<float>(m);
    uint8_t* cs_ = A.take<uint8_t>(m);
    uint8_t* grown = A.take<uint8_t>(m);
    // The compacted pass (coarse or fine, one at a time).
    int64_t* kidx = A.take<int64_t>(n);
    double* kx = A.take<double>(n);
    double* ky = A.take<double>(n);
    double* kdx0 = A.take<double>(n);
    double* kdy0 = A.take<double>(n);
    int64_t* krx = A.take<int64_t>(n);
    int64_t* kry = A.take<int64_t>(n);
    int64_t* kcsx = A.take<int64_t>(n);
    int64_t* kcsy = A.take<int64_t>(n);
    float* kdx = A.take<float>(n);
    float* kdy = A.take<float>(n);
    float* kc = A.take<float>(n);
    uint8_t* ks = A.take<uint8_t>(n);
    if (A.off > A.size) {
        if (errmsg) *errmsg = "multichip scratch too small";
        return cudaErrorInvalidValue;
    }
    const MultichipParams& P = J.P;
    if (P.outliers == 1 && (P.gwindow > kMaxWin || P.gwindow < 1)) {
        if (errmsg) *errmsg = "outlier window above the supported maximum (9)";
        return cudaErrorInvalidValue;
    }
    if (P.fill_window > kMaxWin || P.fill_window < 1) {
        if (errmsg) *errmsg = "fill window above the supported maximum (9)";
        return cudaErrorInvalidValue;
    }
    long long& L = scratch.timer.launches;
    k_init_result<<<blocks(n), kT, 0, s>>>(n, J.dx, J.dy, J.corr, J.chip, J.interp);
    ++L;

    // Gardner / NoOutlierFilter rejection of a field (src/outliers.jl:38-160) into `keep`.
    auto reject = [&](const float* dx, const float* dy, const int64_t* prx, const int64_t* pry,
                      int64_t nr, int64_t nc, int64_t iterations) {
        const int64_t nn = nr * nc;
        k_normalize<<<blocks(nn), kT, 0, s>>>(dx, dy, prx, pry, measured, nn, nx, ny, keep);
        ++L;
        if (P.outliers != 1) return;
        const Win W = window_of(P.gwindow, nr, nc);
        const float needed = static_cast<float>(P.gfrac * static_cast<double>(P.gwindow * P.gwindow));
        const float tol = static_cast<float>(P.gtol);
        for (int64_t it = 0; it < iterations; ++it) {
            k_mask_nan<<<blocks(nn), kT, 0, s>>>(keep, nn, nx, ny);
            k_agree<<<blocks(nn), kT, 0, s>>>(nx, ny, nr, nc, W, tol, needed, keep);
            L += 2;
        }
        const int64_t n2 = std::max<int64_t>(iterations - 1, 1);
        for (int64_t it = 0; it < n2; ++it) {
            k_mask_nan<<<blocks(nn), kT, 0, s>>>(keep, nn, nx, ny);
            k_madtest<<<blocks(nn), kT, 0, s>>>(nx, ny, prx, pry, nr, nc, W, J.P.up, P.gmad, keep);
            L += 2;
        }
    };

    // The level's similarity measure (measure_at, src/types.jl:893-894), set per level below.
    int level_measure = P.measure;

    // A track pass over the searchable points of P only, results scattered back into O.
    // The searchable points are counted per shape bin; when both bins are occupied each runs
    // as its own compacted launch, otherwise the whole pass runs as one.
    auto track_searchable = [&](const DevPoints& P, const DevOutputs& O, int up) {
        k_unmeasured<<<blocks(P.n), kT, 0, s>>>(O, P.n);
        ++L;
        C.zero(2);
        k_count_bins<<<blocks(P.n), kT, 0, s>>>(P.rx, P.ry, P.n, C.dev);
        ++L;
        unsigned long long cnt[2];
        C.read(cnt, 2);
        if (err != cudaSuccess) return;
        const bool split = scratch.shape_bins && cnt[0] > 0 && cnt[1] > 0;
        for (int bin = split ? 0 : -1; bin <= (split ? 1 : -1); ++bin) {
            const int64_t ns = static_cast<int64_t>(bin < 0 ? cnt[0] + cnt[1] : cnt[bin]);
            if (ns == 0) continue;
            if (err == cudaSuccess) err = cudaMemsetAsync(C.dev + 2, 0, 8, s);
            k_compact<<<blocks(P.n), kT, 0, s>>>(P.rx, P.ry, P.n, bin, kidx, C.dev + 2);
            k_gather_points<<<blocks(ns), kT, 0, s>>>(kidx, ns, P, kx, ky, krx, kry, kdx0, kdy0,
                                                       kcsx, kcsy);
            L += 2;
            DevPoints cp{kx, ky, krx, kry, kdx0, kdy0, kcsx, kcsy, ns};
            DevOutputs co{kdx, kdy, kc, ks};
            PassGeometry g;
            if (err == cudaSuccess) err = pass_geometry_device(cp, J.nrows, J.ncols, scratch, s, &g);
            if (err == cudaSuccess)
                err = launch_track(J.dtype, J.ref, J.sec, J.valid, J.nrows, J.ncols, cp, g, up,
                                   level_measure, co, scratch, num_sms, s, errmsg, nullptr,
                                   J.P.rot.count > 0 ? &J.P.rot : nullptr);
            if (err != cudaSuccess) return;
            k_scatter_outputs<<<blocks(ns), kT, 0, s>>>(kidx, ns, co, O);
            ++L;
        }
    };

    std::vector<int64_t> sizes;
    for (int64_t cs = P.chip_base; cs <= P.chip_max; cs *= 2)
        if (cs >= P.chip_min) sizes.push_back(cs);
    unsigned long long unresolved = static_cast<unsigned long long>(n);
    for (size_t li = 0; li < sizes.size(); ++li) {
        const int64_t cs = sizes[li];
        if (unresolved == 0) break;  // any(wanted) || break (src/multichip.jl:130-131)
        level_measure = P.n_level_measures > 0
                            ? P.level_measures[std::min(static_cast<int>(li),
                                                        P.n_level_measures - 1)]
                            : P.measure;
        const int64_t lcsx = cs;
        const int64_t lcsy = 2 * static_cast<int64_t>(std::nearbyint(static_cast<double>(cs) * P.aspect / 2.0));
        C.zero();
        k_level_points<<<blocks(n), kT, 0, s>>>(J.grx, J.gry, J.chip, n, P.min_radius, rx, ry, C.dev);
        k_fill_i64<<<blocks(n), kT, 0, s>>>(csx, n, lcsx);
        k_fill_i64<<<blocks(n), kT, 0, s>>>(csy, n, lcsy);
        L += 3;
        if (C.read1() == 0) continue;

        // Coarse pass (src/multichip.jl:224-288).
        const int64_t w = P.outliers == 1 ? P.gwindow : 0;
        if (!(cr < w || cc < w)) {
            if (m == 0) continue;  // an empty decimated grid has nothing searchable
            C.zero();
            k_coarse_points<<<blocks(m), kT, 0, s>>>(J.gx, J.gy, J.gdx0, J.gdy0, rx, ry, gr, gc, st,
                                                     cr, cc, lcsx, lcsy, cx, cy, cdx0, cdy0, crx,
                                                     cry, ccsx, ccsy, C.dev);
            ++L;
            if (C.read1() == 0) continue;
            DevPoints cp{cx, cy, crx, cry, cdx0, cdy0, ccsx, ccsy, m};
            DevOutputs co{cdx, cdy, ccor, cs_};
            if (err == cudaSuccess) track_searchable(cp, co, 1);
            C.zero();
            k_measured<<<blocks(m), kT, 0, s>>>(cdx, m, measured, C.dev);
            ++L;
            if (C.read1() == 0) continue;
            reject(cdx, cdy, crx, cry, cr, cc, std::max<int64_t>(P.giterations - 1, 1));
            C.zero(2);
            k_gate<<<blocks(m), kT, 0, s>>>(keep, measured, crx, m, C.dev);
            ++L;
            unsigned long long hcounts[2];
            C.read(hcounts, 2);
            if (hcounts[0] == 0 ||
                static_cast<double>(hcounts[1]) / static_cast<double>(hcounts[0]) < P.min_frac)
                continue;
            k_dilate<<<blocks(m), kT, 0, s>>>(keep, cr, cc, P.buffer, grown);
            C.zero();
            k_apply_coarse<<<blocks(n), kT, 0, s>>>(grown, cr, cc, gr, gc, rx, ry, C.dev);
            L += 2;
            if (C.read1() == 0) continue;
        }

        // Fine pass, rejection and filling (src/multichip.jl:182-183, 318-390).
        DevPoints fp{J.gx, J.gy, rx, ry, J.gdx0, J.gdy0, csx, csy, n};
        DevOutputs fo{fdx, fdy, fc, fs};
        if (err == cudaSuccess) track_searchable(fp, fo, static_cast<int>(P.up));
        C.zero();
        k_measured<<<blocks(n), kT, 0, s>>>(fdx, n, measured, C.dev);
        ++L;
        reject(fdx, fdy, rx, ry, gr, gc, P.giterations);
        k_apply_reject<<<blocks(n), kT, 0, s>>>(keep, n, fdx, fdy, fc);
        if (err == cudaSuccess) err = cudaMemsetAsync(filled, 0, n, s);
        // Three two-phase passes; a pass that fills nothing leaves every later pass a no-op.
        float* ax = fdx;
        float* ay = fdy;
        float* bx = gx2;
        float* by = gy2;
        for (int pass = 0; pass < 3; ++pass) {
            k_fill<<<blocks(n), kT, 0, s>>>(ax, ay, gr, gc, static_cast<int>(P.fill_window), bx, by, filled);
            std::swap(ax, bx);
            std::swap(ay, by);
        }
        C.zero();
        k_merge<<<blocks(n), kT, 0, s>>>(ax, ay, fc, filled, n, static_cast<uint16_t>(cs), J.dx, J.dy,
                                         J.corr, J.chip, J.interp, C.dev);
        L += 5;
        unresolved = C.read1();
        if (err == cudaSuccess) err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    if (err == cudaSuccess) err = cudaGetLastError();
    return err;
}

}  // namespace ar
