// CPU oracle for the dense ZNCC tracker -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++17, the algorithm of AutoRIFT.jl's hot path so that the
// CUDA library can be checked against it. It is never linked into the product: only the
// tests, the smoke check and the CPU-baseline leg of the benchmark load it.
//
// Parity pin: the restatement is checked against the reference's own golden vectors
// (test/fixtures/matchtemplate/zncc_*, test/fixtures/pyrup/*, test/fixtures/peak/*, read from
// the reference tree when present) and against golden vectors regenerated with OpenCV in
// tests/golden/make_golden.py.
//
// Every function cites the reference file:line it follows. Arrays are column-major (Julia
// layout: rows fastest), indices are 0-based here and converted where the reference's 1-based
// arithmetic matters (floor of a shifted coordinate, peak offsets).
//
// Floating point: compiled with -ffp-contract=off so that no a*b+c is fused, matching Julia,
// which never contracts without @fastmath/@muladd. The numerator is an FP64 direct sum -- the
// exact value the reference's single-precision FFT approximates (src/correlate.jl:785-848).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum Dtype { OR_U8 = 0, OR_U16 = 1, OR_F32 = 2, OR_I16 = 3, OR_F64 = 4 };
enum Measure { OR_ZNCC = 0, OR_NCC = 1 };

template <class T>
inline double as_f64(T v) { return static_cast<double>(v); }

// ---------------------------------------------------------------------------------------------
// src/correlate.jl:423-453 -- prepare_chip!: FP64 mean, Float32 mean-removed copy, FP64 norm,
// degenerate when the sum of squares is below eps(Float64) * ch * cw.
// `get(i, j)` returns the chip element at row i, column j (0-based).
template <class Get>
bool prepare_chip(Get get, int64_t ch, int64_t cw, float* dst, double* cnorm) {
    double s = 0.0;
    for (int64_t j = 0; j < cw; ++j)
        for (int64_t i = 0; i < ch; ++i) s += get(i, j);
    const double mean = s / static_cast<double>(ch * cw);
    double sq = 0.0;
    for (int64_t j = 0; j < cw; ++j)
        for (int64_t i = 0; i < ch; ++i) {
            const double d = get(i, j) - mean;
            dst[i + j * ch] = static_cast<float>(d);
            sq += d * d;
        }
    *cnorm = std::sqrt(sq);
    return sq > (DBL_EPSILON * static_cast<double>(ch)) * static_cast<double>(cw);
}

// src/integral.jl:141-170 -- integral_both!: per-window summed-area tables of x and x^2, one
// column-major traversal, (m+1) x (n+1) with a zero first row and column.
template <class Get>
void integral_both(Get get, int64_t m, int64_t n, double* S, double* S2) {
    const int64_t ld = m + 1;
    for (int64_t j = 0; j <= n; ++j) { S[0 + j * ld] = 0.0; S2[0 + j * ld] = 0.0; }
    for (int64_t i = 0; i <= m; ++i) { S[i] = 0.0; S2[i] = 0.0; }
    for (int64_t j = 0; j < n; ++j) {
        double run = 0.0, runsq = 0.0;
        for (int64_t i = 0; i < m; ++i) {
            const double v = get(i, j);
            run += v;
            runsq += v * v;
            S[(i + 1) + (j + 1) * ld] = run + S[(i + 1) + j * ld];
            S2[(i + 1) + (j + 1) * ld] = runsq + S2[(i + 1) + j * ld];
        }
    }
}

// src/integral.jl:244-247 -- boxsum, 0-based top-left (i, j) of an h x w block.
inline double boxsum(const double* S, int64_t ld, int64_t i, int64_t j, int64_t h, int64_t w) {
    return ((S[(i + h) + (j + w) * ld] - S[i + (j + w) * ld]) - S[(i + h) + j * ld]) +
           S[i + j * ld];
}

// src/correlate.jl:528-557, 575-630 -- correlate! with the ZNCC or NCC normaliser.
// The numerator is the FP64 direct sum of src/correlate.jl:799-814 (column-major order over
// the chip); the reference evaluates the same quantity with a single-precision FFT.
// Returns false (surface all zeros) for a degenerate chip.
template <class GetW, class GetC>
bool correlate(GetW getw, GetC getc, int64_t ch, int64_t cw, int64_t rx, int64_t ry, int measure,
               float* surface, std::vector<float>& chipbuf, std::vector<double>& S,
               std::vector<double>& S2, std::vector<double>& num) {
    const int64_t nr = 2 * ry, nc = 2 * rx;
    const int64_t wr = ch + 2 * ry - 1, wc = cw + 2 * rx - 1;
    chipbuf.resize(static_cast<size_t>(ch * cw));
    double cnorm = 0.0;
    const bool ok = prepare_chip(getc, ch, cw, chipbuf.data(), &cnorm);
    if (!ok) {
        std::fill(surface, surface + nr * nc, 0.0f);
        return false;
    }
    S.resize(static_cast<size_t>((wr + 1) * (wc + 1)));
    S2.resize(S.size());
    integral_both(getw, wr, wc, S.data(), S2.data());

    // Numerator: each shift accumulates jj-outer, ii-inner exactly as the direct loop; the
    // shifts themselves are independent, so the innermost loop runs over them.
    num.assign(static_cast<size_t>(nr * nc), 0.0);
    std::vector<double> col(static_cast<size_t>(wr));
    for (int64_t j = 0; j < nc; ++j) {
        double* acc = num.data() + j * nr;
        for (int64_t jj = 0; jj < cw; ++jj) {
            for (int64_t r = 0; r < wr; ++r) col[r] = getw(r, j + jj);
            for (int64_t ii = 0; ii < ch; ++ii) {
                const double c = static_cast<double>(chipbuf[ii + jj * ch]);
                const double* w = col.data() + ii;
                for (int64_t i = 0; i < nr; ++i) acc[i] += c * w[i];
            }
        }
    }

    const double n = static_cast<double>(ch * cw);
    const int64_t ld = wr + 1;
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            double den;
            if (measure == OR_NCC) {
                const double wsq = boxsum(S2.data(), ld, i, j, ch, cw);
                den = cnorm * std::sqrt(wsq < 0.0 ? 0.0 : wsq);
            } else {
                const double s1 = boxsum(S.data(), ld, i, j, ch, cw);
                const double s2 = boxsum(S2.data(), ld, i, j, ch, cw);
                double wvar = s2 - s1 * s1 / n;
                if (!(wvar > 0.0)) wvar = 0.0;
                den = cnorm * std::sqrt(wvar);
            }
            surface[i + j * nr] =
                den > 0.0 ? static_cast<float>(num[i + j * nr] / den) : 0.0f;
        }
    return true;
}

// src/peak.jl:32-61 -- row-major first strict maximum, NaN never selected, (0,0) by default.
void peak_index(const float* s, int64_t nr, int64_t nc, int64_t* bi, int64_t* bj) {
    int64_t best_i = 0, best_j = 0;
    float best = -INFINITY;
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            const float v = s[i + j * nr];
            if (v > best || (v == best && (i < best_i || (i == best_i && j < best_j)))) {
                best = v;
                best_i = i;
                best_j = j;
            }
        }
    *bi = best_i;
    *bj = best_j;
}

// src/peak.jl:374-382 -- reflect101_0.
inline int64_t reflect101_0(int64_t p, int64_t n) {
    if (n == 1) return 0;
    const int64_t m = n - 1;
    while (p < 0 || p > m) {
        if (p < 0) p = -p;
        if (p > m) p = 2 * m - p;
    }
    return p;
}

// src/peak.jl:312-324 -- _pyrup_taps, returned 0-based: (minus, centre, plus, ntaps).
inline void pyrup_taps(int64_t k0, int64_t n, int64_t* m, int64_t* c, int64_t* q, int* nt) {
    const int64_t p = k0;  // 0-based upsampled position
    if (p % 2 == 0) {
        *c = p / 2;
        *m = reflect101_0(p - 2, 2 * n) / 2;
        *q = reflect101_0(p + 2, 2 * n) / 2;
        *nt = 3;
    } else {
        *c = reflect101_0(p - 1, 2 * n) / 2;
        *m = *c;
        *q = reflect101_0(p + 1, 2 * n) / 2;
        *nt = 2;
    }
}

// src/peak.jl:297-299 -- the tap weights.
constexpr float W_C = 6.0f / 8;
constexpr float W_S = 1.0f / 8;
constexpr float W_H = 4.0f / 8;

// src/peak.jl:196-294 -- one pyrUp step, vertical then horizontal, Float32 throughout, in the
// reference's operation order: W_C*b + W_S*(a+c) for a sample position, W_H*(b+c) between.
void pyrup(const float* src, int64_t sh, int64_t sw, float* dst, std::vector<float>& tmp) {
    tmp.resize(static_cast<size_t>(2 * sh * sw));
    const int64_t th = 2 * sh;
    for (int64_t j = 0; j < sw; ++j)
        for (int64_t i = 0; i < th; ++i) {
            int64_t m, c, q;
            int nt;
            pyrup_taps(i, sh, &m, &c, &q, &nt);
            const float* s = src + j * sh;
            tmp[i + j * th] = nt == 3 ? W_C * s[c] + W_S * (s[m] + s[q]) : W_H * (s[c] + s[q]);
        }
    for (int64_t j = 0; j < 2 * sw; ++j) {
        int64_t m, c, q;
        int nt;
        pyrup_taps(j, sw, &m, &c, &q, &nt);
        for (int64_t i = 0; i < th; ++i) {
            const float a = tmp[i + m * th], b = tmp[i + c * th], cc = tmp[i + q * th];
            dst[i + j * th] = nt == 3 ? W_C * b + W_S * (a + cc) : W_H * (b + cc);
        }
    }
}

// src/peak.jl:102-106 -- peak_offset (1-based peak index minus the surface origin).
void peak_offset(const float* s, int64_t nr, int64_t nc, int64_t rx, int64_t ry, double* dx,
                 double* dy, float* v) {
    int64_t i, j;
    peak_index(s, nr, nc, &i, &j);
    *dx = static_cast<double>((j + 1) - rx - 1);
    *dy = static_cast<double>((i + 1) - ry - 1);
    *v = s[i + j * nr];
}

// src/peak.jl:456-522 -- subpixel_peak: clamp a 5x5 patch around the integer peak, cascade
// log2(up) pyrUp steps, row-major argmax, convert back to a displacement.
void subpixel_peak(const float* s, int64_t nr, int64_t nc, int64_t rx, int64_t ry, int up,
                   double* dx, double* dy, float* v, std::vector<float>& a,
                   std::vector<float>& b, std::vector<float>& tmp) {
    if (up == 1) { peak_offset(s, nr, nc, rx, ry, dx, dy, v); return; }
    const int64_t p = 5;
    int64_t pi, pj;
    peak_index(s, nr, nc, &pi, &pj);
    // 1-based clamp(pi - half, 1, max(nr - p + 1, 1)), here on 0-based indices.
    const int64_t half = p / 2;
    const int64_t i0 = std::clamp<int64_t>(pi - half, 0, std::max<int64_t>(nr - p, 0));
    const int64_t j0 = std::clamp<int64_t>(pj - half, 0, std::max<int64_t>(nc - p, 0));
    if (nr < p || nc < p) { peak_offset(s, nr, nc, rx, ry, dx, dy, v); return; }
    a.resize(static_cast<size_t>(p * up * p * up));
    b.resize(a.size());
    std::vector<float> patch(static_cast<size_t>(p * p));
    for (int64_t j = 0; j < p; ++j)
        for (int64_t i = 0; i < p; ++i) patch[i + j * p] = s[(i0 + i) + (j0 + j) * nr];
    int64_t n = p;
    int factor = 1;
    const float* cur = patch.data();
    bool use_a = true;
    while (factor < up) {
        float* dst = use_a ? a.data() : b.data();
        pyrup(cur, n, n, dst, tmp);
        n *= 2;
        factor *= 2;
        cur = dst;
        use_a = !use_a;
    }
    int64_t si, sj;
    peak_index(cur, n, n, &si, &sj);
    *v = cur[si + sj * n];
    const double row = static_cast<double>(si) / factor + static_cast<double>(i0);
    const double col = static_cast<double>(sj) / factor + static_cast<double>(j0);
    *dx = col - static_cast<double>(rx);
    *dy = row - static_cast<double>(ry);
}

// ---------------------------------------------------------------------------------------------
// The grid loop: src/track.jl:103-152 (pass set-up), 176-220 (geometry, +0.5 shift, padding),
// 249-305 (per point), src/points.jl:358-395 (chip and window bounds), 116-117, 421-425.

struct Points {
    const double *x, *y, *dx0, *dy0;
    const int64_t *rx, *ry, *csx, *csy;
    int64_t n;
};

// src/track.jl:377-409 -- _rotate_chip: the chip turned by `deg` degrees about its centre
// ((ch + 1) / 2, (cw + 1) / 2 in 1-based coordinates). Each destination pixel reads the source
// by the inverse rotation, interpolates bilinearly in FP64 from its four neighbours, is zero
// where any neighbour falls outside the chip, and is rounded to Float32 (the reference's
// rotation buffer). The angle in radians is deg * (pi / 180), Julia's deg2rad; sin and cos come
// from the C library. Operation order is the reference's, each operation rounded.
template <class Get>
void rotate_chip(Get get, int64_t ch, int64_t cw, double deg, float* dst) {
    const double r = deg * (M_PI / 180.0);
    const double s = std::sin(r), c = std::cos(r);
    const double yc = static_cast<double>(ch + 1) / 2.0, xc = static_cast<double>(cw + 1) / 2.0;
    for (int64_t j = 1; j <= cw; ++j)
        for (int64_t i = 1; i <= ch; ++i) {
            const double dy = static_cast<double>(i) - yc, dx = static_cast<double>(j) - xc;
            const double sy = (yc + c * dy) + s * dx;
            const double sx = (xc - s * dy) + c * dx;
            const double fi = std::floor(sy), fj = std::floor(sx);
            const int64_t i0 = static_cast<int64_t>(fi), j0 = static_cast<int64_t>(fj);
            float v = 0.0f;
            if (!(i0 < 1 || j0 < 1 || i0 + 1 > ch || j0 + 1 > cw)) {
                const double fy = sy - fi, fx = sx - fj;
                const double v00 = get(i0 - 1, j0 - 1), v10 = get(i0, j0 - 1);
                const double v01 = get(i0 - 1, j0), v11 = get(i0, j0);
                v = static_cast<float>((1.0 - fy) * ((1.0 - fx) * v00 + fx * v01) +
                                       fy * ((1.0 - fx) * v10 + fx * v11));
            }
            dst[(i - 1) + (j - 1) * ch] = v;
        }
}

// src/track.jl:313-350 -- _correlate_rotations! with a RotationSearch: correlate the chip
// turned by each angle (the chip itself at an angle of exactly 0), skip the angles whose
// turned chip is degenerate, and keep the surface whose maximum is strictly larger than every
// earlier one. Returns false (surface zero) when every angle is degenerate.
template <class GetW, class GetC>
bool correlate_rotations(GetW getw, GetC getc, int64_t ch, int64_t cw, int64_t rx, int64_t ry,
                         int measure, const double* angles, int nang, float* surface,
                         std::vector<float>& rot, std::vector<float>& hold,
                         std::vector<float>& chipbuf, std::vector<double>& S,
                         std::vector<double>& S2, std::vector<double>& num) {
    const int64_t ns = (2 * ry) * (2 * rx);
    hold.resize(static_cast<size_t>(ns));
    rot.resize(static_cast<size_t>(ch * cw));
    float best = -INFINITY;
    bool found = false;
    for (int a = 0; a < nang; ++a) {
        bool ok;
        if (angles[a] == 0.0) {
            ok = correlate(getw, getc, ch, cw, rx, ry, measure, surface, chipbuf, S, S2, num);
        } else {
            rotate_chip(getc, ch, cw, angles[a], rot.data());
            auto getr = [&](int64_t i, int64_t j) {
                return static_cast<double>(rot[static_cast<size_t>(i + j * ch)]);
            };
            ok = correlate(getw, getr, ch, cw, rx, ry, measure, surface, chipbuf, S, S2, num);
        }
        if (!ok) continue;
        float pk = surface[0];
        for (int64_t e = 1; e < ns; ++e)
            if (surface[e] > pk) pk = surface[e];
        if (pk > best) {
            best = pk;
            std::copy(surface, surface + ns, hold.begin());
            found = true;
        }
    }
    if (!found) {
        std::fill(surface, surface + ns, 0.0f);
        return false;
    }
    std::copy(hold.begin(), hold.end(), surface);
    return true;
}

inline int64_t floor_i(double v) { return static_cast<int64_t>(std::floor(v)); }

// Julia's `÷` on Int truncates toward zero.
inline int64_t jdiv(int64_t a, int64_t b) { return a / b; }

template <class T>
int track_impl(const T* ref, const T* sec, const uint8_t* refv, const uint8_t* secv,
               int64_t nrows, int64_t ncols, Points pts, int up, int measure, float* odx,
               float* ody, float* ocorr, uint8_t* osearched, int nthreads,
               const double* angles = nullptr, int nang = 0) {
    const int64_t n = pts.n;
    for (int64_t k = 0; k < n; ++k) {
        odx[k] = NAN;
        ody[k] = NAN;
        ocorr[k] = NAN;
        osearched[k] = 0;
    }
    // _pass_geometry (src/track.jl:176-197), on the unshifted points.
    int64_t cx = 0, cy = 0, mrx = 0, mry = 0, px = 0, py = 0;
    bool fits = true;
    for (int64_t k = 0; k < n; ++k) {
        if (!(pts.rx[k] > 0 && pts.ry[k] > 0)) continue;
        cx = std::max(cx, pts.csx[k]);
        cy = std::max(cy, pts.csy[k]);
        mrx = std::max(mrx, pts.rx[k]);
        mry = std::max(mry, pts.ry[k]);
        px = std::max(px, jdiv(pts.csx[k], 2) + pts.rx[k] +
                              static_cast<int64_t>(std::ceil(std::fabs(pts.dx0[k]))));
        py = std::max(py, jdiv(pts.csy[k], 2) + pts.ry[k] +
                              static_cast<int64_t>(std::ceil(std::fabs(pts.dy0[k]))));
        // inbounds (src/points.jl:421-425) with search_bounds on the unshifted point.
        const int64_t hx = jdiv(pts.csx[k], 2), hy = jdiv(pts.csy[k], 2);
        const int64_t wcx = floor_i(pts.x[k]), wcy = floor_i(pts.y[k]);
        const bool inb = (wcy - hy - pts.ry[k]) >= 1 && (wcy + hy + pts.ry[k] - 2) <= nrows &&
                         (wcx - hx - pts.rx[k]) >= 1 && (wcx + hx + pts.rx[k] - 2) <= ncols;
        fits = fits && inb;
    }
    if (cx == 0) return 0;
    const int64_t padx = fits ? 0 : px + 2, pady = fits ? 0 : py + 2;
    const int64_t NR = nrows + 2 * pady, NC = ncols + 2 * padx;  // padded extent
    const double shx = static_cast<double>(padx) + 0.5, shy = static_cast<double>(pady) + 0.5;

    // Padded-image readers (1-based padded coordinates): zero / false outside the image.
    auto pix = [&](const T* img, int64_t r1, int64_t c1) -> double {
        const int64_t r = r1 - 1 - pady, c = c1 - 1 - padx;
        if (r < 0 || r >= nrows || c < 0 || c >= ncols) return 0.0;
        return as_f64(img[r + c * nrows]);
    };
    auto okpix = [&](int64_t r1, int64_t c1) -> bool {
        const int64_t r = r1 - 1 - pady, c = c1 - 1 - padx;
        if (r < 0 || r >= nrows || c < 0 || c >= ncols) return false;
        return refv[r + c * nrows] != 0 && secv[r + c * nrows] != 0;
    };

#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        std::vector<float> surface, chipbuf, ba, bb, tmp, rot, hold;
        std::vector<double> S, S2, num;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
        for (int64_t k = 0; k < n; ++k) {
            const int64_t prx = pts.rx[k], pry = pts.ry[k];
            if (!(prx > 0 && pry > 0)) continue;
            const double xs = pts.x[k] + shx, ys = pts.y[k] + shy;
            const int64_t hx = jdiv(pts.csx[k], 2), hy = jdiv(pts.csy[k], 2);
            // chip_bounds (src/points.jl:358-366)
            const int64_t ccx = floor_i(xs - pts.dx0[k]), ccy = floor_i(ys - pts.dy0[k]);
            const int64_t cr0 = ccy - hy, cr1 = ccy + hy - 1, cc0 = ccx - hx, cc1 = ccx + hx - 1;
            // search_bounds (src/points.jl:385-395)
            const int64_t wcx = floor_i(xs), wcy = floor_i(ys);
            const int64_t wr0 = wcy - hy - pry, wr1 = wcy + hy + pry - 2;
            const int64_t wc0 = wcx - hx - prx, wc1 = wcx + hx + prx - 2;
            auto inb = [&](int64_t r0, int64_t r1, int64_t c0, int64_t c1) {
                if (r1 < r0 || c1 < c0) return true;  // empty range: checkbounds is true
                return r0 >= 1 && r1 <= NR && c0 >= 1 && c1 <= NC;
            };
            if (!inb(cr0, cr1, cc0, cc1)) continue;
            if (!inb(wr0, wr1, wc0, wc1)) continue;
            // _any_valid (src/track.jl:416-421)
            bool any = false;
            for (int64_t c = cc0; c <= cc1 && !any; ++c)
                for (int64_t r = cr0; r <= cr1; ++r)
                    if (okpix(r, c)) { any = true; break; }
            if (!any) continue;
            osearched[k] = 1;
            const int64_t ch = 2 * hy, cw = 2 * hx;
            auto getc = [&](int64_t i, int64_t j) { return pix(sec, cr0 + i, cc0 + j); };
            auto getw = [&](int64_t i, int64_t j) { return pix(ref, wr0 + i, wc0 + j); };
            const int64_t nr = 2 * pry, nc = 2 * prx;
            surface.resize(static_cast<size_t>(nr * nc));
            // _correlate_rotations! (src/track.jl:313-350): one correlation, or one per angle
            // with the best kept.
            const bool ok =
                nang == 0
                    ? correlate(getw, getc, ch, cw, prx, pry, measure, surface.data(), chipbuf, S,
                                S2, num)
                    : correlate_rotations(getw, getc, ch, cw, prx, pry, measure, angles, nang,
                                          surface.data(), rot, hold, chipbuf, S, S2, num);
            if (!ok) continue;  // degenerate: searched, no measurement
            double dx, dy;
            float c;
            subpixel_peak(surface.data(), nr, nc, prx, pry, up, &dx, &dy, &c, ba, bb, tmp);
            odx[k] = static_cast<float>(dx + pts.dx0[k]);
            ody[k] = static_cast<float>(dy + pts.dy0[k]);
            ocorr[k] = c;
        }
    }
    return 0;
}

template <class T>
bool correlate_arrays(const T* search, const T* chip, int64_t ch, int64_t cw, int64_t rx,
                      int64_t ry, int measure, float* surface) {
    const int64_t wr = ch + 2 * ry - 1;
    std::vector<float> chipbuf;
    std::vector<double> S, S2, num;
    auto getc = [&](int64_t i, int64_t j) { return as_f64(chip[i + j * ch]); };
    auto getw = [&](int64_t i, int64_t j) { return as_f64(search[i + j * wr]); };
    return correlate(getw, getc, ch, cw, rx, ry, measure, surface, chipbuf, S, S2, num);
}

// ---------------------------------------------------------------------------------------------
// Pre-correlation filters and quantisation: src/preprocess.jl:275-460, 546-592 and the
// sliding-window mean of src/window.jl:228-439 (banded running sums, 16-row bands).

// src/window.jl:632-637 -- window clamped to the array; src/window.jl:254-257 -- margins.
struct Margins { int64_t lx, ly, rx, ry; };
inline Margins margins(int64_t wx, int64_t wy) {
    return {wx / 2, wy / 2, wx - 1 - wx / 2, wy - 1 - wy / 2};
}

// src/window.jl:388-439 -- the dense path: no NaN, counts from the window geometry.
template <class Get>
void windowmean_dense(Get A, int64_t nr, int64_t nc, int64_t wx, int64_t wy, float* out) {
    const Margins m = margins(wx, wy);
    const int64_t nb = std::min<int64_t>(16, nr);
    std::vector<double> sums(static_cast<size_t>(nb * nc)), rowbuf(static_cast<size_t>(nc));
    for (int64_t i0 = 1; i0 <= nr;) {
        const int64_t i1 = std::min(i0 + nb - 1, nr);
        for (int64_t j = 1; j <= nc; ++j) {
            double s = 0.0;
            for (int64_t i = std::max<int64_t>(i0 - m.ly, 1); i <= std::min(i0 + m.ry, nr); ++i)
                s += A(i - 1, j - 1);
            for (int64_t i = i0; i <= i1; ++i) {
                sums[(i - i0) + (j - 1) * nb] = s;
                const int64_t oi = i - m.ly;
                if (1 <= oi && oi <= nr) s -= A(oi - 1, j - 1);
                const int64_t ii = i + m.ry + 1;
                if (ii <= nr) s += A(ii - 1, j - 1);
            }
        }
        for (int64_t i = i0; i <= i1; ++i) {
            const int64_t ci = std::min(i + m.ry, nr) - std::max<int64_t>(i - m.ly, 1) + 1;
            for (int64_t j = 1; j <= nc; ++j) rowbuf[j - 1] = sums[(i - i0) + (j - 1) * nb];
            double s = 0.0;
            for (int64_t j = 1; j <= std::min(m.rx + 1, nc); ++j) s += rowbuf[j - 1];
            for (int64_t j = 1; j <= nc; ++j) {
                const int64_t cj = std::min(j + m.rx, nc) - std::max<int64_t>(j - m.lx, 1) + 1;
                out[(i - 1) + (j - 1) * nr] = static_cast<float>(s / static_cast<double>(ci * cj));
                const int64_t oj = j - m.lx;
                if (1 <= oj && oj <= nc) s -= rowbuf[oj - 1];
                const int64_t jj = j + m.rx + 1;
                if (jj <= nc) s += rowbuf[jj - 1];
            }
        }
        i0 = i1 + 1;
    }
}

// src/window.jl:289-366 -- the masked path: NaN skipped, sums carried with counts.
template <class Get>
void windowmean_masked(Get A, int64_t nr, int64_t nc, int64_t wx, int64_t wy, float* out) {
    const Margins m = margins(wx, wy);
    const int64_t nb = std::min<int64_t>(16, nr);
    std::vector<double> sums(static_cast<size_t>(nb * nc)), rowbuf(static_cast<size_t>(nc));
    std::vector<int32_t> counts(static_cast<size_t>(nb * nc)), cntbuf(static_cast<size_t>(nc));
    for (int64_t i0 = 1; i0 <= nr;) {
        const int64_t i1 = std::min(i0 + nb - 1, nr);
        for (int64_t j = 1; j <= nc; ++j) {
            double s = 0.0;
            int32_t c = 0;
            for (int64_t i = std::max<int64_t>(i0 - m.ly, 1); i <= std::min(i0 + m.ry, nr); ++i) {
                const double v = A(i - 1, j - 1);
                if (!std::isnan(v)) { s += v; c += 1; }
            }
            for (int64_t i = i0; i <= i1; ++i) {
                sums[(i - i0) + (j - 1) * nb] = s;
                counts[(i - i0) + (j - 1) * nb] = c;
                const int64_t oi = i - m.ly;
                if (1 <= oi && oi <= nr) {
                    const double v = A(oi - 1, j - 1);
                    if (!std::isnan(v)) { s -= v; c -= 1; }
                }
                const int64_t ii = i + m.ry + 1;
                if (ii <= nr) {
                    const double v = A(ii - 1, j - 1);
                    if (!std::isnan(v)) { s += v; c += 1; }
                }
            }
        }
        for (int64_t i = i0; i <= i1; ++i) {
            for (int64_t j = 1; j <= nc; ++j) {
                rowbuf[j - 1] = sums[(i - i0) + (j - 1) * nb];
                cntbuf[j - 1] = counts[(i - i0) + (j - 1) * nb];
            }
            double s = 0.0;
            int64_t c = 0;
            for (int64_t j = 1; j <= std::min(m.rx + 1, nc); ++j) { s += rowbuf[j - 1]; c += cntbuf[j - 1]; }
            for (int64_t j = 1; j <= nc; ++j) {
                out[(i - 1) + (j - 1) * nr] =
                    c > 0 ? static_cast<float>(s / static_cast<double>(c)) : NAN;
                const int64_t oj = j - m.lx;
                if (1 <= oj && oj <= nc) { s -= rowbuf[oj - 1]; c -= cntbuf[oj - 1]; }
                const int64_t jj = j + m.rx + 1;
                if (jj <= nc) { s += rowbuf[jj - 1]; c += cntbuf[jj - 1]; }
            }
        }
        i0 = i1 + 1;
    }
}

template <class Get>
void windowmean(Get A, int64_t nr, int64_t nc, int64_t w, bool gaps, float* out) {
    const int64_t wx = std::min(w, nc), wy = std::min(w, nr);
    if (gaps) windowmean_masked(A, nr, nc, wx, wy, out);
    else windowmean_dense(A, nr, nc, wx, wy, out);
}

// src/preprocess.jl:371-399 -- mask-aware box mean.
template <class T>
void masked_boxmean(const T* img, const uint8_t* mask, int64_t nr, int64_t nc, int64_t w,
                    float* out) {
    const int64_t n = nr * nc;
    bool all = true;
    for (int64_t i = 0; i < n; ++i) all = all && mask[i];
    if (all) {
        bool gaps = false;
        for (int64_t i = 0; i < n && !gaps; ++i) gaps = std::isnan(as_f64(img[i]));
        windowmean([&](int64_t i, int64_t j) { return as_f64(img[i + j * nr]); }, nr, nc, w,
                   gaps, out);
        return;
    }
    std::vector<float> masked(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) masked[i] = mask[i] ? static_cast<float>(img[i]) : NAN;
    windowmean([&](int64_t i, int64_t j) { return static_cast<double>(masked[i + j * nr]); },
               nr, nc, w, true, out);
}

// src/preprocess.jl:447-460 -- erosion: valid only where the whole (clamped) window is valid.
void erode_mask(const uint8_t* mask, int64_t nr, int64_t nc, int64_t w, uint8_t* out) {
    const int64_t n = nr * nc;
    bool all = true;
    for (int64_t i = 0; i < n; ++i) all = all && mask[i];
    if (all) { std::memcpy(out, mask, static_cast<size_t>(n)); return; }
    const Margins m = margins(std::min(w, nc), std::min(w, nr));
    std::vector<uint8_t> tmp(static_cast<size_t>(n));
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            uint8_t v = 1;
            for (int64_t q = std::max<int64_t>(i - m.ly, 0); q <= std::min(i + m.ry, nr - 1); ++q)
                v = v && mask[q + j * nr];
            tmp[i + j * nr] = v;
        }
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            uint8_t v = 1;
            for (int64_t q = std::max<int64_t>(j - m.lx, 0); q <= std::min(j + m.rx, nc - 1); ++q)
                v = v && tmp[i + q * nr];
            out[i + j * nr] = v;
        }
}

// src/preprocess.jl:275-288 -- non-finite outputs become zero and invalid; the mask erodes.
void filtered(float* out, const uint8_t* mask, int64_t nr, int64_t nc, int64_t w, uint8_t* vout) {
    erode_mask(mask, nr, nc, w, vout);
    for (int64_t i = 0; i < nr * nc; ++i)
        if (!std::isfinite(out[i])) { out[i] = 0.0f; vout[i] = 0; }
}

// src/preprocess.jl:304-312 -- highpass.
template <class T>
void highpass(const T* img, const uint8_t* mask, int64_t nr, int64_t nc, int64_t w, float* out) {
    masked_boxmean(img, mask, nr, nc, w, out);
    for (int64_t i = 0; i < nr * nc; ++i)
        out[i] = (mask[i] && std::isfinite(out[i])) ? static_cast<float>(img[i]) - out[i] : NAN;
}

// src/preprocess.jl:333-351, 416-438 -- Wallis with the two-pass local deviation.
template <class T>
void wallis(const T* img, const uint8_t* mask, int64_t nr, int64_t nc, int64_t w,
            double min_std, float* out) {
    const int64_t n = nr * nc;
    std::vector<float> mean(static_cast<size_t>(n)), dev2(static_cast<size_t>(n)), msd(static_cast<size_t>(n));
    masked_boxmean(img, mask, nr, nc, w, mean.data());
    bool gaps = false;
    for (int64_t i = 0; i < n; ++i) {
        if (mask[i] && std::isfinite(mean[i])) {
            const float d = static_cast<float>(img[i]) - mean[i];
            const float v = d * d;
            dev2[i] = v;
            gaps = gaps || std::isnan(v);
        } else {
            dev2[i] = NAN;
            gaps = true;
        }
    }
    windowmean([&](int64_t i, int64_t j) { return static_cast<double>(dev2[i + j * nr]); }, nr,
               nc, w, gaps, msd.data());
    // sqrt(max(msd, 0f0)): Julia's max keeps a NaN.
    for (int64_t i = 0; i < n; ++i)
        if (!std::isnan(msd[i])) msd[i] = std::sqrt(std::max(msd[i], 0.0f));
    const float floor_sd = static_cast<float>(min_std);
    for (int64_t i = 0; i < n; ++i) {
        if (!mask[i] || !std::isfinite(mean[i]) || !std::isfinite(msd[i])) { out[i] = NAN; continue; }
        const float s = std::max(msd[i], floor_sd);
        out[i] = s > 0.0f ? (static_cast<float>(img[i]) - mean[i]) / s : NAN;
    }
}

// src/preprocess.jl:546-592 -- _to_uint8: mean +- 3 sd of the valid pixels onto 0..255.
template <class T>
void to_uint8(const T* img, const uint8_t* mask, int64_t n, uint8_t* out) {
    int64_t cnt = 0;
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double v = as_f64(img[i]);
        if (mask[i] && std::isfinite(v)) { ++cnt; s += v; }
    }
    std::memset(out, 0, static_cast<size_t>(n));
    if (cnt == 0) return;
    const double mean = s / static_cast<double>(cnt);
    double ss = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double v = as_f64(img[i]);
        if (mask[i] && std::isfinite(v)) { const double d = v - mean; ss += d * d; }
    }
    const double sd = cnt > 1 ? std::sqrt(ss / static_cast<double>(cnt - 1)) : 0.0;
    if (sd == 0.0) {
        for (int64_t i = 0; i < n; ++i) out[i] = mask[i] ? 0x80 : 0x00;
        return;
    }
    const double lo = mean - 3.0 * sd;
    const double scale = 255.0 / (6.0 * sd);
    for (int64_t i = 0; i < n; ++i) {
        const double v = as_f64(img[i]);
        if (!mask[i] || !std::isfinite(v)) { out[i] = 0; continue; }
        double x = (v - lo) * scale;
        x = x < 0.0 ? 0.0 : (x > 255.0 ? 255.0 : x);
        out[i] = static_cast<uint8_t>(std::nearbyint(x));  // round half to even
    }
}

// One image through preprocess then quantize (src/api.jl:305-306).
// pre: 0 none, 1 highpass, 2 wallis; quant: 0 none, 1 uint8. Output element type: uint8 for
// quant 1; float32 when a filter ran; otherwise the input type (a copy, non-finite floats
// replaced by zero, src/preprocess.jl:492-507).
template <class T>
void prepare_one(const T* img, const uint8_t* mask, int64_t nr, int64_t nc, int pre, int64_t w,
                 double min_std, int quant, void* out, uint8_t* vout) {
    const int64_t n = nr * nc;
    if (pre == 0) {
        std::memcpy(vout, mask, static_cast<size_t>(n));
        if (quant == 1) { to_uint8(img, mask, n, static_cast<uint8_t*>(out)); return; }
        T* o = static_cast<T*>(out);
        for (int64_t i = 0; i < n; ++i) {
            const T v = img[i];
            o[i] = std::isfinite(as_f64(v)) ? v : T(0);
        }
        return;
    }
    std::vector<float> f(static_cast<size_t>(n));
    if (pre == 1) highpass(img, mask, nr, nc, w, f.data());
    else wallis(img, mask, nr, nc, w, min_std, f.data());
    filtered(f.data(), mask, nr, nc, w, vout);
    if (quant == 1) {
        std::vector<uint8_t> v2(vout, vout + n);
        to_uint8(f.data(), v2.data(), n, static_cast<uint8_t*>(out));
    } else {
        std::memcpy(out, f.data(), static_cast<size_t>(n) * 4);
    }
}

// ---------------------------------------------------------------------------------------------
// The multi-chip-size search: src/multichip.jl:106-422, src/outliers.jl:38-172, the window
// reductions of src/window.jl:474-637 and src/resample.jl:56-71, 190-325. Grid fields are
// column-major nr x nc.

struct MCParams {
    int64_t chip_base, chip_min, chip_max;
    double aspect;
    int64_t min_radius, stride, buffer;
    double min_frac;
    int up, measure;
    int outliers;  // 0 NoOutlierFilter, 1 GardnerFilter
    int64_t gwindow, giterations;
    double gfrac, gtol, gmad;
    int64_t fill_window;
    const double* angles;  // RotationSearch chip rotations (degrees), nang of them; 0: none
    int nang;
    int nlev;     // per-level measures (measure_at, src/types.jl:893-894); 0: `measure` always
    int lev[8];
};

// src/window.jl:565-582.
void insertion_sort(float* b, int64_t n) {
    for (int64_t k = 1; k < n; ++k) {
        const float v = b[k];
        int64_t m = k - 1;
        while (m >= 0 && b[m] > v) { b[m + 1] = b[m]; --m; }
        b[m + 1] = v;
    }
}
float sorted_median(const float* b, int64_t n) {
    return (n % 2 == 1) ? b[(n + 1) / 2 - 1] : (b[n / 2 - 1] + b[n / 2]) / 2.0f;
}

// src/window.jl:594-619 -- neighbours within tol of the centre (itself included).
void count_agreeing(const float* A, int64_t nr, int64_t nc, int64_t w, float t, float* out) {
    const Margins m = margins(std::min(w, nc), std::min(w, nr));
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            const float c = A[i + j * nr];
            if (std::isnan(c)) { out[i + j * nr] = 0.0f; continue; }
            int64_t n = 0;
            for (int64_t jj = std::max<int64_t>(j - m.lx, 0); jj <= std::min(j + m.rx, nc - 1); ++jj)
                for (int64_t ii = std::max<int64_t>(i - m.ly, 0); ii <= std::min(i + m.ry, nr - 1); ++ii)
                    if (std::fabs(A[ii + jj * nr] - c) < t) ++n;
            out[i + j * nr] = static_cast<float>(n);
        }
}

// src/window.jl:501-563 -- median and MAD over the window, NaN skipped, NaN when empty.
void windowmedmad(const float* A, int64_t nr, int64_t nc, int64_t w, float* med, float* mad) {
    const Margins m = margins(std::min(w, nc), std::min(w, nr));
    std::vector<float> buf(static_cast<size_t>((m.lx + m.rx + 1) * (m.ly + m.ry + 1)));
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            int64_t n = 0;
            for (int64_t jj = std::max<int64_t>(j - m.lx, 0); jj <= std::min(j + m.rx, nc - 1); ++jj)
                for (int64_t ii = std::max<int64_t>(i - m.ly, 0); ii <= std::min(i + m.ry, nr - 1); ++ii) {
                    const float v = A[ii + jj * nr];
                    if (!std::isnan(v)) buf[n++] = v;
                }
            if (n == 0) { med[i + j * nr] = NAN; mad[i + j * nr] = NAN; continue; }
            insertion_sort(buf.data(), n);
            const float md = sorted_median(buf.data(), n);
            for (int64_t k = 0; k < n; ++k) buf[k] = std::fabs(buf[k] - md);
            insertion_sort(buf.data(), n);
            med[i + j * nr] = md;
            mad[i + j * nr] = sorted_median(buf.data(), n);
        }
}

// src/outliers.jl:38-172 -- which displacements to keep.
void reject_outliers(const float* dx, const float* dy, const int64_t* rx, const int64_t* ry,
                     const uint8_t* valid, int64_t nr, int64_t nc, int up, const MCParams& P,
                     int64_t iterations, uint8_t* keep) {
    const int64_t n = nr * nc;
    for (int64_t i = 0; i < n; ++i) keep[i] = valid[i];
    if (P.outliers == 0) return;
    std::vector<float> nx(n), ny(n), ax(n), ay(n), mx(n), sx(n), my(n), sy(n);
    for (int64_t i = 0; i < n; ++i) {
        nx[i] = rx[i] > 0 ? dx[i] / static_cast<float>(rx[i]) : NAN;
        ny[i] = ry[i] > 0 ? dy[i] / static_cast<float>(ry[i]) : NAN;
    }
    const int64_t w = P.gwindow;
    const float needed = static_cast<float>(P.gfrac * static_cast<double>(w * w));
    const float tol = static_cast<float>(P.gtol);
    auto mask_to_nan = [&]() {
        for (int64_t i = 0; i < n; ++i)
            if (!keep[i]) { nx[i] = NAN; ny[i] = NAN; }
    };
    for (int64_t it = 0; it < iterations; ++it) {
        mask_to_nan();
        count_agreeing(nx.data(), nr, nc, w, tol, ax.data());
        count_agreeing(ny.data(), nr, nc, w, tol, ay.data());
        for (int64_t i = 0; i < n; ++i) keep[i] = (ax[i] >= needed && ay[i] >= needed) ? 1 : 0;
    }
    const int64_t n2 = std::max<int64_t>(iterations - 1, 1);
    for (int64_t it = 0; it < n2; ++it) {
        mask_to_nan();
        windowmedmad(nx.data(), nr, nc, w, mx.data(), sx.data());
        windowmedmad(ny.data(), nr, nc, w, my.data(), sy.data());
        for (int64_t i = 0; i < n; ++i) {
            if (!keep[i]) continue;
            const double floor_x = rx[i] > 0 ? 2.0 / static_cast<double>(up * rx[i]) : INFINITY;
            const double floor_y = ry[i] > 0 ? 2.0 / static_cast<double>(up * ry[i]) : INFINITY;
            const double tolx = std::max(P.gmad * static_cast<double>(sx[i]), floor_x);
            const double toly = std::max(P.gmad * static_cast<double>(sy[i]), floor_y);
            const bool kx = static_cast<double>(std::fabs(nx[i] - mx[i])) <= tolx;
            const bool ky = static_cast<double>(std::fabs(ny[i] - my[i])) <= toly;
            keep[i] = (kx && ky) ? 1 : 0;
        }
    }
}

// src/resample.jl:190-325 -- every position within Euclidean `radius` of a true (the exact
// squared-distance test the transform answers, evaluated directly over the disc).
void dilate_within(const uint8_t* m, int64_t nr, int64_t nc, int64_t radius, uint8_t* out) {
    const int64_t r2 = radius * radius;
    for (int64_t j = 0; j < nc; ++j)
        for (int64_t i = 0; i < nr; ++i) {
            uint8_t v = 0;
            for (int64_t dj = -radius; dj <= radius && !v; ++dj)
                for (int64_t di = -radius; di <= radius; ++di) {
                    if (di * di + dj * dj > r2) continue;
                    const int64_t ii = i + di, jj = j + dj;
                    if (ii < 0 || ii >= nr || jj < 0 || jj >= nc) continue;
                    if (m[ii + jj * nr]) { v = 1; break; }
                }
            out[i + j * nr] = v;
        }
}

// src/resample.jl:56-71 -- nearest, half-sample convention, a mask to a mask.
void resample_nearest(const uint8_t* A, int64_t sr, int64_t sc, int64_t dr, int64_t dc,
                      uint8_t* out) {
    const double ys = static_cast<double>(sr) / static_cast<double>(dr);
    const double xs = static_cast<double>(sc) / static_cast<double>(dc);
    for (int64_t j = 1; j <= dc; ++j) {
        const int64_t sj = std::clamp<int64_t>(floor_i((static_cast<double>(j) - 0.5) * xs) + 1, 1, sc);
        for (int64_t i = 1; i <= dr; ++i) {
            const int64_t si = std::clamp<int64_t>(floor_i((static_cast<double>(i) - 0.5) * ys) + 1, 1, sr);
            out[(i - 1) + (j - 1) * dr] = A[(si - 1) + (sj - 1) * sr];
        }
    }
}

// src/multichip.jl:347-390 -- three passes of two-phase median filling of NaN holes.
void fill_holes(float* dx, float* dy, int64_t nr, int64_t nc, int64_t w, std::vector<uint8_t>& filled) {
    const int64_t lo = w / 2, hi = w - 1 - lo;
    const int64_t needed = 2 * w * w / 3;
    std::vector<float> bx(static_cast<size_t>(w * w)), by(static_cast<size_t>(w * w));
    struct Pend { int64_t idx; float x, y; };
    for (int pass = 0; pass < 3; ++pass) {
        std::vector<Pend> pending;
        for (int64_t j = 0; j < nc; ++j)
            for (int64_t i = 0; i < nr; ++i) {
                if (!std::isnan(dx[i + j * nr])) continue;
                int64_t n = 0;
                for (int64_t jj = std::max<int64_t>(j - lo, 0); jj <= std::min(j + hi, nc - 1); ++jj)
                    for (int64_t ii = std::max<int64_t>(i - lo, 0); ii <= std::min(i + hi, nr - 1); ++ii) {
                        const float v = dx[ii + jj * nr];
                        if (std::isnan(v)) continue;
                        bx[n] = v;
                        by[n] = dy[ii + jj * nr];
                        ++n;
                    }
                if (n < needed) continue;
                insertion_sort(bx.data(), n);
                insertion_sort(by.data(), n);
                pending.push_back({i + j * nr, sorted_median(bx.data(), n), sorted_median(by.data(), n)});
            }
        if (pending.empty()) break;
        for (const auto& q : pending) {
            dx[q.idx] = q.x;
            dy[q.idx] = q.y;
            filled[q.idx] = 1;
        }
    }
}

template <class T>
struct MCImages {
    const T* ref;
    const T* sec;
    const uint8_t* refv;
    const uint8_t* secv;
    int64_t nrows, ncols;
};

template <class T>
void run_track(const MCImages<T>& I, const double* x, const double* y, const int64_t* rx,
               const int64_t* ry, const double* dx0, const double* dy0, const int64_t* csx,
               const int64_t* csy, int64_t n, int up, int measure, float* odx, float* ody,
               float* oc, uint8_t* os, int nthreads, const double* angles, int nang) {
    Points p{x, y, dx0, dy0, rx, ry, csx, csy, n};
    track_impl(I.ref, I.sec, I.refv, I.secv, I.nrows, I.ncols, p, up, measure, odx, ody, oc, os,
               nthreads, angles, nang);
}

// src/multichip.jl:106-422 -- correlate_multichip over a gridded point set (gr x gc).
template <class T>
void multichip(const MCImages<T>& I, const double* gx, const double* gy, const int64_t* grx,
               const int64_t* gry, const double* gdx0, const double* gdy0, int64_t gr, int64_t gc,
               const MCParams& P, float* rdx, float* rdy, float* rcorr, uint16_t* rcs,
               uint8_t* rinterp, int nthreads) {
    const int64_t n = gr * gc;
    for (int64_t i = 0; i < n; ++i) {
        rdx[i] = NAN; rdy[i] = NAN; rcorr[i] = NAN; rcs[i] = 0; rinterp[i] = 0;
    }
    std::vector<int64_t> sizes;
    for (int64_t cs = P.chip_base; cs <= P.chip_max; cs *= 2)
        if (cs >= P.chip_min) sizes.push_back(cs);
    for (size_t li = 0; li < sizes.size(); ++li) {
        const int64_t cs = sizes[li];
        bool any = false;
        for (int64_t i = 0; i < n; ++i) any = any || rcs[i] == 0;
        if (!any) break;
        // measure_at(p, k) (src/types.jl:893-894): the level's entry, the last one repeating.
        const int measure =
            P.nlev > 0 ? P.lev[std::min(static_cast<int>(li), P.nlev - 1)] : P.measure;
        const int64_t csx = cs;
        const int64_t csy = 2 * static_cast<int64_t>(std::nearbyint(static_cast<double>(cs) * P.aspect / 2.0));
        // _level_points (src/multichip.jl:193-213) with sanitize! (src/points.jl:332-346).
        std::vector<int64_t> rx(n), ry(n), vcsx(n, csx), vcsy(n, csy);
        int64_t nsearch = 0;
        for (int64_t i = 0; i < n; ++i) {
            rx[i] = rcs[i] == 0 ? grx[i] : 0;
            ry[i] = rcs[i] == 0 ? gry[i] : 0;
            if (rx[i] <= 0 || ry[i] <= 0) { rx[i] = 0; ry[i] = 0; }
            else { rx[i] = std::max(rx[i], P.min_radius); ry[i] = std::max(ry[i], P.min_radius); ++nsearch; }
        }
        if (nsearch == 0) continue;
        // _coarse_pass (src/multichip.jl:224-288).
        std::vector<uint8_t> cmask(n, 1);
        bool level_off = false;
        {
            const int64_t st = P.stride;
            const int64_t cr = gr / st, cc = gc / st;  // rows stride:stride:gr
            const int64_t w = P.outliers == 1 ? P.gwindow : 0;
            if (!(cr < w || cc < w)) {
                const int64_t m = cr * cc;
                std::vector<double> cx(m), cy(m), cdx0(m), cdy0(m);
                std::vector<int64_t> crx(m), cry(m), ccsx(m, csx), ccsy(m, csy);
                const int64_t lo = st / 2, hi = st - 1 - lo;
                int64_t csearch = 0;
                for (int64_t jo = 0; jo < cc; ++jo)
                    for (int64_t io = 0; io < cr; ++io) {
                        const int64_t i = (io + 1) * st - 1, j = (jo + 1) * st - 1;  // 0-based fine index
                        const int64_t k = io + jo * cr, f = i + j * gr;
                        cx[k] = gx[f]; cy[k] = gy[f]; cdx0[k] = gdx0[f]; cdy0[k] = gdy0[f];
                        int64_t mx = 0, my = 0;
                        for (int64_t jj = std::max<int64_t>(j - lo, 0); jj <= std::min(j + hi, gc - 1); ++jj)
                            for (int64_t ii = std::max<int64_t>(i - lo, 0); ii <= std::min(i + hi, gr - 1); ++ii) {
                                mx = std::max(mx, rx[ii + jj * gr]);
                                my = std::max(my, ry[ii + jj * gr]);
                            }
                        crx[k] = mx; cry[k] = my;
                        if (mx > 0 && my > 0) ++csearch;
                    }
                if (csearch == 0) { level_off = true; }
                else {
                    std::vector<float> cdx(m), cdy(m), ccor(m);
                    std::vector<uint8_t> cs_(m), measured(m), keep(m), grown(m);
                    run_track(I, cx.data(), cy.data(), crx.data(), cry.data(), cdx0.data(), cdy0.data(),
                              ccsx.data(), ccsy.data(), m, 1, measure, cdx.data(), cdy.data(),
                              ccor.data(), cs_.data(), nthreads, P.angles, P.nang);
                    bool anym = false;
                    for (int64_t k = 0; k < m; ++k) { measured[k] = !std::isnan(cdx[k]); anym = anym || measured[k]; }
                    if (!anym) level_off = true;
                    else {
                        // relax(filter): one fewer stage-1 iteration, at least one.
                        const int64_t iters = std::max<int64_t>(P.giterations - 1, 1);
                        reject_outliers(cdx.data(), cdy.data(), crx.data(), cry.data(), measured.data(),
                                        cr, cc, P.up, P, iters, keep.data());
                        int64_t denom = 0, numer = 0;
                        for (int64_t k = 0; k < m; ++k) {
                            if (!measured[k]) keep[k] = 0;
                            if (crx[k] > 0 && measured[k]) { ++denom; if (keep[k]) ++numer; }
                        }
                        if (denom == 0 || static_cast<double>(numer) / static_cast<double>(denom) < P.min_frac)
                            level_off = true;
                        else {
                            dilate_within(keep.data(), cr, cc, P.buffer, grown.data());
                            resample_nearest(grown.data(), cr, cc, gr, gc, cmask.data());
                        }
                    }
                }
            }
        }
        if (level_off) continue;
        nsearch = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (!cmask[i]) { rx[i] = 0; ry[i] = 0; }
            if (rx[i] > 0 && ry[i] > 0) ++nsearch;
        }
        if (nsearch == 0) continue;
        std::vector<float> fdx(n), fdy(n), fc(n);
        std::vector<uint8_t> fs(n), measured(n), keep(n), filled(n, 0);
        run_track(I, gx, gy, rx.data(), ry.data(), gdx0, gdy0, vcsx.data(), vcsy.data(), n, P.up,
                  measure, fdx.data(), fdy.data(), fc.data(), fs.data(), nthreads, P.angles,
                  P.nang);
        // _reject_and_fill! (src/multichip.jl:318-330).
        for (int64_t i = 0; i < n; ++i) measured[i] = !std::isnan(fdx[i]);
        reject_outliers(fdx.data(), fdy.data(), rx.data(), ry.data(), measured.data(), gr, gc, P.up, P,
                        P.giterations, keep.data());
        for (int64_t i = 0; i < n; ++i)
            if (!keep[i]) { fdx[i] = NAN; fdy[i] = NAN; fc[i] = NAN; }
        fill_holes(fdx.data(), fdy.data(), gr, gc, P.fill_window, filled);
        // _merge_level! (src/multichip.jl:401-422).
        for (int64_t i = 0; i < n; ++i) {
            if (rcs[i] != 0) continue;
            if (std::isnan(fdx[i])) continue;
            rdx[i] = fdx[i]; rdy[i] = fdy[i]; rcorr[i] = fc[i];
            rcs[i] = static_cast<uint16_t>(cs);
            rinterp[i] = filled[i];
        }
    }
}

}  // namespace

extern "C" {

// Surface of one chip against one search window (src/correlate.jl:528-557).
// search: (ch+2ry-1) x (cw+2rx-1), chip: ch x cw, surface: 2ry x 2rx, all column-major.
// Returns 1 when the chip is degenerate (surface zero-filled), 0 otherwise, <0 on bad dtype.
int or_correlate(const void* search, const void* chip, int dtype, int64_t ch, int64_t cw,
                 int64_t rx, int64_t ry, int measure, float* surface) {
    bool ok;
    switch (dtype) {
        case OR_U8: ok = correlate_arrays(static_cast<const uint8_t*>(search),
                                          static_cast<const uint8_t*>(chip), ch, cw, rx, ry,
                                          measure, surface); break;
        case OR_U16: ok = correlate_arrays(static_cast<const uint16_t*>(search),
                                           static_cast<const uint16_t*>(chip), ch, cw, rx, ry,
                                           measure, surface); break;
        case OR_F32: ok = correlate_arrays(static_cast<const float*>(search),
                                           static_cast<const float*>(chip), ch, cw, rx, ry,
                                           measure, surface); break;
        case OR_I16: ok = correlate_arrays(static_cast<const int16_t*>(search),
                                           static_cast<const int16_t*>(chip), ch, cw, rx, ry,
                                           measure, surface); break;
        case OR_F64: ok = correlate_arrays(static_cast<const double*>(search),
                                           static_cast<const double*>(chip), ch, cw, rx, ry,
                                           measure, surface); break;
        default: return -1;
    }
    return ok ? 0 : 1;
}

// src/peak.jl:32-61, returned 0-based.
void or_peak_index(const float* surface, int64_t nr, int64_t nc, int64_t* i, int64_t* j) {
    peak_index(surface, nr, nc, i, j);
}

// src/peak.jl:196-294: dst is (2sh) x (2sw).
void or_pyrup(const float* src, int64_t sh, int64_t sw, float* dst) {
    std::vector<float> tmp;
    pyrup(src, sh, sw, dst, tmp);
}

// src/peak.jl:456-522.
void or_subpixel_peak(const float* surface, int64_t nr, int64_t nc, int64_t rx, int64_t ry,
                      int up, double* dx, double* dy, float* v) {
    std::vector<float> a, b, tmp;
    subpixel_peak(surface, nr, nc, rx, ry, up, dx, dy, v, a, b, tmp);
}

// track! over a point set (src/track.jl:103-152). Images and masks are nrows x ncols
// column-major; points are 8 SoA arrays of length n; outputs are prefilled by this call.
// up = 1 is NoRefine, otherwise PyramidRefine(up). nthreads <= 0 uses the OpenMP default.
// `angles` (nang of them, degrees, `about` already subtracted: the reference's angles(m)) turns
// on the rotation search (src/track.jl:313-350); nang = 0 is NoRotationSearch.
int or_track(const void* ref, const void* sec, const uint8_t* refv, const uint8_t* secv,
             int64_t nrows, int64_t ncols, int dtype, const double* x, const double* y,
             const int64_t* rx, const int64_t* ry, const double* dx0, const double* dy0,
             const int64_t* csx, const int64_t* csy, int64_t n, int up, int measure,
             float* dx, float* dy, float* corr, uint8_t* searched, int nthreads,
             const double* angles, int nang) {
    Points p{x, y, dx0, dy0, rx, ry, csx, csy, n};
    auto run = [&](auto* r, auto* s) {
        return track_impl(r, s, refv, secv, nrows, ncols, p, up, measure, dx, dy, corr, searched,
                          nthreads, angles, nang);
    };
    switch (dtype) {
        case OR_U8: return run(static_cast<const uint8_t*>(ref), static_cast<const uint8_t*>(sec));
        case OR_U16:
            return run(static_cast<const uint16_t*>(ref), static_cast<const uint16_t*>(sec));
        case OR_F32: return run(static_cast<const float*>(ref), static_cast<const float*>(sec));
        case OR_I16: return run(static_cast<const int16_t*>(ref), static_cast<const int16_t*>(sec));
        case OR_F64: return run(static_cast<const double*>(ref), static_cast<const double*>(sec));
        default: return -1;
    }
}

// _rotate_chip (src/track.jl:377-409) of one ch x cw chip into `out` (Float32, ch x cw).
int or_rotate_chip(const void* chip, int dtype, int64_t ch, int64_t cw, double deg, float* out) {
    auto run = [&](auto* c) {
        rotate_chip([&](int64_t i, int64_t j) { return as_f64(c[i + j * ch]); }, ch, cw, deg, out);
        return 0;
    };
    switch (dtype) {
        case OR_U8: return run(static_cast<const uint8_t*>(chip));
        case OR_U16: return run(static_cast<const uint16_t*>(chip));
        case OR_F32: return run(static_cast<const float*>(chip));
        case OR_I16: return run(static_cast<const int16_t*>(chip));
        case OR_F64: return run(static_cast<const double*>(chip));
        default: return -1;
    }
}

// preprocess + quantize of one image (src/api.jl:305-306; src/preprocess.jl). `mask` may be
// NULL (finiteness for float types, all-valid otherwise). `out` must hold nrows*ncols
// elements of the output type (uint8 when quant = 1, float32 when a filter ran, else the
// input type); `vout` receives the output mask.
int or_prepare(const void* img, const uint8_t* mask, int64_t nrows, int64_t ncols, int dtype,
               int pre, int64_t width, double min_std, int quant, void* out, uint8_t* vout) {
    const int64_t n = nrows * ncols;
    std::vector<uint8_t> m(static_cast<size_t>(n), 1);
    auto run = [&](auto* p) {
        if (mask) std::memcpy(m.data(), mask, static_cast<size_t>(n));
        else for (int64_t i = 0; i < n; ++i) m[i] = std::isfinite(as_f64(p[i])) ? 1 : 0;
        prepare_one(p, m.data(), nrows, ncols, pre, width, min_std, quant, out, vout);
    };
    switch (dtype) {
        case OR_U8: run(static_cast<const uint8_t*>(img)); break;
        case OR_U16: run(static_cast<const uint16_t*>(img)); break;
        case OR_F32: run(static_cast<const float*>(img)); break;
        case OR_I16: run(static_cast<const int16_t*>(img)); break;
        case OR_F64: run(static_cast<const double*>(img)); break;
        default: return -1;
    }
    return 0;
}

// correlate_multichip (src/multichip.jl:106-137) over a gridded point set of gr x gc points
// (column-major fields). params (doubles): chip_base, chip_min, chip_max, aspect, min_radius,
// stride, buffer, min_frac, up, measure, outliers, window, iterations, min_agree_fraction,
// agree_tolerance, mad_scale, fill_window, the per-level measure count and 8 per-level
// measures. `angles`, `nang`: the rotation search, as or_track.
int or_multichip(const void* ref, const void* sec, const uint8_t* refv, const uint8_t* secv,
                 int64_t nrows, int64_t ncols, int dtype, const double* gx, const double* gy,
                 const int64_t* grx, const int64_t* gry, const double* gdx0, const double* gdy0,
                 int64_t gr, int64_t gc, const double* prm, float* dx, float* dy, float* corr,
                 uint16_t* chip, uint8_t* interp, int nthreads, const double* angles,
                 int nang) {
    MCParams P;
    P.angles = angles;
    P.nang = nang;
    P.chip_base = static_cast<int64_t>(prm[0]);
    P.chip_min = static_cast<int64_t>(prm[1]);
    P.chip_max = static_cast<int64_t>(prm[2]);
    P.aspect = prm[3];
    P.min_radius = static_cast<int64_t>(prm[4]);
    P.stride = static_cast<int64_t>(prm[5]);
    P.buffer = static_cast<int64_t>(prm[6]);
    P.min_frac = prm[7];
    P.up = static_cast<int>(prm[8]);
    P.measure = static_cast<int>(prm[9]);
    P.outliers = static_cast<int>(prm[10]);
    P.gwindow = static_cast<int64_t>(prm[11]);
    P.giterations = static_cast<int64_t>(prm[12]);
    P.gfrac = prm[13];
    P.gtol = prm[14];
    P.gmad = prm[15];
    P.fill_window = static_cast<int64_t>(prm[16]);
    P.nlev = static_cast<int>(prm[17]);
    for (int i = 0; i < 8; ++i) P.lev[i] = static_cast<int>(prm[18 + i]);
    auto run = [&](auto* r, auto* s) {
        using T = std::remove_const_t<std::remove_pointer_t<decltype(r)>>;
        MCImages<T> I{r, s, refv, secv, nrows, ncols};
        multichip(I, gx, gy, grx, gry, gdx0, gdy0, gr, gc, P, dx, dy, corr, chip, interp, nthreads);
    };
    switch (dtype) {
        case OR_U8: run(static_cast<const uint8_t*>(ref), static_cast<const uint8_t*>(sec)); break;
        case OR_U16: run(static_cast<const uint16_t*>(ref), static_cast<const uint16_t*>(sec)); break;
        case OR_F32: run(static_cast<const float*>(ref), static_cast<const float*>(sec)); break;
        case OR_I16: run(static_cast<const int16_t*>(ref), static_cast<const int16_t*>(sec)); break;
        default: return -1;
    }
    return 0;
}

// Gardner / NoOutlierFilter rejection alone (src/outliers.jl:38-160), for tests.
int or_reject_outliers(const float* dx, const float* dy, const int64_t* rx, const int64_t* ry,
                       const uint8_t* valid, int64_t nr, int64_t nc, int up, int outliers,
                       int64_t window, int64_t iterations, double frac, double tol, double mad,
                       uint8_t* keep) {
    MCParams P{};
    P.outliers = outliers; P.gwindow = window; P.giterations = iterations;
    P.gfrac = frac; P.gtol = tol; P.gmad = mad;
    reject_outliers(dx, dy, rx, ry, valid, nr, nc, up, P, iterations, keep);
    return 0;
}

int or_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
