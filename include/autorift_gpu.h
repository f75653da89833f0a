/*
 * autorift_gpu.h -- C ABI of the B200 (sm_100a) dense ZNCC tracker.
 *
 * The drop-in boundary for AutoRIFT.jl's correlator. Every entry point takes plain pointers
 * and sizes, returns an int status (AR_OK = 0), and never retains a caller's host pointer past
 * return. Images, masks and point-set fields use Julia's layout: matrices are column-major
 * (rows fastest), masks are one byte per pixel (Matrix{Bool}, not BitMatrix).
 *
 * Citations are to the AutoRIFT.jl source the entry point replaces. The reference's only FFI
 * is its FFTW binding (src/plans.jl:271-312: const library path, ccall, opaque Ptr{Cvoid}
 * handles, errors raised on the Julia side); these entry points follow the same idiom.
 */
#ifndef AUTORIFT_GPU_H
#define AUTORIFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum {
    AR_OK = 0,
    AR_ERR_ARG = 1,         /* a null pointer or an out-of-range argument */
    AR_ERR_SIZE = 2,        /* array extents that do not agree (Julia DimensionMismatch) */
    AR_ERR_OOM = 3,         /* device allocation failed */
    AR_ERR_TIMEOUT = 4,     /* a bounded wait ran out */
    AR_ERR_CUDA = 5,        /* a CUDA runtime error; ar_last_error has the text */
    AR_ERR_UNSUPPORTED = 6  /* a geometry or element type this build does not handle */
};

/* Element types of an image pair (the T of ImagePair{T}, src/preprocess.jl:41-62). */
enum { AR_U8 = 0, AR_U16 = 1, AR_F32 = 2, AR_I16 = 3, AR_F64 = 4 };

/* Similarity measures (ZNCC, NCC of src/types.jl:104-140). */
enum { AR_ZNCC = 0, AR_NCC = 1 };

typedef struct ar_ctx ar_ctx;   /* one device, its streams and scratch */
typedef struct ar_pair ar_pair; /* a device-resident image pair with its validity mask */

/*
 * A point set: the eight SoA fields of PointSet{N} (src/points.jl:50-74), flattened in
 * Julia's memory order (`scatter`, src/points.jl:276-281). Coordinates are 1-based pixel
 * positions as in Julia. For ar_track the pointers are host memory; for ar_track_device they
 * are device memory.
 */
typedef struct {
    const double* x;
    const double* y;
    const int64_t* radius_x;
    const int64_t* radius_y;
    const double* dx_prior;
    const double* dy_prior;
    const int64_t* chip_size_x;
    const int64_t* chip_size_y;
    int64_t n;
} ar_points;

/* Library version (major * 10000 + minor * 100 + patch). */
int ar_version(void);

/* Create a context on `device` (a CUDA ordinal). Replaces the reference's process-wide FFT
 * plan cache and workspace pools (src/plans.jl:25-47, src/correlate.jl:294-350). */
int ar_ctx_create(int device, ar_ctx** out);
/* Destroy a context. Its pairs live in its memory pool: destroy them first. */
int ar_ctx_destroy(ar_ctx* ctx);

/* Copy the last error message of `ctx` (NUL-terminated, truncated to `size`). */
int ar_last_error(const ar_ctx* ctx, char* buf, size_t size);

/*
 * Upload an image pair (ImagePair, src/preprocess.jl:74-79). `ref` and `sec` are
 * nrows x ncols column-major arrays of `dtype`. `ref_valid`/`sec_valid` may be NULL, which
 * means finiteness for float types and all-valid for integer types, as ImagePair's default.
 * The pair keeps `valid(pair) = ref_valid .& sec_valid` (src/preprocess.jl:106). Returns once
 * the caller's arrays have been copied out (they may be reused at once); the transfers finish
 * in the background, ordered before every later use of the pair on any stream.
 */
int ar_pair_upload(ar_ctx* ctx, const void* ref, const void* sec, const uint8_t* ref_valid,
                   const uint8_t* sec_valid, int64_t nrows, int64_t ncols, int dtype,
                   ar_pair** out);
int ar_pair_destroy(ar_pair* pair);

/* Pre-correlation filter and quantisation methods (src/types.jl:259-499). */
enum { AR_PRE_NONE = 0, AR_PRE_HIGHPASS = 1, AR_PRE_WALLIS = 2 };
enum { AR_QUANT_NONE = 0, AR_QUANT_UINT8 = 1 };

typedef struct {
    int preprocess;  /* AR_PRE_*: NoPreprocess, Highpass(width), Wallis(width, min_std) */
    int width;       /* filter width, odd and >= 3 (ignored for AR_PRE_NONE) */
    double min_std;  /* Wallis divisor floor, >= 0 */
    int quantize;    /* AR_QUANT_*: NoQuantize or QuantizeUInt8 */
} ar_prepare_opts;

/*
 * `_prepare(pair, p)` (src/api.jl:305-311): preprocess then quantize each image of `raw`
 * (src/preprocess.jl:131-160, 275-460, 477-592) into a new device pair. The result's element
 * type is UInt8 under AR_QUANT_UINT8, Float32 when a filter ran without quantisation, else the
 * input type; its masks are the filtered (eroded) masks. `raw` is unchanged. Returns once the
 * work is queued on the context's stream; every later use of the new pair, on any stream, is
 * ordered after it (ar_synchronize waits for it).
 */
int ar_prepare(ar_ctx* ctx, const ar_pair* raw, const ar_prepare_opts* opts, ar_pair** out);

/* Copy a pair's images and masks back to host arrays (any may be NULL). */
int ar_pair_download(ar_ctx* ctx, const ar_pair* pair, void* ref, void* sec, uint8_t* ref_valid,
                     uint8_t* sec_valid);

/* Element type and extents of an uploaded pair. */
int ar_pair_info(const ar_pair* pair, int* dtype, int64_t* nrows, int64_t* ncols);

/*
 * track! (src/track.jl:103-152): correlate `pair` at every searchable point of `pts`.
 * `upsampling` is 1 for NoRefine or a power of two (PyramidRefine, src/types.jl:215-230);
 * `measure` is AR_ZNCC or AR_NCC. Outputs are host arrays of length pts->n, overwritten in
 * full: dx, dy, correlation (NaN where there is no measurement) and searched (0/1), the
 * fields of DisplacementField (src/track.jl:46-62). Host points and outputs are copied in
 * and out inside the call; the call returns when the results are on the host.
 */
int ar_track(ar_ctx* ctx, const ar_pair* pair, const ar_points* pts, int upsampling,
             int measure, float* dx, float* dy, float* correlation, uint8_t* searched);

/*
 * ar_track with the rotation search (_correlate_rotations!, src/track.jl:313-409): every
 * point correlates its chip turned by each of the `count` angles (degrees, the reference's
 * angles(RotationSearch): `about` already subtracted; an angle of exactly 0 is the chip
 * itself), skips angles whose turned chip is degenerate and keeps the surface with the
 * strictly highest peak, first angle first; a point whose every angle is degenerate is
 * searched without a measurement. The turned chip is the reference's bilinear resample about
 * the chip centre (src/track.jl:377-409), rounded to Float32, so these passes correlate in
 * FP32/FP64 on CUDA cores for every element type. count = 0 is ar_track. At most
 * AR_MAX_ROTATION_ANGLES angles, finite and distinct.
 */
enum { AR_MAX_ROTATION_ANGLES = 64 };
int ar_track_rotated(ar_ctx* ctx, const ar_pair* pair, const ar_points* pts, int upsampling,
                     int measure, const double* angles, int count, float* dx, float* dy,
                     float* correlation, uint8_t* searched);

/*
 * As ar_track with device-resident points and outputs, enqueued on `stream` (a
 * cudaStream_t, or NULL for the context's stream). Returns after the kernels are enqueued;
 * one small device-to-host read of the pass geometry (src/track.jl:176-197) synchronises.
 */
int ar_track_device(ar_ctx* ctx, const ar_pair* pair, const ar_points* pts_dev,
                    int upsampling, int measure, float* dx_dev, float* dy_dev,
                    float* correlation_dev, uint8_t* searched_dev, void* stream);

/* ar_track_device with the rotation search of ar_track_rotated (`angles`: host array). */
int ar_track_device_rotated(ar_ctx* ctx, const ar_pair* pair, const ar_points* pts_dev,
                            int upsampling, int measure, const double* angles, int count,
                            float* dx_dev, float* dy_dev, float* correlation_dev,
                            uint8_t* searched_dev, void* stream);

/*
 * ar_track_device without any device allocation. No counterpart in the reference: it exists
 * for callers that cannot allocate device memory when they correlate -- a host that owns the
 * device pool and hands out only planned buffers (a fixed-budget or real-time service), code
 * running under another framework's allocator, or a pipeline that must not hit cudaMalloc's
 * implicit synchronisation. The caller passes device pointers for everything it owns: the
 * images and the combined validity mask (nrows x ncols, column-major, `dtype`), the point
 * set (as in ar_track_device) and the outputs. No context is needed; the kernels run on
 * `stream` (NULL is the legacy default stream) of the current device.
 *
 * The pass's scratch (the sub-pixel refinement queue and the pass-geometry words) lives in a
 * static device array of this library sized for at most 32768 points per call (about 3.8 MB,
 * resident on every GPU that loads the library until the process exits). Larger point sets
 * return AR_ERR_SIZE; split them. Every call shares the array and resets the parts that must
 * start at zero; two calls that overlap on the GPU (other streams or host threads) race on it
 * and must not be issued. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before any stream
 * capture. Like ar_track_device, one small device-to-host read of the pass geometry
 * synchronises the stream; the call then returns once the pass has completed on `stream`,
 * with AR_ERR_TIMEOUT if a bounded device wait ran out (the outputs are then incomplete).
 * `err` (may be NULL) receives a message on failure.
 */
int ar_track_device_static(const void* ref, const void* sec, const uint8_t* valid, int64_t nrows,
                           int64_t ncols, int dtype, const ar_points* pts_dev, int upsampling,
                           int measure, float* dx_dev, float* dy_dev, float* correlation_dev,
                           uint8_t* searched_dev, void* stream, char* err, size_t err_size);

/*
 * Diagnostic: how many device buffers and events the library's track scratch has allocated or
 * created in this process so far. ar_track_device_static never adds to it. No reference
 * counterpart.
 */
int ar_scratch_allocations(int64_t* count);

/* The parameters correlate_multichip reads (Params, src/types.jl:781-829). */
typedef struct {
    int chip_size_base, chip_size_min, chip_size_max; /* levels chip_size_base * 2^k */
    double chip_aspect;
    int min_search_radius, coarse_stride, coarse_buffer;
    double min_coarse_valid_fraction;
    int upsampling;      /* PyramidRefine factor, or 1 for NoRefine */
    int measure;         /* AR_ZNCC or AR_NCC */
    int outliers;        /* 0 NoOutlierFilter, 1 GardnerFilter */
    int outlier_window, outlier_iterations;
    double min_agree_fraction, agree_tolerance, mad_scale;
    int fill_window;
    /* Rotation search (RotationSearch, src/types.jl:529-577): the chip rotations each
     * correlation tries, in degrees with `about` already subtracted (the reference's
     * angles(m)); rotation_count 0 is NoRotationSearch. At most AR_MAX_ROTATION_ANGLES finite,
     * distinct angles. The array is read during the call (ar_submit copies it). */
    int rotation_count;
    const double* rotation_angles;
    /* Per-level similarity (a `similarity` tuple; measure_at, src/types.jl:893-894): level k
     * (1 = finest) uses level_measures[min(k, count) - 1], AR_ZNCC or AR_NCC; count 0 uses
     * `measure` at every level. At most 8 entries, no more than the chip-size levels. */
    int level_measure_count;
    int level_measures[8];
} ar_multichip_params;

/*
 * correlate_multichip (src/multichip.jl:106-137) on a prepared pair over a gridded point set
 * (PointSet{2}, grid_rows x grid_cols, fields flattened column-major; its chip-size fields are
 * ignored: each level sets them). Host grid and host outputs of grid_rows*grid_cols elements:
 * the fields of MultichipResult (src/multichip.jl:74-80) -- dx, dy, correlation (NaN where no
 * level resolved the point), chip_size (0 there) and interpolated (0/1).
 */
int ar_multichip(ar_ctx* ctx, const ar_pair* pair, const ar_points* grid, int64_t grid_rows,
                 int64_t grid_cols, const ar_multichip_params* params, float* dx, float* dy,
                 float* correlation, uint16_t* chip_size, uint8_t* interpolated);

/*
 * ar_multichip with the grid fields and the outputs in device memory, run on `stream` (NULL:
 * the context's stream). The grid coordinates and priors must be finite (not re-checked on
 * the device). Each level reads a few counters back to take the reference's early exits, so
 * the call returns once the search has completed on `stream`.
 */
int ar_multichip_device(ar_ctx* ctx, const ar_pair* pair, const ar_points* grid_dev,
                        int64_t grid_rows, int64_t grid_cols, const ar_multichip_params* params,
                        float* dx_dev, float* dy_dev, float* correlation_dev,
                        uint16_t* chip_size_dev, uint8_t* interpolated_dev, void* stream);

/*
 * Diagnostic: one tensor-core product (tcgen05.mma kind::i8, unsigned 8-bit operands, 32-bit
 * integer accumulator) of two operand images placed in shared memory as given, read through
 * SWIZZLE_NONE K-major descriptors. params = {a_off, a_lbo, a_sbo, a_kstep, b_off, b_lbo,
 * b_sbo, b_kstep, M, N, nk, dstep, mode}: byte offsets and strides (multiples of 16), M in {64, 128},
 * N, and nk K-steps of 32 accumulated, step s reading at offset + s * kstep and, when dstep > 0,
 * adding into accumulator columns [s * dstep, s * dstep + N) of a cleared accumulator. `d_out`
 * receives the accumulator as 128 Tensor Memory lanes x (N + (nk - 1) * dstep) columns (int32,
 * lane-major) for mode 0; for mode 1, row (32 w + t) holds the 16 registers thread t of warp w
 * reads with the 16x256b.x4 pattern from its quarter's first 16 lanes, columns 0..31; mode 2
 * issues no product, so the kernel's bounded completion wait runs out and the call returns
 * AR_ERR_TIMEOUT with the context still usable (the failure path every tensor-core wait takes).
 * Descriptors that would read outside an image are rejected. It validates on a device the
 * operand and accumulator layouts the correlation kernel uses; no reference counterpart.
 */
int ar_tc_selftest(ar_ctx* ctx, const uint8_t* a_img, int a_bytes, const uint8_t* b_img,
                   int b_bytes, const int* params, int32_t* d_out);

/*
 * Serving: whole autorift() requests (src/api.jl:210-274 -- prepare both images, then the
 * multi-chip-size search over `grid`) queued on a context and run with continuous batching.
 * The context starts its request loop on the first ar_submit: AR_OPT_SERVE_SLOTS slots (each
 * a stream with its own scratch and memory, driven by its own host thread; default 4) take
 * requests in submission order as soon as the device memory the running requests hold (an
 * estimate of each request's footprint) leaves room within AR_OPT_SERVE_MEMORY_MB (default:
 * three quarters of the memory free when serving starts); a request larger than the budget
 * runs alone. Requests that arrive while others run overlap with them on the device; each
 * result is bit-identical to the same request run alone (ar_pair_upload, ar_prepare,
 * ar_multichip). Every array a request names -- images, masks (may be NULL), the grid's
 * fields and the outputs (grid_rows * grid_cols each) -- must stay valid until the request
 * has completed. No reference counterpart (the reference serves one pair per call).
 */
typedef struct {
    const void* reference;
    const void* secondary;
    const uint8_t* reference_valid;
    const uint8_t* secondary_valid;
    int64_t nrows, ncols;
    int dtype;
    ar_prepare_opts prepare;
    ar_multichip_params params;
    const ar_points* grid;
    int64_t grid_rows, grid_cols;
    float* dx;
    float* dy;
    float* correlation;
    uint16_t* chip_size;
    uint8_t* interpolated;
} ar_request;

typedef int64_t ar_ticket;

/* Queue a request; `ticket` identifies it. Thread-safe. */
int ar_submit(ar_ctx* ctx, const ar_request* request, ar_ticket* ticket);
/* Non-blocking: *done = 0 while pending; once complete *done = 1 and the request's status is
 * returned (its message through ar_last_error). */
int ar_poll(ar_ctx* ctx, ar_ticket ticket, int* done);
/* Block until the request completes (timeout_ms < 0: no limit) and return its status, or
 * AR_ERR_TIMEOUT if it has not completed within timeout_ms. */
int ar_wait(ar_ctx* ctx, ar_ticket ticket, int timeout_ms);
/* Milliseconds a completed request spent queued and running. */
int ar_request_times(ar_ctx* ctx, ar_ticket ticket, double* queued_ms, double* run_ms);
/* Forget a completed request (its ticket becomes unknown). */
int ar_release(ar_ctx* ctx, ar_ticket ticket);

/*
 * Context options. AR_OPT_TENSOR_CORES (default 1): UInt8 passes whose geometry fits (surface
 * at most 128 columns and 256 rows, chip at most 226 rows) compute the correlation numerator
 * on the tensor cores (exact 8-bit products, bit-identical results); 0 keeps every pass on the
 * CUDA-core kernel (direct FP32 for other element types, the plain method).
 * AR_OPT_SPLIT_BF16 (default 1; applies while AR_OPT_TENSOR_CORES is 1): UInt16, Int16 and
 * Float32 passes whose surfaces are at most 64 x 64 compute the numerator on the tensor cores
 * as split-BF16 products (each operand as two BF16 limbs, hi*hi + hi*lo + lo*hi accumulated in
 * FP32) -- 1 for passes whose chips are 64 px and up, 2 for every chip size, 0 never (direct
 * FP32). Surface values then differ from the FP64 ones by up to a few 1e-6 instead of ~1e-7;
 * the box sums and the normalisation stay FP64.
 * AR_OPT_AUTOTUNE (default 1): for UInt8 passes of 8192 points or more, the kernels that give
 * identical results (the two tensor-core kernels whose plans fit and the CUDA-core kernel) are
 * timed once per pass geometry on a sample of the pass, and the context runs the fastest from
 * then on; 0 always takes the first tensor-core kernel that fits.
 * AR_OPT_SHAPE_BINS (default 1): a multichip pass whose searchable points include both surfaces
 * of at most 64 x 64 and larger ones runs the two groups as separate launches, each planned for
 * its own largest surface (per-point radii); 0 runs every pass as one launch. Results are the
 * same either way.
 * AR_OPT_UINT8_KERNEL (default -1: the autotuner, or the fixed rule above): 2, 1 or 0 runs
 * every UInt8 pass on k_corr_tc2, k_corr_tc or the CUDA-core kernel where that kernel's plan
 * fits the pass (else the usual choice) -- for benchmarks and profiles; results are identical.
 * AR_OPT_SERVE_SLOTS and AR_OPT_SERVE_MEMORY_MB configure the request loop (see ar_submit);
 * they must be set before the first ar_submit. No reference counterpart.
 */
enum { AR_OPT_TENSOR_CORES = 1, AR_OPT_SERVE_SLOTS = 2, AR_OPT_SERVE_MEMORY_MB = 3,
       AR_OPT_SPLIT_BF16 = 4, AR_OPT_AUTOTUNE = 5, AR_OPT_SHAPE_BINS = 6,
       AR_OPT_UINT8_KERNEL = 7 };
int ar_ctx_set_option(ar_ctx* ctx, int option, int value);

/* The context's own CUDA stream (cudaStream_t), on which calls without a stream argument run;
 * for callers that order their own work or timing events after the library's. */
int ar_ctx_stream(ar_ctx* ctx, void** stream);

/*
 * The surface of one chip against one search window (correlate!, src/correlate.jl:528-557),
 * for host arrays: `search` is (ch+2ry-1) x (cw+2rx-1), `chip` ch x cw, `surface` 2ry x 2rx,
 * all column-major of `dtype`/float. `degenerate` receives 1 for a constant chip
 * (src/correlate.jl:571), whose surface is all zeros.
 */
int ar_correlate(ar_ctx* ctx, const void* search, const void* chip, int dtype, int64_t ch,
                 int64_t cw, int64_t rx, int64_t ry, int measure, float* surface,
                 int* degenerate);

/*
 * Sub-pixel refinement of `count` 5x5 patches (the cascade of subpixel_peak,
 * src/peak.jl:456-522, from the patch copy onward): `patches` holds count x 25 floats, each
 * patch column-major. Outputs are the row and column of the peak in the upsampled
 * (5*up) x (5*up) patch (0-based) and its value. Host arrays.
 */
int ar_refine_patches(ar_ctx* ctx, const float* patches, int64_t count, int upsampling,
                      int32_t* row, int32_t* col, float* value);

/*
 * Kernel timing, for benchmarks: when enabled, every track launch records CUDA events on its
 * stream around the correlation kernel and the refinement kernel, and the correlation kernel
 * counts the algorithmic FLOPs of the surfaces it computes (2 * chip area * surface area per
 * point). ar_kernel_times waits for the recorded events and returns the summed milliseconds
 * of each kernel, the number of track launches timed, the number of kernels the library
 * launched and the FLOP count, then resets. No reference counterpart (the reference times
 * from Julia: benchmark/run.jl).
 */
int ar_ctx_set_timing(ar_ctx* ctx, int enable);
int ar_kernel_times(ar_ctx* ctx, double* corr_ms, double* refine_ms, int64_t* tracks,
                    int64_t* launches, double* corr_flops);

/*
 * The UInt8 correlation kernel the autotuner kept for each pass geometry it has timed in this
 * context (AR_OPT_AUTOTUNE): five int32 per geometry -- largest chip rows, chip columns,
 * surface rows, surface columns, then the kernel (2: k_corr_tc2, 1: k_corr_tc, 0: k_corr, the
 * CUDA-core direct sum). Writes up to `cap` geometries to `out`; *count = the number tuned.
 * Diagnostics for benchmarks; no reference counterpart.
 */
int ar_ctx_tuned(ar_ctx* ctx, int32_t* out, int64_t cap, int64_t* count);

/* Block until all work the context enqueued has finished. */
int ar_synchronize(ar_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* AUTORIFT_GPU_H */
