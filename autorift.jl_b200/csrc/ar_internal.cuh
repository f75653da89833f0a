// Internal declarations shared by the CUDA translation units of libautorift_gpu.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "autorift_gpu.h"

namespace ar {

// Dynamic shared memory a kernel is allowed (cudaFuncAttributeMaxDynamicSharedMemorySize). The
// attribute belongs to the function, shared by every context and host thread of the process, so
// it is always set to this one value and each launch checks its own size against it: a launch
// can never find it lowered by a concurrent launch of the same kernel with a smaller plan.
constexpr int kDynSmemCap = 220 * 1024;

// Pass geometry: the summary of a point set that sizes a launch (src/track.jl:176-197).
struct PassGeometry {
    int64_t max_ch = 0, max_cw = 0;  // effective chip extents (2 * (size / 2))
    int64_t max_nr = 0, max_nc = 0;  // surface extents (2 * radius)
    int64_t padx = 0, pady = 0;      // virtual zero padding, 0 when every window fits
    int64_t searchable = 0;          // points with both radii > 0
};

// Device-resident point set (same field order as ar_points).
struct DevPoints {
    const double* x;
    const double* y;
    const int64_t* rx;
    const int64_t* ry;
    const double* dx0;
    const double* dy0;
    const int64_t* csx;
    const int64_t* csy;
    int64_t n;
};

// Rotation search (src/track.jl:313-409): the chip rotations each point of a pass tries, as
// sin and cos of the angle (deg * (pi / 180), C library sin and cos, computed on the host), and
// whether the angle is nonzero (an angle of exactly 0 correlates the chip itself). count 0 is
// NoRotationSearch. Passed to the correlation kernel by value.
constexpr int kMaxAngles = AR_MAX_ROTATION_ANGLES;
struct Rotation {
    int count = 0;
    double sn[kMaxAngles];
    double cs[kMaxAngles];
    unsigned char turn[kMaxAngles];
};

// Checks an angle list (finite, distinct, 1..kMaxAngles of them) and fills `out`; false with a
// message otherwise.
bool make_rotation(const double* deg, int count, Rotation* out, std::string* err);

struct DevOutputs {
    float* dx;
    float* dy;
    float* corr;
    uint8_t* searched;
};

// Scratch the track launch needs, owned by the context and grown on demand.
// Optional per-kernel timing: events recorded on the launch stream around the correlation and
// refinement kernels of each track launch, summed when queried. Off unless enabled.
struct KernelTimer {
    bool enabled = false;
    std::vector<std::array<cudaEvent_t, 3>> recs;  // before corr, after corr, after refine
    std::vector<cudaEvent_t> pool;
    long long launches = 0;  // kernels this library launched since the last query
    unsigned long long* flops = nullptr;  // device counter of surface FLOPs (while enabled)
    cudaEvent_t get();
};

struct TrackScratch {
    int* sub_count = nullptr;       // number of points queued for sub-pixel refinement
    int64_t* sub_point = nullptr;   // point index per queued item
    int32_t* sub_origin = nullptr;  // (i0, j0) of the 5x5 patch, 0-based, per item
    float* sub_patch = nullptr;     // 25 floats per item, column-major
    int64_t capacity = 0;
    int64_t* geom = nullptr;        // device-side pass geometry (8 int64)
    KernelTimer timer;
    // Recorded after the last pass that used these buffers; a pass on another stream waits
    // for it before reusing them.
    cudaEvent_t done = nullptr;
    // Set by a kernel whose bounded wait ran out (read and cleared by the synchronous calls).
    int* status = nullptr;
    // UInt8 passes use the tensor-core correlation when their geometry fits it.
    bool tensor_cores = true;
    // UInt16, Int16 and Float32 passes: 0 direct FP32 on CUDA cores, 1 split-BF16 tensor-core
    // products for chips of 64 px and up, 2 split-BF16 for every chip size (AR_OPT_SPLIT_BF16).
    int split_bf16 = 1;
    // UInt8 passes of at least kTuneMinPoints points: the tensor-core and CUDA-core kernels
    // (identical results) are timed once per pass geometry and the fastest kept in `tuned`
    // (key: chip and surface extents) -- AR_OPT_AUTOTUNE.
    bool autotune = true;
    // AR_OPT_UINT8_KERNEL: -1 the autotuner (or the fixed rule); 2, 1, 0 run k_corr_tc2,
    // k_corr_tc or the CUDA-core kernel on every UInt8 pass whose plan fits it.
    int uint8_kernel = -1;
    // Multichip passes whose searchable points have both small (up to 64 x 64) and larger
    // surfaces run each group as its own launch (AR_OPT_SHAPE_BINS).
    bool shape_bins = true;
    std::map<uint64_t, int> tuned;
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    // When set, the sub-pixel queue grows from this pool in stream order (no device-wide
    // synchronisation when a context first meets a larger pass).
    cudaMemPool_t pool = nullptr;
    // Set for a view of caller-provided memory (the allocation-free entry point): every buffer
    // above is already in place, nothing is ever allocated or created for it, and a pass that
    // would need more fails instead of growing it.
    bool fixed = false;
};

// Number of device buffers and events the track scratch has allocated or created in this
// process (a diagnostic: the allocation-free entry point must never add to it).
long long scratch_allocations();

// Reads and clears the pass status; AR-style: 0 ok, 1 a bounded device wait ran out.
cudaError_t read_status(TrackScratch& scratch, cudaStream_t stream, int* status);

// Host-side pass geometry of a host point set.
PassGeometry pass_geometry_host(const ar_points& p, int64_t nrows, int64_t ncols);

// Enqueue the track kernels. `geom` must describe `pts` (host- or device-computed).
// `surf_out`, when given, receives every searched point's surface (max_nr x max_nc floats per
// point, column-major with leading dimension nr of that point).
cudaError_t launch_track(int dtype, const void* ref, const void* sec, const uint8_t* valid,
                         int64_t nrows, int64_t ncols, const DevPoints& pts,
                         const PassGeometry& geom, int up, int measure, const DevOutputs& out,
                         TrackScratch& scratch, int num_sms, cudaStream_t stream,
                         std::string* err, float* surf_out = nullptr,
                         const Rotation* rot = nullptr);

// Device-side pass geometry for a device point set (one small synchronising read).
cudaError_t pass_geometry_device(const DevPoints& pts, int64_t nrows, int64_t ncols,
                                 TrackScratch& scratch, cudaStream_t stream, PassGeometry* out);

// One image through preprocess then quantize (src/api.jl:305-306) on the device.
// preprocess: 0 none, 1 highpass, 2 Wallis; quantize: 0 none, 1 uint8. `out` holds
// nrows*ncols elements of the output type (uint8 for quantize 1, float32 when a filter ran,
// else the input type); `ftmp` and `mtmp` are float scratch of the same length (ftmp used when
// a filter feeds the quantiser, mtmp by Wallis); `stats` is quant_stats_bytes() of scratch.
struct QuantStats;
struct PrepareJob {
    int dtype;
    const void* img;
    const uint8_t* mask;
    int64_t nrows, ncols;
    int preprocess, width;
    double min_std;
    int quantize;
    void* out;
    uint8_t* vout;
    float* ftmp;
    float* mtmp;
    QuantStats* stats;
};
size_t quant_stats_bytes();
int max_filter_width();
cudaError_t launch_prepare(const PrepareJob& job, cudaStream_t stream, long long* launches);

// The parameters of correlate_multichip (the Params fields src/multichip.jl reads).
struct MultichipParams {
    int64_t chip_base, chip_min, chip_max;
    double aspect;
    int64_t min_radius, stride, buffer;
    double min_frac;
    int up, measure;
    int outliers;  // 0 NoOutlierFilter, 1 GardnerFilter
    int64_t gwindow, giterations;
    double gfrac, gtol, gmad;
    int64_t fill_window;
    Rotation rot;  // the rotation search of every track pass (count 0: none)
    int n_level_measures;  // 0: `measure` at every level
    int level_measures[8];  // measure_at(p, k) = level_measures[min(k, n) - 1]
};

// One multichip run: a prepared pair, a gr x gc point grid (device, column-major), outputs
// (device) and a scratch block of multichip_arena_bytes(gr, gc).
struct MultichipJob {
    int dtype;
    const void* ref;
    const void* sec;
    const uint8_t* valid;
    int64_t nrows, ncols;
    const double* gx;
    const double* gy;
    const int64_t* grx;
    const int64_t* gry;
    const double* gdx0;
    const double* gdy0;
    int64_t gr, gc;
    MultichipParams P;
    float* dx;
    float* dy;
    float* corr;
    uint16_t* chip;
    uint8_t* interp;
    void* arena;
    size_t arena_bytes;
};
size_t multichip_arena_bytes(int64_t gr, int64_t gc);

// The request loop (ar_serve.cu).
struct ServeEngine;
ServeEngine* serve_create(int device, int slots, size_t budget, std::string* err);
void serve_destroy(ServeEngine* engine);
int serve_submit(ServeEngine* engine, const ar_request* req, int64_t* ticket, std::string* err);
int serve_poll(ServeEngine* engine, int64_t ticket, int* done, std::string* err);
int serve_wait(ServeEngine* engine, int64_t ticket, int timeout_ms, std::string* err);
int serve_times(ServeEngine* engine, int64_t ticket, double* queued_ms, double* run_ms);
int serve_release(ServeEngine* engine, int64_t ticket, std::string* err);

// One tensor-core product of two shared-memory operand images (the layout self-test):
// params = {a_off, a_lbo, a_sbo, a_kstep, b_off, b_lbo, b_sbo, b_kstep, M, N, nk, dstep}.
cudaError_t tc_probe(const uint8_t* a_img, int a_bytes, const uint8_t* b_img, int b_bytes,
                     const int* params, int32_t* d_out, int* status, cudaStream_t s,
                     std::string* err);
cudaError_t run_multichip(const MultichipJob& job, TrackScratch& scratch, int num_sms,
                          cudaStream_t stream, std::string* errmsg);

// Refine `count` patches already on the device.
cudaError_t launch_refine_patches(const float* patches, int64_t count, int up, int32_t* row,
                                  int32_t* col, float* value, int num_sms, cudaStream_t stream);

}  // namespace ar
